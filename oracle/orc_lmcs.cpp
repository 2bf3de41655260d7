// CPU oracle (test infrastructure only; see oracle.h): LMCS and joint Cb-Cr
// residuals of the general decoding path.
//   LmcsReshaper16::from_aps          filter.rs:2628-2705
//   apply_forward/inverse_plane_16    filter.rs:2708-2722
//   chroma_scale_for_luma             filter.rs:2725-2735
//   scale_chroma_residual             filter.rs:2740-2749
//   chroma_adj_luma                   decode_general.rs:4803-4835 (one VPDU)
//   joint Cb-Cr combination           decode_general.rs:3932-3955
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "../include/vvcg.h"
#include "oracle.h"

static const int kLmcsFpPrec = 11;  // filter.rs:22

extern "C" int orc_lmcs_build(const vvcg_lmcs_aps* aps, int bit_depth, vvcg_lmcs_tables* t) {
  memset(t, 0, sizeof(*t));
  const int bd = std::min(12, std::max(8, bit_depth));
  const int max_val = (1 << bd) - 1, log2_cw = bd - 4, init_cw = 1 << log2_cw;
  const int min_bin = std::min<int>(aps->min_bin_idx, 15);
  const int max_bin = std::max(std::min<int>(aps->max_bin_idx, 15), min_bin);
  int bin_cw[16] = {0}, input_pivot[17] = {0}, reshape_pivot[17] = {0};
  int fwd_scale[16], inv_scale[16], adj[16];
  for (int i = min_bin; i <= max_bin; i++) bin_cw[i] = std::max(0, init_cw + aps->bin_cw_delta[i]);
  for (int i = 0; i < 16; i++) {
    fwd_scale[i] = inv_scale[i] = adj[i] = 1 << kLmcsFpPrec;
    reshape_pivot[i + 1] = reshape_pivot[i] + bin_cw[i];
    input_pivot[i + 1] = input_pivot[i] + init_cw;
    fwd_scale[i] = ((bin_cw[i] << kLmcsFpPrec) + (1 << (log2_cw - 1))) >> log2_cw;
    if (bin_cw[i] == 0) {
      inv_scale[i] = 0;
      adj[i] = 1 << kLmcsFpPrec;
    } else {
      inv_scale[i] = (init_cw << kLmcsFpPrec) / bin_cw[i];
      const int denom = std::max(1, bin_cw[i] + aps->chroma_res_scaling_offset);
      adj[i] = (init_cw << kLmcsFpPrec) / denom;
    }
  }
  for (int s = 0; s <= max_val; s++) {
    const int iy = std::min(15, s >> log2_cw);
    const int fv = reshape_pivot[iy] + ((fwd_scale[iy] * (s - input_pivot[iy]) + (1 << (kLmcsFpPrec - 1))) >> kLmcsFpPrec);
    t->fwd_lut[s] = (uint16_t)std::min(max_val, std::max(0, fv));
    int ii = min_bin;
    while (ii <= max_bin && !(s < reshape_pivot[ii + 1])) ii++;
    ii = std::min(ii, 15);
    const int iv = input_pivot[ii] + ((inv_scale[ii] * (s - reshape_pivot[ii]) + (1 << (kLmcsFpPrec - 1))) >> kLmcsFpPrec);
    t->inv_lut[s] = (uint16_t)std::min(max_val, std::max(0, iv));
  }
  t->bit_depth = (uint8_t)bd;
  t->min_bin_idx = (uint8_t)min_bin;
  t->max_bin_idx = (uint8_t)max_bin;
  memcpy(t->reshape_pivot, reshape_pivot, sizeof(reshape_pivot));
  memcpy(t->chroma_adj_lut, adj, sizeof(adj));
  return 0;
}

extern "C" void orc_lmcs_map_plane(const vvcg_lmcs_tables* t, int inverse, uint16_t* p, int n) {
  const int cap = (1 << t->bit_depth) - 1;
  const uint16_t* lut = inverse ? t->inv_lut : t->fwd_lut;
  for (int i = 0; i < n; i++) p[i] = lut[std::min<int>(p[i], cap)];
}

static int chroma_scale_for_luma(const vvcg_lmcs_tables* t, int avg) {
  int i = t->min_bin_idx;
  while (i <= t->max_bin_idx && !(avg < t->reshape_pivot[i + 1])) i++;
  return t->chroma_adj_lut[std::min(i, 15)];
}

// chroma_adj_luma for the TU at luma (x, y): the VPDU's left column and top
// row averages, then chroma_scale_for_luma.
extern "C" int orc_lmcs_chroma_scale(const vvcg_lmcs_tables* t, const uint16_t* luma, int stride, int pw, int ph,
                                     int ctu, int x, int y) {
  const int vpdu = ctu == 128 ? 64 : ctu;
  const int vx = (x / vpdu) * vpdu, vy = (y / vpdu) * vpdu;
  const int n = std::min(64, vpdu);
  int sum = 0, count = 0;
  if (vx > 0)
    for (int i = 0; i < n; i++) {
      sum += luma[std::min(vy + i, ph - 1) * stride + vx - 1];
      count++;
    }
  if (vy > 0)
    for (int i = 0; i < n; i++) {
      sum += luma[(vy - 1) * stride + std::min(vx + i, pw - 1)];
      count++;
    }
  const int tz = __builtin_ctz((unsigned)n);
  const int dc = 1 << (std::min(12, std::max(8, (int)t->bit_depth)) - 1);
  int avg = count == 0 ? dc : count == n ? (sum + (1 << (tz - 1))) >> tz
                                          : count == 2 * n ? (sum + (1 << tz)) >> (tz + 1) : dc;
  return chroma_scale_for_luma(t, avg);
}

static inline int16_t sat16(int v) { return (int16_t)std::min(32767, std::max(-32768, v)); }

// One vvcg_cres_rec on int16 residuals in place. The reference keeps these
// residuals in i32; int16 storage saturates, which leaves the reconstruction
// clip(pred + residual, 0, maxVal) unchanged.
extern "C" void orc_chroma_residuals(const vvcg_cres_rec* r, int16_t* res) {
  const int n = (1 << r->log2_w) * (1 << r->log2_h);
  int16_t* cb = res + r->cb_off;
  int16_t* cr = res + r->cr_off;
  const bool single = r->flags & VVCG_CRES_SINGLE;
  if (!single)
    for (int i = 0; i < n; i++) {
      switch (r->joint) {
        case 3: cb[i] = sat16(cr[i] >> 1); break;
        case -3: cb[i] = sat16((-cr[i]) >> 1); break;
        case 1: cr[i] = sat16(cb[i] >> 1); break;
        case -1: cr[i] = sat16((-cb[i]) >> 1); break;
        case 2: cr[i] = cb[i]; break;
        case -2: cr[i] = sat16(-cb[i]); break;
        default: break;
      }
    }
  if (r->flags & VVCG_CRES_SCALE) {
    const int max_val = (1 << std::min(12, std::max(8, (int)r->bit_depth))) - 1;
    for (int c = 0; c < (single ? 1 : 2); c++) {
      int16_t* p = c ? cr : cb;
      for (int i = 0; i < n; i++) {
        const int v = std::min(max_val, std::max(-max_val - 1, (int)p[i]));
        const int sign = v < 0 ? -1 : 1;
        p[i] = sat16((int)(sign * (((int64_t)abs(v) * r->scale + (1 << (kLmcsFpPrec - 1))) >> kLmcsFpPrec)));
      }
    }
  }
}
