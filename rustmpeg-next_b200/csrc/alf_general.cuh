// ALF of the general decoding path (sm_100a), following apply_alf and its
// block functions (crates/rustmpeg-video/src/vvc/decode_general.rs:5225-5660)
// and derive_alf_class_4x4_vb_16 (filter.rs:1558-1691). Every CTU region
// reads only the unfiltered copies (src), so all regions run in parallel:
// one thread per 4x4 luma block (classification + 16 samples), one thread per
// chroma sample (chroma ALF, then CCALF added to it).
#pragma once
#include <stdint.h>

#include "../../include/vvcg.h"
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

struct AlfGenView {
  const uint16_t* p;
  int32_t stride, lw, lh;  // clamp bounds: min(visible, plane)
  __device__ __forceinline__ int get(int x, int y) const {
    return p[(size_t)clampi(y, 0, lh - 1) * stride + clampi(x, 0, lw - 1)];
  }
};

struct AlfGenPass {
  AlfGenView y, u, v;
  uint16_t* dst[3];
  int32_t dstride[3];
  int32_t pw, ph, cw, ch;        // plane sizes (chroma half)
  int32_t vis_w, vis_h, cvis_w, cvis_h;
  int32_t bd, ctu, ctu_cols;
  const vvcg_alf_ctu* ctus;
  const vvcg_alf_params* a;      // device copy
};

__device__ __forceinline__ int alf_clip_val(int bd, int idx) {
  return c_alf_clip[bd >= 12 ? 2 : (bd >= 10 ? 1 : 0)][idx & 3];
}

// filter.rs:1580-1691 derive_alf_class_4x4_vb_samples
__device__ void alf_classify_vb(const AlfGenView& v, int bx, int by, int vb_h, int vb_pos, int bd, int* cls,
                                int* tr) {
  int sv = 0, sh = 0, d0 = 0, d1 = 0;
  const int row_vb = (by % vb_h == vb_pos - 4) ? 1 : (by % vb_h == vb_pos) ? 2 : 0;
  for (int dy = -2; dy < 6; dy += 2) {
    if ((row_vb == 1 && dy == 4) || (row_vb == 2 && dy == -2)) continue;
    for (int dx = -2; dx < 6; dx += 2) {
      const int x = bx + dx, y = by + dy;
      int down = y - 1, up = y + 1, up2 = y + 2;
      if (y > 0) {
        const int yy = y % vb_h;
        if (vb_pos >= 2 && yy == vb_pos - 2) {
          up2 = y + 1;
        } else if (yy == vb_pos) {
          down = y;
        }
      }
      const int y0 = v.get(x, y) << 1, yu = v.get(x + 1, y + 1) << 1;
      sv += abs(y0 - v.get(x, down) - v.get(x, up)) + abs(yu - v.get(x + 1, y) - v.get(x + 1, up2));
      sh += abs(y0 - v.get(x + 1, y) - v.get(x - 1, y)) + abs(yu - v.get(x + 2, y + 1) - v.get(x, y + 1));
      d0 += abs(y0 - v.get(x - 1, down) - v.get(x + 1, up)) + abs(yu - v.get(x, y) - v.get(x + 2, up2));
      d1 += abs(y0 - v.get(x - 1, up) - v.get(x + 1, down)) + abs(yu - v.get(x, up2) - v.get(x + 2, y));
    }
  }
  const int yy = by % vb_h;
  const int scale = (vb_pos >= 4 && (yy == vb_pos - 4 || yy == vb_pos)) ? 96 : 64;
  const int act = clampi(((sv + sh) * scale) >> (bd + 4), 0, 15);
  int c = act == 0 ? 0 : act == 1 ? 1 : act <= 6 ? 2 : act <= 14 ? 3 : 4;
  int hv1, hv0, dhv, dd1, dd0, ddd;
  if (sv > sh) { hv1 = sv; hv0 = sh; dhv = 1; } else { hv1 = sh; hv0 = sv; dhv = 3; }
  if (d0 > d1) { dd1 = d0; dd0 = d1; ddd = 0; } else { dd1 = d1; dd0 = d0; ddd = 2; }
  int h1, h0, md, sd;
  if ((long long)dd1 * hv0 > (long long)hv1 * dd0) { h1 = dd1; h0 = dd0; md = ddd; sd = dhv; }
  else { h1 = hv1; h0 = hv0; md = dhv; sd = ddd; }
  int ds = 0;
  if (h1 > 2 * h0) ds = 1;
  if (h1 * 2 > 9 * h0) ds = 2;
  if (ds > 0) c += (((md & 1) << 1) + ds) * 5;
  *cls = c;
  *tr = (0xDE84 >> (2 * (md * 2 + (sd >> 1)))) & 3;  // {0, 1, 0, 2, 2, 3, 1, 3}
}

// alf_luma_block (decode_general.rs:5411-5565) for the 4x4 block at
// (4 * bx4, 4 * by4); blocks of CTUs without luma ALF, and samples outside
// the visible picture, are copied.
__global__ void __launch_bounds__(128) k_alf_general_luma(AlfGenPass P) {
  const int nbx = (P.pw + 3) >> 2, nby = (P.ph + 3) >> 2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nbx * nby; i += gridDim.x * blockDim.x) {
    const int bx = (i % nbx) * 4, by = (i / nbx) * 4;
    const bool vis = bx < P.vis_w && by < P.vis_h;
    const vvcg_alf_ctu m = vis ? P.ctus[(by / P.ctu) * P.ctu_cols + bx / P.ctu] : vvcg_alf_ctu{};
    const int xe = min(bx + 4, P.pw), ye = min(by + 4, P.ph);
    uint16_t* d = P.dst[0];
    const int ds = P.dstride[0];
    if (!vis || m.luma_mode == VVCG_ALF_OFF) {
      for (int y = by; y < ye; y++)
        for (int x = bx; x < xe; x++) d[(size_t)y * ds + x] = P.y.p[(size_t)y * P.y.stride + x];
      continue;
    }
    const int vb_h = P.ctu, vb_pos = P.ctu - 4, bd = P.bd, maxv = (1 << bd) - 1;
    int cls, tr;
    alf_classify_vb(P.y, bx, by, vb_h, vb_pos, bd, &cls, &tr);
    const vvcg_alf_params& a = *P.a;
    int coeffs[12], clips[12];
    if (m.luma_mode == VVCG_ALF_FIXED) {
      const int fi = c_alf_class_to_filter[min((int)m.luma_set, 15) * 25 + min(cls, 24)];
#pragma unroll
      for (int k = 0; k < 12; k++) {
        coeffs[k] = c_alf_fixed[fi * 13 + k];
        clips[k] = 0;
      }
    } else {
      const int fi = min((int)a.coeff_delta_idx[min(cls, 24)], max(1, (int)a.num_luma_filters) - 1);
      const bool cl = a.luma_clip && fi < a.num_luma_filters;
#pragma unroll
      for (int k = 0; k < 12; k++) {
        coeffs[k] = a.luma_coeff[fi][k];
        clips[k] = cl ? a.luma_clip_idx[fi][k] : 0;
      }
    }
    int fc[12], fcl[12];
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const int p = c_alf_transpose_perm[(tr & 3) * 12 + k];
      fc[k] = coeffs[p];
      fcl[k] = alf_clip_val(bd, clips[p]);
    }
    // the reference filters the block's samples inside the visible CTU region
    const int ctu_x0 = (bx / P.ctu) * P.ctu, ctu_y0 = (by / P.ctu) * P.ctu;
    const int rxe = min(xe, ctu_x0 + min(P.ctu, P.vis_w - ctu_x0));
    const int rye = min(ye, ctu_y0 + min(P.ctu, P.vis_h - ctu_y0));
    for (int y = by; y < ye; y++)
      for (int x = bx; x < xe; x++) {
        const int cur = P.y.p[(size_t)y * P.y.stride + x];
        if (x >= rxe || y >= rye) {
          d[(size_t)y * ds + x] = (uint16_t)cur;
          continue;
        }
        const int c0 = P.y.get(x, y);
        const int yv = y % vb_h;
        int r0 = y, r1 = y + 1, r2 = y - 1, r3 = y + 2, r4 = y - 2, r5 = y + 3, r6 = y - 3;
        if (yv < vb_pos && yv + 4 >= vb_pos) {
          if (yv == vb_pos - 1) { r1 = r0; r2 = r0; }
          if (yv + 2 >= vb_pos) { r3 = r1; r4 = r2; }
          if (yv + 3 >= vb_pos) { r5 = r3; r6 = r4; }
        } else if (yv >= vb_pos && yv <= vb_pos + 3) {
          if (yv == vb_pos) { r2 = r0; r1 = r0; }
          if (yv <= vb_pos + 1) { r4 = r2; r3 = r1; }
          if (yv <= vb_pos + 2) { r6 = r4; r5 = r3; }
        }
        const bool near = (yv < vb_pos && yv + 1 >= vb_pos) || yv == vb_pos;
        auto t = [&](int k, int ax, int ar, int bxo, int br) {
          const int pa = P.y.get(x + ax, ar), pb = P.y.get(x + bxo, br);
          return fc[k] * (clampi(pa - c0, -fcl[k], fcl[k]) + clampi(pb - c0, -fcl[k], fcl[k]));
        };
        int sum = t(0, 0, r5, 0, r6) + t(1, 1, r3, -1, r4) + t(2, 0, r3, 0, r4) + t(3, -1, r3, 1, r4) +
                  t(4, 2, r1, -2, r2) + t(5, 1, r1, -1, r2) + t(6, 0, r1, 0, r2) + t(7, -1, r1, 1, r2) +
                  t(8, -2, r1, 2, r2) + t(9, 3, r0, -3, r0) + t(10, 2, r0, -2, r0) + t(11, 1, r0, -1, r0);
        const int shift = near ? 10 : 7;
        d[(size_t)y * ds + x] = (uint16_t)clampi(c0 + ((sum + (1 << (shift - 1))) >> shift), 0, maxv);
      }
  }
}

// alf_chroma_block (decode_general.rs:5568-5660) then ccalf_block
// (:5348-5408), one thread per chroma sample of both planes.
__global__ void __launch_bounds__(256) k_alf_general_chroma(AlfGenPass P) {
  const int n = P.cw * P.ch;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * n; i += gridDim.x * blockDim.x) {
    const int comp = i < n ? 1 : 2, j = i < n ? i : i - n;
    const int x = j % P.cw, y = j / P.cw;
    const AlfGenView& S = comp == 1 ? P.u : P.v;
    uint16_t* d = P.dst[comp];
    const int ds = P.dstride[comp];
    int out = S.p[(size_t)y * S.stride + x];
    // the luma CTU whose chroma region holds (x, y): regions start at
    // (gx * ctu) / 2 and span max(w / 2, 1) samples of the visible CTU
    const int hc = P.ctu / 2;
    const int gx = x / hc, gy = y / hc;
    if (gx * P.ctu < P.vis_w && gy * P.ctu < P.vis_h) {
      const vvcg_alf_ctu m = P.ctus[gy * P.ctu_cols + gx];
      const int lw = min(P.ctu, P.vis_w - gx * P.ctu), lh = min(P.ctu, P.vis_h - gy * P.ctu);
      const int rw = max(lw / 2, 1), rh = max(lh / 2, 1);
      const int rx = x - gx * hc, ry = y - gy * hc;
      const vvcg_alf_params& a = *P.a;
      const int bd = P.bd, maxv = (1 << bd) - 1;
      const int alt = comp == 1 ? m.cb_alt : m.cr_alt;
      if (alt != 0xFF && a.num_chroma_filters > 0 && rx < rw && ry < rh) {
        const int idx = min(alt, (int)a.num_chroma_filters - 1);
        const int vb_h = hc, vb_pos = hc - 2;
        const int cur = S.get(x, y);
        const int yv = y % vb_h;
        int r0 = y, r1 = y + 1, r2 = y - 1, r3 = y + 2, r4 = y - 2;
        if (yv < vb_pos && yv + 2 >= vb_pos) {
          if (yv + 1 == vb_pos) { r1 = r0; r2 = r0; }
          if (yv + 2 >= vb_pos) { r3 = r1; r4 = r2; }
        } else if (yv >= vb_pos && yv <= vb_pos + 1) {
          if (yv == vb_pos) { r2 = r0; r1 = r0; }
          if (yv <= vb_pos + 1) { r4 = r2; r3 = r1; }
        }
        const bool near = (yv < vb_pos && yv + 1 >= vb_pos) || yv == vb_pos;
        auto t = [&](int k, int ax, int ar, int bxo, int br) {
          const int cl = alf_clip_val(bd, a.chroma_clip ? a.chroma_clip_idx[idx][k] : 0);
          const int pa = S.get(x + ax, ar), pb = S.get(x + bxo, br);
          return (int)a.chroma_coeff[idx][k] * (clampi(pa - cur, -cl, cl) + clampi(pb - cur, -cl, cl));
        };
        const int sum = t(0, 0, r3, 0, r4) + t(1, 1, r1, -1, r2) + t(2, 0, r1, 0, r2) + t(3, -1, r1, 1, r2) +
                        t(4, 2, r0, -2, r0) + t(5, 1, r0, -1, r0);
        const int shift = near ? 10 : 7;
        out = clampi(cur + ((sum + (1 << (shift - 1))) >> shift), 0, maxv);
      }
      const int idc = comp == 1 ? m.cc_cb : m.cc_cr;
      const int nf = comp == 1 ? a.num_cc_cb : a.num_cc_cr;
      if (idc != 0 && idc <= nf && rx < rw && ry < rh && x < P.cvis_w && y < P.cvis_h) {
        const int16_t* co = comp == 1 ? a.cc_cb[idc - 1] : a.cc_cr[idc - 1];
        const int off = 1 << (bd - 1), vbp = max(0, P.ctu - 4);
        const int ly = y * 2, pos = ly & (P.ctu - 1), lx = x * 2;
        int above = ly - 1, below = ly + 1, below2 = ly + 2;
        if (pos == max(0, vbp - 2) || pos == vbp + 1) {
          below2 = ly + 1;
        } else if (pos == max(0, vbp - 1) || pos == vbp) {
          above = ly; below = ly; below2 = ly;
        }
        const int cur = P.y.get(lx, ly);
        int sum = co[0] * (P.y.get(lx, above) - cur);
        sum += co[1] * (P.y.get(lx - 1, ly) - cur);
        sum += co[2] * (P.y.get(lx + 1, ly) - cur);
        sum += co[3] * (P.y.get(lx - 1, below) - cur);
        sum += co[4] * (P.y.get(lx, below) - cur);
        sum += co[5] * (P.y.get(lx + 1, below) - cur);
        sum += co[6] * (P.y.get(lx, below2) - cur);
        out = clampi(out + clampi((sum + 64) >> 7, -off, off - 1), 0, maxv);
      }
    }
    d[(size_t)y * ds + x] = (uint16_t)out;
  }
}

}  // namespace vvcg
