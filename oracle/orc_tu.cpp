// CPU oracle (test infrastructure only; see oracle.h): one transform unit's
// residual path in both directions, composed the way the reference composes it.
//
//   inverse: decode_general.rs:4100-4122 residual_of (transform skip) and
//            :4124-4199 inverse_residual (DQ / regular dequantisation, LFNST,
//            implicit / explicit MTS, zero-out), then the BDPCM step of
//            reconstruct_tu (:4055-4060) with predict.rs:4224-4240.
//   forward: slice.rs:690-760 plan_transform_skip / plan_primary (the level
//            side), with the bit depth, DQ and the intra/inter rounding offset
//            as parameters, as the frame encoder uses them.
#include <string.h>

#include <algorithm>
#include <vector>

#include "oracle.h"

namespace orc {

// decode_general.rs:4205-4214 mts_types
static void mts_types(int idx, int* th, int* tv) {
  static const int T[5][2] = {{kDct2, kDct2}, {kDst7, kDst7}, {kDct8, kDst7}, {kDst7, kDct8}, {kDct8, kDct8}};
  *th = T[idx][0];
  *tv = T[idx][1];
}

// decode_general.rs:4216-4230 primary_skips
static void primary_skips(int w, int h, int th, int tv, int* sw, int* sh) {
  *sw = (w == 32 && th != kDct2) ? 16 : std::max(0, w - 32);
  *sh = (h == 32 && tv != kDct2) ? 16 : std::max(0, h - 32);
}

// decode_general.rs:4233-4237 lfnst_skips
static void lfnst_skips(int w, int h, int* sw, int* sh) {
  int nz = (w == 4 || h == 4) ? 4 : 8;
  *sw = w - std::min(nz, w);
  *sh = h - std::min(nz, h);
}

static void transform_types(const TuRec& r, int w, int h, int* th, int* tv, int* sw, int* sh) {
  const bool used_mts = r.mts_idx != 0;
  if (used_mts) {
    mts_types(r.mts_idx, th, tv);
  } else if ((r.flags & kTuImplicitMts) && r.lfnst_idx == 0) {
    *th = (w >= 4 && w <= 16) ? kDst7 : kDct2;
    *tv = (h >= 4 && h <= 16) ? kDst7 : kDct2;
  } else {
    *th = *tv = kDct2;
  }
  if (r.lfnst_idx > 0 && !used_mts)
    lfnst_skips(w, h, sw, sh);
  else
    primary_skips(w, h, *th, *tv, sw, sh);
}

// predict.rs:4224-4240 apply_bdpcm_inverse
static void bdpcm_inverse(int32_t* v, int w, int h, bool vertical) {
  if (!vertical) {
    for (int y = 0; y < h; y++)
      for (int x = 1; x < w; x++) v[y * w + x] = std::min(32767, std::max(-32768, v[y * w + x] + v[y * w + x - 1]));
  } else {
    for (int y = 1; y < h; y++)
      for (int x = 0; x < w; x++) v[y * w + x] = std::min(32767, std::max(-32768, v[y * w + x] + v[(y - 1) * w + x]));
  }
}

int tu_inverse(const TuRec& r, const int16_t* in, int16_t* out) {
  const int w = 1 << r.log2_w, h = 1 << r.log2_h, n = w * h;
  std::vector<int32_t> lv(in, in + n), res(n, 0);
  if (r.flags & kTuTransformSkip) {
    for (int i = 0; i < n; i++) res[i] = dequantize_ts(lv[i], r.qp);
  } else {
    std::vector<int32_t> scan(n);
    coeff_scan_raster(w, h, scan.data());
    std::vector<int32_t> deq(n);
    int rc = (r.flags & kTuDepQuant) ? dequantize_dep_quant_bd(w, h, lv.data(), scan.data(), r.qp, r.bit_depth, deq.data())
                                     : dequantize_rect_bd(w, h, lv.data(), r.qp, r.bit_depth, deq.data());
    if (rc) return -1;
    if (r.lfnst_idx > 0 && r.mts_idx == 0)
      if (inverse_lfnst_rect(deq.data(), w, h, r.lfnst_idx, r.lfnst_mode)) return -2;
    int th, tv, sw, sh;
    transform_types(r, w, h, &th, &tv, &sw, &sh);
    if (inverse_transform_rect_bd(w, h, deq.data(), th, tv, sw, sh, r.bit_depth, res.data())) return -3;
  }
  if (r.flags & (kTuBdpcmHor | kTuBdpcmVer)) bdpcm_inverse(res.data(), w, h, (r.flags & kTuBdpcmVer) != 0);
  for (int i = 0; i < n; i++) out[i] = (int16_t)res[i];
  return 0;
}

int tu_forward(const TuRec& r, const int16_t* in, int16_t* out) {
  const int w = 1 << r.log2_w, h = 1 << r.log2_h, n = w * h;
  std::vector<int32_t> res(in, in + n), lv(n, 0);
  if (r.flags & kTuTransformSkip) {
    for (int i = 0; i < n; i++) lv[i] = quantize_ts(res[i], r.qp);
  } else {
    if (r.lfnst_idx > 0 && r.mts_idx != 0) return -4;  // slice.rs:701-703
    int th, tv, sw, sh;
    transform_types(r, w, h, &th, &tv, &sw, &sh);
    std::vector<int32_t> co(n);
    if (forward_transform_rect_bd(w, h, res.data(), th, tv, sw, sh, r.bit_depth, co.data())) return -3;
    if (r.lfnst_idx > 0)
      if (forward_lfnst_rect(co.data(), w, h, r.lfnst_idx, r.lfnst_mode)) return -2;
    std::vector<int32_t> scan(n);
    coeff_scan_raster(w, h, scan.data());
    int rc = (r.flags & kTuDepQuant) ? quantize_dep_quant_bd(w, h, co.data(), scan.data(), r.qp, r.bit_depth, lv.data())
                                     : quantize_rect_bd(w, h, co.data(), r.qp, r.bit_depth, !(r.flags & kTuInter), lv.data());
    if (rc) return -1;
  }
  for (int i = 0; i < n; i++) out[i] = (int16_t)lv[i];
  return 0;
}

}  // namespace orc
