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

namespace orc {

// slice.rs:699-760 plan_primary / :671-697 plan_transform_skip on one square
// block of the 8-bit strict encoder: levels and reconstructed samples.
struct BlockPlan {
  std::vector<int32_t> levels;
  std::vector<int32_t> samples;
  bool cbf = false;
};

static void slice_lfnst_skips(int w, int h, int* sw, int* sh) {  // slice.rs:674-682
  if ((w == 4 && h > 4) || (w > 4 && h == 4)) {
    *sw = w - 4;
    *sh = h - 4;
  } else if (w >= 8 && h >= 8) {
    *sw = w - 8;
    *sh = h - 8;
  } else {
    *sw = *sh = 0;
  }
}

static BlockPlan plan_primary(const int32_t* pred, const int32_t* res, int n, int qp, int mts, int lfnst,
                              int mode) {
  BlockPlan p;
  int th, tv;
  mts_types(mts, &th, &tv);
  int sw, sh;
  if (lfnst > 0)
    slice_lfnst_skips(n, n, &sw, &sh);
  else {
    sw = (n == 32 && th != kDct2) ? 16 : 0;  // slice.rs:659-670
    sh = (n == 32 && tv != kDct2) ? 16 : 0;
  }
  std::vector<int32_t> co(n * n), deq(n * n), rec(n * n);
  forward_transform_rect_bd(n, n, res, th, tv, sw, sh, 8, co.data());
  if (lfnst > 0) forward_lfnst_rect(co.data(), n, n, lfnst, mode);
  p.levels.assign(n * n, 0);
  quantize_rect_bd(n, n, co.data(), qp, 8, true, p.levels.data());
  for (int v : p.levels) p.cbf |= v != 0;
  dequantize_rect_bd(n, n, p.levels.data(), qp, 8, deq.data());
  if (lfnst > 0) inverse_lfnst_rect(deq.data(), n, n, lfnst, mode);
  inverse_transform_rect_bd(n, n, deq.data(), th, tv, sw, sh, 8, rec.data());
  p.samples.resize(n * n);
  for (int i = 0; i < n * n; i++) p.samples[i] = std::min(255, std::max(0, pred[i] + rec[i]));
  return p;
}

// slice.rs:935-939 scan_pos_last over CoeffScan(n, n)
static int scan_pos_last(const std::vector<int32_t>& lv, int n) {
  std::vector<int32_t> scan(n * n);
  int ns = coeff_scan_raster(n, n, scan.data());
  for (int s = ns - 1; s >= 0; s--)
    if (lv[scan[s]] != 0) return s;
  return -1;
}

}  // namespace orc

// slice.rs:810-874 encode_luma (after the prediction): the transform choice of
// one n x n luma block by reconstruction SSE. pred / src are n*n raster
// samples; writes the winner's levels and samples; returns (mts_idx << 8) |
// (lfnst_idx << 4) | (ts << 1) | cbf, and the winner's SSE.
extern "C" int orc_luma_tx_search(int n, const int32_t* pred, const int32_t* src, int qp, int mode, int use_ts,
                                  int chroma_can_lfnst, int16_t* levels, int16_t* samples, uint64_t* sse_out) {
  using namespace orc;
  std::vector<int32_t> res(n * n);
  for (int i = 0; i < n * n; i++) res[i] = src[i] - pred[i];
  auto sse_of = [&](const BlockPlan& p) {
    uint64_t s = 0;
    for (int i = 0; i < n * n; i++) {
      int64_t d = (int64_t)src[i] - p.samples[i];
      s += (uint64_t)(d * d);
    }
    return s;
  };
  BlockPlan best;
  int best_mts = 0, best_lfnst = 0, ts = 0;
  uint64_t best_sse;
  if (use_ts) {  // slice.rs:671-697 plan_transform_skip
    best.levels.resize(n * n);
    best.samples.resize(n * n);
    for (int i = 0; i < n * n; i++) {
      int l = quantize_ts(res[i], qp);
      best.levels[i] = l;
      best.cbf |= l != 0;
      best.samples[i] = std::min(255, std::max(0, pred[i] + dequantize_ts(l, qp)));
    }
    best_sse = sse_of(best);
    ts = 1;
  } else {
    best = plan_primary(pred, res.data(), n, qp, 0, 0, mode);
    best_sse = sse_of(best);
    for (int m = 1; m <= 4; m++) {
      BlockPlan p = plan_primary(pred, res.data(), n, qp, m, 0, mode);
      // slice.rs:877-885 mts_candidate_ok
      if (!p.cbf) continue;
      int last = scan_pos_last(p.levels, n);
      bool violates = false;
      for (int i = 0; i < n * n; i++)
        if (p.levels[i] != 0 && ((i % n) / 4 > 3 || (i / n) / 4 > 3)) violates = true;
      if (!(last >= 1 && !violates)) continue;
      uint64_t s = sse_of(p);
      if (s < best_sse) {
        best_sse = s;
        best = p;
        best_mts = m;
      }
    }
    if (chroma_can_lfnst)
      for (int l = 1; l <= 2; l++) {
        BlockPlan p = plan_primary(pred, res.data(), n, qp, 0, l, mode);
        // slice.rs:888-896 lfnst_candidate_ok
        if (!p.cbf) continue;
        int last = scan_pos_last(p.levels, n);
        int max_pos = (n == 4 || n == 8) ? 7 : 15;
        if (!(last >= 1 && last <= max_pos)) continue;
        uint64_t s = sse_of(p);
        if (s < best_sse) {
          best_sse = s;
          best = p;
          best_mts = 0;
          best_lfnst = l;
        }
      }
  }
  for (int i = 0; i < n * n; i++) {
    levels[i] = (int16_t)best.levels[i];
    samples[i] = (int16_t)best.samples[i];
  }
  *sse_out = best_sse;
  return (best_mts << 8) | (best_lfnst << 4) | (ts << 1) | (best.cbf ? 1 : 0);
}
