// CPU oracle (test infrastructure only; see oracle.h): primary transforms,
// scalar / dependent quantisation and the grouped diagonal scan.
//
// Restates crates/rustmpeg-video/src/vvc/dct.rs and transform.rs of the
// reference. Every function keeps the reference's integer widths (i64
// accumulation, int16 clipping of each stage) so results are bit-identical.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../rustmpeg-next_b200/csrc/vvc_tables.h"
#include "oracle.h"

namespace orc {
using namespace vvc_tables;

static const int kMaxLog2TrDynamicRange = 15;  // dct.rs:49
static const int kTransformMatrixShift = 6;     // dct.rs:52

static inline int ilog2(int v) { return __builtin_ctz((unsigned)v); }
static inline int32_t clip_transform(int64_t v) {  // dct.rs:315 clip_transform
  return (int32_t)std::min<int64_t>(32767, std::max<int64_t>(-32768, v));
}
static inline bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

// dct.rs:215-262 dct2_matrix_any / matrix_for / matrix_for_any
const int8_t* matrix_for_any(int tr, int size) {
  if (tr == kDct2) {
    switch (size) {
      case 2: return kDct2N2;
      case 4: return kDct2N4;
      case 8: return kDct2N8;
      case 16: return kDct2N16;
      case 32: return kDct2N32;
      case 64: return kDct2N64;
      default: return nullptr;
    }
  }
  if (tr == kDst7) {
    switch (size) {
      case 4: return kDst7N4;
      case 8: return kDst7N8;
      case 16: return kDst7N16;
      case 32: return kDst7N32;
      default: return nullptr;
    }
  }
  switch (size) {
    case 4: return kDct8N4;
    case 8: return kDct8N8;
    case 16: return kDct8N16;
    case 32: return kDct8N32;
    default: return nullptr;
  }
}

// dct.rs:269-276 is_supported_rect
static bool is_supported_rect(int w, int h) {
  return w >= 1 && w <= 64 && h >= 1 && h <= 64 && w * h >= 2 && is_pow2(w) && is_pow2(h);
}

// Default zero-out: 32-point MTS keeps 16, 64-point DCT-2 keeps 32
// (dct.rs:898-907, :1049-1058).
static int default_skip(int tr, int n) {
  if (tr != kDct2 && n == 32) return 16;
  return n > 32 ? n - 32 : 0;
}

// dct.rs:865-991 forward_transform_rect_bd
int forward_transform_rect_bd(int w, int h, const int32_t* residual, int tr_hor, int tr_ver,
                              int extra_skip_w, int extra_skip_h, int bd, int32_t* out) {
  bd = std::min(12, std::max(8, bd));
  if (w == 1 && h > 1) {
    const int8_t* mv = matrix_for_any(tr_ver, h);
    if (!mv) return -1;
    int skip_h = std::max(default_skip(tr_ver, h), extra_skip_h);
    if (skip_h >= h) return -2;
    int shift = (ilog2(h) + bd + kTransformMatrixShift) - kMaxLog2TrDynamicRange;
    int64_t add = shift > 0 ? (int64_t)1 << (shift - 1) : 0;
    int cutoff_h = h - skip_h;
    for (int i = 0; i < h; i++) out[i] = 0;
    for (int v = 0; v < cutoff_h; v++) {
      int64_t sum = 0;
      for (int y = 0; y < h; y++) sum += (int64_t)mv[v * h + y] * residual[y];
      out[v] = clip_transform(shift >= 0 ? (sum + add) >> shift : sum << (-shift));
    }
    return 0;
  }
  if (h == 1 && w > 1) {
    const int8_t* mh = matrix_for_any(tr_hor, w);
    if (!mh) return -1;
    int skip_w = std::max(default_skip(tr_hor, w), extra_skip_w);
    if (skip_w >= w) return -2;
    int shift = (ilog2(w) + bd + kTransformMatrixShift) - kMaxLog2TrDynamicRange;
    int64_t add = shift > 0 ? (int64_t)1 << (shift - 1) : 0;
    int cutoff_w = w - skip_w;
    for (int i = 0; i < w; i++) out[i] = 0;
    for (int k = 0; k < cutoff_w; k++) {
      int64_t sum = 0;
      for (int n = 0; n < w; n++) sum += (int64_t)mh[k * w + n] * residual[n];
      out[k] = clip_transform(shift >= 0 ? (sum + add) >> shift : sum << (-shift));
    }
    return 0;
  }
  const int8_t* mh = matrix_for_any(tr_hor, w);
  const int8_t* mv = matrix_for_any(tr_ver, h);
  if (!mh || !mv) return -1;
  int skip_w = std::max(default_skip(tr_hor, w), extra_skip_w);
  int skip_h = std::max(default_skip(tr_ver, h), extra_skip_h);
  if (skip_w >= w || skip_h >= h) return -2;
  int shift1 = (ilog2(w) + bd + kTransformMatrixShift) - kMaxLog2TrDynamicRange;
  int shift2 = ilog2(h) + kTransformMatrixShift;
  int64_t add1 = shift1 > 0 ? (int64_t)1 << (shift1 - 1) : 0;
  int64_t add2 = (int64_t)1 << (shift2 - 1);
  int cw = w - skip_w, ch = h - skip_h;
  std::vector<int32_t> tmp((size_t)w * h, 0);
  for (int y = 0; y < h; y++)
    for (int k = 0; k < cw; k++) {
      int64_t sum = 0;
      for (int n = 0; n < w; n++) sum += (int64_t)mh[k * w + n] * residual[y * w + n];
      tmp[k * h + y] = (int32_t)((sum + add1) >> shift1);  // no clip (dct.rs:963)
    }
  for (int i = 0; i < w * h; i++) out[i] = 0;
  for (int v = 0; v < ch; v++)
    for (int k = 0; k < cw; k++) {
      int64_t sum = 0;
      for (int y = 0; y < h; y++) sum += (int64_t)mv[v * h + y] * tmp[k * h + y];
      out[v * w + k] = clip_transform((sum + add2) >> shift2);
    }
  return 0;
}

// dct.rs:996-1109 inverse_transform_rect_bd
int inverse_transform_rect_bd(int w, int h, const int32_t* coeffs, int tr_hor, int tr_ver,
                              int extra_skip_w, int extra_skip_h, int bd, int32_t* out) {
  bd = std::min(12, std::max(8, bd));
  if (w == 1 && h > 1) {
    const int8_t* mv = matrix_for_any(tr_ver, h);
    if (!mv) return -1;
    int skip_h = std::max(default_skip(tr_ver, h), extra_skip_h);
    if (skip_h >= h) return -2;
    int shift = (kTransformMatrixShift + kMaxLog2TrDynamicRange) - bd;
    int64_t add = (int64_t)1 << (shift - 1);
    int cutoff_h = h - skip_h;
    for (int j = 0; j < h; j++) {
      int64_t sum = 0;
      for (int k = 0; k < cutoff_h; k++) sum += (int64_t)mv[k * h + j] * coeffs[k];
      out[j] = clip_transform((sum + add) >> shift);
    }
    return 0;
  }
  if (h == 1 && w > 1) {
    const int8_t* mh = matrix_for_any(tr_hor, w);
    if (!mh) return -1;
    int skip_w = std::max(default_skip(tr_hor, w), extra_skip_w);
    if (skip_w >= w) return -2;
    int shift = (kTransformMatrixShift + kMaxLog2TrDynamicRange) - bd;
    int64_t add = (int64_t)1 << (shift - 1);
    int cutoff_w = w - skip_w;
    for (int x = 0; x < w; x++) {
      int64_t sum = 0;
      for (int k = 0; k < cutoff_w; k++) sum += (int64_t)mh[k * w + x] * coeffs[k];
      out[x] = clip_transform((sum + add) >> shift);
    }
    return 0;
  }
  const int8_t* mh = matrix_for_any(tr_hor, w);
  const int8_t* mv = matrix_for_any(tr_ver, h);
  if (!mh || !mv) return -1;
  int skip_w = std::max(default_skip(tr_hor, w), extra_skip_w);
  int skip_h = std::max(default_skip(tr_ver, h), extra_skip_h);
  if (skip_w >= w || skip_h >= h) return -2;
  int shift1 = kTransformMatrixShift + 1;
  int shift2 = (kTransformMatrixShift + kMaxLog2TrDynamicRange - 1) - bd;
  int64_t add1 = (int64_t)1 << (shift1 - 1);
  int64_t add2 = (int64_t)1 << (shift2 - 1);
  int cw = w - skip_w, ch = h - skip_h;
  std::vector<int32_t> tmp((size_t)w * h, 0);
  for (int i = 0; i < cw; i++)
    for (int j = 0; j < h; j++) {
      int64_t sum = 0;
      for (int k = 0; k < ch; k++) sum += (int64_t)mv[k * h + j] * coeffs[k * w + i];
      tmp[i * h + j] = clip_transform((sum + add1) >> shift1);
    }
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      int64_t sum = 0;
      for (int k = 0; k < cw; k++) sum += (int64_t)mh[k * w + x] * tmp[k * h + y];
      out[y * w + x] = clip_transform((sum + add2) >> shift2);
    }
  return 0;
}

// dct.rs:828-830 transform_shift_rect_bd, plus the sqrt(2) adjustment of
// quantize_rect_bd / dequantize_rect_bd (dct.rs:1127-1129, :1166-1168).
static int tr_shift_q(int w, int h, int bd, bool* needs_sqrt2) {
  *needs_sqrt2 = ((ilog2(w) + ilog2(h)) & 1) == 1;
  return kMaxLog2TrDynamicRange - bd - ((ilog2(w) + ilog2(h)) >> 1) - (*needs_sqrt2 ? 1 : 0);
}

// dct.rs:1113-1147 quantize_rect_bd
int quantize_rect_bd(int w, int h, const int32_t* coeffs, int qp_scaled, int bd, bool is_intra,
                     int32_t* out) {
  if (!is_supported_rect(w, h)) return -1;
  int qp = std::max(4, qp_scaled);
  int qp_per = qp / 6, qp_rem = qp % 6;
  bool s2;
  int tr_shift = tr_shift_q(w, h, bd, &s2);
  int qbits = 14 + qp_per + tr_shift;
  int64_t off = is_intra ? 171 : 85;
  int64_t add = off << std::max(0, qbits - 9);
  int64_t scale = kQuantScale[s2 ? 1 : 0][qp_rem];
  for (int i = 0; i < w * h; i++) {
    int32_t c = coeffs[i];
    int64_t level = ((int64_t)std::abs(c) * scale + add) >> std::max(0, qbits);
    out[i] = clip_transform(c < 0 ? -level : level);
  }
  return 0;
}

// dct.rs:1151-1187 dequantize_rect_bd
int dequantize_rect_bd(int w, int h, const int32_t* levels, int qp_scaled, int bd, int32_t* out) {
  if (!is_supported_rect(w, h)) return -1;
  int qp = std::max(4, qp_scaled);
  int qp_per = qp / 6, qp_rem = qp % 6;
  bool s2;
  int tr_shift = tr_shift_q(w, h, bd, &s2);
  int right_shift = 6 - (tr_shift + qp_per);
  int64_t scale = kInvQuantScale[s2 ? 1 : 0][qp_rem];
  for (int i = 0; i < w * h; i++) {
    int64_t value = (int64_t)levels[i] * scale;
    int64_t scaled = right_shift > 0 ? (value + ((int64_t)1 << (right_shift - 1))) >> right_shift
                                     : value << (-right_shift);
    out[i] = clip_transform(scaled);
  }
  return 0;
}

// dct.rs:1191-1248 dequantize_dep_quant_bd
int dequantize_dep_quant_bd(int w, int h, const int32_t* levels, const int32_t* scan, int qp_scaled,
                            int bd, int32_t* out) {
  if (!is_supported_rect(w, h)) return -1;
  int n = w * h;
  for (int i = 0; i < n; i++) out[i] = 0;
  int nscan = coeff_scan_raster(w, h, nullptr);
  int last = -1;
  for (int s = nscan - 1; s >= 0; s--) {
    int r = scan[s];
    if (r < n && levels[r] != 0) {
      last = s;
      break;
    }
  }
  if (last < 0) return 0;
  int qp_dq = std::max(4, qp_scaled) + 1;
  int qp_per = qp_dq / 6, qp_rem = qp_dq % 6;
  bool s2;
  int tr_shift = tr_shift_q(w, h, bd, &s2);
  int shift = 7 - qp_per - tr_shift;
  int64_t inv_q = kInvQuantScale[s2 ? 1 : 0][qp_rem];
  if (shift < 0) inv_q <<= -shift;
  int64_t add = shift > 0 ? (int64_t)1 << (shift - 1) : 0;
  int rshift = std::max(0, shift);
  int state = 0;
  for (int s = last; s >= 0; s--) {
    int r = scan[s];
    int32_t level = levels[r];
    if (level != 0) {
      int64_t q_idx = (int64_t)(2 * level + (level > 0 ? -(state >> 1) : (state >> 1)));
      out[r] = clip_transform((q_idx * inv_q + add) >> rshift);
    }
    state = (32040 >> ((state << 2) + ((level & 1) << 1))) & 3;
  }
  return 0;
}

// dct.rs:1252-1301 quantize_dep_quant_bd
int quantize_dep_quant_bd(int w, int h, const int32_t* coeffs, const int32_t* scan, int qp_scaled,
                          int bd, int32_t* out) {
  if (!is_supported_rect(w, h)) return -1;
  int n = w * h;
  int qp_dq = std::max(4, qp_scaled) + 1;
  int qp_per = qp_dq / 6, qp_rem = qp_dq % 6;
  bool s2;
  int tr_shift = tr_shift_q(w, h, bd, &s2);
  int q_shift = 13 + qp_per + tr_shift;
  int64_t q_scale = kQuantScale[s2 ? 1 : 0][qp_rem];
  int64_t half = (int64_t)1 << std::max(0, q_shift - 1);
  for (int i = 0; i < n; i++) out[i] = 0;
  int nscan = coeff_scan_raster(w, h, nullptr);
  int state = 0;
  for (int s = nscan - 1; s >= 0; s--) {
    int r = scan[s];
    if (r >= n) continue;
    int32_t c = coeffs[r];
    int64_t q_idx_est = ((int64_t)std::abs(c) * q_scale + half) >> std::max(0, q_shift);
    int64_t offset = state >> 1;
    int32_t abs_level = q_idx_est <= offset ? 0 : (int32_t)((q_idx_est + offset + 1) >> 1);
    int32_t level = c < 0 ? -abs_level : abs_level;
    level = std::min(32767, std::max(-32768, level));
    out[r] = level;
    state = (32040 >> ((state << 2) + ((level & 1) << 1))) & 3;
  }
  return 0;
}

// transform.rs:100-171 coefficient_group_log2 (VTM g_log2TxSubblockSize)
static void cg_log2(int w, int h, int* lw, int* lh) {
  static const uint8_t T[8][8][2] = {
      {{0, 0}, {0, 1}, {0, 2}, {0, 3}, {0, 4}, {0, 4}, {0, 4}, {0, 4}},
      {{1, 0}, {1, 1}, {1, 1}, {1, 3}, {1, 3}, {1, 3}, {1, 3}, {1, 3}},
      {{2, 0}, {1, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{3, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
  };
  int a = std::min(7, ilog2(w)), b = std::min(7, ilog2(h));
  *lw = T[a][b][0];
  *lh = T[a][b][1];
}

// transform.rs:175-198 diagonal_scan (VTM ScanGenerator, DIAG)
static void diagonal_scan(int w, int h, std::vector<std::pair<int, int>>& out) {
  out.clear();
  if (w == 0 || h == 0) return;
  int line = 0, column = 0;
  for (int i = 0; i < w * h; i++) {
    out.push_back({column, line});
    if (column == w - 1 || line == 0) {
      line += column + 1;
      column = 0;
      if (line >= h) {
        column += line - (h - 1);
        line = h - 1;
      }
    } else {
      column += 1;
      line -= 1;
    }
  }
}

// transform.rs:43-80 CoeffScan::new (raster indices only)
int coeff_scan_raster(int w, int h, int32_t* raster) {
  int lw, lh;
  cg_log2(w, h, &lw, &lh);
  int cgw = 1 << lw, cgh = 1 << lh;
  int capped_w = std::min(w, 32), capped_h = std::min(h, 32);
  int wg = capped_w >> lw, hg = capped_h >> lh;
  if (!raster) return capped_w * capped_h;
  std::vector<std::pair<int, int>> groups, inner;
  diagonal_scan(wg, hg, groups);
  diagonal_scan(cgw, cgh, inner);
  int k = 0;
  for (auto& g : groups)
    for (auto& in : inner) raster[k++] = (g.second * cgh + in.second) * w + g.first * cgw + in.first;
  return k;
}

// transform.rs:214-226 quantize_ts
int32_t quantize_ts(int32_t residual, int qp) {
  qp = std::max(4, qp);
  int qp_per = qp / 6, qp_rem = qp % 6;
  int qbits = 14 + qp_per;
  int64_t add = (int64_t)171 << (qbits - 9);
  int sign = (residual > 0) - (residual < 0);
  int32_t level = (int32_t)(((int64_t)std::abs(residual) * kQuantScale[0][qp_rem] + add) >> qbits);
  return std::min(32767, std::max(-32768, sign * level));
}

// transform.rs:229-246 dequantize_ts
int32_t dequantize_ts(int32_t level, int qp) {
  qp = std::max(4, qp);
  int qp_per = qp / 6, qp_rem = qp % 6;
  int right_shift = 6 - qp_per;
  int64_t value = (int64_t)level * kInvQuantScale[0][qp_rem];
  int64_t scaled = right_shift > 0 ? (value + ((int64_t)1 << (right_shift - 1))) >> right_shift
                                   : value << (-right_shift);
  int32_t t = (int32_t)(uint32_t)(uint64_t)scaled;  // Rust `as i32` truncation
  return std::min(32767, std::max(-32768, t));
}

// hls.rs:787-792 scaled_luma_qp_bd
int scaled_luma_qp_bd(int qpy, int bd) {
  bd = std::min(12, std::max(8, bd));
  int off = 6 * (bd - 8);
  return std::min(63 + off, std::max(0, qpy + off));
}

// hls.rs:796-802 derived_chroma_qp_bd
int derived_chroma_qp_bd(int qpy, int bd, int cqo) {
  bd = std::min(12, std::max(8, bd));
  int off = 6 * (bd - 8);
  int qpi = std::min(63, std::max(-off, qpy));
  int mapped = qpi <= 26 ? qpi : qpi - 1;
  int base = std::min(63, std::max(-off, mapped + cqo)) + off;
  return std::min(63 + off, std::max(0, base));
}

// hls.rs:778-781 derived_chroma_qp
int derived_chroma_qp(int qp) {
  int qpi = std::min(63, std::max(0, qp));
  return qpi <= 26 ? qpi : qpi - 1;
}

}  // namespace orc
