// Function-level transform-unit kernels of libvvcg (sm_100a): levels ->
// residual (dequantisation, inverse LFNST, inverse DCT-2 / DST-7 / DCT-8,
// BDPCM) and residual -> levels (forward transform, forward LFNST,
// quantisation). One warp per transform unit; the host bins units by size so
// each warp's two shared tiles fit the largest unit of its bin.
//
// Every sum is exact: the inverse stages and the forward first stage stay
// below 2^31 (int16 inputs, |matrix| <= 90, at most 64 terms); the forward
// second stage, whose inputs are not clipped, accumulates in 64 bits.
#pragma once
#include <stdint.h>

#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

// Grouped diagonal scans of every (log2 w, log2 h) in 0..6, raster indices of
// the top-left min(w,32) x min(h,32) (transform.rs:43-80 CoeffScan::new).
constexpr int kTuScanTotal = 95 * 95;
__device__ int16_t g_tu_scan[kTuScanTotal];
__device__ int32_t g_tu_scan_off[49];
// LFNST kernels (tr_tables.rs LFNST_8X8 / LFNST_4X4 / LFNST_LUT).
__device__ int8_t g_lfnst8[4 * 2 * 16 * 48];
__device__ int8_t g_lfnst4[4 * 2 * 16 * 16];
__device__ uint8_t g_lfnst_lut[95];

constexpr int kTuPad = 64;   // tiles are padded by one sample per row or column

// Transform types and zero-out of a unit (decode_general.rs:4165-4198 with
// mts_types :4205, primary_skips :4216, lfnst_skips :4233).
struct TuShape {
  int w, h, lw, lh, n;
  int th, tv;  // 0 DCT-2, 1 DST-7, 2 DCT-8
  int sw, sh;  // zero-out width / height (at least the default of the types)
};

__host__ __device__ __forceinline__ int tu_default_skip(int tr, int n) {
  return (tr != 0 && n == 32) ? 16 : (n > 32 ? n - 32 : 0);
}

__host__ __device__ __forceinline__ void tu_shape(const vvcg_tu_rec& r, TuShape& s) {
  s.lw = r.log2_w;
  s.lh = r.log2_h;
  s.w = 1 << s.lw;
  s.h = 1 << s.lh;
  s.n = s.w * s.h;
  const bool mts = r.mts_idx != 0;
  if (mts) {
    s.th = (r.mts_idx == 1 || r.mts_idx == 3) ? 1 : 2;
    s.tv = (r.mts_idx == 1 || r.mts_idx == 2) ? 1 : 2;
  } else if ((r.flags & VVCG_TU_IMPLICIT_MTS) && r.lfnst_idx == 0) {
    s.th = (s.w >= 4 && s.w <= 16) ? 1 : 0;
    s.tv = (s.h >= 4 && s.h <= 16) ? 1 : 0;
  } else {
    s.th = s.tv = 0;
  }
  int sw, sh;
  if (r.lfnst_idx > 0 && !mts) {
    const int nz = (s.w == 4 || s.h == 4) ? 4 : 8;
    sw = s.w - (nz < s.w ? nz : s.w);
    sh = s.h - (nz < s.h ? nz : s.h);
  } else {
    sw = tu_default_skip(s.th, s.w);
    sh = tu_default_skip(s.tv, s.h);
  }
  const int dw = tu_default_skip(s.th, s.w), dh = tu_default_skip(s.tv, s.h);
  s.sw = sw > dw ? sw : dw;
  s.sh = sh > dh ? sh : dh;
}

__device__ __forceinline__ const int8_t* tu_matrix(int tr, int log2n) {
  if (tr == 0) return g_dct2_m[log2n - 1];
  return tr == 1 ? g_dst7_m[log2n - 2] : g_dct8_m[log2n - 2];
}

__device__ __forceinline__ const int16_t* tu_scan(int lw, int lh) { return g_tu_scan + g_tu_scan_off[lw * 7 + lh]; }

// dct.rs:828-830 transform shift with the sqrt(2) flag of the quantisers.
__device__ __forceinline__ int tu_tr_shift(int lw, int lh, int bd, bool* s2) {
  *s2 = ((lw + lh) & 1) != 0;
  return 15 - bd - ((lw + lh) >> 1) - (*s2 ? 1 : 0);
}

// transform.rs:229-246 dequantize_ts (with the reference's `as i32` truncation)
__device__ __forceinline__ int tu_dequant_ts(int level, int qp) {
  qp = max(4, qp);
  const int qp_per = qp / 6, rs = 6 - qp_per;
  const long long v = (long long)level * c_inv_quant_scale[0][qp % 6];
  const long long s = rs > 0 ? (v + (1ll << (rs - 1))) >> rs : v << (-rs);
  return clip16i((int32_t)(uint32_t)(unsigned long long)s);
}

// transform.rs:214-226 quantize_ts
__device__ __forceinline__ int tu_quant_ts(int res, int qp) {
  qp = max(4, qp);
  const int qbits = 14 + qp / 6;
  const long long add = 171ll << (qbits - 9);
  const long long a = ((long long)abs(res) * c_quant_scale[0][qp % 6] + add) >> qbits;
  const int sign = (res > 0) - (res < 0);
  return clip16((long long)sign * a);
}

// One 4-state step of dependent quantisation (dct.rs:1238, table 32040).
__device__ __forceinline__ int dq_next(int st, int level) { return (32040 >> ((st << 2) + ((level & 1) << 1))) & 3; }

// Splits scan positions [0, last] into 32 chunks walked from the end: lane 0
// takes the highest positions. Returns this lane's chunk [lo, hi].
__device__ __forceinline__ void dq_chunk(int last, int lane, int& lo, int& hi) {
  const int cs = (last + 32) >> 5;
  hi = last - lane * cs;
  lo = max(hi - cs + 1, 0);
}

// Entry state of each lane's chunk from per-lane state maps (2 bits per
// state): an inclusive warp scan of map compositions, shifted by one lane.
__device__ __forceinline__ int dq_entry_state(uint32_t map, int lane) {
  uint32_t pre = map;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t other = __shfl_up_sync(0xffffffffu, pre, o);
    if (lane >= o) {
      uint32_t comp = 0;
      for (int s = 0; s < 4; s++) comp |= ((pre >> (2 * ((other >> (2 * s)) & 3))) & 3) << (2 * s);
      pre = comp;
    }
  }
  const uint32_t excl = __shfl_up_sync(0xffffffffu, pre, 1);
  return lane == 0 ? 0 : (int)(excl & 3);
}

// dct.rs:1191-1248 dequantize_dep_quant_bd, in place on the level tile A
// (raster, stride w).
__device__ void tu_dq_dequant(int32_t* A, const TuShape& S, int qp_scaled, int bd, int lane) {
  const int16_t* scan = tu_scan(S.lw, S.lh);
  const int ns = min(S.w, 32) * min(S.h, 32);
  int last = -1;
  for (int s = lane; s < ns; s += 32)
    if (A[scan[s]] != 0) last = max(last, s);
  last = __reduce_max_sync(0xffffffffu, last);
  __syncwarp();
  if (last < 0) {
    for (int i = lane; i < S.n; i += 32) A[i] = 0;
    __syncwarp();
    return;
  }
  int lo, hi;
  dq_chunk(last, lane, lo, hi);
  uint32_t map = 0;
  for (int st0 = 0; st0 < 4; st0++) {
    int st = st0;
    for (int s = hi; s >= lo; s--) st = dq_next(st, A[scan[s]]);
    map |= (uint32_t)st << (2 * st0);
  }
  int st = dq_entry_state(map, lane);
  const int qp_dq = max(4, qp_scaled) + 1;
  bool s2;
  const int tr_shift = tu_tr_shift(S.lw, S.lh, bd, &s2);
  const int shift = 7 - qp_dq / 6 - tr_shift;
  long long inv_q = c_inv_quant_scale[s2 ? 1 : 0][qp_dq % 6];
  if (shift < 0) inv_q <<= -shift;
  const long long add = shift > 0 ? (1ll << (shift - 1)) : 0;
  const int rsh = max(0, shift);
  // Each lane rewrites only its own chunk, reading every level before writing
  // it; positions past `last` hold zero levels already. Raster positions
  // outside the scan (64-point units) are zero in the reference's output.
  if (ns < S.n)
    for (int i = lane; i < S.n; i += 32) {
      const int y = i >> S.lw, x = i & (S.w - 1);
      if (x >= 32 || y >= 32) A[i] = 0;
    }
  for (int s = hi; s >= lo; s--) {
    int32_t* p = &A[scan[s]];
    const int L = *p;
    if (L != 0) {
      const long long q = (long long)(2 * L + (L > 0 ? -(st >> 1) : (st >> 1)));
      *p = clip16((q * inv_q + add) >> rsh);
    }
    st = dq_next(st, L);
  }
  __syncwarp();
}

// dct.rs:1252-1301 quantize_dep_quant_bd: coefficients A (raster) -> levels,
// written to `out` (raster; zero outside the scan). `out` may be A itself:
// each lane reads a coefficient before it writes that position's level.
template <class OutT>
__device__ void tu_dq_quant(const int32_t* A, const TuShape& S, int qp_scaled, int bd, OutT* out,
                            int lane) {
  const int16_t* scan = tu_scan(S.lw, S.lh);
  const int ns = min(S.w, 32) * min(S.h, 32);
  const int qp_dq = max(4, qp_scaled) + 1;
  bool s2;
  const int tr_shift = tu_tr_shift(S.lw, S.lh, bd, &s2);
  const int q_shift = 13 + qp_dq / 6 + tr_shift;
  const long long q_scale = c_quant_scale[s2 ? 1 : 0][qp_dq % 6];
  const long long half = 1ll << max(0, q_shift - 1);
  auto qest = [&](int c) -> long long { return ((long long)abs(c) * q_scale + half) >> max(0, q_shift); };
  auto level_of = [&](long long est, int c, int st) -> int {
    const long long off = st >> 1;
    const int a = est <= off ? 0 : (int)((est + off + 1) >> 1);
    return clampi(c < 0 ? -a : a, -32768, 32767);
  };
  int lo, hi;
  dq_chunk(ns - 1, lane, lo, hi);
  uint32_t map = 0;
  for (int st0 = 0; st0 < 4; st0++) {
    int st = st0;
    for (int s = hi; s >= lo; s--) {
      const int c = A[scan[s]];
      st = dq_next(st, level_of(qest(c), c, st));
    }
    map |= (uint32_t)st << (2 * st0);
  }
  int st = dq_entry_state(map, lane);
  for (int s = hi; s >= lo; s--) {
    const int c = A[scan[s]];
    const int L = level_of(qest(c), c, st);
    out[scan[s]] = (OutT)L;
    st = dq_next(st, L);
  }
  if (ns < S.n)
    for (int i = lane; i < S.n; i += 32) {
      const int y = i >> S.lw, x = i & (S.w - 1);
      if (x >= 32 || y >= 32) out[i] = 0;
    }
}

// Position (row, column) in the unit of LFNST element j (lfnst.rs:253-292):
// the non-transposed layout fills rows of sb (first 4 rows) then 4; the
// transposed one fills columns.
__device__ __forceinline__ int lfnst_pos(int j, int sb, bool transposed, int w) {
  int y, x;
  if (!transposed) {
    if (sb == 4) {
      y = j >> 2;
      x = j & 3;
    } else if (j < 32) {
      y = j >> 3;
      x = j & 7;
    } else {
      y = 4 + ((j - 32) >> 2);
      x = (j - 32) & 3;
    }
  } else {
    if (sb == 4) {
      y = j & 3;
      x = j >> 2;
    } else if (j < 32) {
      y = j & 7;
      x = j >> 3;
    } else {
      y = (j - 32) & 3;
      x = 4 + ((j - 32) >> 2);
    }
  }
  return y * w + x;
}

struct LfnstParams {
  int sb, tr, zo;
  const int8_t* m;  // [16][tr] rows of the selected kernel
  bool transposed;
};

__device__ __forceinline__ LfnstParams lfnst_params(const TuShape& S, int idx, int mode) {
  LfnstParams p;
  p.sb = (S.w >= 8 && S.h >= 8) ? 8 : 4;
  const bool small = (S.w == 4 && S.h == 4) || (S.w == 8 && S.h == 8);
  p.tr = p.sb == 4 ? 16 : 48;
  p.zo = small ? 8 : 16;
  const int set = g_lfnst_lut[mode];
  p.m = p.sb == 4 ? g_lfnst4 + (set * 2 + idx - 1) * 16 * 16 : g_lfnst8 + (set * 2 + idx - 1) * 16 * 48;
  p.transposed = (mode >= 35 && mode < 67) || mode >= 81;
  return p;
}

// lfnst.rs:219-294 inverse_lfnst_rect, in place on A (raster, stride w).
__device__ void tu_lfnst_inverse(int32_t* A, const TuShape& S, int idx, int mode, int lane) {
  const LfnstParams p = lfnst_params(S, idx, mode);
  const int16_t* scan8 = tu_scan(3, 3);
  int src[16];
#pragma unroll
  for (int i = 0; i < 16; i++) {
    const int r = scan8[i];
    src[i] = A[(r >> 3) * S.w + (r & 7)];
  }
  int o[2];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int j = lane + 32 * q;
    int s = 0;
    if (j < p.tr)
      for (int i = 0; i < p.zo; i++) s += src[i] * (int)p.m[i * p.tr + j];
    o[q] = clip16i((s + 64) >> 7);
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int j = lane + 32 * q;
    if (j < p.tr) A[lfnst_pos(j, p.sb, p.transposed, S.w)] = o[q];
  }
  __syncwarp();
}

// lfnst.rs:131-205 forward_lfnst_rect, in place on A (raster, stride w).
__device__ void tu_lfnst_forward(int32_t* A, const TuShape& S, int idx, int mode, int lane) {
  const LfnstParams p = lfnst_params(S, idx, mode);
  const int16_t* scan8 = tu_scan(3, 3);
  // lane j holds src[j] and src[j + 32]
  int s0 = lane < p.tr ? A[lfnst_pos(lane, p.sb, p.transposed, S.w)] : 0;
  int s1 = lane + 32 < p.tr ? A[lfnst_pos(lane + 32, p.sb, p.transposed, S.w)] : 0;
  int out = 0;  // lane j < zo: output j
  for (int i = 0; i < p.tr; i++) {
    const int v = __shfl_sync(0xffffffffu, i < 32 ? s0 : s1, i & 31);
    if (lane < p.zo) out += v * (int)p.m[lane * p.tr + i];
  }
  out = (out + 64) >> 7;
  __syncwarp();
  if (lane < p.tr) {
    const int r = scan8[lane];
    A[(r >> 3) * S.w + (r & 7)] = lane < p.zo ? out : 0;
  }
  if (lane + 32 < p.tr) {
    const int r = scan8[lane + 32];
    A[(r >> 3) * S.w + (r & 7)] = 0;
  }
  __syncwarp();
}

// dct.rs:996-1109 inverse_transform_rect_bd: A (dequantised, raster) -> A
// (residual, raster), B as the transposed intermediate (stride h + 1).
__device__ void tu_inverse_transform(int32_t* A, int32_t* B, const TuShape& S, int bd, int lane) {
  if (S.w == 1 || S.h == 1) {
    const bool col = S.w == 1;
    const int len = col ? S.h : S.w, lg = col ? S.lh : S.lw;
    const int8_t* m = tu_matrix(col ? S.tv : S.th, lg);
    const int cut = len - (col ? S.sh : S.sw);
    const int shift = 21 - bd, add = 1 << (shift - 1);
    int r[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int j = lane + 32 * q;
      int s = 0;
      if (j < len)
        for (int k = 0; k < cut; k++) s += (int)m[k * len + j] * A[k];
      r[q] = clip16i((s + add) >> shift);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; q++)
      if (lane + 32 * q < len) A[lane + 32 * q] = r[q];
    __syncwarp();
    return;
  }
  const int8_t* mv = tu_matrix(S.tv, S.lh);
  const int8_t* mh = tu_matrix(S.th, S.lw);
  const int cw = S.w - S.sw, ch = S.h - S.sh;
  const int hs = S.h + 1;
  for (int id = lane; id < cw * S.h; id += 32) {
    const int i = id >> S.lh, j = id & (S.h - 1);
    int s = 0;
    for (int k = 0; k < ch; k++) s += (int)mv[k * S.h + j] * A[k * S.w + i];
    B[i * hs + j] = clip16i((s + 64) >> 7);
  }
  __syncwarp();
  const int sh2 = 20 - bd, add2 = 1 << (sh2 - 1);
  for (int id = lane; id < S.n; id += 32) {
    const int y = id >> S.lw, x = id & (S.w - 1);
    int s = 0;
    for (int k = 0; k < cw; k++) s += (int)mh[k * S.w + x] * B[k * hs + y];
    A[id] = clip16i((s + add2) >> sh2);
  }
  __syncwarp();
}

// dct.rs:865-991 forward_transform_rect_bd: A (residual, row stride w + 1)
// -> A (coefficients, raster, zero outside the kept region), B intermediate.
__device__ void tu_forward_transform(int32_t* A, int32_t* B, const TuShape& S, int bd, int lane) {
  const int ws = S.w + 1;
  if (S.w == 1 || S.h == 1) {
    const bool col = S.w == 1;
    const int len = col ? S.h : S.w, lg = col ? S.lh : S.lw;
    const int8_t* m = tu_matrix(col ? S.tv : S.th, lg);
    const int cut = len - (col ? S.sh : S.sw);
    const int shift = lg + bd + 6 - 15;
    const int add = shift > 0 ? 1 << (shift - 1) : 0;
    int r[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int v = lane + 32 * q;
      int s = 0;
      if (v < cut)
        for (int k = 0; k < len; k++) s += (int)m[v * len + k] * A[col ? k * ws : k];
      r[q] = v < cut ? clip16(shift >= 0 ? (long long)((s + add) >> shift) : (long long)s << (-shift)) : 0;
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; q++)
      if (lane + 32 * q < len) A[lane + 32 * q] = r[q];
    __syncwarp();
    return;
  }
  const int8_t* mh = tu_matrix(S.th, S.lw);
  const int8_t* mv = tu_matrix(S.tv, S.lh);
  const int cw = S.w - S.sw, ch = S.h - S.sh;
  const int hs = S.h + 1;
  const int sh1 = S.lw + bd + 6 - 15;
  const int add1 = sh1 > 0 ? 1 << (sh1 - 1) : 0;
  for (int id = lane; id < cw * S.h; id += 32) {
    const int k = id >> S.lh, y = id & (S.h - 1);
    int s = 0;
    for (int x = 0; x < S.w; x++) s += (int)mh[k * S.w + x] * A[y * ws + x];
    B[k * hs + y] = (s + add1) >> sh1;  // not clipped (dct.rs:963)
  }
  __syncwarp();
  for (int i = lane; i < S.n; i += 32) A[i] = 0;
  __syncwarp();
  const int sh2 = S.lh + 6;
  const long long add2 = 1ll << (sh2 - 1);
  for (int id = lane; id < ch * cw; id += 32) {
    const int v = id / cw, k = id - v * cw;
    long long s = 0;
    for (int y = 0; y < S.h; y++) s += (long long)mv[v * S.h + y] * B[k * hs + y];
    A[v * S.w + k] = clip16((s + add2) >> sh2);
  }
  __syncwarp();
}

// One warp: levels -> residual of one unit (decode_general.rs:4100-4199 and
// the BDPCM of :4055-4060). The residual goes to `out` with row stride
// `ostride` (0: the unit's width).
__device__ void warp_tu_inverse(const vvcg_tu_rec& r, const int16_t* __restrict__ in,
                                int16_t* __restrict__ out, int32_t* A, int32_t* B, int lane, int ostride = 0) {
  TuShape S;
  tu_shape(r, S);
  const int bd = r.bit_depth, qp = r.qp;
  if (r.flags & VVCG_TU_TRANSFORM_SKIP) {
    for (int i = lane; i < S.n; i += 32) A[i] = tu_dequant_ts(in[i], qp);
    __syncwarp();
  } else {
    for (int i = lane; i < S.n; i += 32) A[i] = in[i];
    __syncwarp();
    if (r.flags & VVCG_TU_DEP_QUANT) {
      tu_dq_dequant(A, S, qp, bd, lane);
    } else {
      // dct.rs:1151-1187 dequantize_rect_bd
      const int q = max(4, qp);
      bool s2;
      const int tr_shift = tu_tr_shift(S.lw, S.lh, bd, &s2);
      const int rs = 6 - (tr_shift + q / 6);
      const long long scale = c_inv_quant_scale[s2 ? 1 : 0][q % 6];
      for (int i = lane; i < S.n; i += 32) {
        const long long v = (long long)A[i] * scale;
        A[i] = clip16(rs > 0 ? (v + (1ll << (rs - 1))) >> rs : v << (-rs));
      }
      __syncwarp();
    }
    if (r.lfnst_idx > 0 && r.mts_idx == 0) tu_lfnst_inverse(A, S, r.lfnst_idx, r.lfnst_mode, lane);
    tu_inverse_transform(A, B, S, bd, lane);
  }
  if (r.flags & (VVCG_TU_BDPCM_HOR | VVCG_TU_BDPCM_VER)) {
    // predict.rs:4224-4240: saturating running sums, one lane per row / column
    const bool vert = (r.flags & VVCG_TU_BDPCM_VER) != 0;
    const int lines = vert ? S.w : S.h, len = vert ? S.h : S.w;
    const int step = vert ? S.w : 1, lstep = vert ? 1 : S.w;
    for (int l = lane; l < lines; l += 32) {
      int acc = A[l * lstep];
      for (int k = 1; k < len; k++) {
        int* p = &A[l * lstep + k * step];
        acc = clampi(*p + acc, -32768, 32767);
        *p = acc;
      }
    }
    __syncwarp();
  }
  if (ostride == 0)
    for (int i = lane; i < S.n; i += 32) out[i] = (int16_t)A[i];
  else
    for (int i = lane; i < S.n; i += 32) out[(size_t)(i >> S.lw) * ostride + (i & (S.w - 1))] = (int16_t)A[i];
  __syncwarp();
}

// One warp: residual -> levels of one unit (slice.rs:690-760, level side).
__device__ void warp_tu_forward(const vvcg_tu_rec& r, const int16_t* __restrict__ in,
                                int16_t* __restrict__ out, int32_t* A, int32_t* B, int lane) {
  TuShape S;
  tu_shape(r, S);
  const int bd = r.bit_depth, qp = r.qp;
  if (r.flags & VVCG_TU_TRANSFORM_SKIP) {
    for (int i = lane; i < S.n; i += 32) out[i] = (int16_t)tu_quant_ts(in[i], qp);
    return;
  }
  const int ws = S.w + 1;
  for (int i = lane; i < S.n; i += 32) A[(i >> S.lw) * ws + (i & (S.w - 1))] = in[i];
  __syncwarp();
  tu_forward_transform(A, B, S, bd, lane);
  if (r.lfnst_idx > 0) tu_lfnst_forward(A, S, r.lfnst_idx, r.lfnst_mode, lane);
  if (r.flags & VVCG_TU_DEP_QUANT) {
    tu_dq_quant(A, S, qp, bd, out, lane);
  } else {
    // dct.rs:1113-1147 quantize_rect_bd
    const int q = max(4, qp);
    bool s2;
    const int tr_shift = tu_tr_shift(S.lw, S.lh, bd, &s2);
    const int qbits = 14 + q / 6 + tr_shift;
    const long long add = (long long)((r.flags & VVCG_TU_INTER) ? 85 : 171) << max(0, qbits - 9);
    const long long scale = c_quant_scale[s2 ? 1 : 0][q % 6];
    for (int i = lane; i < S.n; i += 32) {
      const int c = A[i];
      const long long lv = ((long long)abs(c) * scale + add) >> max(0, qbits);
      out[i] = (int16_t)clip16(c < 0 ? -lv : lv);
    }
  }
}

// Grid: ceil(units / warps); each warp takes idx[blockIdx.x * warps + warp].
template <int kMax, int kWarps, bool kForward>
__global__ void __launch_bounds__(kWarps * 32)
k_tu(const vvcg_tu_rec* __restrict__ recs, const uint32_t* __restrict__ idx, uint32_t n,
     const int16_t* __restrict__ in, int16_t* __restrict__ out) {
  extern __shared__ __align__(16) int32_t tu_smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t t = blockIdx.x * kWarps + wid;
  if (t >= n) return;
  int32_t* A = tu_smem + wid * 2 * (kMax + kTuPad);
  int32_t* B = A + kMax + kTuPad;
  const vvcg_tu_rec r = recs[idx[t]];
  if (kForward)
    warp_tu_forward(r, in + r.in_off, out + r.out_off, A, B, lane);
  else
    warp_tu_inverse(r, in + r.in_off, out + r.out_off, A, B, lane);
}

template <int kMax, int kWarps>
constexpr size_t tu_smem_bytes() {
  return (size_t)kWarps * 2 * (kMax + kTuPad) * sizeof(int32_t);
}

// True when TB c of a coding unit with tu_tools `t` leaves the frame path's
// DCT-2 residual kernel: transform skip, or (luma) explicit MTS / LFNST.
__host__ __device__ __forceinline__ bool tb_uses_tu_tools(uint32_t t, int c) {
  return ((t >> c) & 1) || (c == 0 && (t >> VVCG_CU_MTS_SHIFT) != 0);
}

constexpr int kResToolWarps = 4;

// The frame path's TBs with per-TB transform choices (pictures with
// VVCG_TOOL_TU_TOOLS; slice.rs:1050-1097 reconstruct_block, residual part):
// one warp per coding unit runs each such coded TB through the TU path above
// (transform-skip dequantisation, or dequantisation, inverse LFNST with the
// CU's luma mode, inverse DCT-2 / DST-7 / DCT-8 with the zero-out) into the
// scratch planes, where the reconstruction adds it to the prediction.
// Records outside the ranges of vvcg_cu_rec.tu_tools, or with levels past the
// pool, set the bad-record status and are skipped.
// Grid: (ceil(max CUs per picture / kResToolWarps), pictures).
// A sparse TB's (raster index, level) pairs expanded into n dense levels;
// false when an index is outside the TB or not above the one before it.
__device__ bool expand_sparse(const int16_t* __restrict__ lv, int count, int n, int16_t* dense, int lane) {
  for (int i = lane; i < n; i += 32) dense[i] = 0;
  __syncwarp();
  const uint32_t* pr = reinterpret_cast<const uint32_t*>(lv + 2);
  bool ok = true;
  int prev_last = -1;
  for (int base = 0; base < count; base += 32) {
    const int i = base + lane;
    const bool have = i < count;
    const uint32_t e = have ? pr[i] : (uint32_t)n;
    const int pos = (int)(e & 0xFFFFu);
    int prev = __shfl_up_sync(0xffffffffu, pos, 1);
    if (lane == 0) prev = prev_last;
    if (have) {
      if (pos >= n || pos <= prev)
        ok = false;
      else
        dense[pos] = (int16_t)(e >> 16);
    }
    prev_last = __shfl_sync(0xffffffffu, pos, 31);
  }
  __syncwarp();
  return __all_sync(0xffffffffu, ok);
}

__global__ void __launch_bounds__(kResToolWarps * 32)
k_residual_tools(const DevPic* __restrict__ pics, const int16_t* __restrict__ levels, uint64_t n_levels,
                 uint32_t* status) {
  __shared__ __align__(16) int32_t ws[kResToolWarps][2][1024 + kTuPad];
  __shared__ __align__(16) int16_t dense[kResToolWarps][1024];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const DevPic& P = pics[blockIdx.y];
  if (!(P.tools & VVCG_TOOL_TU_TOOLS)) return;
  const int cu = blockIdx.x * kResToolWarps + wid;
  if (cu >= P.grid_w * P.grid_h) return;
  const vvcg_cu_rec rec = P.cus[cu];
  const uint32_t t = rec.tu_tools;
  if (!t) return;
  const int mts = (t >> VVCG_CU_MTS_SHIFT) & 7, lfnst = t >> VVCG_CU_LFNST_SHIFT;
  const bool bad_tools = mts > 4 || lfnst > 2 || (mts && lfnst) || ((t & VVCG_CU_TS_Y) && (mts || lfnst));
  const bool sparse = (P.tools & VVCG_TOOL_SPARSE_LEVELS) != 0;
  const int gx = cu % P.grid_w, gy = cu / P.grid_w;
  for (int c = 0; c < (P.cf ? 3 : 1); c++) {
    if (!tb_uses_tu_tools(t, c) || !((rec.cbf >> c) & 1)) continue;
    const int off = rec.level_off[c];
    if (off < 0) continue;
    const int w = c ? P.tb_cw : P.tb, h = c ? P.tb_ch : P.tb;
    const int16_t* src = levels + off;
    if (sparse) {  // count at levels[off], pairs from off + 2 (off even)
      const int cnt = (off & 1) || (uint64_t)off + 2 > n_levels ? -1 : levels[off];
      if (bad_tools || cnt < 0 || cnt > w * h || (uint64_t)off + 2 + 2 * (uint64_t)cnt > n_levels ||
          !expand_sparse(levels + off, cnt, w * h, dense[wid], lane)) {
        if (lane == 0) atomicOr(status, kStatusBadRecord);
        continue;
      }
      src = dense[wid];
    } else if (bad_tools || (uint64_t)off + (uint64_t)(w * h) > n_levels) {
      if (lane == 0) atomicOr(status, kStatusBadRecord);
      continue;
    }
    const bool ts = (t >> c) & 1;
    const int q = c ? P.cqp : P.lqp;
    vvcg_tu_rec r;
    r.log2_w = (uint8_t)ilog2(w);
    r.log2_h = (uint8_t)ilog2(h);
    r.bit_depth = (uint8_t)P.bd;
    r.qp = (uint8_t)(ts ? max(4, q) : q);
    r.flags = ts ? VVCG_TU_TRANSFORM_SKIP : ((P.tools & VVCG_TOOL_DEP_QUANT) ? VVCG_TU_DEP_QUANT : 0);
    r.mts_idx = (uint8_t)(c ? 0 : mts);
    r.lfnst_idx = (uint8_t)(c ? 0 : lfnst);
    r.lfnst_mode = rec.luma_mode;
    r.in_off = r.out_off = 0;
    const int x0 = c ? gx * P.tb / P.sub_w : gx * P.tb, y0 = c ? gy * P.tb / P.sub_h : gy * P.tb;
    int16_t* out = reinterpret_cast<int16_t*>(P.scratch[c]) + (size_t)y0 * P.stride[c] + x0;
    warp_tu_inverse(r, src, out, ws[wid][0], ws[wid][1], lane, P.stride[c]);
  }
}

}  // namespace vvcg
