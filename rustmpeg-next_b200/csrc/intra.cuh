// Warp-cooperative intra prediction of the 8..12-bit frame path: reference
// gathering with coded-unit availability, [1 2 1] smoothing, planar / DC /
// 65 angular modes with PDPC, and CCLM, fused with the residual add, clip and
// store. Integer arithmetic only; each function follows the reference function
// named beside it (crates/rustmpeg-video/src/vvc/predict.rs), bit for bit.
#pragma once
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

constexpr int kMaxBlk = 32;                                // largest TB of the frame path

// 4-tap cubic intra interpolation taps, one packed word per 1/32 position,
// staged in shared memory by the kernels that predict (lane-divergent indices
// would serialise constant-memory reads).
__shared__ uint32_t s_cubic_taps[32];
__device__ __forceinline__ void load_cubic_taps() {
  for (int i = threadIdx.x; i < 32; i += blockDim.x)
    s_cubic_taps[i] = (uint32_t)(uint8_t)c_chroma_taps4[4 * i] | ((uint32_t)(uint8_t)c_chroma_taps4[4 * i + 1] << 8) |
                      ((uint32_t)(uint8_t)c_chroma_taps4[4 * i + 2] << 16) |
                      ((uint32_t)(uint8_t)c_chroma_taps4[4 * i + 3] << 24);
  __syncthreads();
}
constexpr int kRefBuf = (kMaxBlk + 4) + 2 * kMaxBlk + 64;  // predict.rs:3251 buf_len

struct IntraWs {
  int16_t above[2 * kMaxBlk];
  int16_t left[2 * kMaxBlk];
  int16_t fabove[2 * kMaxBlk];
  int16_t fleft[2 * kMaxBlk];
  int16_t ref_above[kRefBuf];
  int16_t ref_left[kRefBuf];
  int16_t ds_top[kMaxBlk];   // CCLM luma templates
  int16_t ds_left[kMaxBlk];
  int16_t lcol[kMaxBlk];      // CCLM: luma column left of the CU
  int top_left, ftop_left;
  int dc;
};

// Position of the CU at tb-grid cell (gx, gy) in the coding order of the
// frame path: CTU raster scan, quadtree z-order inside a CTU (slice.rs:164-187).
__device__ __forceinline__ uint32_t cu_order(const DevPic& P, int gx, int gy) {
  int sh = P.ctu_log2 - ilog2(P.tb);
  int cx = gx >> sh, cy = gy >> sh;
  int lx = gx & ((1 << sh) - 1), ly = gy & ((1 << sh) - 1);
  uint32_t z = 0;
  for (int b = 0; b < sh; b++) z |= (((lx >> b) & 1) << (2 * b)) | (((ly >> b) & 1) << (2 * b + 1));
  return ((uint32_t)(cy * P.ctu_w + cx) << (2 * sh)) | z;
}

// CodedUnits::is_coded_luma (slice.rs:218-223) for the CU being coded at cur_order.
__device__ __forceinline__ bool is_coded_luma(const DevPic& P, int lx, int ly, uint32_t cur_order) {
  int gx = lx / P.tb, gy = ly / P.tb;
  if (gx >= P.grid_w || gy >= P.grid_h) return false;
  return cu_order(P, gx, gy) <= cur_order;
}

// AngularParams of predict.rs:1608-1685 (no ISP, no MRL).
struct AngP {
  int pred_mode, angle, abs_inv, scale;
  bool is_ver, ref_filter, interp, pdpc;
};
__device__ __forceinline__ AngP angular_params(int dir, int w, int h, bool is_luma) {
  AngP p;
  int mode = dir;
  // predict.rs:1405-1422 get_modified_wide_angle
  if (dir > 1 && dir <= 66) {
    int delta = abs(floor_log2(w) - floor_log2(h));
    if (delta < 6) {
      const int shifts[6] = {0, 6, 10, 12, 14, 15};
      int s = shifts[delta];
      if (w > h && dir < 2 + s)
        mode = dir + 65;
      else if (h > w && dir > 66 - s)
        mode = dir - 65;
    }
  }
  p.pred_mode = mode;
  p.is_ver = mode >= 34;
  p.pdpc = w >= 4 && h >= 4;
  int am = p.is_ver ? mode - 50 : -(mode - 18);
  int absm = min(31, abs(am));
  int abs_ang = c_ang_table[absm];
  p.abs_inv = c_inv_ang_table[absm];
  p.angle = (am < 0 ? -1 : 1) * abs_ang;
  p.scale = 0;
  if (am < 0) {
    p.pdpc = false;
  } else if (am > 0) {
    int side = p.is_ver ? h : w;
    int inv_term = floor_log2((unsigned)max(1, 3 * p.abs_inv - 2)) - 8;
    p.scale = min(2, floor_log2((unsigned)side) - inv_term);
    if (p.scale < 0) p.pdpc = false;
  }
  p.ref_filter = false;
  p.interp = false;
  if (is_luma && dir != 1 && dir != 0) {
    int diff = min(abs(mode - 18), abs(mode - 50));
    int l2 = (floor_log2(w) + floor_log2(h)) >> 1;
    if (diff > c_intra_filter_thr[min(7, l2)]) {
      bool integer = (abs_ang & 0x1F) == 0;
      p.ref_filter = integer;
      p.interp = !integer;
    }
  }
  return p;
}


__device__ __forceinline__ int ldp(const uint16_t* p) { return __ldcg(p); }

// Reference samples with the frame path's availability rules:
// gather_references_16 (predict.rs:3016-3076) followed by the coded-unit
// substitution of predict_coded_block_16 (predict.rs:3101-3135); `plain`
// leaves the substitution out (predict_block_16, which the encoder's mode
// decisions use: h left samples, 2w above whether coded or not).
// All loads of a lane are issued before any is used (one L2 round trip);
// reads go to L2 (ld.cg) because the samples were written by other SMs.
__device__ void warp_gather_refs(const DevPic& P, int comp, int x, int y, int w, int h,
                                 uint32_t cur_order, IntraWs& S, bool plain) {
  const int lane = threadIdx.x & 31;
  const uint16_t* pl = P.plane[comp];
  const int st = P.stride[comp], pw = P.pw[comp], ph = P.ph[comp];
  const int def = 1 << (P.bd - 1);
  const bool ha = y > 0, hl = x > 0;
  const int sx = comp ? P.sub_w : 1, sy = comp ? P.sub_h : 1;
  // positions: up to 2 above and 2 left samples per lane (2w, 2h <= 64), and the corner
  const uint16_t* pa[2] = {nullptr, nullptr};
  const uint16_t* pll[2] = {nullptr, nullptr};
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int i = lane + 32 * t;
    if (ha && i < 2 * w) {
      int avail = min(pw - x, 2 * w);
      int px = x + (i < avail ? i : avail - 1);
      if (!plain && i >= w && x + i < pw && !is_coded_luma(P, (x + i) * sx, (y - 1) * sy, cur_order))
        px = x + w - 1;
      pa[t] = &pl[(size_t)(y - 1) * st + px];
    }
    const int j = lane + 32 * t;
    if (hl && j < 2 * h) {
      int avail = min(ph - y, h);
      int py = y + (j < avail ? j : avail - 1);
      if (!plain && j >= h && y + j < ph && is_coded_luma(P, (x - 1) * sx, (y + j) * sy, cur_order))
        py = y + j;
      pll[t] = &pl[(size_t)py * st + x - 1];
    }
  }
  const uint16_t* ptl = ha && hl ? &pl[(size_t)(y - 1) * st + x - 1]
                                 : (ha ? &pl[(size_t)(y - 1) * st + x] : (hl ? &pl[(size_t)y * st + x - 1] : nullptr));
  int va[2], vl[2], tl;
#pragma unroll
  for (int t = 0; t < 2; t++) {
    va[t] = pa[t] ? ldp(pa[t]) : def;
    vl[t] = pll[t] ? ldp(pll[t]) : def;
  }
  tl = ptl ? ldp(ptl) : def;
  // gather_references_16's fills when only one side exists
  const int a0 = __shfl_sync(0xffffffffu, va[0], 0);
  const int l0 = __shfl_sync(0xffffffffu, vl[0], 0);
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int i = lane + 32 * t;
    if (i < 2 * w) S.above[i] = (int16_t)(!ha && hl ? l0 : va[t]);
    if (i < 2 * h) S.left[i] = (int16_t)(ha && !hl ? a0 : vl[t]);
  }
  if (lane == 0) S.top_left = tl;
  __syncwarp();
}

// ReferenceSamples16::filtered (predict.rs:2970-3005) into fabove/fleft/ftop_left.
__device__ void warp_filter_refs(int w, int h, IntraWs& S) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < 2 * w; i += 32) {
    int v = S.above[i];
    if (i + 1 < 2 * w) v = ((i == 0 ? S.top_left : S.above[i - 1]) + 2 * v + S.above[i + 1] + 2) >> 2;
    S.fabove[i] = (int16_t)v;
  }
  for (int j = lane; j < 2 * h; j += 32) {
    int v = S.left[j];
    if (j + 1 < 2 * h) v = ((j == 0 ? S.top_left : S.left[j - 1]) + 2 * v + S.left[j + 1] + 2) >> 2;
    S.fleft[j] = (int16_t)v;
  }
  if (lane == 0) S.ftop_left = (2 * S.top_left + S.above[0] + S.left[0] + 2) >> 2;
  __syncwarp();
}

// The samples of a block that other blocks read while they are predicted:
// the bottom `rows` rows and the right `cols` columns. For luma that is 2 rows
// and 5 columns: the above/left reference samples and the corner, the 2 rows /
// 3 columns the neighbours' CCLM templates downsample, and the columns this
// CU's own CCLM needs for its right chroma column pair; for chroma 1 and 1. Phase 1 reconstructs
// those, phase 2 the rest, phase 0 everything.
__device__ __forceinline__ bool in_phase(int phase, int x, int y, int w, int h, int rows, int cols) {
  if (phase == 0) return true;
  const bool edge = y >= h - rows || x + 1 >= w - cols;  // pair (x, x+1)
  return phase == 1 ? edge : !edge;
}

// Reconstruction of the pairs of one w x h block that belong to `phase`:
// `pred(x, y)` gives the prediction of sample (x, y), called for the two
// samples of a pair in a loop kept rolled (instruction-cache misses, not
// arithmetic, limit the wavefront kernels); the
// lane's residual pairs (int16 in a plane-strided buffer, nullable) are all
// fetched before the first is used, then clip(pred + res) is stored with
// 32-bit stores (into the plane when `store`). `keep` (nullable) receives the
// samples (int16 raster, width w).
constexpr int kPairChunk = 1;  // pairs per lane fetched and emitted together
template <class F>
__device__ __forceinline__ void emit_block(const DevPic& P, int comp, int x0, int y0, int w, int h,
                                           const int16_t* res, int16_t* keep, bool store, int phase,
                                           int rows, int cols, F&& pred) {
  const int lane = threadIdx.x & 31;
  const int maxv = (1 << P.bd) - 1;
  const int lw = ilog2(w);
  const int npair = (w * h) >> 1;
  const int st = P.stride[comp];
  uint16_t* base = P.plane[comp] + (size_t)y0 * st + x0;
#pragma unroll 1
  for (int k0 = 0; 32 * k0 < npair; k0 += kPairChunk) {
    uint32_t rv[kPairChunk];
#pragma unroll
    for (int k = 0; k < kPairChunk; k++) {
      const int q = lane + 32 * (k0 + k);
      const int y = (2 * q) >> lw, x = (2 * q) & (w - 1);
      rv[k] = 0;
      if (res && q < npair && in_phase(phase, x, y, w, h, rows, cols))
        rv[k] = __ldcs(reinterpret_cast<const unsigned int*>(res + (size_t)y * st + x));
    }
#pragma unroll
    for (int k = 0; k < kPairChunk; k++) {
      const int q = lane + 32 * (k0 + k);
      const int y = (2 * q) >> lw, x = (2 * q) & (w - 1);
      if (q < npair && in_phase(phase, x, y, w, h, rows, cols)) {
        int pv[2];
#pragma unroll 1
        for (int t = 0; t < 2; t++) pv[t] = pred(x + t, y);
        const int v0 = clampi(pv[0] + (int)(int16_t)(rv[k] & 0xFFFFu), 0, maxv);
        const int v1 = clampi(pv[1] + (int)(int16_t)(rv[k] >> 16), 0, maxv);
        const uint32_t pk = (uint32_t)v0 | ((uint32_t)v1 << 16);
        if (store) *reinterpret_cast<uint32_t*>(base + (size_t)y * st + x) = pk;
        if (keep) *reinterpret_cast<uint32_t*>(&keep[y * w + x]) = pk;
      }
    }
  }
  __syncwarp();
}

// Gathers the references of one block and prepares what its prediction needs
// in S: filtered references (planar, angular with the [1 2 1] filter), the DC
// value, and the extended main/side reference arrays of angular modes
// (predict_angular_16, predict.rs:3240-3305).
__device__ __noinline__ void prep_intra(const DevPic& P, int comp, int x0, int y0, int w, int h, bool is_luma,
                           int mode, uint32_t order, IntraWs& S, bool plain = false) {
  const int lane = threadIdx.x & 31;
  const int bd = P.bd, maxv = (1 << bd) - 1;
  const int lw = ilog2(w), lh = ilog2(h);
  warp_gather_refs(P, comp, x0, y0, w, h, order, S, plain);
  if (mode == 0) {
    if (is_luma && w * h > 32) warp_filter_refs(w, h, S);
    return;
  }
  if (mode == 1) {
    unsigned st = 0, sl = 0;
    for (int i = lane; i < w; i += 32) st += (unsigned)S.above[i];
    for (int j = lane; j < h; j += 32) sl += (unsigned)S.left[j];
    st = __reduce_add_sync(0xffffffffu, st);
    sl = __reduce_add_sync(0xffffffffu, sl);
    unsigned dcu;
    if (w == h)
      dcu = (st + sl + (unsigned)w) >> (lw + 1);
    else if (w > h)
      dcu = (st + ((unsigned)w >> 1)) >> lw;
    else
      dcu = (sl + ((unsigned)h >> 1)) >> lh;
    if (lane == 0) S.dc = (int)min(dcu & 0xFFFFu, (unsigned)maxv);
    __syncwarp();
    return;
  }
  if (mode < 2 || mode > 66) return;
  const AngP p = angular_params(mode, w, h, is_luma);
  if (p.ref_filter) warp_filter_refs(w, h, S);
  const int16_t* A = p.ref_filter ? S.fabove : S.above;
  const int16_t* L = p.ref_filter ? S.fleft : S.left;
  const int tl = p.ref_filter ? S.ftop_left : S.top_left;
  const int def = 1 << (bd - 1);
  const int mx = max(w, h);
  const int base = mx + 4;
  const int buf_len = base + 2 * mx + 64;
  const int lim_a = p.angle < 0 ? w + 1 : 2 * w;
  const int lim_l = p.angle < 0 ? h + 1 : 2 * h;
  for (int i = lane; i < buf_len; i += 32) {
    int k = i - base;
    int va = def, vl = def;
    if (k >= 0 && k <= lim_a) va = k == 0 ? tl : A[min(k, 2 * w) - 1];
    if (k >= 0 && k <= lim_l) vl = k == 0 ? tl : L[min(k, 2 * h) - 1];
    S.ref_above[i] = (int16_t)va;
    S.ref_left[i] = (int16_t)vl;
  }
  __syncwarp();
  if (p.angle < 0) {
    const int size_side = p.is_ver ? h : w;
    for (int k = -size_side + lane; k <= -1; k += 32) {
      int proj = min((-k * p.abs_inv + 256) >> 9, size_side);
      if (p.is_ver)
        S.ref_above[base + k] = S.ref_left[base + proj];
      else
        S.ref_left[base + k] = S.ref_above[base + proj];
    }
  } else if (lane == 0) {
    if (p.is_ver) {
      int16_t v = S.ref_above[base + 2 * w];
      S.ref_above[base + 2 * w + 1] = v;
      S.ref_above[base + 2 * w + 2] = v;
    } else {
      int16_t v = S.ref_left[base + 2 * h];
      S.ref_left[base + 2 * h + 1] = v;
      S.ref_left[base + 2 * h + 2] = v;
    }
  }
  __syncwarp();
}

// Intra prediction of one block (prepared by prep_intra) fused with
// reconstruction, for the pairs of `phase`: planar / DC are
// predict_from_refs_16 + apply_pdpc_16 (predict.rs:3138-3215), angular is
// predict_angular_16 (:3223-3410), other mode values predict zeros
// (predict.rs:3194). `keep` (optional) receives the reconstructed samples;
// without `store` only `keep` is written (a prediction, when `res` is null).
__device__ __noinline__ void emit_intra(const DevPic& P, int comp, int x0, int y0, int w, int h, bool is_luma,
                           int mode, const IntraWs& S, const int16_t* res, int16_t* keep, int phase,
                           int rows, int cols, bool store = true) {
  const int bd = P.bd, maxv = (1 << bd) - 1;
  const int lw = ilog2(w), lh = ilog2(h);
  if (mode == 0) {
    const bool filt = is_luma && w * h > 32;
    const int16_t* A = filt ? S.fabove : S.above;
    const int16_t* L = filt ? S.fleft : S.left;
    const int shift = lw + lh + 1;
    const int tr = A[w], bl = L[h];
    const int sc = (lw + lh >= 2 ? lw + lh - 2 : 0) >> 2;
    emit_block(P, comp, x0, y0, w, h, res, keep, store, phase, rows, cols, [&](int rx, int ry) -> int {
      const int left = L[ry];
      const int wt = 32 >> min(31, (ry * 2) >> sc);
      // exact in int32 for bd <= 12 and w, h <= 64
      int ver = (h - 1 - ry) * A[rx] + (ry + 1) * bl;
      int hor = (w - 1 - rx) * left + (rx + 1) * tr;
      int val = clampi(((ver << lw) + (hor << lh) + (1 << (shift - 1))) >> shift, 0, maxv);
      int wl = 32 >> min(31, (rx * 2) >> sc);
      return clampi(val + ((wl * (left - val) + wt * (A[rx] - val) + 32) >> 6), 0, maxv);
    });
    return;
  }
  if (mode == 1) {
    const int dc = S.dc;
    const int sc = (lw + lh >= 2 ? lw + lh - 2 : 0) >> 2;
    emit_block(P, comp, x0, y0, w, h, res, keep, store, phase, rows, cols, [&](int rx, int ry) -> int {
      const int wt = 32 >> min(31, (ry * 2) >> sc);
      const int wl = 32 >> min(31, (rx * 2) >> sc);
      return clampi(dc + ((wl * (S.left[ry] - dc) + wt * (S.above[rx] - dc) + 32) >> 6), 0, maxv);
    });
    return;
  }
  if (mode < 2 || mode > 66) {
    emit_block(P, comp, x0, y0, w, h, res, keep, store, phase, rows, cols, [&](int, int) -> int { return 0; });
    return;
  }
  const AngP p = angular_params(mode, w, h, is_luma);
  const int mx = max(w, h);
  const int base = mx + 4;
  const int buf_len = base + 2 * mx + 64;
  const int16_t* rm = p.is_ver ? S.ref_above : S.ref_left;
  const int16_t* rs = p.is_ver ? S.ref_left : S.ref_above;
  const int ww = p.is_ver ? w : h, wh = p.is_ver ? h : w;
  if (p.angle == 0) {
    const int sc0 = (ilog2(ww) + ilog2(wh) - 2) >> 2;
    const int lim = p.pdpc ? min(3 << sc0, ww) : 0;
    auto sample = [&](int x, int yy) -> int {
      int val = rm[base + x + 1];
      if (x < lim) {
        int wl = 32 >> ((2 * x) >> sc0);
        val = clampi(val + ((wl * (rs[base + 1 + yy] - rm[base]) + 32) >> 6), 0, maxv);
      }
      return val;
    };
    emit_block(P, comp, x0, y0, w, h, res, keep, store, phase, rows, cols, [&](int ox, int oy) -> int {
      return p.is_ver ? sample(ox, oy) : sample(oy, ox);
    });
    return;
  }
  // Every non-zero-angle case is one 4-tap filter over rm[j..j+3], j = base + di + x:
  // integer slopes take rm[j+1] (taps 0,64,0,0: (64v + 32) >> 6 == v); chroma's
  // linear p0 + ((f (p1 - p0) + 16) >> 5) with p0 = rm[j+1] equals taps
  // 0, 2(32-f), 2f, 0; luma non-integer slopes use the Gaussian or cubic taps.
  const int kind = (abs(p.angle) & 0x1F) == 0 ? 0 : (!is_luma ? 1 : (p.interp ? 2 : 3));
  const int sca = max(0, p.scale);
  const int lim = p.pdpc ? min(3 << sca, ww) : 0;
  auto sample = [&](int x, int yy) -> int {
    const int dp = p.angle * (yy + 1);
    const int di = dp >> 5, fr = dp & 31;
    int f0, f1, f2, f3;
    if (kind == 0) {
      f0 = 0; f1 = 64; f2 = 0; f3 = 0;
    } else if (kind == 1) {
      f0 = 0; f1 = 2 * (32 - fr); f2 = 2 * fr; f3 = 0;
    } else if (kind == 2) {
      f0 = 16 - (fr >> 1); f1 = 32 - (fr >> 1); f2 = 16 + (fr >> 1); f3 = fr >> 1;
    } else {
      const uint32_t t = s_cubic_taps[fr];
      f0 = (int8_t)t;
      f1 = (int8_t)(t >> 8);
      f2 = (int8_t)(t >> 16);
      f3 = (int8_t)(t >> 24);
    }
    const int j = base + di + x;
    int val = clampi((f0 * rm[j] + f1 * rm[j + 1] + f2 * rm[j + 2] + f3 * rm[j + 3] + 32) >> 6, 0, maxv);
    if (x < lim) {
      const int inv_sum = 256 + (x + 1) * p.abs_inv;
      const int wl = 32 >> ((2 * x) >> sca);
      const int li = min(base + yy + (inv_sum >> 9) + 1, buf_len - 1);
      val = clampi(val + ((wl * (rs[li] - val) + 32) >> 6), 0, maxv);
    }
    return val;
  };
  emit_block(P, comp, x0, y0, w, h, res, keep, store, phase, rows, cols, [&](int ox, int oy) -> int {
      return p.is_ver ? sample(ox, oy) : sample(oy, ox);
    });
}

// CCLM templates and linear models for both chroma components of the chroma
// block at (bxc, byc): the luma templates of downsample_luma_for_cclm_format_16
// (predict.rs:3869-3990) go to L.ds_top / L.ds_left, the luma column left of the
// CU (x = lbx - 1) to L.lcol, and each component's (a, b, shift) of
// predict_cclm_with_format_16 (predict.rs:3996-4066) and
// derive_cclm_params_from_4_samples (:2088-2177) to Sc[c].dc / ftop_left /
// top_left. All plane loads of a lane are independent (one round trip).
__device__ __noinline__ void prep_cclm(const DevPic& P, int bxc, int byc, int cw, int ch, int lbx, int lby, int tb,
                          int cclm_mode, IntraWs& L, IntraWs* Sc) {
  const int lane = threadIdx.x & 31;
  const uint16_t* lp = P.plane[0];
  const int lst = P.stride[0], lwid = P.pw[0], lhei = P.ph[0];
  const int bd = P.bd, mid = 1 << (bd - 1);
  const int cf = P.cf;
  const int bx = bxc * P.sub_w, by = byc * P.sub_h;
  auto gp = [&](int x, int y) -> int {  // plane read, coordinates clamped
    return ldp(&lp[(size_t)clampi(y, 0, lhei - 1) * lst + clampi(x, 0, lwid - 1)]);
  };
  // luma column lbx - 1 next to the tile, rows lby .. lby + tb - 1
  if (lbx > 0)
    for (int r = lane; r < tb; r += 32) L.lcol[r] = (int16_t)gp(lbx - 1, lby + r);
  int vt = mid, vl = mid;
  const int x = lane, y = lane;
  if (x < cw) {
    if (cf == 1) {
      const bool first_row = (by & (P.ctu - 1)) == 0;
      if (by > 0 && first_row) {
        int lx = bx + 2 * x, yy = by - 1;
        int x0 = clampi(lx, 0, lwid - 1), xr = clampi(lx + 1, 0, lwid - 1);
        int xl = ((x == 0 && bx == 0) || x0 == 0) ? x0 : x0 - 1;
        int a = gp(x0, yy), b = gp(xl, yy), c = gp(xr, yy);
        vt = (2 * a + b + c + 2) >> 2;
      } else if (by >= 2) {
        int lx = bx + 2 * x, ly = by - 2;
        int lxl = (x == 0 && !(bx > 0)) ? lx : lx - 1;
        int a = gp(lx, ly), b = gp(lxl, ly), c = gp(lx + 1, ly);
        int d = gp(lx, ly + 1), e = gp(lxl, ly + 1), f = gp(lx + 1, ly + 1);
        vt = (2 * a + b + c + 2 * d + e + f + 4) >> 3;
      }
    } else if (cf == 2) {
      if (by > 0) {
        int lx = bx + 2 * x, ly = by - 1;
        int lxl = (x == 0 && bx == 0) ? lx : lx - 1;
        int a = gp(lx, ly), b = gp(lxl, ly), c = gp(lx + 1, ly);
        vt = (2 * a + b + c + 2) >> 2;
      }
    } else if (by > 0) {
      vt = gp(bx + x, by - 1);
    }
  }
  if (y < ch) {
    if (cf == 1) {
      if (bx >= 2) {
        int lx = bx - 2, ly = by + 2 * y;
        int a = gp(lx, ly), b = gp(lx - 1, ly), c = gp(lx + 1, ly);
        int d = gp(lx, ly + 1), e = gp(lx - 1, ly + 1), f = gp(lx + 1, ly + 1);
        vl = (2 * a + b + c + 2 * d + e + f + 4) >> 3;
      }
    } else if (cf == 2) {
      if (bx > 0) {
        int ly = by + y, lx = bx - 2;
        int lxl = bx >= 2 ? lx - 1 : lx;
        int a = gp(max(0, lx), ly), b = gp(max(0, lxl), ly), c = gp(bx - 1, ly);
        vl = (2 * a + b + c + 2) >> 2;
      }
    } else if (bx > 0) {
      vl = gp(bx - 1, by + y);
    }
  }
  if (x < cw) L.ds_top[x] = (int16_t)vt;
  if (y < ch) L.ds_left[y] = (int16_t)vl;
  __syncwarp();
  const bool ha = byc > 0, hl = bxc > 0;
  const bool has_top = ha && cclm_mode != 1;
  const bool has_left = hl && cclm_mode != 2;
  // template positions of the LM derivation (same for both components)
  int idx[4] = {0, 0, 0, 0}, from_top[4] = {0, 0, 0, 0};
  int cnt = 0;
  if (has_top && has_left) {
    idx[0] = cw / 4; idx[1] = (3 * cw) / 4; idx[2] = ch / 4; idx[3] = (3 * ch) / 4;
    from_top[0] = from_top[1] = 1;
    cnt = 4;
  } else if (has_top) {
    for (int i = 0; i < min(4, cw); i++) {
      idx[i] = min(((2 * i + 1) * cw) / 8, cw - 1);
      from_top[i] = 1;
      cnt++;
    }
  } else if (has_left) {
    for (int i = 0; i < min(4, ch); i++) {
      idx[i] = min(((2 * i + 1) * ch) / 8, ch - 1);
      cnt++;
    }
  }
  // lanes 0..3: component 1, lanes 4..7: component 2 fetch one chroma template sample
  int tv = mid;
  if (lane < 8) {
    const int c = 1 + (lane >> 2), i = lane & 3;
    const uint16_t* pl = P.plane[c];
    const int st = P.stride[c], pw = P.pw[c], ph = P.ph[c];
    if (i < cnt) {
      if (from_top[i]) {  // gather_references_16 above row
        tv = ha ? ldp(&pl[(size_t)(byc - 1) * st + min(bxc + idx[i], pw - 1)])
                : (hl ? ldp(&pl[(size_t)byc * st + bxc - 1]) : mid);
      } else {  // left column
        tv = hl ? ldp(&pl[(size_t)min(byc + idx[i], ph - 1) * st + bxc - 1])
                : (ha ? ldp(&pl[(size_t)(byc - 1) * st + bxc]) : mid);
      }
    }
  }
  for (int c = 1; c <= 2; c++) {
    int sl[4], sc[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      sl[i] = i < cnt ? (from_top[i] ? L.ds_top[idx[i]] : L.ds_left[idx[i]]) : mid;
      sc[i] = __shfl_sync(0xffffffffu, tv, (c - 1) * 4 + i);
      if (i >= cnt) sc[i] = mid;
    }
    int a = 0, b = mid, shift = 0;
    if (cnt == 0) {
      a = 0;
      b = 1 << (bd - 1);
      shift = 0;
    } else {
      if (cnt == 2) {
        sl[3] = sl[0]; sc[3] = sc[0];
        sl[2] = sl[1]; sc[2] = sc[1];
        sl[0] = sl[1]; sc[0] = sc[1];
        sl[1] = sl[3]; sc[1] = sc[3];
      }
      int mn0 = 0, mn1 = 2, mx0 = 1, mx1 = 3, t;
      if (sl[mn0] > sl[mn1]) { t = mn0; mn0 = mn1; mn1 = t; }
      if (sl[mx0] > sl[mx1]) { t = mx0; mx0 = mx1; mx1 = t; }
      if (sl[mn0] > sl[mx1]) {
        t = mn0; mn0 = mx0; mx0 = t;
        t = mn1; mn1 = mx1; mx1 = t;
      }
      if (sl[mn1] > sl[mx0]) { t = mn1; mn1 = mx0; mx0 = t; }
      int min_l = (sl[mn0] + sl[mn1] + 1) >> 1, min_c = (sc[mn0] + sc[mn1] + 1) >> 1;
      int max_l = (sl[mx0] + sl[mx1] + 1) >> 1, max_c = (sc[mx0] + sc[mx1] + 1) >> 1;
      int diff = max_l - min_l;
      if (diff > 0) {
        int diff_c = max_c - min_c;
        int xx = floor_log2((unsigned)diff);
        int norm = ((diff << 4) >> xx) & 15;
        int vv = (int)c_cclm_div_sig[norm] | 8;
        if (norm != 0) xx += 1;
        int yy = diff_c == 0 ? 1 : floor_log2((unsigned)abs(diff_c)) + 1;
        int add = (1 << yy) >> 1;
        a = (diff_c * vv + add) >> yy;
        shift = 3 + xx - yy;
        if (shift < 1) {
          shift = 1;
          a = a == 0 ? 0 : (a < 0 ? -15 : 15);
        }
        b = min_c - ((a * min_l) >> shift);
      } else {
        a = 0;
        b = min_c;
        shift = 0;
      }
    }
    if (lane == 0) {
      Sc[c - 1].dc = a;
      Sc[c - 1].ftop_left = b;
      Sc[c - 1].top_left = shift;
    }
  }
  __syncwarp();
}

// CCLM prediction of one chroma component fused with reconstruction, for the
// pairs of `phase`; the downsampled luma of each sample is formed from the
// CU's reconstructed luma tile (tb x tb at (lbx, lby)) and the prefetched
// column left of it (L.lcol), as downsample_luma_for_cclm_format_16 does.
__device__ __noinline__ void emit_cclm(const DevPic& P, int comp, int bxc, int byc, int cw, int ch, int lbx,
                          int lby, int tb, const IntraWs& L, const IntraWs& S, const int16_t* tile,
                          const int16_t* res, int phase, int16_t* keep = nullptr, bool store = true) {
  const int maxv = (1 << P.bd) - 1;
  const int cf = P.cf;
  const int a = S.dc, b = S.ftop_left, shift = S.top_left;
  const int bx = bxc * P.sub_w, by = byc * P.sub_h;
  auto T = [&](int x, int y) -> int {  // x >= lbx - 1; y inside the tile
    return x < lbx ? L.lcol[y - lby] : tile[(y - lby) * tb + (x - lbx)];
  };
  auto ds = [&](int x, int y) -> int {
    if (cf == 1) {
      int lx = bx + 2 * x, ly = by + 2 * y;
      int lxl = (x == 0 && bx == 0) ? lx : lx - 1;
      int r0 = 2 * T(lx, ly) + T(lxl, ly) + T(lx + 1, ly);
      int r1 = 2 * T(lx, ly + 1) + T(lxl, ly + 1) + T(lx + 1, ly + 1);
      return (r0 + r1 + 4) >> 3;
    }
    if (cf == 2) {
      int lx = bx + 2 * x, ly = by + y;
      int lxl = (x == 0 && bx == 0) ? lx : lx - 1;
      return (2 * T(lx, ly) + T(lxl, ly) + T(lx + 1, ly) + 2) >> 2;
    }
    return T(bx + x, by + y);
  };
  emit_block(P, comp, bxc, byc, cw, ch, res, keep, store, phase, 1, 1, [&](int x, int y) -> int {
    return clampi(((ds(x, y) * a) >> shift) + b, 0, maxv);
  });
}

}  // namespace vvcg
