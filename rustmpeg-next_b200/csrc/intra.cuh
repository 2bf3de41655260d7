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
constexpr int kRefBuf = (kMaxBlk + 4) + 2 * kMaxBlk + 64;  // predict.rs:3251 buf_len

struct IntraWs {
  int16_t above[2 * kMaxBlk];
  int16_t left[2 * kMaxBlk];
  int16_t fabove[2 * kMaxBlk];
  int16_t fleft[2 * kMaxBlk];
  int16_t ref_above[kRefBuf];
  int16_t ref_left[kRefBuf];
  int16_t ds_top[kMaxBlk];
  int16_t ds_left[kMaxBlk];
  int top_left, ftop_left;
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
// substitution of predict_coded_block_16 (predict.rs:3101-3135). Reads go to
// L2 (ld.cg): the samples were written by other SMs.
__device__ void warp_gather_refs(const DevPic& P, int comp, int x, int y, int w, int h,
                                 uint32_t cur_order, IntraWs& S) {
  const int lane = threadIdx.x & 31;
  const uint16_t* pl = P.plane[comp];
  const int st = P.stride[comp], pw = P.pw[comp], ph = P.ph[comp];
  const int def = 1 << (P.bd - 1);
  const bool ha = y > 0, hl = x > 0;
  const int sx = comp ? P.sub_w : 1, sy = comp ? P.sub_h : 1;
  for (int i = lane; i < 2 * w; i += 32) {
    int v = def;
    if (ha) {
      int avail = min(pw - x, 2 * w);
      v = ldp(&pl[(size_t)(y - 1) * st + x + (i < avail ? i : avail - 1)]);
      if (i >= w && x + i < pw && !is_coded_luma(P, (x + i) * sx, (y - 1) * sy, cur_order))
        v = ldp(&pl[(size_t)(y - 1) * st + x + w - 1]);
    }
    S.above[i] = (int16_t)v;
  }
  for (int j = lane; j < 2 * h; j += 32) {
    int v = def;
    if (hl) {
      int avail = min(ph - y, h);
      v = ldp(&pl[(size_t)(y + (j < avail ? j : avail - 1)) * st + x - 1]);
      if (j >= h && y + j < ph && is_coded_luma(P, (x - 1) * sx, (y + j) * sy, cur_order))
        v = ldp(&pl[(size_t)(y + j) * st + x - 1]);
    }
    S.left[j] = (int16_t)v;
  }
  int tl = def;
  if (ha && hl)
    tl = ldp(&pl[(size_t)(y - 1) * st + x - 1]);
  else if (ha)
    tl = ldp(&pl[(size_t)(y - 1) * st + x]);
  else if (hl)
    tl = ldp(&pl[(size_t)y * st + x - 1]);
  __syncwarp();
  if (ha && !hl) {
    int16_t a0 = S.above[0];
    for (int j = lane; j < 2 * h; j += 32) S.left[j] = a0;
  } else if (!ha && hl) {
    int16_t l0 = S.left[0];
    for (int i = lane; i < 2 * w; i += 32) S.above[i] = l0;
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

// Writes clip(pred + res) for sample pairs (x, x+1) of row y as one 32-bit
// store. `res` (nullable) points at the block's residual in a plane-strided
// int16 buffer; `keep` (nullable) receives the block (int16 raster, width w).
__device__ __forceinline__ void store_pair(const DevPic& P, int comp, int x0, int y0, int w, int x,
                                           int y, int p0, int p1, const int16_t* res, int16_t* keep,
                                           int maxv) {
  if (res) {
    uint32_t rv = __ldcs(reinterpret_cast<const unsigned int*>(res + (size_t)y * P.stride[comp] + x));
    p0 += (int)(int16_t)(rv & 0xFFFFu);
    p1 += (int)(int16_t)(rv >> 16);
  }
  const int v0 = clampi(p0, 0, maxv), v1 = clampi(p1, 0, maxv);
  uint16_t* dst = P.plane[comp] + (size_t)(y0 + y) * P.stride[comp] + x0 + x;
  *reinterpret_cast<uint32_t*>(dst) = (uint32_t)v0 | ((uint32_t)v1 << 16);
  if (keep) *reinterpret_cast<uint32_t*>(&keep[y * w + x]) = (uint32_t)v0 | ((uint32_t)v1 << 16);
}

// Intra prediction of one block fused with reconstruction: gathers the
// references, predicts (planar / DC: predict_from_refs_16 + apply_pdpc_16,
// predict.rs:3138-3215; angular: predict_angular_16, :3223-3410; other mode
// values predict zeros as in predict.rs:3194), adds the residual, clips and
// stores. `keep` (optional) receives the reconstructed block (int16 raster).
__device__ void warp_predict_store(const DevPic& P, int comp, int x0, int y0, int w, int h,
                                   bool is_luma, int mode, uint32_t order, IntraWs& S,
                                   const int16_t* res, int16_t* keep) {
  const int lane = threadIdx.x & 31;
  const int bd = P.bd, maxv = (1 << bd) - 1;
  const int lw = ilog2(w), lh = ilog2(h);
  const int npair = (w * h) >> 1;
  warp_gather_refs(P, comp, x0, y0, w, h, order, S);
  if (mode == 0) {
    const bool filt = is_luma && w * h > 32;
    if (filt) warp_filter_refs(w, h, S);
    const int16_t* A = filt ? S.fabove : S.above;
    const int16_t* L = filt ? S.fleft : S.left;
    const int shift = lw + lh + 1;
    const int tr = A[w], bl = L[h];
    const int sc = (lw + lh >= 2 ? lw + lh - 2 : 0) >> 2;
    for (int q = lane; q < npair; q += 32) {
      const int ry = (2 * q) >> lw, rx0 = (2 * q) & (w - 1);
      const int left = L[ry];
      const int wt = 32 >> min(31, (ry * 2) >> sc);
      int v[2];
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const int rx = rx0 + t;
        // (h-1-ry)*A + (ry+1)*bl and (w-1-rx)*L + (rx+1)*tr fit in int32 for bd <= 12, w,h <= 64
        int ver = (h - 1 - ry) * A[rx] + (ry + 1) * bl;
        int hor = (w - 1 - rx) * left + (rx + 1) * tr;
        int val = ((ver << lw) + (hor << lh) + (1 << (shift - 1))) >> shift;
        val = clampi(val, 0, maxv);
        int wl = 32 >> min(31, (rx * 2) >> sc);
        v[t] = clampi(val + ((wl * (left - val) + wt * (A[rx] - val) + 32) >> 6), 0, maxv);
      }
      store_pair(P, comp, x0, y0, w, rx0, ry, v[0], v[1], res, keep, maxv);
    }
    __syncwarp();
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
    const int dc = (int)min(dcu & 0xFFFFu, (unsigned)maxv);
    const int sc = (lw + lh >= 2 ? lw + lh - 2 : 0) >> 2;
    for (int q = lane; q < npair; q += 32) {
      const int ry = (2 * q) >> lw, rx0 = (2 * q) & (w - 1);
      const int wt = 32 >> min(31, (ry * 2) >> sc);
      int v[2];
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const int rx = rx0 + t;
        int wl = 32 >> min(31, (rx * 2) >> sc);
        v[t] = clampi(dc + ((wl * (S.left[ry] - dc) + wt * (S.above[rx] - dc) + 32) >> 6), 0, maxv);
      }
      store_pair(P, comp, x0, y0, w, rx0, ry, v[0], v[1], res, keep, maxv);
    }
    __syncwarp();
    return;
  }
  if (mode < 2 || mode > 66) {
    for (int q = lane; q < npair; q += 32) {
      const int ry = (2 * q) >> lw, rx0 = (2 * q) & (w - 1);
      store_pair(P, comp, x0, y0, w, rx0, ry, 0, 0, res, keep, maxv);
    }
    __syncwarp();
    return;
  }
  // ---- angular ----
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
  const int16_t* rm = p.is_ver ? S.ref_above : S.ref_left;
  const int16_t* rs = p.is_ver ? S.ref_left : S.ref_above;
  const int ww = p.is_ver ? w : h, wh = p.is_ver ? h : w;
  if (p.angle == 0) {
    const int sc0 = (ilog2(ww) + ilog2(wh) - 2) >> 2;
    const int lim = p.pdpc ? min(3 << sc0, ww) : 0;
    for (int q = lane; q < npair; q += 32) {
      const int oy = (2 * q) >> lw, ox0 = (2 * q) & (w - 1);
      int v[2];
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const int ox = ox0 + t;
        const int x = p.is_ver ? ox : oy, yy = p.is_ver ? oy : ox;  // work coordinates
        int val = rm[base + x + 1];
        if (x < lim) {
          int wl = 32 >> ((2 * x) >> sc0);
          val = clampi(val + ((wl * (rs[base + 1 + yy] - rm[base]) + 32) >> 6), 0, maxv);
        }
        v[t] = val;
      }
      store_pair(P, comp, x0, y0, w, ox0, oy, v[0], v[1], res, keep, maxv);
    }
    __syncwarp();
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
      f0 = c_chroma_taps4[fr * 4 + 0];
      f1 = c_chroma_taps4[fr * 4 + 1];
      f2 = c_chroma_taps4[fr * 4 + 2];
      f3 = c_chroma_taps4[fr * 4 + 3];
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
  for (int q = lane; q < npair; q += 32) {
    const int oy = (2 * q) >> lw, ox0 = (2 * q) & (w - 1);
    int v0, v1;
    if (p.is_ver) {
      v0 = sample(ox0, oy);
      v1 = sample(ox0 + 1, oy);
    } else {
      v0 = sample(oy, ox0);
      v1 = sample(oy, ox0 + 1);
    }
    store_pair(P, comp, x0, y0, w, ox0, oy, v0, v1, res, keep, maxv);
  }
  __syncwarp();
}

// CCLM luma downsampling (downsample_luma_for_cclm_format_16, predict.rs:3869-3990)
// for the chroma block at (bxc, byc): `ds` (cw*ch int16) gets the block, S.ds_top /
// S.ds_left the templates. The CU's own reconstructed luma comes from `tile`
// (tb x tb at luma (lbx, lby)); everything else is read from the plane.
__device__ void warp_cclm_downsample(const DevPic& P, int bxc, int byc, int cw, int ch, int lbx,
                                     int lby, int tb, const int16_t* tile, IntraWs& S, int16_t* ds) {
  const int lane = threadIdx.x & 31;
  const uint16_t* lp = P.plane[0];
  const int lst = P.stride[0], lwid = P.pw[0], lhei = P.ph[0];
  const int mid = 1 << (P.bd - 1);
  const int cf = P.cf;
  const int bx = bxc * P.sub_w, by = byc * P.sub_h;
  auto gy = [&](int x, int y) -> int {
    x = clampi(x, 0, lwid - 1);
    y = clampi(y, 0, lhei - 1);
    if (x >= lbx && x < lbx + tb && y >= lby && y < lby + tb) return tile[(y - lby) * tb + (x - lbx)];
    return ldp(&lp[(size_t)y * lst + x]);
  };
  for (int i = lane; i < cw * ch; i += 32) {
    int x = i % cw, y = i / cw;
    int v;
    if (cf == 1) {
      int lx = bx + 2 * x, ly = by + 2 * y;
      int lxl = (x == 0 && !(bx > 0)) ? lx : lx - 1;
      int r0 = 2 * gy(lx, ly) + gy(lxl, ly) + gy(lx + 1, ly);
      int r1 = 2 * gy(lx, ly + 1) + gy(lxl, ly + 1) + gy(lx + 1, ly + 1);
      v = (r0 + r1 + 4) >> 3;
    } else if (cf == 2) {
      int lx = bx + 2 * x, ly = by + y;
      int lxl = (x == 0 && bx == 0) ? lx : lx - 1;
      v = (2 * gy(lx, ly) + gy(lxl, ly) + gy(lx + 1, ly) + 2) >> 2;
    } else {
      v = gy(bx + x, by + y);
    }
    ds[i] = (int16_t)v;
  }
  for (int x = lane; x < cw; x += 32) {
    int v = mid;
    if (cf == 1) {
      const bool first_row = (by & (P.ctu - 1)) == 0;
      if (by > 0 && first_row) {
        int lx = bx + 2 * x, yy = by - 1;
        int x0 = clampi(lx, 0, lwid - 1), xr = clampi(lx + 1, 0, lwid - 1);
        int xl = ((x == 0 && bx == 0) || x0 == 0) ? x0 : x0 - 1;
        v = (2 * gy(x0, yy) + gy(xl, yy) + gy(xr, yy) + 2) >> 2;
      } else if (by >= 2) {
        int lx = bx + 2 * x, ly = by - 2;
        int lxl = (x == 0 && !(bx > 0)) ? lx : lx - 1;
        int r0 = 2 * gy(lx, ly) + gy(lxl, ly) + gy(lx + 1, ly);
        int r1 = 2 * gy(lx, ly + 1) + gy(lxl, ly + 1) + gy(lx + 1, ly + 1);
        v = (r0 + r1 + 4) >> 3;
      }
    } else if (cf == 2) {
      if (by > 0) {
        int lx = bx + 2 * x, ly = by - 1;
        int lxl = (x == 0 && bx == 0) ? lx : lx - 1;
        v = (2 * gy(lx, ly) + gy(lxl, ly) + gy(lx + 1, ly) + 2) >> 2;
      }
    } else if (by > 0) {
      v = gy(bx + x, by - 1);
    }
    S.ds_top[x] = (int16_t)v;
  }
  for (int y = lane; y < ch; y += 32) {
    int v = mid;
    if (cf == 1) {
      if (bx >= 2) {
        int lx = bx - 2, ly = by + 2 * y;
        int r0 = 2 * gy(lx, ly) + gy(lx - 1, ly) + gy(lx + 1, ly);
        int r1 = 2 * gy(lx, ly + 1) + gy(lx - 1, ly + 1) + gy(lx + 1, ly + 1);
        v = (r0 + r1 + 4) >> 3;
      }
    } else if (cf == 2) {
      if (bx > 0) {
        int ly = by + y, lx = bx - 2;
        int lxl = bx >= 2 ? lx - 1 : lx;
        v = (2 * gy(max(0, lx), ly) + gy(max(0, lxl), ly) + gy(bx - 1, ly) + 2) >> 2;
      }
    } else if (bx > 0) {
      v = gy(bx - 1, by + y);
    }
    S.ds_left[y] = (int16_t)v;
  }
  __syncwarp();
}

// predict_cclm_with_format_16 (predict.rs:3996-4066) for one chroma component
// from a prepared downsampling, fused with add / clip / store.
// cclm_mode 0 LM, 1 LM-L, 2 LM-T. Chroma templates come from a plain gather.
__device__ void warp_cclm_predict_store(const DevPic& P, int comp, int bxc, int byc, int cw, int ch,
                                        int cclm_mode, IntraWs& S, const int16_t* ds,
                                        const int16_t* res) {
  const int lane = threadIdx.x & 31;
  const int bd = P.bd, maxv = (1 << bd) - 1, mid = 1 << (bd - 1);
  const uint16_t* pl = P.plane[comp];
  const int st = P.stride[comp], pw = P.pw[comp], ph = P.ph[comp];
  const bool ha = byc > 0, hl = bxc > 0;
  // template samples at the positions the LM derivation reads
  auto above = [&](int i) -> int {
    if (ha) return ldp(&pl[(size_t)(byc - 1) * st + min(bxc + i, pw - 1)]);
    if (hl) return ldp(&pl[(size_t)byc * st + bxc - 1]);
    return mid;
  };
  auto left = [&](int j) -> int {
    if (hl) return ldp(&pl[(size_t)min(byc + j, ph - 1) * st + bxc - 1]);
    if (ha) return ldp(&pl[(size_t)(byc - 1) * st + bxc]);
    return mid;
  };
  int a = 0, b = mid, shift = 0;
  {
    const bool has_top = byc > 0 && cclm_mode != 1;
    const bool has_left = bxc > 0 && cclm_mode != 2;
    int sl[4] = {mid, mid, mid, mid}, sc[4] = {mid, mid, mid, mid};
    int cnt = 0;
    if (has_top && has_left) {
      int x0 = cw / 4, x1 = (3 * cw) / 4, y0 = ch / 4, y1 = (3 * ch) / 4;
      sl[0] = S.ds_top[x0]; sl[1] = S.ds_top[x1]; sl[2] = S.ds_left[y0]; sl[3] = S.ds_left[y1];
      sc[0] = above(x0); sc[1] = above(x1); sc[2] = left(y0); sc[3] = left(y1);
      cnt = 4;
    } else if (has_top) {
      for (int i = 0; i < min(4, cw); i++) {
        int idx = min(((2 * i + 1) * cw) / 8, cw - 1);
        sl[i] = S.ds_top[idx];
        sc[i] = above(idx);
        cnt++;
      }
    } else if (has_left) {
      for (int i = 0; i < min(4, ch); i++) {
        int idx = min(((2 * i + 1) * ch) / 8, ch - 1);
        sl[i] = S.ds_left[idx];
        sc[i] = left(idx);
        cnt++;
      }
    }
    // derive_cclm_params_from_4_samples (predict.rs:2088-2177); every lane
    // evaluates it on the same values
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
  }
  const int lw = ilog2(cw);
  for (int q = lane; q < (cw * ch) >> 1; q += 32) {
    const int y = (2 * q) >> lw, x = (2 * q) & (cw - 1);
    int p0 = clampi(((ds[y * cw + x] * a) >> shift) + b, 0, maxv);
    int p1 = clampi(((ds[y * cw + x + 1] * a) >> shift) + b, 0, maxv);
    store_pair(P, comp, bxc, byc, cw, x, y, p0, p1, res, nullptr, maxv);
  }
  __syncwarp();
}

}  // namespace vvcg
