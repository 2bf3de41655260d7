// Cooperative (one CTA per block) intra prediction of the 8..12-bit frame
// path: reference gathering with coded-unit availability, [1 2 1] smoothing,
// planar / DC / 65 angular modes with PDPC, and CCLM. Integer arithmetic
// only; each function follows the reference function named beside it
// (crates/rustmpeg-video/src/vvc/predict.rs) so results are bit-identical.
#pragma once
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

constexpr int kMaxBlk = 32;                        // largest TB of the frame path
constexpr int kRefBuf = (kMaxBlk + 4) + 2 * kMaxBlk + 64;  // predict.rs:3251 buf_len

struct IntraSmem {
  int above[2 * kMaxBlk];
  int left[2 * kMaxBlk];
  int fabove[2 * kMaxBlk];
  int fleft[2 * kMaxBlk];
  int ref_above[kRefBuf];
  int ref_left[kRefBuf];
  int top_left, ftop_left;
  int dc;
  int cclm_a, cclm_b, cclm_shift;
  int ds_top[kMaxBlk];
  int ds_left[kMaxBlk];
  int ds_blk[kMaxBlk * kMaxBlk];
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

// Reference samples with the frame path's availability rules:
// gather_references_16 (predict.rs:3016-3076) followed by the coded-unit
// substitution of predict_coded_block_16 (predict.rs:3101-3135) when `coded`.
__device__ void gather_refs(const DevPic& P, int comp, int x, int y, int w, int h, bool coded,
                            uint32_t cur_order, IntraSmem& S) {
  const uint16_t* pl = P.plane[comp];
  const int st = P.stride[comp], pw = P.pw[comp], ph = P.ph[comp];
  const int def = 1 << (P.bd - 1);
  const bool ha = y > 0, hl = x > 0;
  const int sx = comp ? P.sub_w : 1, sy = comp ? P.sub_h : 1;
  for (int i = threadIdx.x; i < 2 * w; i += blockDim.x) {
    int v = def;
    if (ha) {
      int avail = min(pw - x, 2 * w);
      int px = x + (i < avail ? i : avail - 1);
      v = __ldcg(&pl[(size_t)(y - 1) * st + px]);
      if (coded && i >= w && x + i < pw && !is_coded_luma(P, (x + i) * sx, (y - 1) * sy, cur_order))
        v = __ldcg(&pl[(size_t)(y - 1) * st + x + w - 1]);
    }
    S.above[i] = v;
  }
  for (int j = threadIdx.x; j < 2 * h; j += blockDim.x) {
    int v = def;
    if (hl) {
      int avail = min(ph - y, h);
      int py = y + (j < avail ? j : avail - 1);
      v = __ldcg(&pl[(size_t)py * st + x - 1]);
      if (coded && j >= h && y + j < ph && is_coded_luma(P, (x - 1) * sx, (y + j) * sy, cur_order))
        v = __ldcg(&pl[(size_t)(y + j) * st + x - 1]);
    }
    S.left[j] = v;
  }
  __syncthreads();
  if (ha && !hl) {
    int a0 = S.above[0];
    for (int j = threadIdx.x; j < 2 * h; j += blockDim.x) S.left[j] = a0;
  } else if (!ha && hl) {
    int l0 = S.left[0];
    for (int i = threadIdx.x; i < 2 * w; i += blockDim.x) S.above[i] = l0;
  }
  if (threadIdx.x == 0) {
    if (ha && hl)
      S.top_left = __ldcg(&pl[(size_t)(y - 1) * st + x - 1]);
    else if (ha)
      S.top_left = __ldcg(&pl[(size_t)(y - 1) * st + x]);
    else if (hl)
      S.top_left = __ldcg(&pl[(size_t)y * st + x - 1]);
    else
      S.top_left = def;
  }
  __syncthreads();
}

// ReferenceSamples16::filtered (predict.rs:2970-3005) into fabove/fleft/ftop_left.
__device__ void filter_refs(int w, int h, IntraSmem& S) {
  for (int i = threadIdx.x; i < 2 * w; i += blockDim.x) {
    int v = S.above[i];
    if (i + 1 < 2 * w) {
      int prev = i == 0 ? S.top_left : S.above[i - 1];
      v = (prev + 2 * S.above[i] + S.above[i + 1] + 2) >> 2;
    }
    S.fabove[i] = v;
  }
  for (int j = threadIdx.x; j < 2 * h; j += blockDim.x) {
    int v = S.left[j];
    if (j + 1 < 2 * h) {
      int prev = j == 0 ? S.top_left : S.left[j - 1];
      v = (prev + 2 * S.left[j] + S.left[j + 1] + 2) >> 2;
    }
    S.fleft[j] = v;
  }
  if (threadIdx.x == 0) S.ftop_left = (2 * S.top_left + S.above[0] + S.left[0] + 2) >> 2;
  __syncthreads();
}

// Prediction of one block into `pred` (shared, w*h ints, raster).
// Planar / DC: predict_from_refs_16 (predict.rs:3138-3196) + apply_pdpc_16
// (:3200); angular: predict_angular_16 (:3223-3410). Other mode values
// predict zeros, as the reference does (predict.rs:3194).
__device__ void predict_intra(int w, int h, bool is_luma, int mode, int bd, IntraSmem& S,
                              int* pred) {
  const int maxv = (1 << bd) - 1;
  const int lw = ilog2(w), lh = ilog2(h);
  const int n = w * h;
  if (mode == 0) {
    bool filt = is_luma && n > 32;
    if (filt) filter_refs(w, h, S);
    const int* A = filt ? S.fabove : S.above;
    const int* L = filt ? S.fleft : S.left;
    const int shift = lw + lh + 1;
    const int tr = A[w], bl = L[h];
    const int sc = (lw + lh >= 2 ? lw + lh - 2 : 0) >> 2;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int rx = i & (w - 1), ry = i >> lw;
      long long ver = (long long)(h - 1 - ry) * A[rx] + (long long)(ry + 1) * bl;
      long long hor = (long long)(w - 1 - rx) * L[ry] + (long long)(rx + 1) * tr;
      long long v = ((ver << lw) + (hor << lh) + (1ll << (shift - 1))) >> shift;
      int val = (int)(v < 0 ? 0 : (v > maxv ? maxv : v));
      int wt = 32 >> min(31, (ry * 2) >> sc), wl = 32 >> min(31, (rx * 2) >> sc);
      pred[i] = clampi(val + ((wl * (L[ry] - val) + wt * (A[rx] - val) + 32) >> 6), 0, maxv);
    }
    __syncthreads();
    return;
  }
  if (mode == 1) {
    if (threadIdx.x < 32) {
      unsigned st = 0, sl = 0;
      for (int i = threadIdx.x; i < w; i += 32) st += S.above[i];
      for (int j = threadIdx.x; j < h; j += 32) sl += S.left[j];
      for (int o = 16; o > 0; o >>= 1) {
        st += __shfl_xor_sync(0xffffffffu, st, o);
        sl += __shfl_xor_sync(0xffffffffu, sl, o);
      }
      if (threadIdx.x == 0) {
        unsigned dc;
        if (w == h)
          dc = (st + sl + (unsigned)w) >> (lw + 1);
        else if (w > h)
          dc = (st + ((unsigned)w >> 1)) >> lw;
        else
          dc = (sl + ((unsigned)h >> 1)) >> lh;
        dc &= 0xFFFFu;
        S.dc = (int)min(dc, (unsigned)maxv);
      }
    }
    __syncthreads();
    const int dc = S.dc;
    const int sc = (lw + lh >= 2 ? lw + lh - 2 : 0) >> 2;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int rx = i & (w - 1), ry = i >> lw;
      int wt = 32 >> min(31, (ry * 2) >> sc), wl = 32 >> min(31, (rx * 2) >> sc);
      pred[i] = clampi(dc + ((wl * (S.left[ry] - dc) + wt * (S.above[rx] - dc) + 32) >> 6), 0, maxv);
    }
    __syncthreads();
    return;
  }
  if (mode < 2 || mode > 66) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) pred[i] = 0;
    __syncthreads();
    return;
  }
  // ---- angular ----
  const AngP p = angular_params(mode, w, h, is_luma);
  if (p.ref_filter) filter_refs(w, h, S);
  const int* A = p.ref_filter ? S.fabove : S.above;
  const int* L = p.ref_filter ? S.fleft : S.left;
  const int tl = p.ref_filter ? S.ftop_left : S.top_left;
  const int def = 1 << (bd - 1);
  const int mx = max(w, h);
  const int base = mx + 4;
  const int buf_len = base + 2 * mx + 64;
  // row_above = [tl, A[0..2w)], row_left = [tl, L[0..2h)]; index clamps at the end
  for (int i = threadIdx.x; i < buf_len; i += blockDim.x) {
    int k = i - base;
    int va = def, vl = def;
    int lim_a = p.angle < 0 ? w + 1 : 2 * w;
    int lim_l = p.angle < 0 ? h + 1 : 2 * h;
    if (k >= 0 && k <= lim_a) va = k == 0 ? tl : A[min(k, 2 * w) - 1];
    if (k >= 0 && k <= lim_l) vl = k == 0 ? tl : L[min(k, 2 * h) - 1];
    S.ref_above[i] = va;
    S.ref_left[i] = vl;
  }
  __syncthreads();
  if (p.angle < 0) {
    int size_side = p.is_ver ? h : w;
    for (int k = -size_side + (int)threadIdx.x; k <= -1; k += blockDim.x) {
      int proj = min((-k * p.abs_inv + 256) >> 9, size_side);
      if (p.is_ver)
        S.ref_above[base + k] = S.ref_left[base + proj];
      else
        S.ref_left[base + k] = S.ref_above[base + proj];
    }
  } else if (threadIdx.x == 0) {
    if (p.is_ver) {
      int v = S.ref_above[base + 2 * w];
      S.ref_above[base + 2 * w + 1] = v;
      S.ref_above[base + 2 * w + 2] = v;
    } else {
      int v = S.ref_left[base + 2 * h];
      S.ref_left[base + 2 * h + 1] = v;
      S.ref_left[base + 2 * h + 2] = v;
    }
  }
  __syncthreads();
  const int* rm = p.is_ver ? S.ref_above : S.ref_left;
  const int* rs = p.is_ver ? S.ref_left : S.ref_above;
  const int ww = p.is_ver ? w : h, wh = p.is_ver ? h : w;
  const int lww = ilog2(ww);
  const bool int_slope = (abs(p.angle) & 0x1F) == 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int x = i & (ww - 1), yy = i >> lww;  // work coordinates
    int v;
    if (p.angle == 0) {
      v = rm[base + x + 1];
      int sc = (ilog2(ww) + ilog2(wh) - 2) >> 2;
      if (p.pdpc && x < min(3 << sc, ww)) {
        int wl = 32 >> ((2 * x) >> sc);
        v = clampi(v + ((wl * (rs[base + 1 + yy] - rm[base]) + 32) >> 6), 0, maxv);
      }
    } else {
      int dp = p.angle * (yy + 1);
      int di = dp >> 5, fr = dp & 31;
      if (!int_slope) {
        if (is_luma) {
          int f0, f1, f2, f3;
          if (p.interp) {
            f0 = 16 - (fr >> 1);
            f1 = 32 - (fr >> 1);
            f2 = 16 + (fr >> 1);
            f3 = fr >> 1;
          } else {
            f0 = c_chroma_taps4[fr * 4 + 0];
            f1 = c_chroma_taps4[fr * 4 + 1];
            f2 = c_chroma_taps4[fr * 4 + 2];
            f3 = c_chroma_taps4[fr * 4 + 3];
          }
          int j = base + di + x;
          int s = f0 * rm[j] + f1 * rm[j + 1] + f2 * rm[j + 2] + f3 * rm[j + 3];
          v = clampi((s + 32) >> 6, 0, maxv);
        } else {
          int j = base + di + x + 1;
          int p0 = rm[j], p1 = rm[j + 1];
          v = clampi(p0 + ((fr * (p1 - p0) + 16) >> 5), 0, maxv);
        }
      } else {
        v = clampi(rm[base + di + x + 1], 0, maxv);
      }
      if (p.pdpc) {
        int sc = max(0, p.scale);
        if (x < min(3 << sc, ww)) {
          int inv_sum = 256 + (x + 1) * p.abs_inv;
          int wl = 32 >> ((2 * x) >> sc);
          int li = min(base + yy + (inv_sum >> 9) + 1, buf_len - 1);
          v = clampi(v + ((wl * (rs[li] - v) + 32) >> 6), 0, maxv);
        }
      }
    }
    int ox = p.is_ver ? x : yy, oy = p.is_ver ? yy : x;
    pred[oy * w + ox] = v;
  }
  __syncthreads();
}

// CCLM for the frame path: downsample_luma_for_cclm_format_16 (predict.rs:3869-3990)
// and predict_cclm_with_format_16 (:3996-4066). cclm_mode 0 LM, 1 LM-L, 2 LM-T.
// Chroma references come from a plain gather (no coded-unit substitution).
__device__ void predict_cclm(const DevPic& P, int comp, int bxc, int byc, int cw, int ch,
                             int cclm_mode, IntraSmem& S, int* pred) {
  const uint16_t* ly = P.plane[0];
  const int lst = P.stride[0], lwid = P.pw[0], lhei = P.ph[0];
  const int bd = P.bd, maxv = (1 << bd) - 1, mid = 1 << (bd - 1);
  const int cf = P.cf;
  const int bx = bxc * P.sub_w, by = byc * P.sub_h;
  auto gy = [&](int x, int y) -> int {
    return __ldcg(&ly[(size_t)clampi(y, 0, lhei - 1) * lst + clampi(x, 0, lwid - 1)]);
  };
  const int n = cw * ch;
  // downsampled block
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int x = i % cw, y = i / cw;
    int v;
    if (cf == 1) {
      int lx = bx + 2 * x, lyy = by + 2 * y;
      int lxl = (x == 0 && !(bx > 0)) ? lx : lx - 1;
      int r0 = 2 * gy(lx, lyy) + gy(lxl, lyy) + gy(lx + 1, lyy);
      int r1 = 2 * gy(lx, lyy + 1) + gy(lxl, lyy + 1) + gy(lx + 1, lyy + 1);
      v = (r0 + r1 + 4) >> 3;
    } else if (cf == 2) {
      int lx = bx + 2 * x, lyy = by + y;
      int lxl = (x == 0 && bx == 0) ? lx : lx - 1;
      v = (2 * gy(lx, lyy) + gy(lxl, lyy) + gy(lx + 1, lyy) + 2) >> 2;
    } else {
      v = gy(bx + x, by + y);
    }
    S.ds_blk[i] = v;
  }
  for (int x = threadIdx.x; x < cw; x += blockDim.x) {
    int v = mid;
    if (cf == 1) {
      bool first_row = (by & (P.ctu - 1)) == 0;
      if (by > 0 && first_row) {
        int lx = bx + 2 * x, yy = by - 1;
        int x0 = clampi(lx, 0, lwid - 1), xr = clampi(lx + 1, 0, lwid - 1);
        int xl = ((x == 0 && bx == 0) || x0 == 0) ? x0 : x0 - 1;
        v = (2 * gy(x0, yy) + gy(xl, yy) + gy(xr, yy) + 2) >> 2;
      } else if (by >= 2) {
        int lx = bx + 2 * x, lyy = by - 2;
        int lxl = (x == 0 && !(bx > 0)) ? lx : lx - 1;
        int r0 = 2 * gy(lx, lyy) + gy(lxl, lyy) + gy(lx + 1, lyy);
        int r1 = 2 * gy(lx, lyy + 1) + gy(lxl, lyy + 1) + gy(lx + 1, lyy + 1);
        v = (r0 + r1 + 4) >> 3;
      }
    } else if (cf == 2) {
      if (by > 0) {
        int lx = bx + 2 * x, lyy = by - 1;
        int lxl = (x == 0 && bx == 0) ? lx : lx - 1;
        v = (2 * gy(lx, lyy) + gy(lxl, lyy) + gy(lx + 1, lyy) + 2) >> 2;
      }
    } else if (by > 0) {
      v = gy(bx + x, by - 1);
    }
    S.ds_top[x] = v;
  }
  for (int y = threadIdx.x; y < ch; y += blockDim.x) {
    int v = mid;
    if (cf == 1) {
      if (bx >= 2) {
        int lx = bx - 2, lyy = by + 2 * y;
        int r0 = 2 * gy(lx, lyy) + gy(lx - 1, lyy) + gy(lx + 1, lyy);
        int r1 = 2 * gy(lx, lyy + 1) + gy(lx - 1, lyy + 1) + gy(lx + 1, lyy + 1);
        v = (r0 + r1 + 4) >> 3;
      }
    } else if (cf == 2) {
      if (bx > 0) {
        int lyy = by + y, lx = bx - 2;
        int lxl = bx >= 2 ? lx - 1 : lx;
        v = (2 * gy(max(0, lx), lyy) + gy(max(0, lxl), lyy) + gy(bx - 1, lyy) + 2) >> 2;
      }
    } else if (bx > 0) {
      v = gy(bx - 1, by + y);
    }
    S.ds_left[y] = v;
  }
  __syncthreads();
  // chroma template: plain gather_references_16 of this component
  {
    const uint16_t* pl = P.plane[comp];
    const int st = P.stride[comp], pw = P.pw[comp], ph = P.ph[comp];
    const bool ha = byc > 0, hl = bxc > 0;
    for (int i = threadIdx.x; i < cw; i += blockDim.x) {
      int v = mid;
      if (ha) v = __ldcg(&pl[(size_t)(byc - 1) * st + min(bxc + i, pw - 1)]);
      else if (hl) v = __ldcg(&pl[(size_t)byc * st + bxc - 1]);
      S.above[i] = v;
    }
    for (int j = threadIdx.x; j < ch; j += blockDim.x) {
      int v = mid;
      if (hl) v = __ldcg(&pl[(size_t)min(byc + j, ph - 1) * st + bxc - 1]);
      else if (ha) v = __ldcg(&pl[(size_t)(byc - 1) * st + bxc]);
      S.left[j] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const bool has_top = byc > 0 && cclm_mode != 1;
    const bool has_left = bxc > 0 && cclm_mode != 2;
    int sl[4] = {mid, mid, mid, mid}, sc[4] = {mid, mid, mid, mid};
    int cnt = 0;
    if (has_top && has_left) {
      int x0 = cw / 4, x1 = (3 * cw) / 4, y0 = ch / 4, y1 = (3 * ch) / 4;
      sl[0] = S.ds_top[x0]; sl[1] = S.ds_top[x1]; sl[2] = S.ds_left[y0]; sl[3] = S.ds_left[y1];
      sc[0] = S.above[x0]; sc[1] = S.above[x1]; sc[2] = S.left[y0]; sc[3] = S.left[y1];
      cnt = 4;
    } else if (has_top) {
      for (int i = 0; i < min(4, cw); i++) {
        int idx = min(((2 * i + 1) * cw) / 8, cw - 1);
        sl[i] = S.ds_top[idx];
        sc[i] = S.above[idx];
        cnt++;
      }
    } else if (has_left) {
      for (int i = 0; i < min(4, ch); i++) {
        int idx = min(((2 * i + 1) * ch) / 8, ch - 1);
        sl[i] = S.ds_left[idx];
        sc[i] = S.left[idx];
        cnt++;
      }
    }
    // derive_cclm_params_from_4_samples (predict.rs:2088-2177)
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
    S.cclm_a = a;
    S.cclm_b = b;
    S.cclm_shift = shift;
  }
  __syncthreads();
  const int a = S.cclm_a, b = S.cclm_b, shift = S.cclm_shift;
  for (int i = threadIdx.x; i < n; i += blockDim.x) pred[i] = clampi(((S.ds_blk[i] * a) >> shift) + b, 0, maxv);
  __syncthreads();
}

}  // namespace vvcg
