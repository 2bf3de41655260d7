// Reconstruction of the 8..12-bit frame path on the GPU: a persistent
// wavefront kernel. One work item is a CTU; items are handed out by an atomic
// counter in wavefront order (CTU diagonal t = cx + 2*cy across all pictures
// of the batch), so a CTA only ever waits on items that running CTAs already
// hold and the schedule cannot deadlock. Per CTU, the CTA first dequantises
// and inverse-transforms its residual (independent of neighbours), then waits
// (bounded) for the left and top-right CTUs, then predicts, adds and clips.
//
// Follows slice::decode_vvc_frame_picture_with_chroma_qp (slice.rs:4834-4988):
// predict_coded_block_16 / CCLM prediction, dequantize_rect_bd or
// dequantize_dep_quant_bd (dct.rs:1151, :1191), inverse_transform_rect_bd
// (dct.rs:996) with DCT-II in both directions, and the add/clip to 0..2^bd-1.
#pragma once
#include "intra.cuh"
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

struct ResidSmem {
  int coef[kMaxBlk * kMaxBlk];
  int tmp[kMaxBlk * kMaxBlk];
  int maxr, maxc, last;
};

// The DCT-II matrices of the frame path's TB sizes (16 and 32), staged in
// shared memory once per CTA of the persistent kernel.
struct MatSmem {
  int16_t m32[32 * 32];
  int16_t m16[16 * 16];
};

__device__ __forceinline__ const int16_t* dct2_smem(const MatSmem& M, int n) {
  return n == 32 ? M.m32 : M.m16;
}

// Dequantisation (regular or dependent) and 2-D inverse DCT-II of a w x h TB
// (w, h in {16, 32}) whose int16 raster levels start at `lv`; the residual is
// left in `res` (w*h ints). Zero rows/columns beyond the last nonzero level
// are skipped, which does not change any sum.
__device__ void residual_dct2(const int16_t* __restrict__ lv, int w, int h, int qp_scaled, int bd,
                              bool dq, const MatSmem& M, ResidSmem& R, int* res) {
  const int n = w * h, lw = ilog2(w), lh = ilog2(h);
  if (threadIdx.x == 0) {
    R.maxr = -1;
    R.maxc = -1;
    R.last = -1;
  }
  __syncthreads();
  const bool s2 = ((lw + lh) & 1) != 0;
  const int tr_shift = 15 - bd - ((lw + lh) >> 1) - (s2 ? 1 : 0);
  int lmaxr = -1, lmaxc = -1;
  if (!dq) {
    // dequantize_rect_bd (dct.rs:1151-1187)
    const int qp = max(4, qp_scaled);
    const int qp_per = qp / 6, qp_rem = qp % 6;
    const int rs = 6 - (tr_shift + qp_per);
    const long long scale = c_inv_quant_scale[s2 ? 1 : 0][qp_rem];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int L = lv[i];
      int v = 0;
      if (L != 0) {
        lmaxr = max(lmaxr, i >> lw);
        lmaxc = max(lmaxc, i & (w - 1));
        long long val = (long long)L * scale;
        long long sc = rs > 0 ? (val + (1ll << (rs - 1))) >> rs : val << (-rs);
        v = clip16(sc);
      }
      R.coef[i] = v;
    }
  } else {
    // dequantize_dep_quant_bd (dct.rs:1191-1248): the 4-state machine walks
    // the grouped diagonal scan backwards from the last nonzero level. The
    // walk is split into 32 chunks; each lane composes its chunk's state
    // transitions, a warp scan of the compositions gives each chunk's entry
    // state, then every lane replays its chunk.
    const int16_t* scan = g_scan + g_scan_off[(lw - 1) * 6 + (lh - 1)];
    const int ns = min(w, 32) * min(h, 32);
    int llast = -1;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int L = lv[i];
      R.coef[i] = L;
      if (L != 0) {
        lmaxr = max(lmaxr, i >> lw);
        lmaxc = max(lmaxc, i & (w - 1));
      }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < ns; s += blockDim.x)
      if (R.coef[scan[s]] != 0) llast = max(llast, s);
    llast = __reduce_max_sync(0xffffffffu, llast);
    if ((threadIdx.x & 31) == 0 && llast >= 0) atomicMax(&R.last, llast);
    __syncthreads();
    const int last = R.last;
    if (threadIdx.x < 32 && last >= 0) {
      const int lane = threadIdx.x;
      const int cs = (last + 32) >> 5;  // ceil((last + 1) / 32)
      const int hi = last - lane * cs;  // first scan position of this chunk
      const int lo = max(hi - cs + 1, 0);
      // composite map of this chunk: 2 bits per start state
      uint32_t map = 0;
      for (int st0 = 0; st0 < 4; st0++) {
        int st = st0;
        for (int s = hi; s >= lo; s--) {
          int L = R.coef[scan[s]];
          st = (32040 >> ((st << 2) + ((L & 1) << 1))) & 3;
        }
        map |= (uint32_t)st << (2 * st0);
      }
      if (hi < 0) map = 0xE4u;  // identity (3,2,1,0) for empty chunks
      // inclusive scan: P_L = f_L o f_{L-1} o ... o f_0
      uint32_t pre = map;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t other = __shfl_up_sync(0xffffffffu, pre, o);
        if (lane >= o) {
          uint32_t comp = 0;  // pre o other
          for (int s = 0; s < 4; s++) {
            int mid = (other >> (2 * s)) & 3;
            comp |= ((pre >> (2 * mid)) & 3) << (2 * s);
          }
          pre = comp;
        }
      }
      uint32_t excl = __shfl_up_sync(0xffffffffu, pre, 1);
      int st = lane == 0 ? 0 : (int)(excl & 3);  // P_{L-1}(0)
      const int qp_dq = max(4, qp_scaled) + 1;
      const int qp_per = qp_dq / 6, qp_rem = qp_dq % 6;
      const int shift = 7 - qp_per - tr_shift;
      long long inv_q = c_inv_quant_scale[s2 ? 1 : 0][qp_rem];
      if (shift < 0) inv_q <<= -shift;
      const long long add = shift > 0 ? (1ll << (shift - 1)) : 0;
      const int rsh = max(0, shift);
      for (int s = hi; s >= lo; s--) {
        int r = scan[s];
        int L = R.coef[r];
        if (L != 0) {
          long long q = (long long)(2 * L + (L > 0 ? -(st >> 1) : (st >> 1)));
          R.coef[r] = clip16((q * inv_q + add) >> rsh);
        }
        st = (32040 >> ((st << 2) + ((L & 1) << 1))) & 3;
      }
    }
  }
  lmaxr = __reduce_max_sync(0xffffffffu, lmaxr);
  lmaxc = __reduce_max_sync(0xffffffffu, lmaxc);
  if ((threadIdx.x & 31) == 0) {
    if (lmaxr >= 0) atomicMax(&R.maxr, lmaxr);
    if (lmaxc >= 0) atomicMax(&R.maxc, lmaxc);
  }
  __syncthreads();
  const int maxr = R.maxr, maxc = R.maxc;
  if (maxr < 0) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) res[i] = 0;
    __syncthreads();
    return;
  }
  // inverse_transform_rect_bd (dct.rs:1075-1108): columns, then rows
  const int16_t* mv = dct2_smem(M, h);
  const int16_t* mh = dct2_smem(M, w);
  const int ncol = maxc + 1;
  for (int t = threadIdx.x; t < ncol * h; t += blockDim.x) {
    int i = t >> lh, j = t & (h - 1);
    int sum = 0;
    for (int k = 0; k <= maxr; k++) sum += (int)mv[k * h + j] * R.coef[k * w + i];
    R.tmp[i * h + j] = clip16i((sum + 64) >> 7);
  }
  __syncthreads();
  const int sh2 = 20 - bd;
  const int add2 = 1 << (sh2 - 1);
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    int x = t & (w - 1), y = t >> lw;
    int sum = 0;
    for (int k = 0; k < ncol; k++) sum += (int)mh[k * w + x] * R.tmp[k * h + y];
    res[t] = clip16i((sum + add2) >> sh2);
  }
  __syncthreads();
}

struct ReconSmem {
  MatSmem M;
  ResidSmem R;
  IntraSmem S;
  int res[3][kMaxBlk * kMaxBlk];
  int pred[kMaxBlk * kMaxBlk];
  DevPic P;
  uint32_t item;
  int timed_out;
};

// Residuals of the three TBs of one CU into sm.res (zeros without levels).
__device__ void cu_residuals(const DevPic& P, const vvcg_cu_rec& rec, const int16_t* levels,
                             uint64_t n_levels, uint32_t* status, ReconSmem& sm) {
  const bool dq = (P.tools & VVCG_TOOL_DEP_QUANT) != 0;
  const int ncomp = P.cf ? 3 : 1;
  for (int c = 0; c < ncomp; c++) {
    const int w = c ? P.tb_cw : P.tb, h = c ? P.tb_ch : P.tb;
    const int off = rec.level_off[c];
    const bool has = ((rec.cbf >> c) & 1) && off >= 0;
    if (has && (uint64_t)off + (uint64_t)(w * h) > n_levels) {
      if (threadIdx.x == 0) atomicOr(status, kStatusBadRecord);
    }
    if (has && (uint64_t)off + (uint64_t)(w * h) <= n_levels) {
      residual_dct2(levels + off, w, h, c ? P.cqp : P.lqp, P.bd, dq, sm.M, sm.R, sm.res[c]);
    } else {
      for (int i = threadIdx.x; i < w * h; i += blockDim.x) sm.res[c][i] = 0;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void store_block(const DevPic& P, int comp, int x0, int y0, int w, int h,
                                            const int* pred, const int* res) {
  uint16_t* pl = P.plane[comp];
  const int st = P.stride[comp];
  const int maxv = (1 << P.bd) - 1;
  const int lw = ilog2(w);
  for (int i = threadIdx.x; i < w * h; i += blockDim.x) {
    int x = i & (w - 1), y = i >> lw;
    pl[(size_t)(y0 + y) * st + x0 + x] = (uint16_t)clampi(pred[i] + res[i], 0, maxv);
  }
}

// Bounded wait for a CTU flag; returns false when the poll limit ran out.
__device__ __forceinline__ bool wait_flag(const uint32_t* flag, uint32_t epoch, uint32_t limit) {
  uint32_t ns = 32;
  for (uint32_t it = 0; it < limit; it++) {
    if (ld_acquire(flag) == epoch) return true;
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
  return ld_acquire(flag) == epoch;
}

__global__ void __launch_bounds__(256, 2)
k_recon_wavefront(const DevPic* __restrict__ pics, const CtuItem* __restrict__ items,
                  uint32_t n_items, uint32_t* counter, const int16_t* __restrict__ levels,
                  uint64_t n_levels, uint32_t epoch, uint32_t spin_limit, uint32_t* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ReconSmem& sm = *reinterpret_cast<ReconSmem*>(smem_raw);
  for (int i = threadIdx.x; i < 32 * 32; i += blockDim.x) sm.M.m32[i] = g_dct2_m[4][i];
  for (int i = threadIdx.x; i < 16 * 16; i += blockDim.x) sm.M.m16[i] = g_dct2_m[3][i];
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) sm.item = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t it = sm.item;
    if (it >= n_items) break;
    const CtuItem item = items[it];
    if (threadIdx.x < sizeof(DevPic) / 4)
      reinterpret_cast<uint32_t*>(&sm.P)[threadIdx.x] =
          reinterpret_cast<const uint32_t*>(&pics[item.pic])[threadIdx.x];
    __syncthreads();
    const DevPic& P = sm.P;
    const int cx = item.cx, cy = item.cy;
    const int sh = P.ctu_log2 - ilog2(P.tb);
    const int ncu = 1 << (2 * sh);
    for (int k = 0; k < ncu; k++) {
      int lx = 0, ly = 0;
      for (int b = 0; b < sh; b++) {
        lx |= ((k >> (2 * b)) & 1) << b;
        ly |= ((k >> (2 * b + 1)) & 1) << b;
      }
      const int gx = (cx << sh) + lx, gy = (cy << sh) + ly;
      const vvcg_cu_rec rec = P.cus[gy * P.grid_w + gx];
      cu_residuals(P, rec, levels, n_levels, status, sm);
      if (k == 0) {
        if (threadIdx.x == 0) {
          // Once any wait has given up the batch result is void: skip further
          // waits so the kernel drains in bounded time.
          bool ok = (ld_acquire(status) & kStatusTimeout) == 0;
          if (ok && cx > 0) ok = wait_flag(&P.ctu_done[cy * P.ctu_w + cx - 1], epoch, spin_limit);
          if (ok && cy > 0) {
            int tx = cx + 1 < P.ctu_w ? cx + 1 : cx;
            ok = wait_flag(&P.ctu_done[(cy - 1) * P.ctu_w + tx], epoch, spin_limit);
          }
          if (!ok) atomicOr(status, kStatusTimeout);
          sm.timed_out = !ok;
        }
        __syncthreads();
      }
      const int bx = gx * P.tb, by = gy * P.tb;
      const uint32_t order = cu_order(P, gx, gy);
      // luma
      const int lm = rec.luma_mode <= 69 ? rec.luma_mode : 0;
      gather_refs(P, 0, bx, by, P.tb, P.tb, true, order, sm.S);
      predict_intra(P.tb, P.tb, true, lm, P.bd, sm.S, sm.pred);
      store_block(P, 0, bx, by, P.tb, P.tb, sm.pred, sm.res[0]);
      __syncthreads();
      if (P.cf) {
        const int cxp = bx / P.sub_w, cyp = by / P.sub_h;
        const int chm = rec.chroma_mode;
        for (int c = 1; c <= 2; c++) {
          if (chm >= 81 && chm <= 83) {
            predict_cclm(P, c, cxp, cyp, P.tb_cw, P.tb_ch, chm - 81, sm.S, sm.pred);
          } else {
            gather_refs(P, c, cxp, cyp, P.tb_cw, P.tb_ch, true, order, sm.S);
            predict_intra(P.tb_cw, P.tb_ch, false, chm <= 69 ? chm : 0, P.bd, sm.S, sm.pred);
          }
          store_block(P, c, cxp, cyp, P.tb_cw, P.tb_ch, sm.pred, sm.res[c]);
          __syncthreads();
        }
      }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) st_release(&P.ctu_done[cy * P.ctu_w + cx], epoch);
  }
}

}  // namespace vvcg
