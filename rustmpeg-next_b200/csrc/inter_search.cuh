// Motion estimation of the reference encoders' hook estimate_inter_block
// (crates/rustmpeg-video/src/vvc/inter.rs:1866-2003) on 8-bit luma planes,
// one CTA per block. Each trial (a merge candidate, a diamond or a
// quarter-sample vector) is scored by luma SAD: every thread forms the
// prediction of its samples directly from the reference (the 8-tap filters of
// interpolate_luma_block, inter.rs:896-1051, with its intermediate rounding;
// bi-prediction through weighted_average_bi, inter.rs:1189-1201) and the CTA
// sums the absolute differences. The search order and its tie rules follow
// the reference: every decision is taken from CTA-wide sums, so all threads
// take the same path.
#pragma once
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

constexpr int kMeThreads = 128;
constexpr int kMeMaxRefs = 16;

struct MeArgs {
  const uint8_t* src;
  int64_t stride;
  int32_t width, height;
  const uint8_t* l0[kMeMaxRefs];
  const uint8_t* l1[kMeMaxRefs];
  int32_t n0, n1;
  const vvcg_mv_cand* cands;
  const vvcg_me_req* reqs;
  int32_t n;
  vvcg_me_res* res;
};

// sample (x, y) of a reference, coordinates clamped to the plane (get_p)
__device__ __forceinline__ int me_px(const MeArgs& A, const uint8_t* r, int x, int y) {
  return __ldg(&r[(int64_t)clampi(y, 0, A.height - 1) * A.stride + clampi(x, 0, A.width - 1)]);
}

__device__ __forceinline__ int me_tap(int frac, int k, bool alt) {
  return (alt && frac == 8) ? c_luma_alt_hpel[k] : (int)c_luma_taps8[frac * 8 + k];
}

// interpolate_luma_block (8-bit) at block sample (X, Y): the final sample
// (bi false) or the 14-bit intermediate minus 2^13 (bi true)
__device__ int me_interp(const MeArgs& A, const uint8_t* r, int X, int Y, int mvx, int mvy, bool bi, bool alt) {
  constexpr int head = 6, offs = 1 << 13;
  const int ix = X + (mvx >> 4), iy = Y + (mvy >> 4), fx = mvx & 15, fy = mvy & 15;
  if (fx == 0 && fy == 0) {
    const int s = me_px(A, r, ix, iy);
    return bi ? (s << head) - offs : s;
  }
  if (fy == 0 || fx == 0) {
    const int f = fy == 0 ? fx : fy;
    int s = 0;
    for (int k = 0; k < 8; k++)
      s += (fy == 0 ? me_px(A, r, ix - 3 + k, iy) : me_px(A, r, ix, iy - 3 + k)) * me_tap(f, k, alt);
    return bi ? s - offs : clampi((s + 32) >> 6, 0, 255);
  }
  int s = 0;
  for (int j = 0; j < 8; j++) {
    int t = 0;
    for (int k = 0; k < 8; k++) t += me_px(A, r, ix - 3 + k, iy - 3 + j) * me_tap(fx, k, alt);
    s += (t - offs) * me_tap(fy, j, alt);
  }
  return bi ? s >> 6 : clampi((s + (1 << 11) + (offs << 6)) >> 12, 0, 255);
}

// predict_inter_pu's luma sample (inter.rs:1733-1847; BDOF and DMVR off)
__device__ int me_pred(const MeArgs& A, const vvcg_mv_cand& c, int X, int Y) {
  const bool has0 = (c.inter_dir & 1) && c.ref_idx[0] >= 0 && A.n0 > 0;
  const bool has1 = (c.inter_dir & 2) && c.ref_idx[1] >= 0 && A.n1 > 0;
  const bool alt = c.alt_hpel != 0;
  if (has0 && has1) {
    const int p0 = me_interp(A, A.l0[min((int)c.ref_idx[0], A.n0 - 1)], X, Y, c.mv[0][0], c.mv[0][1], true, alt);
    const int p1 = me_interp(A, A.l1[min((int)c.ref_idx[1], A.n1 - 1)], X, Y, c.mv[1][0], c.mv[1][1], true, alt);
    const int w1 = c_bcw_weights[min((int)c.bcw_idx, 4)];
    return clampi((p0 * (8 - w1) + p1 * w1 + (1 << 8) + ((1 << 13) << 3)) >> 9, 0, 255);
  }
  if (has0) return me_interp(A, A.l0[min((int)c.ref_idx[0], A.n0 - 1)], X, Y, c.mv[0][0], c.mv[0][1], false, alt);
  if (has1) return me_interp(A, A.l1[min((int)c.ref_idx[1], A.n1 - 1)], X, Y, c.mv[1][0], c.mv[1][1], false, alt);
  return 128;
}

// CTA-wide sum (every thread returns it); red: kMeThreads / 32 words of shared memory
__device__ uint64_t me_cta_sum(uint64_t v, uint64_t* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  uint64_t t = 0;
#pragma unroll
  for (int w = 0; w < kMeThreads / 32; w++) t += red[w];
  __syncthreads();
  return t;
}

// luma SAD of the block against pred(X, Y)
template <class F>
__device__ uint64_t me_sad(const MeArgs& A, const vvcg_me_req& q, uint64_t* red, F&& pred) {
  uint64_t s = 0;
  for (int i = threadIdx.x; i < (int)q.w * q.h; i += kMeThreads) {
    const int X = (int)q.x + i % q.w, Y = (int)q.y + i / q.w;
    s += (uint64_t)abs((int)__ldg(&A.src[(int64_t)Y * A.stride + X]) - pred(X, Y));
  }
  return me_cta_sum(s, red);
}

__global__ void __launch_bounds__(kMeThreads) k_inter_search_8(MeArgs A) {
  __shared__ uint64_t red[kMeThreads / 32];
  for (int r = blockIdx.x; r < A.n; r += gridDim.x) {
    const vvcg_me_req q = A.reqs[r];
    // merge list (first lowest SAD wins); InterMergeCand::default without one
    vvcg_mv_cand best_merge{};
    best_merge.inter_dir = 1;
    best_merge.ref_idx[0] = 0;
    best_merge.ref_idx[1] = -1;
    best_merge.bcw_idx = 2;
    if (q.num_cands) best_merge = A.cands[q.cand_off];
    uint64_t best_merge_sad = ~0ull;
    int best_idx = 0;
    for (int i = 0; i < q.num_cands; i++) {
      const vvcg_mv_cand c = A.cands[q.cand_off + i];
      const uint64_t s = me_sad(A, q, red, [&](int X, int Y) { return me_pred(A, c, X, Y); });
      if (s < best_merge_sad) {
        best_merge_sad = s;
        best_idx = i;
        best_merge = c;
      }
    }
    vvcg_me_res out{};
    out.cand = best_merge;
    out.is_merge = 1;
    out.merge_idx = (uint16_t)best_idx;
    out.sad = best_merge_sad;
    if (A.n0 > 0) {
      const uint8_t* r0 = A.l0[0];
      auto sad_at = [&](int mx, int my) {
        return me_sad(A, q, red, [&](int X, int Y) { return me_interp(A, r0, X, Y, mx, my, false, false); });
      };
      // integer diamond around the AMVP predictor
      int bmx = (q.amvp[0] >> 4) * 16, bmy = (q.amvp[1] >> 4) * 16;
      uint64_t best = sad_at(bmx, bmy);
      const int rounds = max((int)q.search_range, 1);
      for (int it = 0; it < rounds; it++) {
        const int cx = bmx >> 4, cy = bmy >> 4;
        bool improved = false;
        for (int k = 0; k < 4; k++) {
          const int tx = (cx + (k == 0 ? 1 : k == 1 ? -1 : 0)) * 16;
          const int ty = (cy + (k == 2 ? 1 : k == 3 ? -1 : 0)) * 16;
          const uint64_t s = sad_at(tx, ty);
          if (s < best) {
            best = s;
            bmx = tx;
            bmy = ty;
            improved = true;
          }
        }
        if (!improved) break;
      }
      // quarter-sample refinement around the integer result
      const int ix = bmx, iy = bmy;
      for (int k = 0; k < 4; k++) {
        const int tx = ix + (k == 0 ? 4 : k == 1 ? -4 : 0), ty = iy + (k == 2 ? 4 : k == 3 ? -4 : 0);
        const uint64_t s = sad_at(tx, ty);
        if (s < best) {
          best = s;
          bmx = tx;
          bmy = ty;
        }
      }
      if (!(best_merge_sad <= best)) {
        vvcg_mv_cand c{};
        c.inter_dir = 1;
        c.mv[0][0] = bmx;
        c.mv[0][1] = bmy;
        c.ref_idx[0] = 0;
        c.ref_idx[1] = -1;
        c.bcw_idx = 2;
        out.cand = c;
        out.is_merge = 0;
        out.merge_idx = 0;
        out.sad = best;
      }
    }
    if (threadIdx.x == 0) A.res[r] = out;
  }
}

}  // namespace vvcg
