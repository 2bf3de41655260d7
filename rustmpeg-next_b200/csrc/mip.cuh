// Matrix-based intra prediction (sm_100a): predict_mip_bd
// (crates/rustmpeg-video/src/vvc/predict.rs:2461-2611, through predict_mip_16
// :4109) and the SAD search over every (transposed, mode) pair of
// choose_best_mip_mode_16 (:4166-4199). One warp per block.
//
// The reference upsamples the reduced prediction in two separable passes
// (mip_prediction_upsampling_1d, :2393-2429): rows (uv - 1) + j * uv first,
// horizontally from the left boundary, then every column vertically from the
// top boundary. Each output sample here evaluates the same two linear
// interpolations directly: H(j, x) between the reduced row's neighbours (or
// left[(j + 1) * uv - 1]), then between H(j - 1, x) (or above[x]) and H(j, x).
#pragma once
#include <stdint.h>

#include "../../include/vvcg.h"
#include "vvcg_device.cuh"

namespace vvcg {

__device__ uint8_t g_mip4[16 * 16 * 4];   // [mode][output][input]
__device__ uint8_t g_mip8[8 * 16 * 8];
__device__ uint8_t g_mip16[6 * 64 * 7];

constexpr int kMipWarps = 4;

struct MipWs {
  int red[64];  // reduced prediction (after the transpose)
  int top[4], left[4];
};

__host__ __device__ __forceinline__ int mip_size_id(int w, int h) {
  return (w == 4 && h == 4) ? 0 : (w == 4 || h == 4 || (w == 8 && h == 8)) ? 1 : 2;
}
__host__ __device__ __forceinline__ int mip_num_modes(int w, int h) {
  const int s = mip_size_id(w, h);
  return s == 0 ? 16 : (s == 1 ? 8 : 6);
}

// Reduced boundaries (mip_boundary_downsampling_1d) of one block into W.top / W.left.
__device__ void mip_boundaries(const int16_t* above, const int16_t* left, int w, int h, MipWs& W, int lane) {
  const int rbs = mip_size_id(w, h) == 0 ? 2 : 4;
  if (lane < 2 * rbs) {
    const bool is_top = lane < rbs;
    const int d = is_top ? lane : lane - rbs;
    const int len = is_top ? w : h;
    const int16_t* src = is_top ? above : left;
    int v;
    if (rbs < len) {
      const int f = len / rbs, lf = __ffs(f) - 1;
      int s = 0;
      for (int k = 0; k < f; k++) s += src[d * f + k];
      v = (s + (1 << (lf - 1))) >> lf;
    } else {
      v = src[d];
    }
    if (is_top) W.top[d] = v; else W.left[d] = v;
  }
  __syncwarp();
}

// Reduced prediction of (mode, transposed) into W.red (transposed back).
__device__ void mip_reduced(int w, int h, int mode, bool tr, int bd, MipWs& W, int lane) {
  const int sid = mip_size_id(w, h);
  const int rbs = sid == 0 ? 2 : 4, rps = sid == 2 ? 8 : 4, np = rps * rps;
  int b[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    int v = 0;
    if (i < 2 * rbs) {
      const bool first = i < rbs;
      const int k = first ? i : i - rbs;
      v = (first != tr) ? W.top[k] : W.left[k];
    }
    b[i] = v;
  }
  const int in_off = b[0];
  const int centre = 1 << (bd - 1), maxv = (1 << bd) - 1;
  b[0] = sid != 2 ? centre - in_off : 0;
  int sum = b[0];
#pragma unroll
  for (int i = 1; i < 8; i++) {
    if (i < 2 * rbs) b[i] -= in_off;
    sum += i < 2 * rbs ? b[i] : 0;
  }
  const int offset = 32 - 32 * sum;
  const int m = mode % mip_num_modes(w, h);
  for (int pos = lane; pos < np; pos += 32) {
    int dot = 0;
    if (sid == 0) {
      const uint8_t* row = g_mip4 + (m * 16 + pos) * 4;
#pragma unroll
      for (int i = 0; i < 4; i++) dot += b[i] * (int)row[i];
    } else if (sid == 1) {
      const uint8_t* row = g_mip8 + (m * 16 + pos) * 8;
#pragma unroll
      for (int i = 0; i < 8; i++) dot += b[i] * (int)row[i];
    } else {
      const uint8_t* row = g_mip16 + (m * 64 + pos) * 7;
#pragma unroll
      for (int i = 0; i < 7; i++) dot += b[i + 1] * (int)row[i];
    }
    const int v = clampi(((dot + offset) >> 6) + in_off, 0, maxv);
    const int y = pos / rps, x = pos - y * rps;  // raw index pos = y * rps + x
    W.red[tr ? x * rps + y : pos] = v;
  }
  __syncwarp();
}

// Upsampled prediction sample (x, y).
__device__ __forceinline__ int mip_sample(const int16_t* above, const int16_t* left, int w, int h, const MipWs& W,
                                          int x, int y) {
  const int rps = mip_size_id(w, h) == 2 ? 8 : 4;
  const int uh = w / rps, uv = h / rps;
  const int luh = __ffs(uh) - 1, luv = __ffs(uv) - 1;
  auto H = [&](int j) -> int {  // horizontally upsampled row j at column x
    if (uh == 1) return W.red[j * rps + x];
    const int i = x >> luh, p = (x & (uh - 1)) + 1;
    const int before = i == 0 ? left[(j + 1) * uv - 1] : W.red[j * rps + i - 1];
    const int behind = W.red[j * rps + i];
    return (before * (uh - p) + behind * p + (uh >> 1)) >> luh;
  };
  if (uv == 1) return H(y);
  const int j = y >> luv, q = (y & (uv - 1)) + 1;
  const int before = j == 0 ? above[x] : H(j - 1);
  return (before * (uv - q) + H(j) * q + (uv >> 1)) >> luv;
}

// Grid: ceil(n / kMipWarps); warp per request.
__global__ void __launch_bounds__(kMipWarps * 32)
k_mip(const vvcg_mip_req* __restrict__ reqs, uint32_t n, const int16_t* __restrict__ refs,
      const int16_t* __restrict__ src, int16_t* __restrict__ pred, vvcg_mip_res* __restrict__ res) {
  __shared__ MipWs ws[kMipWarps];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t k = blockIdx.x * kMipWarps + wid;
  if (k >= n) return;
  MipWs& W = ws[wid];
  const vvcg_mip_req q = reqs[k];
  const int w = 1 << q.log2_w, h = 1 << q.log2_h, bd = clampi(q.bit_depth, 8, 12);
  const int16_t* above = refs + q.ref_off;
  const int16_t* left = above + w;
  int16_t* out = pred + q.out_off;
  mip_boundaries(above, left, w, h, W, lane);
  int mode = q.mode, tr = q.transposed;
  if (q.mode == VVCG_MIP_SEARCH) {
    const int16_t* s = src + q.out_off;
    unsigned long long best = ~0ull;
    const int nm = mip_num_modes(w, h);
    for (int t = 0; t < 2; t++)
      for (int m = 0; m < nm; m++) {
        mip_reduced(w, h, m, t != 0, bd, W, lane);
        unsigned sad = 0;  // <= 4096 * 4095
        for (int i = lane; i < w * h; i += 32) {
          const int y = i / w, x = i - y * w;
          sad += (unsigned)abs((int)(uint16_t)s[i] - mip_sample(above, left, w, h, W, x, y));
        }
        sad = __reduce_add_sync(0xffffffffu, sad);
        if (sad < best) {
          best = sad;
          mode = m;
          tr = t;
        }
        __syncwarp();
      }
    if (lane == 0) {
      vvcg_mip_res r;
      r.sad = best;
      r.mode = (uint8_t)mode;
      r.transposed = (uint8_t)tr;
      for (int i = 0; i < 6; i++) r.reserved[i] = 0;
      res[k] = r;
    }
  }
  mip_reduced(w, h, mode, tr != 0, bd, W, lane);
  for (int i = lane; i < w * h; i += 32) {
    const int y = i / w, x = i - y * w;
    out[i] = (int16_t)mip_sample(above, left, w, h, W, x, y);
  }
}

}  // namespace vvcg
