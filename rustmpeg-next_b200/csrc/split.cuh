// Quadrant-mean partition decision of the reference encoders' split hook,
// choose_qt_mtt_partition_rdo_16 / choose_qt_mtt_partition_rdo
// (crates/rustmpeg-video/src/vvc/slice.rs:4111-4167), one warp per region.
// Samples are rounded to 8 bits as Plane16::to_plane_8bit does
// (predict.rs:2914-2926); a quadrant's mean is its sum over the samples
// inside the plane divided by the full quadrant area (integer division).
#pragma once
#include "vvcg_device.cuh"

namespace vvcg {

constexpr int kSplitWarps = 8;

struct SplitArgs {
  const uint16_t* plane;
  int64_t stride;
  int32_t width, height, bd, n;
  const vvcg_split_req* reqs;
  uint8_t* res;
};

// Sum of the 8-bit-rounded samples of the quadrant (qx, qy, qw, qh) that lie
// inside the plane, reduced over the warp (every lane returns it).
__device__ uint64_t split_quad_sum(const SplitArgs& A, int64_t qx, int64_t qy, int64_t qw, int64_t qh) {
  const int lane = threadIdx.x & 31;
  const int shift = A.bd - 8;
  const uint32_t add = shift > 0 ? 1u << (shift - 1) : 0u;
  const int64_t cw = min(qx + qw, (int64_t)A.width) - qx, ch = min(qy + qh, (int64_t)A.height) - qy;
  uint64_t s = 0;
  if (cw > 0 && ch > 0)
    for (int64_t i = lane; i < cw * ch; i += 32) {
      const int64_t y = qy + i / cw, x = qx + i % cw;
      const uint32_t v = min((uint32_t)__ldg(&A.plane[y * A.stride + x]) + add, 65535u) >> shift;
      s += min(v, 255u);
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

__global__ void __launch_bounds__(kSplitWarps * 32) k_qt_mtt_split(SplitArgs A) {
  const int lane = threadIdx.x & 31;
  for (int r = blockIdx.x * kSplitWarps + (threadIdx.x >> 5); r < A.n; r += gridDim.x * kSplitWarps) {
    const vvcg_split_req q = A.reqs[r];
    const int64_t w = q.w, h = q.h, lim = max((int64_t)q.min_cb, (int64_t)8);
    uint8_t out = VVCG_SPLIT_NONE;
    if (w > lim && h > lim) {
      const int64_t hw = w / 2, hh = h / 2, area = max(hw * hh, (int64_t)1);
      const int64_t x = q.x, y = q.y;
      const int64_t m00 = (int64_t)(split_quad_sum(A, x, y, hw, hh) / (uint64_t)area);
      const int64_t m10 = (int64_t)(split_quad_sum(A, x + hw, y, hw, hh) / (uint64_t)area);
      const int64_t m01 = (int64_t)(split_quad_sum(A, x, y + hh, hw, hh) / (uint64_t)area);
      const int64_t m11 = (int64_t)(split_quad_sum(A, x + hw, y + hh, hw, hh) / (uint64_t)area);
      const int64_t hor = llabs(m00 - m01) + llabs(m10 - m11);
      const int64_t ver = llabs(m00 - m10) + llabs(m01 - m11);
      const int64_t thr = max((int)q.qp, 4) / 2 + 8;
      if (w == h && hor > thr && ver > thr)
        out = VVCG_SPLIT_QT;
      else if (hor > ver && hor > thr)
        out = VVCG_SPLIT_BT_H;
      else if (ver > thr)
        out = VVCG_SPLIT_BT_V;
    }
    if (lane == 0) A.res[r] = out;
  }
}

}  // namespace vvcg
