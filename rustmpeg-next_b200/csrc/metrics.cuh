// Plane distortion metrics (SSE, SAD, sample count) of libvvcg (sm_100a):
// CpuFrameMetrics::plane_metrics (crates/rustmpeg-video/src/accelerator.rs:258-292)
// for 8-bit planes, and the same sums for the library's 16-bit planes.
// Integer sums are order independent, so the result is exact and
// deterministic whatever the grid.
#pragma once
#include <stdint.h>

namespace vvcg {

// Grid-stride over rows; each thread takes 16-byte chunks of a row (scalar
// tail), a block reduction, one 64-bit atomic per block and quantity.
// out[0] += SSE, out[1] += SAD.
template <typename T>
__global__ void __launch_bounds__(256) k_plane_metrics(const T* __restrict__ a, uint64_t sa,
                                                      const T* __restrict__ b, uint64_t sb, uint32_t w,
                                                      uint32_t h, unsigned long long* out) {
  constexpr int kPer = 16 / sizeof(T);  // samples per 16-byte chunk
  unsigned long long sse = 0, sad = 0;
  const uint32_t chunks = w / kPer;
  const bool vec = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15) == 0 &&
                   ((sa | sb) * sizeof(T)) % 16 == 0;
  const uint64_t total = (uint64_t)h * (vec ? chunks : 0);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t y = (uint32_t)(i / chunks), c = (uint32_t)(i % chunks);
    const uint4 va = *reinterpret_cast<const uint4*>(a + y * sa + (uint64_t)c * kPer);
    const uint4 vb = *reinterpret_cast<const uint4*>(b + y * sb + (uint64_t)c * kPer);
    const T* pa = reinterpret_cast<const T*>(&va);
    const T* pb = reinterpret_cast<const T*>(&vb);
    uint32_t s2 = 0, s1 = 0;  // a chunk's sums fit in 32 bits
#pragma unroll
    for (int k = 0; k < kPer; k++) {
      const uint32_t d = (uint32_t)abs((int)pa[k] - (int)pb[k]);
      s2 += d * d;
      s1 += d;
    }
    sse += s2;
    sad += s1;
  }
  // scalar part: the whole plane when unaligned, else the tail of each row
  const uint32_t x0 = vec ? chunks * kPer : 0, tail = w - x0;
  const uint64_t ntail = (uint64_t)h * tail;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ntail;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t y = (uint32_t)(i / tail), x = x0 + (uint32_t)(i % tail);
    const uint64_t d = (uint64_t)abs((int)a[y * sa + x] - (int)b[y * sb + x]);
    sse += d * d;
    sad += d;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sse += __shfl_xor_sync(0xffffffffu, sse, o);
    sad += __shfl_xor_sync(0xffffffffu, sad, o);
  }
  __shared__ unsigned long long s_sse[8], s_sad[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    s_sse[wid] = sse;
    s_sad[wid] = sad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t2 = 0, t1 = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
      t2 += s_sse[i];
      t1 += s_sad[i];
    }
    atomicAdd(&out[0], t2);
    atomicAdd(&out[1], t1);
  }
}

}  // namespace vvcg
