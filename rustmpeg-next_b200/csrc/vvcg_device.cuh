// Device-side data layout and helpers shared by the reconstruction and
// loop-filter kernels of libvvcg (sm_100a).
#pragma once
#include <stdint.h>

#include "../../include/vvcg.h"

namespace vvcg {

// Status word bits written by kernels (read back by vvcg_batch_sync).
enum : uint32_t {
  kStatusTimeout = 1u << 0,      // a wavefront wait ran out of polls
  kStatusBadRecord = 1u << 1,    // a record or level offset was out of range
  kStatusAlfAbort = 1u << 2,     // fixed-filter ALF reached class >= 16 (the reference aborts)
  kStatusSaoAbort = 1u << 3,     // SAO edge class 3 on the first/last row (the reference aborts)
};

// One picture as the kernels see it (built on the host, copied to HBM).
struct DevPic {
  uint16_t* plane[3];       // coded-size reconstructed planes (Y, Cb, Cr)
  uint16_t* scratch[3];     // same-size planes for the pre-SAO / pre-ALF copies
  int32_t stride[3];        // samples
  int32_t pw[3], ph[3];     // plane widths / heights
  const vvcg_cu_rec* cus;   // the picture's records, tb-grid raster order
  const vvcg_ctu_filter* ctus;
  uint64_t* row_done;       // per CTU row: (epoch << 32) | CTUs finished; 128-byte stride
  int32_t bd, cf, ctu_log2, ctu, tb, tb_cw, tb_ch, sub_w, sub_h;
  int32_t grid_w, grid_h, ctu_w, ctu_h;
  int32_t lqp, cqp, slice_qp, tools, aps;
  // encoder: level pool and the picture's first slot in it (one slot of
  // tb*tb + 2*tb_cw*tb_ch levels per CU, raster order)
  int16_t* lv_pool;
  int32_t lv_base;
};

// Work item of the wavefront: one CTU row of a picture.
struct RowItem {
  uint32_t pic;
  uint32_t cy;
};

constexpr int kRowFlagStride = 16;  // uint64 per row flag: one 128-byte line each

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ int ilog2(int v) { return __ffs(v) - 1; }
__device__ __forceinline__ int floor_log2(unsigned v) { return 31 - __clz(v); }
__device__ __forceinline__ int clip16(long long v) {
  return (int)(v < -32768 ? -32768 : (v > 32767 ? 32767 : v));
}
__device__ __forceinline__ int clip16i(int v) { return v < -32768 ? -32768 : (v > 32767 ? 32767 : v); }

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_relaxed64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release64(uint64_t* p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

}  // namespace vvcg
