// Tensor-memory-accelerator (TMA) staging of sample tiles: 2-D tiled
// cp.async.bulk.tensor loads from a plane in this GPU's own memory into shared
// memory, completed on an mbarrier as transaction bytes. No cluster
// multicast: every CTA fetches its own tile.
//
// A tensor map describes one 16-bit plane (width x height samples, row pitch
// in bytes) and the box a load copies. The copy's x coordinate times 2 bytes
// must be a multiple of 16 (x a multiple of 8 samples); callers only issue
// boxes that lie inside the plane, so no fill value is ever read.
#pragma once
#include <cuda.h>  // CUtensorMap and its enums; the encoder is fetched from the driver at run time
#include <stdint.h>

#include "umma.cuh"

namespace vvcg {

__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes)
               : "memory");
}

// Makes mbarrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Box of `map` whose first element is (x, y) -> shared memory at dst (128-byte
// aligned); completes `bytes` transaction bytes on mbar.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(mbar))
      : "memory");
}

// Orders this thread's tensor-map reads after the map's last generic-proxy
// write (the host's copy of the map into device memory).
__device__ __forceinline__ void tma_acquire_map(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
               : "memory");
}

}  // namespace vvcg
