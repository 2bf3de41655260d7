// Blackwell (sm_100a) tensor-core plumbing: shared-memory matrix descriptors,
// the kind::f16 instruction descriptor, TMEM allocation, tcgen05.mma issue /
// commit, bounded mbarrier waits and tcgen05.ld, as inline PTX.
//
// Operands are K-major without swizzle ("interleaved"): a core matrix is 8
// rows x 16 bytes stored contiguously (128 B); SBO is the byte distance
// between core matrices adjacent in M (or N), LBO between the two core
// matrices of one instruction's K = 16 (bf16). D is fp32 in TMEM: row m of an
// M = 128 tile is TMEM lane m, column n is TMEM column (base + n).
#pragma once
#include <stdint.h>

namespace vvcg {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// SM100 shared-memory descriptor: start >> 4 in [0,14), LBO >> 4 in [16,30),
// SBO >> 4 in [32,46), version 1 in [46,48), layout type 0 (no swizzle).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: fp32 D, bf16 A and B, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// D (+)= A * B^T for one M x N x 16 step; issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"((uint32_t)accumulate));
}

// The mbarrier gets one arrival when every MMA this thread issued so far is done.
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar)));
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count));
}

// Waits for the phase with the given parity to complete; gives up after
// max_polls polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t max_polls) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t i = 0; i < max_polls; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 lanes x 16 columns of fp32 from TMEM (lane = the warp's quarter).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// ---- self-test: one 128 x 32 x 16 bf16 MMA ---------------------------------

// A (128 x 16) and B (32 x 16) row-major bf16 in global memory, D (128 x 32)
// fp32 out. status[0] is set to 1 when the completion wait gave up.
__global__ void __launch_bounds__(128) k_umma_selftest(const uint16_t* a, const uint16_t* b, float* d,
                                                       uint32_t* status) {
  __shared__ __align__(128) uint16_t sa[128 * 16];
  __shared__ __align__(128) uint16_t sb[32 * 16];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  // canonical K-major: (m, k) at (m / 8) * 128 + (k / 8) * LBO + (m % 8) * 16 + (k % 8) * 2 bytes,
  // LBO = rows * 16 (the second K half after all M core matrices)
  for (int i = t; i < 128 * 16; i += blockDim.x) {
    const int m = i / 16, k = i % 16;
    sa[((m >> 3) * 128 + (k >> 3) * 2048 + (m & 7) * 16 + (k & 7) * 2) / 2] = a[i];
  }
  for (int i = t; i < 32 * 16; i += blockDim.x) {
    const int n = i / 16, k = i % 16;
    sb[((n >> 3) * 128 + (k >> 3) * 512 + (n & 7) * 16 + (k & 7) * 2) / 2] = b[i];
  }
  if (warp == 0) {
    tmem_alloc(&tbase, 32);
    tmem_relinquish();
  }
  if (t == 0) mbar_init(&mbar, 1);
  fence_async_smem();
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;
  if (t == 0) {
    umma_bf16(tmem, umma_desc(smem_u32(sa), 2048, 128), umma_desc(smem_u32(sb), 512, 128), umma_idesc_bf16(128, 32),
              false);
    umma_commit(&mbar);
  }
  const bool ok = __syncthreads_and(mbar_wait(&mbar, 0, 1u << 24));
  if (!ok && lane == 0) atomicExch(status, 1u);
  tc_fence_after();
  if (ok) {
    float v[16];
    for (int c = 0; c < 32; c += 16) {
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, v);
      for (int i = 0; i < 16; i++) d[(warp * 32 + lane) * 32 + c + i] = v[i];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 32);
}

}  // namespace vvcg
