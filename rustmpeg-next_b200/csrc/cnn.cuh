// The CNN pruner of the GPU encoder: 32x32 luma blocks (samples / max value,
// rounded to bf16) -> conv 3x3 1->32 + ReLU -> 3 x (conv 3x3 32->32 + ReLU)
// -> global average -> 67 intra-mode logits and 6 split logits.
//
// Forward: one CTA per block (persistent over blocks). The block's
// activations stay in shared memory as two ping-pong images of 34 x 34
// pixels (a zero halo around 32 x 32) in four planes of 8 channels, 16 bytes
// per pixel, so each layer's 3x3 convolution is 144 tcgen05 MMAs
// (M = 128 pixels, N = 32 output channels, K = 16 input channels of one tap)
// whose A operand points straight into the image: the 8 rows of a core
// matrix are 8 neighbouring pixels of an image row (16 B apart), SBO steps
// one image row, LBO one channel plane, and a tap is an address offset. The
// 8 tiles of a layer accumulate in 256 TMEM columns; 8 warps read them back,
// add the bias, apply ReLU and write the next image (or the average).
// The first layer (one input channel) runs on the CUDA cores.
#pragma once
#include "umma.cuh"

namespace vvcg {

constexpr int kCnnCh = 32, kCnnModes = 67, kCnnSplits = 6, kCnnOut = kCnnModes + kCnnSplits;
constexpr int kCnnConvW = kCnnCh * kCnnCh * 9;  // 9216
// fp32 parameter vector: W1 [co][tap], b1, then per layer 2..4 W [co][ci][tap]
// and b, then the heads W [out][ch] and b.
constexpr int kOffW1 = 0, kOffB1 = 288;
__host__ __device__ constexpr int cnn_off_w(int layer) { return 320 + (layer - 2) * (kCnnConvW + kCnnCh); }
__host__ __device__ constexpr int cnn_off_b(int layer) { return cnn_off_w(layer) + kCnnConvW; }
constexpr int kOffWi = cnn_off_w(5), kOffBi = kOffWi + kCnnModes * kCnnCh;
constexpr int kOffWs = kOffBi + kCnnModes, kOffBs = kOffWs + kCnnSplits * kCnnCh;
constexpr int kCnnParams = kOffBs + kCnnSplits;  // 30473

constexpr int kImgW = 34;                 // 32 + halo
constexpr int kPlane = kImgW * kImgW * 16;  // one plane of 8 channels, bytes
constexpr int kImg = 4 * kPlane;            // 73984
constexpr int kPackL = 36 * 32 * 16;        // packed bf16 weights of one layer: [tap*4 + ci/8][co][ci%8]
constexpr int kCnnThreads = 256;
constexpr uint32_t kCnnIdesc = umma_idesc_bf16(128, 32);
constexpr int kCnnMisc = (288 + 32 + 96 + 8 * 32 + 1024 + 32) * 4;
constexpr int kCnnSmem = 2 * kImg + 3 * kPackL + kCnnMisc + 64;

__device__ __forceinline__ uint16_t f2bf(float f) {  // round to nearest even
  const uint32_t u = __float_as_uint(f);
  return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}
__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// pack[layer][tap*4 + ci/8][co][ci%8] = bf16(W[co][ci][tap]) (forward), or with
// flip the weights of the transposed convolution: [tap*4 + co/8][ci][co%8] =
// bf16(W[co][ci][8 - tap]).
__global__ void k_cnn_pack(const float* __restrict__ params, uint16_t* __restrict__ pack, bool flip) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * kCnnConvW) return;
  const int l = i / kCnnConvW, r = i % kCnnConvW;
  const int kg = r / 256, n = (r / 8) % 32, j = r % 8;
  const int tap = kg / 4, g = kg % 4;
  const float* W = params + cnn_off_w(2 + l);
  float v;
  if (!flip)
    v = W[(n * kCnnCh + g * 8 + j) * 9 + tap];  // n = co, input channel g*8+j
  else
    v = W[((g * 8 + j) * kCnnCh + n) * 9 + (8 - tap)];  // n = ci, output channel g*8+j
  pack[i] = f2bf(v);
}

struct CnnFwdArgs {
  const uint16_t* plane;
  int64_t stride;
  int32_t width, height, maxv, n;
  const uint32_t* ctu_xy;  // n (x, y) pairs
  const float* params;
  const uint16_t* pack;
  float* logits;     // n x 73
  float* gap_out;    // n x 32, or null
  uint16_t* acts;    // n x 4 x 1024 x 32 bf16 (layer, pixel, channel), or null
  uint32_t* status;  // bit 0: a completion wait gave up; bit 1: a block outside the plane
};

// Issues the 144 MMAs of one 3x3 32->32 layer reading image `xin` with the
// packed weights `w` into TMEM columns tile * 32, then commits to mbar.
__device__ __forceinline__ void cnn_issue_layer(uint32_t tmem, uint32_t xin, uint32_t w, uint64_t* mbar) {
  for (int tile = 0; tile < 8; tile++) {
    const int xg = tile & 3, yh = tile >> 2;
    for (int tap = 0; tap < 9; tap++) {
      const int dy = tap / 3, dx = tap % 3;
      for (int h = 0; h < 2; h++) {
        const uint32_t a = xin + 2 * h * kPlane + ((16 * yh + dy) * kImgW + 8 * xg + dx) * 16;
        const uint32_t b = w + (tap * 4 + 2 * h) * 32 * 16;
        umma_bf16(tmem + tile * 32, umma_desc(a, kPlane, kImgW * 16), umma_desc(b, 512, 128), kCnnIdesc,
                  (tap | h) != 0);
      }
    }
  }
  umma_commit(mbar);
}

__global__ void __launch_bounds__(kCnnThreads, 1) k_cnn_forward(const __grid_constant__ CnnFwdArgs A) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* X0 = smem;
  uint8_t* X1 = smem + kImg;
  uint8_t* W = smem + 2 * kImg;
  float* w1 = (float*)(W + 3 * kPackL);
  float* b1 = w1 + 288;
  float* bias = b1 + 32;   // [3][32]
  float* gpart = bias + 96;  // [8 warps][32]
  float* xin = gpart + 256;  // 32 x 32 input
  float* gap = xin + 1024;   // [32]
  uint64_t* mbar = (uint64_t*)(gap + 32);
  uint32_t* tslot = (uint32_t*)(mbar + 1);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;

  // weights, zero images (the halos stay zero), TMEM, barrier
  for (int i = t; i < 3 * kPackL / 16; i += kCnnThreads) ((uint4*)W)[i] = ((const uint4*)A.pack)[i];
  for (int i = t; i < 2 * kImg / 16; i += kCnnThreads) ((uint4*)X0)[i] = make_uint4(0, 0, 0, 0);
  for (int i = t; i < 288; i += kCnnThreads) w1[i] = A.params[kOffW1 + i];
  if (t < 32) b1[t] = A.params[kOffB1 + t];
  if (t < 96) bias[t] = A.params[cnn_off_b(2 + t / 32) + t % 32];
  if (warp == 0) {
    tmem_alloc(tslot, 256);
    tmem_relinquish();
  }
  if (t == 0) {
    mbar_init(mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  uint32_t phase = 0;
  bool ok = true;

  for (int blk = blockIdx.x; blk < A.n && ok; blk += gridDim.x) {
    const uint32_t ux = A.ctu_xy[2 * blk], uy = A.ctu_xy[2 * blk + 1];
    if (ux > (uint32_t)A.width - 32 || uy > (uint32_t)A.height - 32 || A.width < 32 || A.height < 32) {
      // a block outside the plane: NaN logits, flagged, nothing read
      if (t < kCnnOut) A.logits[(size_t)blk * kCnnOut + t] = __int_as_float(0x7FC00000);
      if (t == 0) atomicOr(A.status, 2u);
      continue;
    }
    const int bx = (int)ux, by = (int)uy;
    const float inv = 1.0f / (float)A.maxv;
    for (int i = t; i < 1024; i += kCnnThreads)
      xin[i] = bf2f(f2bf((float)A.plane[(int64_t)(by + (i >> 5)) * A.stride + bx + (i & 31)] * inv));
    __syncthreads();
    // layer 1 on the CUDA cores: 4 pixels per thread
    for (int p = t; p < 1024; p += kCnnThreads) {
      const int iy = p >> 5, ix = p & 31;
      float in[9];
#pragma unroll
      for (int tap = 0; tap < 9; tap++) {
        const int y = iy + tap / 3 - 1, x = ix + tap % 3 - 1;
        in[tap] = (y >= 0 && y < 32 && x >= 0 && x < 32) ? xin[y * 32 + x] : 0.0f;
      }
      uint32_t pk[16];
#pragma unroll
      for (int c = 0; c < 32; c += 2) {
        float s0 = b1[c], s1 = b1[c + 1];
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
          s0 = fmaf(w1[c * 9 + tap], in[tap], s0);
          s1 = fmaf(w1[(c + 1) * 9 + tap], in[tap], s1);
        }
        pk[c / 2] = (uint32_t)f2bf(fmaxf(s0, 0.0f)) | ((uint32_t)f2bf(fmaxf(s1, 0.0f)) << 16);
      }
      const int off = ((iy + 1) * kImgW + ix + 1) * 16;
#pragma unroll
      for (int g = 0; g < 4; g++)
        *(uint4*)(X0 + g * kPlane + off) = make_uint4(pk[4 * g], pk[4 * g + 1], pk[4 * g + 2], pk[4 * g + 3]);
      if (A.acts) {
        uint4* dst = (uint4*)(A.acts + (((size_t)blk * 4 + 0) * 1024 + p) * 32);
#pragma unroll
        for (int g = 0; g < 4; g++) dst[g] = make_uint4(pk[4 * g], pk[4 * g + 1], pk[4 * g + 2], pk[4 * g + 3]);
      }
    }
    float acc[32];
#pragma unroll
    for (int c = 0; c < 32; c++) acc[c] = 0.0f;
    for (int l = 0; l < 3 && ok; l++) {
      uint8_t* xi = (l & 1) ? X1 : X0;
      uint8_t* xo = (l & 1) ? X0 : X1;
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      if (t == 0) cnn_issue_layer(tmem, smem_u32(xi), smem_u32(W) + l * kPackL, mbar);
      ok = __syncthreads_and(mbar_wait(mbar, phase, 1u << 26));
      phase ^= 1;
      tc_fence_after();
      if (!ok) break;
      const int q = warp & 3;
      for (int k = 0; k < 4; k++) {
        const int tile = (warp >> 2) + 2 * k;
        const int m = 32 * q + lane, j = m >> 3, r = m & 7;
        const int iy = 16 * (tile >> 2) + j, ix = 8 * (tile & 3) + r;
        float v[32];
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + tile * 32, v);
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + tile * 32 + 16, v + 16);
#pragma unroll
        for (int c = 0; c < 32; c++) v[c] = fmaxf(v[c] + bias[l * 32 + c], 0.0f);
        if (l < 2 || A.acts) {
          uint32_t pk[16];
#pragma unroll
          for (int c = 0; c < 32; c += 2) pk[c / 2] = (uint32_t)f2bf(v[c]) | ((uint32_t)f2bf(v[c + 1]) << 16);
          if (l < 2) {
            const int off = ((iy + 1) * kImgW + ix + 1) * 16;
#pragma unroll
            for (int g = 0; g < 4; g++)
              *(uint4*)(xo + g * kPlane + off) = make_uint4(pk[4 * g], pk[4 * g + 1], pk[4 * g + 2], pk[4 * g + 3]);
          }
          if (A.acts) {
            uint4* dst = (uint4*)(A.acts + (((size_t)blk * 4 + l + 1) * 1024 + iy * 32 + ix) * 32);
#pragma unroll
            for (int g = 0; g < 4; g++) dst[g] = make_uint4(pk[4 * g], pk[4 * g + 1], pk[4 * g + 2], pk[4 * g + 3]);
          }
        }
        if (l == 2) {
#pragma unroll
          for (int c = 0; c < 32; c++) acc[c] += v[c];
        }
      }
    }
    if (!ok) break;
    // global average: the warp's 128 pixels, then the 8 warps
#pragma unroll
    for (int c = 0; c < 32; c++) {
      float s = acc[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
      if (lane == 0) gpart[warp * 32 + c] = s;
    }
    tc_fence_before();
    __syncthreads();
    if (t < 32) {
      float s = 0.0f;
      for (int w = 0; w < 8; w++) s += gpart[w * 32 + t];
      gap[t] = s * (1.0f / 1024.0f);
      if (A.gap_out) A.gap_out[(size_t)blk * 32 + t] = gap[t];
    }
    __syncthreads();
    if (t < kCnnOut) {
      const float* Wh = t < kCnnModes ? A.params + kOffWi + t * 32 : A.params + kOffWs + (t - kCnnModes) * 32;
      float s = t < kCnnModes ? A.params[kOffBi + t] : A.params[kOffBs + t - kCnnModes];
      for (int c = 0; c < 32; c++) s = fmaf(Wh[c], gap[c], s);
      A.logits[(size_t)blk * kCnnOut + t] = s;
    }
  }
  if (!ok && t == 0) atomicOr(A.status, 1u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

}  // namespace vvcg
