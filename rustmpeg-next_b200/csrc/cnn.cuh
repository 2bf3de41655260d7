// The CNN pruner of the GPU encoder: 32x32 luma blocks (samples / max value,
// rounded to bf16) with a second, constant input plane QP / 63 (the split
// decision depends on lambda) -> conv 3x3 2->32 + ReLU -> 3 x (conv 3x3
// 32->32 + ReLU) -> global average -> 67 intra-mode logits and 6 split logits.
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
// The first layer (two input channels) runs on the CUDA cores.
#pragma once
#include "umma.cuh"

namespace vvcg {

constexpr int kCnnCh = 32, kCnnModes = 67, kCnnSplits = 6, kCnnOut = kCnnModes + kCnnSplits;
constexpr int kCnnConvW = kCnnCh * kCnnCh * 9;  // 9216
// fp32 parameter vector: W1 [co][2 inputs][tap], b1, then per layer 2..4
// W [co][ci][tap] and b, then the heads W [out][ch] and b.
constexpr int kOffW1 = 0, kOffB1 = 576;
__host__ __device__ constexpr int cnn_off_w(int layer) { return 608 + (layer - 2) * (kCnnConvW + kCnnCh); }
__host__ __device__ constexpr int cnn_off_b(int layer) { return cnn_off_w(layer) + kCnnConvW; }
constexpr int kOffWi = cnn_off_w(5), kOffBi = kOffWi + kCnnModes * kCnnCh;
constexpr int kOffWs = kOffBi + kCnnModes, kOffBs = kOffWs + kCnnSplits * kCnnCh;
constexpr int kCnnParams = kOffBs + kCnnSplits;  // 30761

constexpr int kImgW = 34;                 // 32 + halo
constexpr int kPlane = kImgW * kImgW * 16;  // one plane of 8 channels, bytes
constexpr int kImg = 4 * kPlane;            // 73984
constexpr int kPackL = 36 * 32 * 16;        // packed bf16 weights of one layer: [tap*4 + ci/8][co][ci%8]
constexpr int kCnnThreads = 256;
constexpr uint32_t kCnnIdesc = umma_idesc_bf16(128, 32);
constexpr int kCnnMisc = (576 + 32 + 96 + 8 * 32 + 1024 + 32) * 4;
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
  float qp_in;             // the QP plane's value, QP / 63 rounded to bf16
  const uint32_t* ctu_xy;  // n (x, y) pairs
  const float* params;
  const uint16_t* pack;
  float* logits;     // n x 73
  float* gap_out;    // n x 32, or null
  uint16_t* acts;    // n x 4 x 1024 x 32 bf16 (layer, pixel, channel), or null
  uint32_t* status;  // bit 0: a completion wait gave up; bit 1: a block outside the plane
};

// Issues the 144 MMAs of one 3x3 32->32 layer reading image `xin` with the
// packed weights `w` into TMEM columns tile * 32, then (with commit) commits
// to mbar.
__device__ __forceinline__ void cnn_issue_layer(uint32_t tmem, uint32_t xin, uint32_t w, uint64_t* mbar,
                                                bool commit = true) {
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
  if (commit) umma_commit(mbar);
}

__global__ void __launch_bounds__(kCnnThreads, 1) k_cnn_forward(const __grid_constant__ CnnFwdArgs A) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* X0 = smem;
  uint8_t* X1 = smem + kImg;
  uint8_t* W = smem + 2 * kImg;
  float* w1 = (float*)(W + 3 * kPackL);
  float* b1 = w1 + 576;
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
  for (int i = t; i < 576; i += kCnnThreads) w1[i] = A.params[kOffW1 + i];
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
      float in[9], iq[9];
#pragma unroll
      for (int tap = 0; tap < 9; tap++) {
        const int y = iy + tap / 3 - 1, x = ix + tap % 3 - 1;
        const bool inside = y >= 0 && y < 32 && x >= 0 && x < 32;
        in[tap] = inside ? xin[y * 32 + x] : 0.0f;
        iq[tap] = inside ? A.qp_in : 0.0f;
      }
      uint32_t pk[16];
#pragma unroll
      for (int c = 0; c < 32; c += 2) {
        float s0 = b1[c], s1 = b1[c + 1];
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
          s0 = fmaf(w1[c * 18 + tap], in[tap], s0);
          s1 = fmaf(w1[(c + 1) * 18 + tap], in[tap], s1);
        }
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
          s0 = fmaf(w1[c * 18 + 9 + tap], iq[tap], s0);
          s1 = fmaf(w1[(c + 1) * 18 + 9 + tap], iq[tap], s1);
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

namespace vvcg {

// ---------------------------------------------------------------- backward --
//
// One CTA per block (persistent). From the forward's activations a1..a4,
// gap and logits: the head gradients, then per layer l = 4, 3, 2 the
// gradient dZ_l (w.r.t. the layer's pre-activation) held as a bf16 image:
//  * its input gradient dA_{l-1} = conv(dZ_l, flipped W_l) is 144 tcgen05
//    MMAs exactly as in the forward pass (the taps of the transposed
//    convolution are the mirrored address offsets);
//  * behind them, the weight gradient
//    dW_l[co][ci][tap] = sum_p dZ_l[p][co] a_{l-1}[p + tap][ci] is 576 more
//    MMAs (cnn_issue_dw): the 1024 pixels are the K dimension and both
//    images are MN-major operands as they lie;
//  * the epilogue masks dA_{l-1} by a_{l-1} > 0 into dZ_{l-1}, in place of
//    a_{l-1}.
// Layer 1's weight gradient uses the bf16 input. Gradients and the loss
// accumulate in the CTA's own slice of `partial` (no atomics); a second
// kernel sums the slices.
struct CnnBwdArgs {
  const uint16_t* plane;
  int64_t stride;
  int32_t width, height, maxv, n;
  float qp_in;
  const uint32_t* ctu_xy;
  const uint8_t* labels;  // n x (mode, split)
  const float* params;
  const float* soft;       // optional n x kCnnModes target distribution of the mode head (else the label)
  const uint16_t* packT;  // flipped packed weights of layers 2..4
  const float* logits;
  const float* gap;
  const uint16_t* acts;
  float* partial;  // [gridDim.x][kCnnParams + 1]: gradients, then the loss sum
  float inv_batch;
  uint32_t* status;
};
constexpr int kXPad = 34 * 34;  // the input zero-padded by one pixel
constexpr int kCnnBwdMisc = (2 * kXPad + 32 + 32 * 8 + 96) * 4;
// M = 64, N = 32, both operands MN-major
constexpr uint32_t kCnnIdescW = umma_idesc_bf16(64, 32) | (1u << 15) | (1u << 16);
constexpr int kCnnBwdCols = 512;  // dA_{l-1}: columns 0..255; dW_l: 256..415

// Issues the weight-gradient MMAs of one 3x3 32->32 layer and returns
// without committing. Per tap t, D_t (M = 64, N = 32) += L * H_t^T over the
// 1024 pixels, 16 of one image row per MMA (K), with L the image at `lo`
// and H the one at `hi`: as MN-major operands without swizzle a core matrix
// is 8 pixels (K, 16 B apart) x 8 channels (16 B), LBO = 128 B steps the
// next 8 pixels and SBO = one channel plane the next 8 channels. Only L's
// 32 channels are rows of interest: rows 32..63 read the 4 planes that
// follow L, which must be the other image (lo is the lower of the two
// buffers), and are never read back. The tap's pixel offset applies to the
// activation image: to L when lo_tap, else to H. D_t sits in the TMEM lanes
// 16 (t & 1) + {0..15, 32..47} of columns (t >> 1) * 32 + 0..31 (two M = 64
// accumulators share columns in the two half sub-partitions).
__device__ __forceinline__ void cnn_issue_dw(uint32_t tmem, uint32_t lo, uint32_t hi, bool lo_tap) {
  // the start address is the descriptor's low field in 16-byte units (one
  // pixel): every operand is a base descriptor plus a pixel offset
  const uint64_t da0 = umma_desc(lo, 128, kPlane), db0 = umma_desc(hi, 128, kPlane);
  for (int y = 0; y < 32; y++)
    for (int h = 0; h < 2; h++) {
      const int base = (y + 1) * kImgW + 1 + 16 * h;
#pragma unroll
      for (int tap = 0; tap < 9; tap++) {
        const int sh = (tap / 3 - 1) * kImgW + tap % 3 - 1;
        umma_bf16(tmem + ((uint32_t)(16 * (tap & 1)) << 16) + (tap >> 1) * 32,
                  da0 + (uint64_t)(base + (lo_tap ? sh : 0)), db0 + (uint64_t)(base + (lo_tap ? 0 : sh)),
                  kCnnIdescW, (y | h) != 0);
      }
    }
}
constexpr int kCnnBwdSmem = 2 * kImg + kPackL + kCnnBwdMisc + 64;

// Loads activation image `layer` (0..3) of block blk from global into an
// image buffer (interior only; the halo stays zero).
__device__ __forceinline__ void cnn_load_act(uint8_t* img, const uint16_t* acts, int blk, int layer) {
  const uint4* src = (const uint4*)(acts + ((size_t)blk * 4 + layer) * 1024 * 32);
  for (int i0 = threadIdx.x; i0 < 1024 * 4; i0 += 4 * kCnnThreads) {
    uint4 v[4];  // four loads in flight before the stores
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = src[i0 + k * kCnnThreads];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int i = i0 + k * kCnnThreads, p = i >> 2, g = i & 3;
      *(uint4*)(img + g * kPlane + (((p >> 5) + 1) * kImgW + (p & 31) + 1) * 16) = v[k];
    }
  }
}

__global__ void __launch_bounds__(kCnnThreads, 1) k_cnn_backward(const __grid_constant__ CnnBwdArgs A) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* P = smem;
  uint8_t* Q = smem + kImg;
  uint8_t* Wt = smem + 2 * kImg;
  // (bf16-rounded normalised input, 1) inside the block, (0, 0) in the halo
  float2* xpad = (float2*)(Wt + kPackL);
  float* dgap = (float*)(xpad + kXPad);
  float* dbp = dgap + 32;   // [8 warps][32] bias-gradient partials
  float* dlog = dbp + 256;  // [73] logit gradients (+ pad)
  uint64_t* mbar = (uint64_t*)(dlog + 96);
  uint32_t* tslot = (uint32_t*)(mbar + 1);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  float* part = A.partial + (size_t)blockIdx.x * (kCnnParams + 1);
  for (int i = t; i < kCnnParams + 1; i += kCnnThreads) part[i] = 0.0f;
  for (int i = t; i < 2 * kImg / 16; i += kCnnThreads) ((uint4*)P)[i] = make_uint4(0, 0, 0, 0);
  for (int i = t; i < kXPad; i += kCnnThreads) xpad[i] = make_float2(0.0f, 0.0f);
  if (warp == 0) {
    tmem_alloc(tslot, kCnnBwdCols);
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
    if (ux > (uint32_t)A.width - 32 || uy > (uint32_t)A.height - 32 || A.width < 32 || A.height < 32 ||
        A.labels[2 * blk] >= kCnnModes || A.labels[2 * blk + 1] >= kCnnSplits) {
      if (t == 0) atomicOr(A.status, 2u);  // skipped: outside the plane or a label out of range
      continue;
    }
    // heads: softmax cross-entropy of both heads, mean over the batch
    if (warp == 0 || warp == 1) {
      const float* lg = A.logits + (size_t)blk * kCnnOut;
      const int n_out = warp == 0 ? kCnnModes : kCnnSplits, base = warp == 0 ? 0 : kCnnModes;
      const int label = A.labels[2 * blk + warp];
      float mx = -INFINITY;
      for (int j = lane; j < n_out; j += 32) mx = fmaxf(mx, lg[base + j]);
      for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
      float se = 0.0f;
      for (int j = lane; j < n_out; j += 32) se += __expf(lg[base + j] - mx);
      for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xFFFFFFFFu, se, o);
      // soft targets of the mode head: cross-entropy against the given
      // distribution, the loss summed in a fixed order (shuffles of lanes)
      const float* tg = (warp == 0 && A.soft) ? A.soft + (size_t)blk * kCnnModes : nullptr;
      float ce = 0.0f;
      for (int j = lane; j < n_out; j += 32) {
        const float pj = __expf(lg[base + j] - mx) / se;
        const float yj = tg ? tg[j] : (j == label ? 1.0f : 0.0f);
        dlog[base + j] = (pj - yj) * A.inv_batch;
        if (tg) ce += yj * (logf(se) + mx - lg[base + j]);
      }
      if (tg)
        for (int o = 16; o > 0; o >>= 1) ce += __shfl_xor_sync(0xFFFFFFFFu, ce, o);
      if (lane == 0) dlog[kCnnOut + warp] = (tg ? ce : (logf(se) + mx - lg[base + label])) * A.inv_batch;
    }
    __syncthreads();
    // the two heads' losses, added in a fixed order (training is deterministic)
    if (t == 0) part[kCnnParams] += dlog[kCnnOut] + dlog[kCnnOut + 1];
    const float inv = 1.0f / (float)A.maxv;
    const int bx = (int)ux, by = (int)uy;
    {
      uint16_t pv[1024 / kCnnThreads];  // the loads first, then the stores
#pragma unroll
      for (int u = 0; u < 1024 / kCnnThreads; u++) {
        const int i = t + u * kCnnThreads;
        pv[u] = A.plane[(int64_t)(by + (i >> 5)) * A.stride + bx + (i & 31)];
      }
#pragma unroll
      for (int u = 0; u < 1024 / kCnnThreads; u++) {
        const int i = t + u * kCnnThreads;
        xpad[((i >> 5) + 1) * 34 + (i & 31) + 1] = make_float2(bf2f(f2bf((float)pv[u] * inv)), 1.0f);
      }
    }
    __syncthreads();
    const float* gp = A.gap + (size_t)blk * 32;
    if (t < 32) {
      float s = 0.0f;
      for (int j = 0; j < kCnnModes; j++) s = fmaf(A.params[kOffWi + j * 32 + t], dlog[j], s);
      for (int j = 0; j < kCnnSplits; j++) s = fmaf(A.params[kOffWs + j * 32 + t], dlog[kCnnModes + j], s);
      dgap[t] = s;
    }
    {
      constexpr int kR = (kCnnOut * 32 + kCnnThreads - 1) / kCnnThreads;
      float o[kR];  // the loads first, then the stores
#pragma unroll
      for (int k = 0; k < kR; k++) {
        const int i = t + k * kCnnThreads;
        if (i < kCnnOut * 32) o[k] = part[((i >> 5) < kCnnModes ? kOffWi : kOffWs - kCnnModes * 32) + i];
      }
#pragma unroll
      for (int k = 0; k < kR; k++) {
        const int i = t + k * kCnnThreads, j = i >> 5;
        if (i < kCnnOut * 32) part[(j < kCnnModes ? kOffWi : kOffWs - kCnnModes * 32) + i] = o[k] + dlog[j] * gp[i & 31];
      }
    }
    if (t < kCnnOut) part[t < kCnnModes ? kOffBi + t : kOffBs + t - kCnnModes] += dlog[t];
    __syncthreads();
    // dZ4 into P (a4 > 0 passes dgap / 1024), a3 into Q
    {
      const uint4* a4 = (const uint4*)(A.acts + ((size_t)blk * 4 + 3) * 1024 * 32);
      float dbs[8];
      for (int k = 0; k < 8; k++) dbs[k] = 0.0f;
      for (int i0 = t; i0 < 1024 * 4; i0 += 8 * kCnnThreads) {
        uint4 avs[8];  // eight loads in flight
#pragma unroll
        for (int u = 0; u < 8; u++) avs[u] = a4[i0 + u * kCnnThreads];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int i = i0 + u * kCnnThreads, p = i >> 2, g = i & 3;  // g is fixed per thread (stride 256)
          const uint32_t aw[4] = {avs[u].x, avs[u].y, avs[u].z, avs[u].w};
          uint32_t o[4];
          for (int k = 0; k < 4; k++) {
            const float d0 = (aw[k] & 0xFFFFu) && !(aw[k] & 0x8000u) ? dgap[g * 8 + 2 * k] * (1.0f / 1024.0f) : 0.0f;
            const float d1 =
                (aw[k] >> 16) && !(aw[k] & 0x80000000u) ? dgap[g * 8 + 2 * k + 1] * (1.0f / 1024.0f) : 0.0f;
            dbs[2 * k] += d0;
            dbs[2 * k + 1] += d1;
            o[k] = (uint32_t)f2bf(d0) | ((uint32_t)f2bf(d1) << 16);
          }
          *(uint4*)(P + g * kPlane + (((p >> 5) + 1) * kImgW + (p & 31) + 1) * 16) =
              make_uint4(o[0], o[1], o[2], o[3]);
        }
      }
      // the 64 threads with the same g hold that plane's sums: reduced over
      // the warp's lanes of equal g, then over the warps in a fixed order
      for (int k = 0; k < 8; k++) {
        float s2 = dbs[k];
        for (int o2 = 4; o2 < 32; o2 <<= 1) s2 += __shfl_xor_sync(0xFFFFFFFFu, s2, o2);
        if (lane < 4) dbp[warp * 32 + lane * 8 + k] = s2;
      }
      __syncthreads();
      if (t < 32) {
        float s2 = 0.0f;
        for (int w2 = 0; w2 < 8; w2++) s2 += dbp[w2 * 32 + t];
        part[cnn_off_b(4) + t] += s2;
      }
    }
    cnn_load_act(Q, A.acts, blk, 2);
    uint8_t* dz = P;  // dZ_l
    uint8_t* act = Q; // a_{l-1}, becomes dZ_{l-1}
    for (int layer = 4; layer >= 2 && ok; layer--) {
      const int li = layer - 2;
      {
        constexpr int kN = kPackL / 16, kU = (kN + kCnnThreads - 1) / kCnnThreads;
        const uint4* src = (const uint4*)(A.packT + (size_t)li * (kPackL / 2));
        uint4 wv[kU];  // the loads first, then the stores
#pragma unroll
        for (int u = 0; u < kU; u++)
          if (t + u * kCnnThreads < kN) wv[u] = src[t + u * kCnnThreads];
#pragma unroll
        for (int u = 0; u < kU; u++)
          if (t + u * kCnnThreads < kN) ((uint4*)Wt)[t + u * kCnnThreads] = wv[u];
      }
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      if (t == 0) {
        cnn_issue_layer(tmem, smem_u32(dz), smem_u32(Wt), mbar, false);
        cnn_issue_dw(tmem + 256, smem_u32(P), smem_u32(Q), act == P);
        umma_commit(mbar);
      }
      ok = __syncthreads_and(mbar_wait(mbar, phase, 1u << 26));
      phase ^= 1;
      tc_fence_after();
      if (!ok) break;
      // weight gradient out of TMEM: warps of lane quarters 0 and 1 hold
      // rows 0..31 (the channels of the image at P); a thread takes tap
      // 2g + lane / 16 of row 16 q + lane % 16 and its 32 columns (the other
      // image's channels)
      if ((warp & 3) < 2) {
        float* gw = part + cnn_off_w(layer);
        const bool rows_co = dz == P;
        const int r = 16 * (warp & 3) + (lane & 15);
        for (int g = warp < 4 ? 0 : 3; g < (warp < 4 ? 3 : 5); g++) {
          const int tp = 2 * g + (lane >> 4);
          const uint32_t ta = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + 256 + g * 32;
          float v[32];
          tmem_ld16(ta, v);
          tmem_ld16(ta + 16, v + 16);
          if (tp < 9) {  // the 32 loads first, then the 32 stores (one round trip, not 32)
            float* g0 = gw + (rows_co ? r * kCnnCh * 9 : r * 9) + tp;
            const int st = rows_co ? 9 : kCnnCh * 9;
            float o[32];
#pragma unroll
            for (int n = 0; n < 32; n++) o[n] = g0[n * st];
#pragma unroll
            for (int n = 0; n < 32; n++) g0[n * st] = o[n] + v[n];
          }
        }
      }
      // epilogue: dZ_{l-1} = dA_{l-1} where a_{l-1} > 0, in place of a_{l-1}
      float dbs[32];
      for (int c = 0; c < 32; c++) dbs[c] = 0.0f;
      const int q = warp & 3;
      for (int k = 0; k < 4; k++) {
        const int tile = (warp >> 2) + 2 * k;
        const int m = 32 * q + lane, j = m >> 3, r = m & 7;
        const int iy = 16 * (tile >> 2) + j, ix = 8 * (tile & 3) + r;
        float v[32];
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + tile * 32, v);
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + tile * 32 + 16, v + 16);
        const int off = ((iy + 1) * kImgW + ix + 1) * 16;
        for (int g = 0; g < 4; g++) {
          uint4 av = *(const uint4*)(act + g * kPlane + off);
          uint32_t aw[4] = {av.x, av.y, av.z, av.w}, o[4];
          for (int k2 = 0; k2 < 4; k2++) {
            const int c = g * 8 + 2 * k2;
            const float d0 = ((aw[k2] & 0xFFFFu) && !(aw[k2] & 0x8000u)) ? v[c] : 0.0f;
            const float d1 = ((aw[k2] >> 16) && !(aw[k2] & 0x80000000u)) ? v[c + 1] : 0.0f;
            dbs[c] += d0;
            dbs[c + 1] += d1;
            o[k2] = (uint32_t)f2bf(d0) | ((uint32_t)f2bf(d1) << 16);
          }
          *(uint4*)(act + g * kPlane + off) = make_uint4(o[0], o[1], o[2], o[3]);
        }
      }
      for (int c = 0; c < 32; c++) {
        float s = dbs[c];
        for (int o2 = 16; o2 > 0; o2 >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o2);
        if (lane == 0) dbp[warp * 32 + c] = s;
      }
      tc_fence_before();
      __syncthreads();
      if (t < 32) {
        float s = 0.0f;
        for (int w2 = 0; w2 < 8; w2++) s += dbp[w2 * 32 + t];
        part[layer == 2 ? kOffB1 + t : cnn_off_b(layer - 1) + t] += s;
      }
      // next layer: the old dZ_l buffer takes a_{l-2}
      if (layer > 2) cnn_load_act(dz, A.acts, blk, layer - 3);
      uint8_t* tmp = dz;
      dz = act;
      act = tmp;
      __syncthreads();
    }
    if (!ok) break;
    // layer 1: dW1[co][input][tap] = sum_p dZ1[p][co] in[p + tap] (dZ1 is in
    // dz; the second input is the constant QP plane, zero in the halo). Warp
    // w takes rows 4w..4w+3 and lane the output channel, over a sliding 3x3
    // window of (input, inside) pairs; the 8 row groups' sums meet in the
    // weight buffer (free until the next block) and are added in a fixed order.
    {
      const uint8_t* zp = dz + (lane >> 3) * kPlane + (lane & 7) * 2;
      float sx[9], sq[9];
#pragma unroll
      for (int k = 0; k < 9; k++) sx[k] = sq[k] = 0.0f;
      for (int y = 4 * warp; y < 4 * warp + 4; y++) {
        float2 w[3][3];
#pragma unroll
        for (int dy = 0; dy < 3; dy++)
#pragma unroll
          for (int dx = 0; dx < 2; dx++) w[dy][dx + 1] = xpad[(y + dy) * 34 + dx];
        for (int x = 0; x < 32; x++) {
#pragma unroll
          for (int dy = 0; dy < 3; dy++) {
            w[dy][0] = w[dy][1];
            w[dy][1] = w[dy][2];
            w[dy][2] = xpad[(y + dy) * 34 + x + 2];
          }
          const float z = bf2f(*(const uint16_t*)(zp + ((y + 1) * kImgW + x + 1) * 16));
#pragma unroll
          for (int k = 0; k < 9; k++) {
            sx[k] = fmaf(z, w[k / 3][k % 3].x, sx[k]);
            sq[k] = fmaf(z, w[k / 3][k % 3].y, sq[k]);
          }
        }
      }
      float* red = (float*)Wt;  // [8 row groups][32 channels][18]
#pragma unroll
      for (int k = 0; k < 9; k++) {
        red[(warp * 32 + lane) * 18 + k] = sx[k];
        red[(warp * 32 + lane) * 18 + 9 + k] = sq[k];
      }
      __syncthreads();
      for (int o = t; o < 32 * 18; o += kCnnThreads) {
        float v = 0.0f;
        for (int g = 0; g < 8; g++) v += red[g * 32 * 18 + o];
        part[kOffW1 + o] += (o % 18) < 9 ? v : v * A.qp_in;
      }
    }
    __syncthreads();
  }
  if (!ok && t == 0) atomicOr(A.status, 1u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kCnnBwdCols);
}

// grads[i] = sum over the CTA slices; loss[0] = sum of the loss slots.
__global__ void k_cnn_reduce(const float* __restrict__ partial, int slices, float* __restrict__ grads,
                             float* __restrict__ loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > kCnnParams) return;
  float s = 0.0f;
  for (int k = 0; k < slices; k++) s += partial[(size_t)k * (kCnnParams + 1) + i];
  if (i < kCnnParams)
    grads[i] = s;
  else
    loss[0] = s;
}

// Adam (bias-corrected) on the fp32 parameter vector.
__global__ void k_cnn_adam(float* __restrict__ params, const float* __restrict__ grads, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCnnParams) return;
  const float g = grads[i];
  const float mi = b1 * m[i] + (1.0f - b1) * g, vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace vvcg
