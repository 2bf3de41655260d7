// LMCS sample mapping, chroma residual scale derivation and joint Cb-Cr
// residuals of the general decoding path (sm_100a), each following the
// reference function named beside it (crates/rustmpeg-video/src/vvc/).
#pragma once
#include <stdint.h>

#include "../../include/vvcg.h"
#include "vvcg_device.cuh"

namespace vvcg {

constexpr int kLmcsFpPrec = 11;  // filter.rs:22 LMCS_FP_PREC

// apply_inverse_plane_16 / apply_forward_plane_16 (filter.rs:2708-2722): the
// LUT (1 << bd entries) is staged in shared memory; 4 samples per thread with
// 8-byte accesses when the row allows, scalar otherwise.
__global__ void __launch_bounds__(256) k_lut_plane(const uint16_t* __restrict__ lut, int bd, uint16_t* plane,
                                                   uint32_t stride, uint32_t w, uint32_t h) {
  __shared__ uint16_t s_lut[4096];
  const int n = 1 << bd, cap = n - 1;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_lut[i] = lut[i];
  __syncthreads();
  const uint32_t qw = (w + 3) >> 2;
  const bool vec = (stride & 3) == 0 && (reinterpret_cast<uintptr_t>(plane) & 7) == 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (uint64_t)qw * h;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t y = (uint32_t)(i / qw), x = (uint32_t)(i % qw) * 4;
    uint16_t* p = plane + (uint64_t)y * stride + x;
    if (vec && x + 4 <= w) {
      uint2 v = *reinterpret_cast<uint2*>(p);
      const uint32_t a = s_lut[min((int)(v.x & 0xFFFFu), cap)], b = s_lut[min((int)(v.x >> 16), cap)];
      const uint32_t c = s_lut[min((int)(v.y & 0xFFFFu), cap)], d = s_lut[min((int)(v.y >> 16), cap)];
      *reinterpret_cast<uint2*>(p) = make_uint2(a | (b << 16), c | (d << 16));
    } else {
      for (uint32_t k = 0; k < 4 && x + k < w; k++) p[k] = s_lut[min((int)p[k], cap)];
    }
  }
}

// chroma_adj_luma (decode_general.rs:4803-4835) for the VPDU holding luma
// position (x, y), then chroma_scale_for_luma (filter.rs:2725-2735). One warp
// per position; `t` is the device copy of the tables.
__global__ void __launch_bounds__(256) k_lmcs_chroma_scales(const vvcg_lmcs_tables* __restrict__ t,
                                                            const uint16_t* __restrict__ luma, uint32_t stride,
                                                            int pw, int ph, int ctu, const uint32_t* __restrict__ pos,
                                                            uint32_t num, int32_t* out) {
  const int lane = threadIdx.x & 31;
  const uint32_t k = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (k >= num) return;
  const int vpdu = ctu == 128 ? 64 : ctu;
  const int vx = ((int)pos[2 * k] / vpdu) * vpdu, vy = ((int)pos[2 * k + 1] / vpdu) * vpdu;
  const int n = min(64, vpdu);
  int sum = 0;
  for (int i = lane; i < n; i += 32) {
    if (vx > 0) sum += luma[(uint64_t)min(vy + i, ph - 1) * stride + vx - 1];
    if (vy > 0) sum += luma[(uint64_t)(vy - 1) * stride + min(vx + i, pw - 1)];
  }
  sum = __reduce_add_sync(0xffffffffu, sum);
  if (lane == 0) {
    const int count = (vx > 0 ? n : 0) + (vy > 0 ? n : 0);
    const int tz = __ffs(n) - 1;
    const int dc = 1 << (clampi(t->bit_depth, 8, 12) - 1);
    const int avg = count == 0 ? dc : count == n ? (sum + (1 << (tz - 1))) >> tz
                                                 : (sum + (1 << tz)) >> (tz + 1);
    int i = t->min_bin_idx;
    while (i <= t->max_bin_idx && !(avg < t->reshape_pivot[i + 1])) i++;
    out[k] = t->chroma_adj_lut[min(i, 15)];
  }
}

__device__ __forceinline__ int16_t sat16(int v) { return (int16_t)clampi(v, -32768, 32767); }

// Joint Cb-Cr derivation (decode_general.rs:3932-3955) and
// scale_chroma_residual (filter.rs:2740-2749), one warp per record. int16
// results saturate (the reference keeps i32; the reconstruction that clips
// pred + residual to [0, maxVal] is the same).
__global__ void __launch_bounds__(256) k_chroma_residuals(const vvcg_cres_rec* __restrict__ recs, uint32_t num,
                                                          int16_t* res) {
  const int lane = threadIdx.x & 31;
  const uint32_t k = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (k >= num) return;
  const vvcg_cres_rec r = recs[k];
  const int n = (1 << r.log2_w) * (1 << r.log2_h);
  int16_t* cb = res + r.cb_off;
  int16_t* cr = res + r.cr_off;
  const bool single = (r.flags & VVCG_CRES_SINGLE) != 0;
  const bool scale = (r.flags & VVCG_CRES_SCALE) != 0;
  const int max_val = (1 << clampi(r.bit_depth, 8, 12)) - 1;
  auto sc = [&](int v) -> int16_t {
    v = clampi(v, -max_val - 1, max_val);
    const long long a = ((long long)abs(v) * r.scale + (1 << (kLmcsFpPrec - 1))) >> kLmcsFpPrec;
    return sat16((int)(v < 0 ? -a : a));
  };
  for (int i = lane; i < n; i += 32) {
    int b = cb[i], c = single ? 0 : cr[i];
    if (!single) {
      switch (r.joint) {
        case 3: b = c >> 1; break;
        case -3: b = (-c) >> 1; break;
        case 1: c = b >> 1; break;
        case -1: c = (-b) >> 1; break;
        case 2: c = b; break;
        case -2: c = b == -32768 ? 32767 : -b; break;  // -b saturated to int16
        default: break;
      }
    }
    if (scale) {
      b = sc(b);
      c = sc(c);
    }
    cb[i] = (int16_t)b;
    if (!single) cr[i] = (int16_t)c;
  }
}

}  // namespace vvcg
