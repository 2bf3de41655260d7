// Motion-compensation interpolation on 16-bit planes (8..12-bit samples):
// 1/16-pel 8-tap luma and 1/32-pel 4-tap chroma, uni-prediction output or
// 14-bit bi-prediction intermediates, and the BCW weighted bi average.
// Follows interpolate_luma_block_16 (inter.rs:2010-2134),
// interpolate_chroma_block_format_16 (:2543-2672) and weighted_average_bi_16
// (:2676-2698) of the reference, including the uni-prediction second-stage
// shift `12 - bd` for 2-D fractional positions (inter.rs:2051 / :2583); and
// the 8-bit functions interpolate_luma_block (inter.rs:896-1051) and
// interpolate_chroma_block_420 (:1056-1182), which read 8-bit planes and use
// the second stage (sum + 2^11) >> 12 for 2-D uni-prediction.
//
// Each CTA computes one block in 32x32 output tiles: the tile's reference
// window (clamped to the plane, as the reference's get_p does) is staged in
// shared memory, the horizontal pass fills a 32 x (32 + taps - 1) buffer, and
// the vertical pass produces the outputs.
#pragma once
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

constexpr int kMcT = 32;

struct McParams {
  const uint16_t* ref;
  const uint8_t* ref8;  // 8-bit plane of the 8-bit functions (then ref is unused and bd is 8)
  int32_t w, h, stride, bd;
  int32_t chroma;   // 0 = luma (8 taps), else chroma format (4 taps)
};

__global__ void __launch_bounds__(256) k_mc(McParams Pm, const vvcg_mc_block* __restrict__ blocks,
                                           uint32_t n, int32_t* __restrict__ out,
                                           uint32_t* status) {
  __shared__ int win[kMcT + 7][kMcT + 7];
  __shared__ int tmp[kMcT + 7][kMcT];
  const uint32_t bi_ = blockIdx.x;
  if (bi_ >= n) return;
  const vvcg_mc_block B = blocks[bi_];
  const bool luma = Pm.chroma == 0;
  const bool bi = (B.flags & VVCG_MC_BI) != 0;
  const int bd = clampi(Pm.bd, 8, 12), maxv = (1 << bd) - 1;
  int dx, dy, fx, fy;
  if (luma) {
    dx = B.mv_x >> 4;
    dy = B.mv_y >> 4;
    fx = B.mv_x & 15;
    fy = B.mv_y & 15;
  } else {
    const int sw = (Pm.chroma == 1 || Pm.chroma == 2) ? 2 : 1, shh = Pm.chroma == 1 ? 2 : 1;
    const int mx = B.mv_x * (sw == 1 ? 2 : 1), my = B.mv_y * (shh == 1 ? 2 : 1);
    dx = mx >> 5;
    dy = my >> 5;
    fx = mx & 31;
    fy = my & 31;
  }
  const int ntap = luma ? 8 : 4, half = luma ? 3 : 1;
  int fh[8], fv[8];
  for (int k = 0; k < ntap; k++) {
    if (luma) {
      if (B.flags & VVCG_MC_AFFINE) {
        fh[k] = c_affine_taps8[fx * 8 + k];
        fv[k] = c_affine_taps8[fy * 8 + k];
      } else {
        fh[k] = ((B.flags & VVCG_MC_ALT_HPEL) && fx == 8) ? c_luma_alt_hpel[k] : c_luma_taps8[fx * 8 + k];
        fv[k] = ((B.flags & VVCG_MC_ALT_HPEL) && fy == 8) ? c_luma_alt_hpel[k] : c_luma_taps8[fy * 8 + k];
      }
    } else {
      fh[k] = c_chroma_taps4[fx * 4 + k];
      fv[k] = c_chroma_taps4[fy * 4 + k];
    }
  }
  const int head = max(14 - bd, 2);
  const int shift1 = 6 - head;
  const int shift2 = bi ? 6 : 12 - bd;
  // The reference's release build masks the shift count to 5 bits (1 << 31 at
  // 12 bit, where shift2 is 0) and wraps the addition below.
  const int add2 = bi ? 0 : (int)(1u << ((unsigned)(shift2 - 1) & 31));
  const int offs = 1 << (bd + head - 1);
  const int bw = B.w, bh = B.h;
  int32_t* o = out + B.out_offset;
  for (int ty0 = 0; ty0 < bh; ty0 += kMcT)
    for (int tx0 = 0; tx0 < bw; tx0 += kMcT) {
      const int tw = min(kMcT, bw - tx0), th = min(kMcT, bh - ty0);
      // reference window: rows y - half .. y + th + (ntap - half - 1), same for x
      const int wx0 = B.x + tx0 + dx - half, wy0 = B.y + ty0 + dy - half;
      const int ww = tw + ntap - 1, wh = th + ntap - 1;
      __syncthreads();
      for (int i = threadIdx.x; i < ww * wh; i += blockDim.x) {
        int yy = i / ww, xx = i % ww;
        int gx = clampi(wx0 + xx, 0, Pm.w - 1), gy = clampi(wy0 + yy, 0, Pm.h - 1);
        win[yy][xx] = Pm.ref8 ? (int)Pm.ref8[(size_t)gy * Pm.stride + gx] : (int)Pm.ref[(size_t)gy * Pm.stride + gx];
      }
      __syncthreads();
      if (fx == 0 && fy == 0) {
        for (int i = threadIdx.x; i < tw * th; i += blockDim.x) {
          int x = i % tw, y = i / tw;
          int s = win[y + half][x + half];
          o[(size_t)(ty0 + y) * bw + tx0 + x] = bi ? (s << head) - offs : s;
        }
      } else if (fy == 0 || fx == 0) {
        const bool hor = fy == 0;
        for (int i = threadIdx.x; i < tw * th; i += blockDim.x) {
          int x = i % tw, y = i / tw;
          int s = 0;
          for (int k = 0; k < ntap; k++)
            s += hor ? fh[k] * win[y + half][x + k] : fv[k] * win[y + k][x + half];
          o[(size_t)(ty0 + y) * bw + tx0 + x] = bi ? (s >> shift1) - offs : clampi((s + 32) >> 6, 0, maxv);
        }
      } else {
        for (int i = threadIdx.x; i < tw * wh; i += blockDim.x) {
          int x = i % tw, yy = i / tw;
          int s = 0;
          for (int k = 0; k < ntap; k++) s += fh[k] * win[yy][x + k];
          tmp[yy][x] = s >> shift1;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < tw * th; i += blockDim.x) {
          int x = i % tw, y = i / tw;
          int s = 0;
          for (int k = 0; k < ntap; k++) s += fv[k] * tmp[y + k][x];
          // 8-bit functions: (sum of taps x (tmp - 2^13) + 2^11 + 2^13 x 64) >> 12,
          // which is (s + 2^11) >> 12 because every filter's taps sum to 64
          o[(size_t)(ty0 + y) * bw + tx0 + x] =
              bi ? (s >> shift2) - offs
                 : (Pm.ref8 ? clampi((s + 2048) >> 12, 0, 255)
                            : clampi((int)((unsigned)s + (unsigned)add2) >> shift2, 0, maxv));
        }
      }
    }
}

// weighted_average_bi_16 (inter.rs:2676-2698)
__global__ void k_bi_average(const int32_t* __restrict__ p0, const int32_t* __restrict__ p1,
                             uint64_t n, int bcw, int bd, uint16_t* __restrict__ out) {
  bd = clampi(bd, 8, 12);
  const int maxv = (1 << bd) - 1;
  const int w1 = c_bcw_weights[min(bcw, 4)], w0 = 8 - w1;
  const int head = max(14 - bd, 2), sn = head + 3;
  const int off = (1 << (sn - 1)) + ((1 << (bd + head - 1)) << 3);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint16_t)clampi((p0[i] * w0 + p1[i] * w1 + off) >> sn, 0, maxv);
}

}  // namespace vvcg
