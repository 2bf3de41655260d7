// Reconstruction of the 8..12-bit frame path on the GPU: a persistent
// wavefront kernel in which every warp works on its own CTU.
//
// Work items are CTUs handed out by an atomic counter in wavefront order
// (diagonal t = cx + 2*cy, across all pictures of the batch), so a warp only
// ever waits on items that running warps already hold and the schedule
// cannot deadlock. For each coding unit the warp first dequantises and
// inverse-transforms the residuals of its three TBs (independent of the
// neighbours, so this overlaps the wait), then waits (bounded) for the left
// and top-right CTUs, then predicts, adds, clips and stores.
//
// Follows slice::decode_vvc_frame_picture_with_chroma_qp (slice.rs:4834-4988):
// predict_coded_block_16 / predict_cclm_with_format_16 prediction (see
// intra.cuh), dequantize_rect_bd or dequantize_dep_quant_bd (dct.rs:1151,
// :1191), inverse_transform_rect_bd (dct.rs:996) with DCT-II both ways, and the
// add/clip to 0..2^bd-1. All sums are exact in int32, so reassociating the
// matrix products (dp2a pairs) gives the reference's results bit for bit.
#pragma once
#include "intra.cuh"
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

constexpr int kWarpsPerCta = 8;
constexpr int kTS = 34;  // row stride (int16) of the transposed coefficient tiles

// Per-warp shared workspace. res_c holds two chroma TBs of up to kMaxCArea
// samples; the coefficient tiles are reused as the CU's luma tile for CCLM.
struct WarpWs {
  DevPic P;  // the item's picture, copied once per item
  int16_t res_y[32 * 32];
  int16_t ct[32 * kTS];  // coefficients, transposed: ct[col * kTS + row]
  int16_t tt[32 * kTS];  // stage-1 output, transposed: tt[row * kTS + col]
  IntraWs in;
  // followed by int16_t res_c[2][max chroma TB area]
};

// Matrix columns held in registers: lane j keeps M[k][j] of the 32-point
// DCT-II for k = 0..31 (8 words of 4 int8) and M[k][j & 15] of the 16-point
// DCT-II for k = 0..15 (4 words).
struct MatRegs {
  int m32[8];
  int m16[4];
};

__device__ __forceinline__ void load_mat_regs(MatRegs& R) {
  const int lane = threadIdx.x & 31;
  const int8_t* a = g_dct2_m[4];
  const int8_t* b = g_dct2_m[3];
#pragma unroll
  for (int g = 0; g < 8; g++) {
    uint32_t v = 0;
#pragma unroll
    for (int t = 0; t < 4; t++) v |= (uint32_t)(uint8_t)a[(4 * g + t) * 32 + lane] << (8 * t);
    R.m32[g] = (int)v;
  }
#pragma unroll
  for (int g = 0; g < 4; g++) {
    uint32_t v = 0;
#pragma unroll
    for (int t = 0; t < 4; t++) v |= (uint32_t)(uint8_t)b[(4 * g + t) * 16 + (lane & 15)] << (8 * t);
    R.m16[g] = (int)v;
  }
}

// sum_k M[k][j] * v[k] for k < 4*ng, with v given as int16 pairs in a
// transposed tile row (v[k] at row[k]); M from the lane's registers.
template <int N>
__device__ __forceinline__ int dot_col(const MatRegs& R, const int16_t* row, int ng) {
  const uint32_t* r2 = reinterpret_cast<const uint32_t*>(row);
  int acc = 0;
  if (N == 32) {
#pragma unroll
    for (int g = 0; g < 8; g++)
      if (g < ng) {
        acc = __dp2a_lo((int)r2[2 * g], R.m32[g], acc);
        acc = __dp2a_hi((int)r2[2 * g + 1], R.m32[g], acc);
      }
  } else {
#pragma unroll
    for (int g = 0; g < 4; g++)
      if (g < ng) {
        acc = __dp2a_lo((int)r2[2 * g], R.m16[g], acc);
        acc = __dp2a_hi((int)r2[2 * g + 1], R.m16[g], acc);
      }
  }
  return acc;
}

// Dequantisation (regular or dependent) and 2-D inverse DCT-II of a w x h TB
// (w, h in {16, 32}) whose int16 raster levels start at `lv`; the residual is
// written to `res` (int16, raster). Rows/columns past the last nonzero level
// hold zeros and are skipped without changing any sum.
__device__ void warp_residual(const int16_t* __restrict__ lv, int w, int h, int qp_scaled, int bd,
                              bool dq, const MatRegs& R, WarpWs& W, int16_t* res) {
  const int lane = threadIdx.x & 31;
  const int n = w * h, lw = ilog2(w), lh = ilog2(h);
  const bool s2 = ((lw + lh) & 1) != 0;
  const int tr_shift = 15 - bd - ((lw + lh) >> 1) - (s2 ? 1 : 0);
  int maxr = -1, maxc = -1;
  // All of the TB's levels are fetched up front (streaming 16-byte loads, one
  // round trip), while the coefficient tile is cleared.
  uint4 buf[4];
  const int nvec = n >> 8;  // uint4 per lane: 4 (1024 levels), 2 (512), 1 (256)
  const bool vec_ok = ((reinterpret_cast<uintptr_t>(lv) & 15) == 0) && (n & 255) == 0;
  if (vec_ok) {
    const uint4* lv4 = reinterpret_cast<const uint4*>(lv);
#pragma unroll
    for (int v = 0; v < 4; v++)
      if (v < nvec) buf[v] = __ldcs(lv4 + lane + 32 * v);
  }
  // clear the coefficient tile rows that the dot products read (k < 32)
  for (int i = lane; i < w * (kTS / 2); i += 32) reinterpret_cast<uint32_t*>(W.ct)[i] = 0;
  __syncwarp();
  if (!dq) {
    const int qp = max(4, qp_scaled);
    const int qp_per = qp / 6, qp_rem = qp % 6;
    const int rs = 6 - (tr_shift + qp_per);
    const long long scale = c_inv_quant_scale[s2 ? 1 : 0][qp_rem];
    auto put = [&](int i, int L) {
      int r = i >> lw, c = i & (w - 1);
      maxr = max(maxr, r);
      maxc = max(maxc, c);
      long long val = (long long)L * scale;
      long long sc = rs > 0 ? (val + (1ll << (rs - 1))) >> rs : val << (-rs);
      W.ct[c * kTS + r] = (int16_t)clip16(sc);
    };
    if (vec_ok) {
#pragma unroll
      for (int v = 0; v < 4; v++)
        if (v < nvec) {
          const uint32_t wv[4] = {buf[v].x, buf[v].y, buf[v].z, buf[v].w};
#pragma unroll
          for (int e = 0; e < 8; e++) {
            int L = (int)(int16_t)(wv[e >> 1] >> (16 * (e & 1)));
            if (L != 0) put(8 * (lane + 32 * v) + e, L);
          }
        }
    } else {
      for (int i = lane; i < n; i += 32) {
        int L = lv[i];
        if (L != 0) put(i, L);
      }
    }
  } else {
    // dequantize_dep_quant_bd (dct.rs:1191-1248): the 4-state machine walks the
    // grouped diagonal scan backwards from the last nonzero level. The walk is
    // split into 32 chunks; each lane composes its chunk's state transitions,
    // a warp scan of the compositions gives each chunk's entry state, then
    // every lane replays its chunk.
    const int16_t* scan = g_scan + g_scan_off[(lw - 1) * 6 + (lh - 1)];
    const int ns = min(w, 32) * min(h, 32);
    int last = -1;
    auto put = [&](int i, int L) {
      int r = i >> lw, c = i & (w - 1);
      maxr = max(maxr, r);
      maxc = max(maxc, c);
      W.ct[c * kTS + r] = (int16_t)L;
    };
    if (vec_ok) {
#pragma unroll
      for (int v = 0; v < 4; v++)
        if (v < nvec) {
          const uint32_t wv[4] = {buf[v].x, buf[v].y, buf[v].z, buf[v].w};
#pragma unroll
          for (int e = 0; e < 8; e++) {
            int L = (int)(int16_t)(wv[e >> 1] >> (16 * (e & 1)));
            if (L != 0) put(8 * (lane + 32 * v) + e, L);
          }
        }
    } else {
      for (int i = lane; i < n; i += 32) {
        int L = lv[i];
        if (L != 0) put(i, L);
      }
    }
    __syncwarp();
    for (int s = lane; s < ns; s += 32) {
      int r = scan[s];
      if (W.ct[(r & (w - 1)) * kTS + (r >> lw)] != 0) last = max(last, s);
    }
    last = __reduce_max_sync(0xffffffffu, last);
    if (last >= 0) {
      const int cs = (last + 32) >> 5;
      const int hi = last - lane * cs;
      const int lo = max(hi - cs + 1, 0);
      uint32_t map = 0;
      for (int st0 = 0; st0 < 4; st0++) {
        int st = st0;
        for (int s = hi; s >= lo; s--) {
          int r = scan[s];
          int L = W.ct[(r & (w - 1)) * kTS + (r >> lw)];
          st = (32040 >> ((st << 2) + ((L & 1) << 1))) & 3;
        }
        map |= (uint32_t)st << (2 * st0);
      }
      uint32_t pre = map;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t other = __shfl_up_sync(0xffffffffu, pre, o);
        if (lane >= o) {
          uint32_t comp = 0;
          for (int s = 0; s < 4; s++) comp |= ((pre >> (2 * ((other >> (2 * s)) & 3))) & 3) << (2 * s);
          pre = comp;
        }
      }
      uint32_t excl = __shfl_up_sync(0xffffffffu, pre, 1);
      int st = lane == 0 ? 0 : (int)(excl & 3);
      const int qp_dq = max(4, qp_scaled) + 1;
      const int qp_per = qp_dq / 6, qp_rem = qp_dq % 6;
      const int shift = 7 - qp_per - tr_shift;
      long long inv_q = c_inv_quant_scale[s2 ? 1 : 0][qp_rem];
      if (shift < 0) inv_q <<= -shift;
      const long long add = shift > 0 ? (1ll << (shift - 1)) : 0;
      const int rsh = max(0, shift);
      __syncwarp();
      for (int s = hi; s >= lo; s--) {
        int r = scan[s];
        int16_t* p = &W.ct[(r & (w - 1)) * kTS + (r >> lw)];
        int L = *p;
        if (L != 0) {
          long long q = (long long)(2 * L + (L > 0 ? -(st >> 1) : (st >> 1)));
          *p = (int16_t)clip16((q * inv_q + add) >> rsh);
        }
        st = (32040 >> ((st << 2) + ((L & 1) << 1))) & 3;
      }
    }
  }
  maxr = __reduce_max_sync(0xffffffffu, maxr);
  maxc = __reduce_max_sync(0xffffffffu, maxc);
  __syncwarp();
  if (maxr < 0) {
    for (int i = lane; i < n / 2; i += 32) reinterpret_cast<uint32_t*>(res)[i] = 0;
    __syncwarp();
    return;
  }
  // Stage 1, columns (dct.rs:1075-1087): tt[j][i] = clip16((sum_k Mv[k][j] ct[i][k] + 64) >> 7)
  const int ngr = (maxr + 4) >> 2;
  if (h == 32) {
    for (int i = 0; i <= maxc; i++) {
      int acc = dot_col<32>(R, &W.ct[i * kTS], ngr);
      W.tt[lane * kTS + i] = (int16_t)clip16i((acc + 64) >> 7);
    }
  } else {  // h == 16: two columns per pass
    const int j = lane & 15;
    for (int i0 = 0; i0 <= maxc; i0 += 2) {
      int i = i0 + (lane >> 4);
      if (i <= maxc) {
        int acc = dot_col<16>(R, &W.ct[i * kTS], ngr);
        W.tt[j * kTS + i] = (int16_t)clip16i((acc + 64) >> 7);
      }
    }
  }
  // tt columns past maxc must read as zero in stage 2
  if (maxc + 1 < w)
    for (int i = lane; i < h * 4; i += 32) {
      int row = i >> 2, c = maxc + 1 + (i & 3);
      if (c < ((maxc + 4) & ~3)) W.tt[row * kTS + c] = 0;
    }
  __syncwarp();
  // Stage 2, rows (dct.rs:1089-1106): res[y][x] = clip16((sum_k Mh[k][x] tt[y][k] + add) >> (20 - bd))
  const int sh2 = 20 - bd, add2 = 1 << (sh2 - 1);
  const int ngc = (maxc + 4) >> 2;
  if (w == 32) {
    for (int y = 0; y < h; y++) {
      int acc = dot_col<32>(R, &W.tt[y * kTS], ngc);
      res[y * 32 + lane] = (int16_t)clip16i((acc + add2) >> sh2);
    }
  } else {
    const int x = lane & 15;
    for (int y0 = 0; y0 < h; y0 += 2) {
      int y = y0 + (lane >> 4);
      int acc = dot_col<16>(R, &W.tt[y * kTS], ngc);
      res[y * 16 + x] = (int16_t)clip16i((acc + add2) >> sh2);
    }
  }
  __syncwarp();
}

// Bounded wait for a CTU flag; returns false when the poll limit ran out.
__device__ __forceinline__ bool wait_flag(const uint32_t* flag, uint32_t epoch, uint32_t limit) {
  uint32_t ns = 32;
  for (uint32_t it = 0; it < limit; it++) {
    if (ld_acquire(flag) == epoch) return true;
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
  return ld_acquire(flag) == epoch;
}

__global__ void __launch_bounds__(kWarpsPerCta * 32, 3)
k_recon_wavefront(const DevPic* __restrict__ pics, const CtuItem* __restrict__ items,
                  uint32_t n_items, uint32_t* counter, const int16_t* __restrict__ levels,
                  uint64_t n_levels, uint32_t epoch, uint32_t spin_limit, uint32_t* status,
                  uint32_t ws_bytes, uint32_t c_area) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  WarpWs& W = *reinterpret_cast<WarpWs*>(smem_raw + (size_t)wid * ws_bytes);
  int16_t* res_c0 = reinterpret_cast<int16_t*>(smem_raw + (size_t)wid * ws_bytes + sizeof(WarpWs));
  int16_t* res_c1 = res_c0 + c_area;
  MatRegs R;
  load_mat_regs(R);
  for (;;) {
    uint32_t it = 0;
    if (lane == 0) it = atomicAdd(counter, 1u);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= n_items) break;
    const CtuItem item = items[it];
    static_assert(sizeof(DevPic) % 4 == 0 && sizeof(DevPic) <= 64 * 4, "DevPic copy");
    for (int i = lane; i < (int)(sizeof(DevPic) / 4); i += 32)
      reinterpret_cast<uint32_t*>(&W.P)[i] = reinterpret_cast<const uint32_t*>(&pics[item.pic])[i];
    __syncwarp();
    const DevPic& P = W.P;
    const int cx = item.cx, cy = item.cy;
    const int tb = P.tb, ctu_log2 = P.ctu_log2, sh = ctu_log2 - ilog2(tb);
    const int ncu = 1 << (2 * sh);
    const int cf = P.cf, bd = P.bd;
    const bool dq = (P.tools & VVCG_TOOL_DEP_QUANT) != 0;
    for (int k = 0; k < ncu; k++) {
      int lx = 0, ly = 0;
      for (int b = 0; b < sh; b++) {
        lx |= ((k >> (2 * b)) & 1) << b;
        ly |= ((k >> (2 * b + 1)) & 1) << b;
      }
      const int gx = (cx << sh) + lx, gy = (cy << sh) + ly;
      const vvcg_cu_rec rec = P.cus[gy * P.grid_w + gx];
      // residuals of the three TBs
      for (int c = 0; c < (cf ? 3 : 1); c++) {
        const int w = c ? P.tb_cw : tb, h = c ? P.tb_ch : tb;
        int16_t* res = c == 0 ? W.res_y : (c == 1 ? res_c0 : res_c1);
        const int off = rec.level_off[c];
        const bool has = ((rec.cbf >> c) & 1) && off >= 0;
        if (has && (uint64_t)off + (uint64_t)(w * h) <= n_levels) {
          warp_residual(levels + off, w, h, c ? P.cqp : P.lqp, bd, dq, R, W, res);
        } else {
          if (has && lane == 0) atomicOr(status, kStatusBadRecord);
          for (int i = lane; i < w * h / 2; i += 32) reinterpret_cast<uint32_t*>(res)[i] = 0;
          __syncwarp();
        }
      }
      if (k == 0) {
        int ok = 1;
        if (lane == 0) {
          // once any wait has given up the batch result is void: skip the rest
          ok = (ld_acquire(status) & kStatusTimeout) == 0;
          if (ok && cx > 0) ok = wait_flag(&P.ctu_done[cy * P.ctu_w + cx - 1], epoch, spin_limit);
          if (ok && cy > 0) {
            int tx = cx + 1 < P.ctu_w ? cx + 1 : cx;
            ok = wait_flag(&P.ctu_done[(cy - 1) * P.ctu_w + tx], epoch, spin_limit);
          }
          if (!ok) atomicOr(status, kStatusTimeout);
        }
        __syncwarp();
      }
      const int bx = gx * tb, by = gy * tb;
      const uint32_t order = cu_order(P, gx, gy);
      // luma; the reconstructed block is also kept in W.ct for CCLM
      int16_t* luma_tile = W.ct;
      warp_predict_store(P, 0, bx, by, tb, tb, true, rec.luma_mode <= 69 ? rec.luma_mode : 0, order,
                         W.in, W.res_y, luma_tile);
      if (cf) {
        const int cxp = bx / P.sub_w, cyp = by / P.sub_h;
        const int chm = rec.chroma_mode;
        if (chm >= 81 && chm <= 83) {
          warp_cclm_downsample(P, cxp, cyp, P.tb_cw, P.tb_ch, bx, by, tb, luma_tile, W.in, W.tt);
          for (int c = 1; c <= 2; c++)
            warp_cclm_predict_store(P, c, cxp, cyp, P.tb_cw, P.tb_ch, chm - 81, W.in, W.tt,
                                    c == 1 ? res_c0 : res_c1);
        } else {
          for (int c = 1; c <= 2; c++)
            warp_predict_store(P, c, cxp, cyp, P.tb_cw, P.tb_ch, false, chm <= 69 ? chm : 0, order,
                               W.in, c == 1 ? res_c0 : res_c1, nullptr);
        }
      }
    }
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release(&P.ctu_done[cy * P.ctu_w + cx], epoch);
  }
}

}  // namespace vvcg
