// Reconstruction of the 8..12-bit frame path on the GPU, in two kernels.
//
// k_residual: every coded TB of the batch is dequantised and inverse
// transformed by one warp, with no dependencies between TBs; the int16
// residual goes to the picture's scratch planes (free until SAO runs).
//
// k_recon_rows: a persistent kernel in which every warp walks one CTU row at a
// time. Rows are handed out by an atomic counter, row-major across the
// pictures of the batch, so a warp only ever waits on the row above, which a
// running warp took earlier, and the schedule cannot deadlock. Before each CTU
// the warp waits (bounded) until the row above has finished the CTU
// above-right of it; the left neighbour is its own previous CTU. It then
// predicts every coding unit, adds the residual, clips, stores, and publishes
// the row's progress word.
//
// Follows slice::decode_vvc_frame_picture_with_chroma_qp (slice.rs:4834-4988):
// predict_coded_block_16 / predict_cclm_with_format_16 prediction (intra.cuh),
// dequantize_rect_bd or dequantize_dep_quant_bd (dct.rs:1151, :1191),
// inverse_transform_rect_bd (dct.rs:996) with DCT-II both ways, and the add /
// clip to 0..2^bd-1. All sums are exact in int32, so reassociating the matrix
// products (dp2a pairs) gives the reference's results bit for bit.
#pragma once
#include "intra.cuh"
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

constexpr int kWarpsPerCta = 8;
constexpr int kTS = 34;  // row stride (int16) of the transposed coefficient tiles

struct ResidWs {
  int16_t ct[32 * kTS];  // coefficients, transposed: ct[col * kTS + row]
  int16_t tt[32 * kTS];  // stage-1 output, transposed: tt[row * kTS + col]
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

// sum_k M[k][j] * v[k] for k < 4*ng, v given as int16 pairs (a transposed tile
// row, v[k] at row[k]), M from the lane's registers.
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
// (w, h in {16, 32}) whose levels start at `lv`: int16 raster levels, or with
// kSparse the sparse form (lv[2..] holds nsparse (raster index, level) int16
// pairs, 4-byte aligned). The residual is stored to `out` (int16, row
// stride `ostride`). Rows/columns past the last nonzero level hold zeros and
// are skipped without changing any sum. Returns false when a sparse entry's
// index lies outside the TB or does not rise above the entry before it (the
// entry is skipped).
template <bool kSparse>
__device__ bool warp_residual(const int16_t* __restrict__ lv, int w, int h, int qp_scaled, int bd,
                              bool dq, const MatRegs& R, ResidWs& W, int16_t* out, int ostride, int nsparse) {
  const int lane = threadIdx.x & 31;
  const int n = w * h, lw = ilog2(w), lh = ilog2(h);
  const bool s2 = ((lw + lh) & 1) != 0;
  const int tr_shift = 15 - bd - ((lw + lh) >> 1) - (s2 ? 1 : 0);
  int maxr = -1, maxc = -1;
  int lastpos = -1;  // dependent quantisation: largest scan position of a nonzero level
  // All of the TB's levels are fetched up front (streaming 16-byte loads, one
  // round trip), while the coefficient tile is cleared.
  uint4 buf[4];
  const int nvec = n >> 8;  // uint4 per lane: 4 (1024 levels), 2 (512), 1 (256)
  const bool vec_ok = !kSparse && ((reinterpret_cast<uintptr_t>(lv) & 15) == 0) && (n & 255) == 0;
  bool ok = true;
  if (vec_ok) {
    const uint4* lv4 = reinterpret_cast<const uint4*>(lv);
#pragma unroll
    for (int v = 0; v < 4; v++)
      if (v < nvec) buf[v] = __ldcs(lv4 + lane + 32 * v);
  }
  for (int i = lane; i < w * (kTS / 2); i += 32) reinterpret_cast<uint32_t*>(W.ct)[i] = 0;
  __syncwarp();
  // level -> tile (regular dequantisation applied here, dct.rs:1151-1187)
  const int qp = max(4, qp_scaled);
  const int rs = 6 - (tr_shift + qp / 6);
  const int scale = c_inv_quant_scale[s2 ? 1 : 0][qp % 6];
  const int scan_off = g_scan_off[(lw - 1) * 6 + (lh - 1)];
  auto put = [&](int i, int L) {
    int r = i >> lw, c = i & (w - 1);
    maxr = max(maxr, r);
    maxc = max(maxc, c);
    if (dq) lastpos = max(lastpos, (int)g_scan_pos[scan_off + i]);
    int v = L;
    if (!dq) {
      long long val = (long long)L * scale;
      v = clip16(rs > 0 ? (val + (1ll << (rs - 1))) >> rs : val << (-rs));
    }
    W.ct[c * kTS + r] = (int16_t)v;
  };
  if (kSparse) {
    // (raster index, level) pairs, little-endian int16 pairs read as one
    // word; the indices must rise strictly (each checked against the entry
    // before it, so that no two entries land on one coefficient)
    const uint32_t* pr = reinterpret_cast<const uint32_t*>(lv + 2);
    int prev_last = -1;
    for (int base = 0; base < nsparse; base += 32) {
      const int i = base + lane;
      const bool have = i < nsparse;
      const uint32_t e = have ? __ldcs(pr + i) : (uint32_t)n;
      const int pos = (int)(e & 0xFFFFu), L = (int)(int16_t)(e >> 16);
      int prev = __shfl_up_sync(0xffffffffu, pos, 1);
      if (lane == 0) prev = prev_last;
      if (have) {
        if (pos >= n || pos <= prev)
          ok = false;
        else if (L != 0)
          put(pos, L);
      }
      prev_last = __shfl_sync(0xffffffffu, pos, 31);
    }
    ok = __all_sync(0xffffffffu, ok);
  } else if (vec_ok) {
#pragma unroll
    for (int v = 0; v < 4; v++)
      if (v < nvec) {
        uint32_t x0 = buf[v].x, x1 = buf[v].y, x2 = buf[v].z, x3 = buf[v].w;
        if ((x0 | x1 | x2 | x3) == 0) continue;  // 8 zero levels (most of a TB)
#pragma unroll 1
        for (int e = 0; e < 8; e++) {
          int L = (int)(int16_t)(x0 & 0xFFFFu);
          if (L != 0) put(8 * (lane + 32 * v) + e, L);
          x0 = __funnelshift_r(x0, x1, 16);
          x1 = __funnelshift_r(x1, x2, 16);
          x2 = __funnelshift_r(x2, x3, 16);
          x3 >>= 16;
        }
      }
  } else {
    for (int i = lane; i < n; i += 32) {
      int L = lv[i];
      if (L != 0) put(i, L);
    }
  }
  if (dq) {
    // dequantize_dep_quant_bd (dct.rs:1191-1248): the 4-state machine walks the
    // grouped diagonal scan backwards from the last nonzero level. The walk is
    // split into 32 chunks; each lane composes its chunk's state transitions,
    // a warp scan of the compositions gives each chunk's entry state, then
    // every lane replays its chunk.
    // The transitions (32040 >> ((st << 2) + ((L & 1) << 1))) & 3 are: for
    // an even level, swap the two bits of the state (0 1 2 3 -> 0 2 1 3);
    // for an odd one, swap and flip the high bit (-> 2 0 3 1). A chunk's
    // composition of all 4 entry states, packed 2 bits each, therefore
    // updates with a few bit operations per position, in one pass.
    __syncwarp();
    const int16_t* scan = g_scan + scan_off;
    const int last = __reduce_max_sync(0xffffffffu, lastpos);
    if (last >= 0) {
      const int cs = (last + 32) >> 5;
      const int hi = last - lane * cs;
      const int lo = max(hi - cs + 1, 0);
      uint32_t map = 0xE4u;  // entry state s -> field s holds s
      for (int s = hi; s >= lo; s--) {
        int r = scan[s];
        int L = W.ct[(r & (w - 1)) * kTS + (r >> lw)];
        map = (((map & 0x55u) << 1) | ((map >> 1) & 0x55u)) ^ ((L & 1) ? 0xAAu : 0u);
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
        st = (((st & 1) << 1) | (st >> 1)) ^ ((L & 1) << 1);
      }
    }
  }
  maxr = __reduce_max_sync(0xffffffffu, maxr);
  maxc = __reduce_max_sync(0xffffffffu, maxc);
  __syncwarp();
  if (maxr < 0) {  // all levels zero (cbf set without levels): residual 0
    for (int i = lane; i < n / 2; i += 32) {
      int y = (2 * i) >> lw, x = (2 * i) & (w - 1);
      *reinterpret_cast<uint32_t*>(&out[(size_t)y * ostride + x]) = 0;
    }
    return ok;
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
  // tt columns past maxc that stage 2 reads must be zero
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
      out[(size_t)y * ostride + lane] = (int16_t)clip16i((acc + add2) >> sh2);
    }
  } else {
    const int x = lane & 15;
    for (int y0 = 0; y0 < h; y0 += 2) {
      int y = y0 + (lane >> 4);
      int acc = dot_col<16>(R, &W.tt[y * kTS], ngc);
      out[(size_t)y * ostride + x] = (int16_t)clip16i((acc + add2) >> sh2);
    }
  }
  __syncwarp();
  return ok;
}

// One warp per coding unit: the residuals of its coded TBs go to the scratch
// planes at the TB's position. Grid: (ceil(max CUs per picture / 8), pictures).
__global__ void __launch_bounds__(kWarpsPerCta * 32, 4)
k_residual(const DevPic* __restrict__ pics, const int16_t* __restrict__ levels, uint64_t n_levels,
           uint32_t* status) {
  __shared__ ResidWs ws[kWarpsPerCta];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const DevPic& P = pics[blockIdx.y];
  const int cu = blockIdx.x * kWarpsPerCta + wid;
  if (cu >= P.grid_w * P.grid_h) return;
  MatRegs R;
  load_mat_regs(R);
  const vvcg_cu_rec rec = P.cus[cu];
  const int gx = cu % P.grid_w, gy = cu / P.grid_w;
  const bool dq = (P.tools & VVCG_TOOL_DEP_QUANT) != 0;
  const bool sparse = (P.tools & VVCG_TOOL_SPARSE_LEVELS) != 0;
  // TBs with transform skip, MTS or LFNST belong to k_residual_tools
  const uint32_t tu_tools = (P.tools & VVCG_TOOL_TU_TOOLS) ? rec.tu_tools : 0;
  for (int c = 0; c < (P.cf ? 3 : 1); c++) {
    if (!((rec.cbf >> c) & 1)) continue;
    if (((tu_tools >> c) & 1) || (c == 0 && (tu_tools >> VVCG_CU_MTS_SHIFT))) continue;
    const int off = rec.level_off[c];
    if (off < 0) continue;
    const int w = c ? P.tb_cw : P.tb, h = c ? P.tb_ch : P.tb;
    int nsp = -1;
    if (sparse) {  // count at levels[off], pairs from off + 2 (off even)
      nsp = (off & 1) || (uint64_t)off + 2 > n_levels ? -2 : levels[off];
      if (nsp < 0 || nsp > w * h || (uint64_t)off + 2 + 2 * (uint64_t)nsp > n_levels) {
        if (lane == 0) atomicOr(status, kStatusBadRecord);
        continue;
      }
    } else if ((uint64_t)off + (uint64_t)(w * h) > n_levels) {
      if (lane == 0) atomicOr(status, kStatusBadRecord);
      continue;
    }
    const int x0 = c ? gx * P.tb / P.sub_w : gx * P.tb, y0 = c ? gy * P.tb / P.sub_h : gy * P.tb;
    int16_t* out = reinterpret_cast<int16_t*>(P.scratch[c]) + (size_t)y0 * P.stride[c] + x0;
    const bool ok = sparse ? warp_residual<true>(levels + off, w, h, c ? P.cqp : P.lqp, P.bd, dq, R, ws[wid], out,
                                                 P.stride[c], nsp)
                           : warp_residual<false>(levels + off, w, h, c ? P.cqp : P.lqp, P.bd, dq, R, ws[wid], out,
                                                  P.stride[c], 0);
    if (!ok && lane == 0) atomicOr(status, kStatusBadRecord);
  }
}

// Per-warp shared workspace of the wavefront kernel.
struct WaveWs {
  DevPic P;                        // the item's picture, copied once per item
  IntraWs in[3];                   // prediction state per colour component
  int16_t luma[32 * 32];           // the CU's reconstructed luma (for CCLM)
};

// Luma keeps 2 rows / 5 columns for neighbours and CCLM; chroma 1 / 1.
constexpr int kLumaRows = 2, kLumaCols = 5, kChromaRows = 1, kChromaCols = 1;

// Reconstructs one coding unit in `phase` (0 all samples, 1 the samples other
// CUs read, 2 the rest). Phase 1 also prepares the prediction state (refs,
// CCLM models) that phase 2 reuses.
__device__ void recon_cu(const DevPic& P, const vvcg_cu_rec& rec, int gx, int gy, WaveWs& W, int phase) {
  const int tb = P.tb;
  const int bx = gx * tb, by = gy * tb;
  const uint32_t order = cu_order(P, gx, gy);
  auto resid = [&](int c, int x0, int y0) -> const int16_t* {
    return ((rec.cbf >> c) & 1) && rec.level_off[c] >= 0
               ? reinterpret_cast<const int16_t*>(P.scratch[c]) + (size_t)y0 * P.stride[c] + x0
               : nullptr;
  };
  const int lm = rec.luma_mode <= 69 ? rec.luma_mode : 0;
  if (phase != 2) prep_intra(P, 0, bx, by, tb, tb, true, lm, order, W.in[0]);
  emit_intra(P, 0, bx, by, tb, tb, true, lm, W.in[0], resid(0, bx, by), W.luma, phase, kLumaRows,
             kLumaCols);
  if (!P.cf) return;
  const int cxp = bx / P.sub_w, cyp = by / P.sub_h;
  const int cw = P.tb_cw, ch = P.tb_ch;
  const int chm = rec.chroma_mode;
  if (chm >= 81 && chm <= 83) {
    if (phase != 2) prep_cclm(P, cxp, cyp, cw, ch, bx, by, tb, chm - 81, W.in[0], &W.in[1]);
    for (int c = 1; c <= 2; c++)
      emit_cclm(P, c, cxp, cyp, cw, ch, bx, by, tb, W.in[0], W.in[c], W.luma, resid(c, cxp, cyp), phase);
  } else {
    const int cm = chm <= 69 ? chm : 0;
    for (int c = 1; c <= 2; c++) {
      if (phase != 2) prep_intra(P, c, cxp, cyp, cw, ch, false, cm, order, W.in[c]);
      emit_intra(P, c, cxp, cyp, cw, ch, false, cm, W.in[c], resid(c, cxp, cyp), nullptr, phase,
                 kChromaRows, kChromaCols);
    }
  }
}

// Bounded wait until the CTU row above has finished `need` CTUs in this run
// (its progress word is (epoch << 32) | count); false when the poll limit ran out.
__device__ __forceinline__ bool wait_row(const uint64_t* row, uint32_t epoch, uint32_t need,
                                         uint32_t limit) {
  uint32_t ns = 64;
  for (uint32_t it = 0;; it++) {
    const uint64_t v = ld_relaxed64(row);
    if ((uint32_t)(v >> 32) == epoch && (uint32_t)v >= need) {
      fence_acq_rel();
      return true;
    }
    if (it >= limit) return false;
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
  }
}

// The CTU-row wavefront, shared by reconstruction and encoding: one warp per
// CTU row. Rows are handed out by an atomic counter row-major across the
// pictures of the batch, so a warp only ever waits on the row above, which a
// running warp took earlier, and the schedule cannot deadlock. Walking its row
// left to right, the warp codes a CTU once the row above has finished the CTU
// above-right of it (or the last CTU of the row), then publishes its own
// progress. The left neighbour is the warp's own previous CTU, so only the row
// above needs synchronisation. `cu(gx, gy)` codes one CU with W.P set.
template <class Ws, class CuFn>
__device__ __forceinline__ void wavefront_rows(const DevPic* __restrict__ pics, const RowItem* __restrict__ rows,
                                               uint32_t n_rows, uint32_t* counter, uint32_t epoch,
                                               uint32_t spin_limit, uint32_t* status, Ws& W, CuFn&& cu) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    uint32_t it = 0;
    if (lane == 0) it = atomicAdd(counter, 1u);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= n_rows) break;
    const RowItem item = rows[it];
    static_assert(sizeof(DevPic) % 4 == 0 && sizeof(DevPic) <= 64 * 4, "DevPic copy");
    for (int i = lane; i < (int)(sizeof(DevPic) / 4); i += 32)
      reinterpret_cast<uint32_t*>(&W.P)[i] = reinterpret_cast<const uint32_t*>(&pics[item.pic])[i];
    __syncwarp();
    const DevPic& P = W.P;
    const int cy = (int)item.cy;
    const int sh = P.ctu_log2 - ilog2(P.tb);
    const int ncu = 1 << (2 * sh);
    const uint64_t* above = cy > 0 ? P.row_done + (size_t)(cy - 1) * kRowFlagStride : nullptr;
    uint64_t* mine = P.row_done + (size_t)cy * kRowFlagStride;
    uint32_t have = 0;  // CTUs of the row above known to be finished
    for (int cx = 0; cx < P.ctu_w; cx++) {
      if (above) {
        const uint32_t need = (uint32_t)min(cx + 2, P.ctu_w);
        if (have < need) {
          int ok = 1;
          if (lane == 0) {
            // once any wait has given up the batch result is void: skip the rest
            ok = (ld_acquire(status) & kStatusTimeout) == 0 && wait_row(above, epoch, need, spin_limit);
            if (!ok) atomicOr(status, kStatusTimeout);
          }
          ok = __shfl_sync(0xffffffffu, ok, 0);
          __syncwarp();
          have = ok ? need : (uint32_t)P.ctu_w;
        }
      }
      for (int k = 0; k < ncu; k++) {
        int lx = 0, ly = 0;
        for (int b = 0; b < sh; b++) {
          lx |= ((k >> (2 * b)) & 1) << b;
          ly |= ((k >> (2 * b + 1)) & 1) << b;
        }
        cu((cx << sh) + lx, (cy << sh) + ly);
      }
      // publish: every lane's stores are ordered before the progress word
      __threadfence();
      __syncwarp();
      if (lane == 0) st_release64(mine, ((uint64_t)epoch << 32) | (uint32_t)(cx + 1));
    }
  }
}

// Reconstruction wavefront over the batch's CTU rows.
__global__ void __launch_bounds__(kWarpsPerCta * 32, 3)
k_recon_rows(const DevPic* __restrict__ pics, const RowItem* __restrict__ rows, uint32_t n_rows,
             uint32_t* counter, uint32_t epoch, uint32_t spin_limit, uint32_t* status) {
  extern __shared__ __align__(16) unsigned char wave_smem[];
  const int wid = threadIdx.x >> 5;
  WaveWs& W = reinterpret_cast<WaveWs*>(wave_smem)[wid];
  load_cubic_taps();
  wavefront_rows(pics, rows, n_rows, counter, epoch, spin_limit, status, W, [&](int gx, int gy) {
    recon_cu(W.P, W.P.cus[gy * W.P.grid_w + gx], gx, gy, W, 0);
  });
}

}  // namespace vvcg
