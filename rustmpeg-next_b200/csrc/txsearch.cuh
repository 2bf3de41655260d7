// Luma transform search of the 8-bit strict encoder (slice.rs:810-874
// encode_luma, after the prediction): DCT-2, the four explicit MTS pairs and
// the two LFNST kernels are each forward transformed, quantised, dequantised,
// inverse transformed and reconstructed; an MTS or LFNST candidate replaces
// the current best only when its signalling is possible (mts_candidate_ok /
// lfnst_candidate_ok, slice.rs:877-896) and its reconstruction SSE is
// strictly lower, in that order. One CTA per block, one warp per candidate.
#pragma once
#include "tu.cuh"

namespace vvcg {

constexpr int kTxsWarps = 7;

struct TxsWarpWs {
  int32_t A[1024 + kTuPad], B[1024 + kTuPad];
  int16_t levels[1024];
  int16_t samples[1024];
};

struct TxsWs {
  int16_t pred[1024];
  int16_t src[1024];
  unsigned long long sse[kTxsWarps];
  int ok[kTxsWarps];
  int cbf[kTxsWarps];
  TxsWarpWs w[kTxsWarps];
};

// Candidate c of one block: 0 DCT-2, 1..4 mts_idx, 5..6 lfnst_idx 1..2; or
// transform skip (c = 0 with ts). Leaves levels / samples in W and returns
// through ok / cbf / sse whether it may be chosen.
__device__ void txs_candidate(const vvcg_tx_search_req& q, int c, bool ts, TxsWs& S, TxsWarpWs& W, int lane) {
  const int lg = q.log2_size, n = 1 << lg, nn = n * n;
  const int qp = q.qp;
  unsigned sse = 0;  // <= 1024 * 255^2
  bool nz = false;
  if (ts) {
    // slice.rs:671-697 plan_transform_skip
    for (int i = lane; i < nn; i += 32) {
      const int l = tu_quant_ts(S.src[i] - S.pred[i], qp);
      W.levels[i] = (int16_t)l;
      nz |= l != 0;
      const int v = clampi(S.pred[i] + tu_dequant_ts(l, qp), 0, 255);
      W.samples[i] = (int16_t)v;
      const int d = S.src[i] - v;
      sse += (unsigned)(d * d);
    }
  } else {
    // slice.rs:699-760 plan_primary (8-bit)
    vvcg_tu_rec r;
    r.log2_w = r.log2_h = (uint8_t)lg;
    r.bit_depth = 8;
    r.qp = (uint8_t)qp;
    r.flags = 0;
    r.mts_idx = (uint8_t)(c >= 1 && c <= 4 ? c : 0);
    r.lfnst_idx = (uint8_t)(c >= 5 ? c - 4 : 0);
    r.lfnst_mode = q.mode;
    TuShape sh;
    tu_shape(r, sh);
    for (int i = lane; i < nn; i += 32) W.A[(i >> lg) * (n + 1) + (i & (n - 1))] = S.src[i] - S.pred[i];
    __syncwarp();
    tu_forward_transform(W.A, W.B, sh, 8, lane);
    if (r.lfnst_idx) tu_lfnst_forward(W.A, sh, r.lfnst_idx, r.lfnst_mode, lane);
    bool s2;
    const int q4 = max(4, qp);
    const int tr_shift = tu_tr_shift(lg, lg, 8, &s2);
    const int qbits = 14 + q4 / 6 + tr_shift;
    const long long add = 171ll << max(0, qbits - 9);
    const long long qs = c_quant_scale[s2 ? 1 : 0][q4 % 6];
    const int rs = 6 - (tr_shift + q4 / 6);
    const long long iqs = c_inv_quant_scale[s2 ? 1 : 0][q4 % 6];
    for (int i = lane; i < nn; i += 32) {
      const int co = W.A[i];
      const long long a = ((long long)abs(co) * qs + add) >> max(0, qbits);
      const int l = clip16(co < 0 ? -a : a);
      W.levels[i] = (int16_t)l;
      nz |= l != 0;
      const long long v = (long long)l * iqs;
      W.A[i] = clip16(rs > 0 ? (v + (1ll << (rs - 1))) >> rs : v << (-rs));
    }
    __syncwarp();
    if (r.lfnst_idx) tu_lfnst_inverse(W.A, sh, r.lfnst_idx, r.lfnst_mode, lane);
    tu_inverse_transform(W.A, W.B, sh, 8, lane);
    for (int i = lane; i < nn; i += 32) {
      const int v = clampi(S.pred[i] + W.A[i], 0, 255);
      W.samples[i] = (int16_t)v;
      const int d = S.src[i] - v;
      sse += (unsigned)(d * d);
    }
  }
  const bool cbf = __any_sync(0xffffffffu, nz);
  sse = __reduce_add_sync(0xffffffffu, sse);
  __syncwarp();
  // scan_pos_last (slice.rs:935-939) and the signalling checks
  int last = -1;
  bool violates = false;
  const int16_t* scan = tu_scan(lg, lg);
  for (int s = lane; s < nn; s += 32) {
    const int ri = scan[s];
    if (W.levels[ri] != 0) {
      last = max(last, s);
      if ((ri & (n - 1)) >= 16 || (ri >> lg) >= 16) violates = true;
    }
  }
  last = __reduce_max_sync(0xffffffffu, last);
  violates = __any_sync(0xffffffffu, violates);
  bool ok = true;
  if (c >= 1 && c <= 4) ok = cbf && last >= 1 && !violates;
  if (c >= 5) ok = cbf && last >= 1 && last <= ((n == 4 || n == 8) ? 7 : 15);
  if (lane == 0) {
    S.sse[c] = sse;
    S.ok[c] = ok;
    S.cbf[c] = cbf;
  }
}

// Grid: one CTA (7 warps) per request.
__global__ void __launch_bounds__(kTxsWarps * 32)
k_luma_tx_search(const vvcg_tx_search_req* __restrict__ reqs, const int16_t* __restrict__ pred,
                 const int16_t* __restrict__ src, int16_t* __restrict__ levels, int16_t* __restrict__ samples,
                 vvcg_tx_search_res* __restrict__ res) {
  extern __shared__ __align__(16) unsigned char txs_smem[];
  TxsWs& S = *reinterpret_cast<TxsWs*>(txs_smem);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const vvcg_tx_search_req q = reqs[blockIdx.x];
  const int n = 1 << q.log2_size, nn = n * n;
  for (int i = threadIdx.x; i < nn; i += blockDim.x) {
    S.pred[i] = pred[q.in_off + i];
    S.src[i] = src[q.in_off + i];
  }
  __syncthreads();
  const bool ts = (q.flags & VVCG_TXS_TRANSFORM_SKIP) != 0;
  const bool lfnst = (q.flags & VVCG_TXS_LFNST) != 0;
  const bool active = ts ? wid == 0 : (wid <= 4 || lfnst);
  if (active) txs_candidate(q, wid, ts, S, S.w[wid], lane);
  __syncthreads();
  int best = 0;
  if (!ts) {
    for (int c = 1; c <= (lfnst ? 6 : 4); c++)
      if (S.ok[c] && S.sse[c] < S.sse[best]) best = c;
  }
  const TxsWarpWs& B = S.w[best];
  for (int i = threadIdx.x; i < nn; i += blockDim.x) {
    levels[q.out_off + i] = B.levels[i];
    samples[q.out_off + i] = B.samples[i];
  }
  if (threadIdx.x == 0) {
    vvcg_tx_search_res r;
    r.sse = S.sse[best];
    r.mts_idx = (uint8_t)(best >= 1 && best <= 4 ? best : 0);
    r.lfnst_idx = (uint8_t)(best >= 5 ? best - 4 : 0);
    r.transform_skip = ts ? 1 : 0;
    r.cbf = (uint8_t)S.cbf[best];
    r.reserved = 0;
    res[blockIdx.x] = r;
  }
}

}  // namespace vvcg
