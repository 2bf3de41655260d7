// The frame-path encoder of libvvcg (sm_100a): slice::encode_vvc_frame_picture
// (crates/rustmpeg-video/src/vvc/slice.rs:4171-4634) without its CABAC writes.
// Each CU is coded by one warp inside the CTU-row wavefront: the 7-mode luma
// SAD decision, prediction, forward DCT-2, regular or dependent quantisation
// and the encoder's own reconstruction, then the chroma mode decision (DM or
// CCLM by SAD) and the same chain for Cb and Cr. The reconstruction feeds the
// next CUs' predictions, exactly as the reference's sequential CTU loop does.
#pragma once
#include "intra.cuh"
#include "recon.cuh"
#include "tu.cuh"

namespace vvcg {

constexpr int kEncWarps = 4;

// Per-warp shared workspace of the encoder.
struct EncWs {
  DevPic P;
  IntraWs in[3];
  int16_t luma[32 * 32];  // the CU's reconstructed luma (CCLM)
  int16_t src[32 * 32];   // source samples of the block being coded
  int16_t pred[32 * 32];  // prediction of the block being coded
  int32_t A[1024 + kTuPad], B[1024 + kTuPad];  // transform tiles
};

// Source block of component c (coded-size source copy in P.scratch) into dst
// (raster, width w).
__device__ __forceinline__ void load_src(const DevPic& P, int c, int x0, int y0, int w, int h, int16_t* dst) {
  const int lane = threadIdx.x & 31;
  const int lw = ilog2(w), st = P.stride[c];
  const uint16_t* base = P.scratch[c] + (size_t)y0 * st + x0;
  for (int q = lane; q < (w * h) >> 1; q += 32) {
    const int y = (2 * q) >> lw, x = (2 * q) & (w - 1);
    *reinterpret_cast<uint32_t*>(&dst[2 * q]) = *reinterpret_cast<const uint32_t*>(base + (size_t)y * st + x);
  }
  __syncwarp();
}

// Sum of absolute differences of two int16 rasters of n samples (< 2^32 for
// n <= 1024 and 12-bit samples).
__device__ __forceinline__ uint32_t block_sad(const int16_t* a, const int16_t* b, int n) {
  const int lane = threadIdx.x & 31;
  uint32_t s = 0;
  for (int i = lane; i < n; i += 32) s += (uint32_t)abs((int)(uint16_t)a[i] - (int)(uint16_t)b[i]);
  return __reduce_add_sync(0xffffffffu, s);
}

// Forward transform, quantisation and the encoder's own reconstruction of one
// TB (slice.rs:4298-4346 for luma, :4442-4553 for chroma): DCT-2 both ways,
// no zero-out at these sizes, intra rounding offset. Writes the levels to
// lv_out when any is nonzero and the reconstruction to the plane (and keep).
// Returns the cbf.
__device__ bool code_block(const DevPic& P, int comp, int x0, int y0, int w, int h, int qp, bool dq,
                           const int16_t* src, const int16_t* pred, int32_t* A, int32_t* B, int16_t* lv_out,
                           int16_t* keep) {
  const int lane = threadIdx.x & 31;
  const int bd = P.bd;
  TuShape S;
  S.w = w;
  S.h = h;
  S.lw = ilog2(w);
  S.lh = ilog2(h);
  S.n = w * h;
  S.th = S.tv = 0;
  S.sw = S.sh = 0;
  const int n = S.n, ws = w + 1;
  for (int i = lane; i < n; i += 32)
    A[(i >> S.lw) * ws + (i & (w - 1))] = (int)(uint16_t)src[i] - (int)(uint16_t)pred[i];
  __syncwarp();
  tu_forward_transform(A, B, S, bd, lane);
  if (dq) {
    tu_dq_quant(A, S, qp, bd, A, lane);
  } else {
    // dct.rs:1113-1147 quantize_rect_bd, intra offset
    const int q = max(4, qp);
    bool s2;
    const int tr_shift = tu_tr_shift(S.lw, S.lh, bd, &s2);
    const int qbits = 14 + q / 6 + tr_shift;
    const long long add = 171ll << max(0, qbits - 9);
    const long long scale = c_quant_scale[s2 ? 1 : 0][q % 6];
    for (int i = lane; i < n; i += 32) {
      const int c = A[i];
      const long long lv = ((long long)abs(c) * scale + add) >> max(0, qbits);
      A[i] = clip16(c < 0 ? -lv : lv);
    }
  }
  __syncwarp();
  bool nz = false;
  for (int i = lane; i < n; i += 32) nz |= A[i] != 0;
  const bool cbf = __any_sync(0xffffffffu, nz);
  if (cbf) {
    for (int i = lane; i < n; i += 32) lv_out[i] = (int16_t)A[i];
    if (dq) {
      tu_dq_dequant(A, S, qp, bd, lane);
    } else {
      // dct.rs:1151-1187 dequantize_rect_bd
      const int q = max(4, qp);
      bool s2;
      const int tr_shift = tu_tr_shift(S.lw, S.lh, bd, &s2);
      const int rs = 6 - (tr_shift + q / 6);
      const long long scale = c_inv_quant_scale[s2 ? 1 : 0][q % 6];
      for (int i = lane; i < n; i += 32) {
        const long long v = (long long)A[i] * scale;
        A[i] = clip16(rs > 0 ? (v + (1ll << (rs - 1))) >> rs : v << (-rs));
      }
      __syncwarp();
    }
    tu_inverse_transform(A, B, S, bd, lane);
  }
  // reconstruction: clip(pred + residual); a TB without levels adds zeros
  const int maxv = (1 << bd) - 1;
  const int st = P.stride[comp];
  uint16_t* base = P.plane[comp] + (size_t)y0 * st + x0;
  for (int q = lane; q < n >> 1; q += 32) {
    const int i = 2 * q, y = i >> S.lw, x = i & (w - 1);
    const int v0 = clampi((int)(uint16_t)pred[i] + (cbf ? A[i] : 0), 0, maxv);
    const int v1 = clampi((int)(uint16_t)pred[i + 1] + (cbf ? A[i + 1] : 0), 0, maxv);
    const uint32_t pk = (uint32_t)v0 | ((uint32_t)v1 << 16);
    *reinterpret_cast<uint32_t*>(base + (size_t)y * st + x) = pk;
    if (keep) *reinterpret_cast<uint32_t*>(&keep[i]) = pk;
  }
  __syncwarp();
  return cbf;
}

// Luma candidates of choose_intra_mode_16 (predict.rs:4069-4105), in order:
// a later candidate wins only with a strictly lower SAD.
__device__ __forceinline__ int enc_candidate(int c) {
  return c == 0 ? 0 : c == 1 ? 1 : c == 2 ? 18 : c == 3 ? 50 : c == 4 ? 2 : c == 5 ? 34 : 66;
}

// One CU of slice::encode_vvc_frame_picture (slice.rs:4240-4560).
__device__ void encode_cu(const DevPic& P, int gx, int gy, EncWs& W) {
  const int lane = threadIdx.x & 31;
  const int tb = P.tb, bx = gx * tb, by = gy * tb;
  const uint32_t order = cu_order(P, gx, gy);
  const bool dq = (P.tools & VVCG_TOOL_DEP_QUANT) != 0;
  const int k = gy * P.grid_w + gx;
  const int cw = P.tb_cw, ch = P.tb_ch;
  const int32_t off0 = P.lv_base + k * (tb * tb + 2 * cw * ch);
  int16_t* lv = P.lv_pool + off0;
  // slice.rs:4264-4274: luma mode by SAD of the plain prediction against the source
  load_src(P, 0, bx, by, tb, tb, W.src);
  int best = 0;
  uint32_t best_sad = 0xffffffffu;
  for (int c = 0; c < 7; c++) {
    const int mode = enc_candidate(c);
    prep_intra(P, 0, bx, by, tb, tb, true, mode, order, W.in[0], true);
    emit_intra(P, 0, bx, by, tb, tb, true, mode, W.in[0], nullptr, W.pred, 0, 0, 0, false);
    const uint32_t sad = block_sad(W.src, W.pred, tb * tb);
    if (sad < best_sad) {
      best_sad = sad;
      best = mode;
    }
  }
  const int luma_mode = (P.tools & VVCG_TOOL_ENC_FULL_INTRA) ? best : (best <= 1 ? best : 0);
  prep_intra(P, 0, bx, by, tb, tb, true, luma_mode, order, W.in[0]);
  emit_intra(P, 0, bx, by, tb, tb, true, luma_mode, W.in[0], nullptr, W.pred, 0, 0, 0, false);
  const bool cbf_y = code_block(P, 0, bx, by, tb, tb, P.lqp, dq, W.src, W.pred, W.A, W.B, lv, W.luma);
  int chroma_mode = luma_mode;
  bool cbf_c[2] = {false, false};
  if (P.cf) {
    const int cxp = bx / P.sub_w, cyp = by / P.sub_h;
    if (P.tools & VVCG_TOOL_ENC_CCLM) {
      // slice.rs:4362-4397: DM (plain prediction) against LM / LM-L / LM-T on Cb
      load_src(P, 1, cxp, cyp, cw, ch, W.src);
      prep_intra(P, 1, cxp, cyp, cw, ch, false, luma_mode, order, W.in[1], true);
      emit_intra(P, 1, cxp, cyp, cw, ch, false, luma_mode, W.in[1], nullptr, W.pred, 0, 0, 0, false);
      uint32_t bsad = block_sad(W.src, W.pred, cw * ch);
      for (int m = 0; m < 3; m++) {
        prep_cclm(P, cxp, cyp, cw, ch, bx, by, tb, m, W.in[0], &W.in[1]);
        emit_cclm(P, 1, cxp, cyp, cw, ch, bx, by, tb, W.in[0], W.in[1], W.luma, nullptr, 0, W.pred, false);
        const uint32_t sad = block_sad(W.src, W.pred, cw * ch);
        if (sad < bsad) {
          bsad = sad;
          chroma_mode = 81 + m;
        }
      }
    }
    const bool cclm = chroma_mode >= 81 && chroma_mode <= 83;
    if (cclm) prep_cclm(P, cxp, cyp, cw, ch, bx, by, tb, chroma_mode - 81, W.in[0], &W.in[1]);
    const int cm = chroma_mode <= 69 ? chroma_mode : 0;
    for (int c = 1; c <= 2; c++) {
      load_src(P, c, cxp, cyp, cw, ch, W.src);
      if (cclm) {
        emit_cclm(P, c, cxp, cyp, cw, ch, bx, by, tb, W.in[0], W.in[c], W.luma, nullptr, 0, W.pred, false);
      } else {
        prep_intra(P, c, cxp, cyp, cw, ch, false, cm, order, W.in[c]);
        emit_intra(P, c, cxp, cyp, cw, ch, false, cm, W.in[c], nullptr, W.pred, 0, 0, 0, false);
      }
      cbf_c[c - 1] = code_block(P, c, cxp, cyp, cw, ch, P.cqp, dq, W.src, W.pred, W.A, W.B,
                                lv + tb * tb + (c - 1) * cw * ch, nullptr);
    }
  }
  if (lane == 0) {
    vvcg_cu_rec r;
    r.luma_mode = (uint8_t)luma_mode;
    r.chroma_mode = (uint8_t)chroma_mode;
    r.cbf = (uint8_t)((cbf_y ? 1 : 0) | (cbf_c[0] ? 2 : 0) | (cbf_c[1] ? 4 : 0));
    r.tu_tools = 0;
    r.level_off[0] = cbf_y ? off0 : -1;
    r.level_off[1] = cbf_c[0] ? off0 + tb * tb : -1;
    r.level_off[2] = cbf_c[1] ? off0 + tb * tb + cw * ch : -1;
    const_cast<vvcg_cu_rec*>(P.cus)[k] = r;
  }
  __syncwarp();
}

// Encoder wavefront over the batch's CTU rows.
__global__ void __launch_bounds__(kEncWarps * 32, 2)
k_encode_rows(const DevPic* __restrict__ pics, const RowItem* __restrict__ rows, uint32_t n_rows,
              uint32_t* counter, uint32_t epoch, uint32_t spin_limit, uint32_t* status) {
  extern __shared__ __align__(16) unsigned char enc_smem[];
  const int wid = threadIdx.x >> 5;
  EncWs& W = reinterpret_cast<EncWs*>(enc_smem)[wid];
  load_cubic_taps();
  wavefront_rows(pics, rows, n_rows, counter, epoch, spin_limit, status, W,
                 [&](int gx, int gy) { encode_cu(W.P, gx, gy, W); });
}

}  // namespace vvcg
