// Deblocking of the general decoding path (crates/rustmpeg-video/src/vvc/
// decode_general.rs:4977-5187 apply_deblock) on 4:2:0 16-bit planes.
//
// The reference walks the edges one at a time, gathering each 4-line (luma)
// or 2-line (chroma) segment with clamped coordinates, filtering it and
// writing it back. Here one thread takes one segment, and all segments of one
// direction run at once. That gives the serial result because of the filter
// lengths the transform sizes allow (luma_lens, decode_general.rs:4916):
//  * an edge next to a transform block of 4 or fewer samples has lengths 1/1;
//    it reads p2..q2 and changes at most p0 and q0, so two such edges 4
//    samples apart never meet;
//  * otherwise the block on each side spans 8 (32) or more samples and the
//    edge changes at most 3 (7) samples of it, reading at most 4 (8), which
//    stops short of what the edge on the block's far side changes;
//  * chroma edges are 8 samples apart and change at most 3 samples per side.
// Each segment stores only the samples its filter may change; a sample that
// the gather reached through clamping more than once takes the value of its
// last occurrence, as the reference's in-order write-back leaves it.
#pragma once
#include "filters.cuh"

namespace vvcg {

struct DbkGenArgs {
  uint16_t* plane[3];
  int32_t stride[3];
  int32_t vis_w, vis_h, cw, ch, bd, ctu;
  const vvcg_dbk_cell* cells;
  int32_t cols, rows;
  const vvcg_dbk_ccell* cc;
  int32_t ccols, crows;
  vvcg_dbk_params prm;
};

// the `field` closure of deblock_bs (decode_general.rs:4950-4957) with
// Gen::ref_poc (:497-504, unwrap_or(0))
__device__ __forceinline__ void dbk_field(const vvcg_dbk_cell& c, bool valid, const vvcg_dbk_params& prm, int* mh,
                                          int* mv, int* poc) {
  *mh = *mv = *poc = 0;
  if (!valid) return;
  for (int l = 0; l < 2; l++) {
    const int idx = c.ref_idx[l];
    if (idx >= 0) {
      *mh = c.mv[l][0];
      *mv = c.mv[l][1];
      *poc = (idx < prm.num_ref[l] && idx < 16) ? prm.ref_poc[l][idx] : 0;
      return;
    }
  }
}

// deblock_bs (decode_general.rs:4939-4975) over derive_boundary_strength
// (filter.rs:202-226) for the cells on both sides of a luma edge
__device__ __forceinline__ int dbk_bs(const vvcg_dbk_cell& p, const vvcg_dbk_cell& q, const vvcg_dbk_params& prm) {
  const bool pv = p.flags & VVCG_DBK_CODED, qv = q.flags & VVCG_DBK_CODED;
  if ((pv && (p.flags & VVCG_DBK_INTRA)) || (qv && (q.flags & VVCG_DBK_INTRA))) return 2;
  if ((p.flags & VVCG_DBK_CBF) || (q.flags & VVCG_DBK_CBF)) return 1;  // every edge here is a TU edge
  int ph, pm, pr, qh, qm, qr;
  dbk_field(p, pv, prm, &ph, &pm, &pr);
  dbk_field(q, qv, prm, &qh, &qm, &qr);
  return (pr != qr || abs(ph - qh) >= 8 || abs(pm - qm) >= 8) ? 1 : 0;
}

// One direction of the luma and chroma passes; blockIdx.y is the component.
template <bool kVertical>
__global__ void __launch_bounds__(128) k_dbk_general(const __grid_constant__ DbkGenArgs A) {
  const int comp = blockIdx.y;
  const int maxv = (1 << A.bd) - 1;
  uint16_t* const pl = A.plane[comp];
  const int st = A.stride[comp];
  if (comp == 0) {
    const int w = A.vis_w, h = A.vis_h;
    // edges at 4, 8, .. below the extent; segments every 4 samples along them
    const int n_edges = ((kVertical ? w : h) - 1) / 4, n_segs = ((kVertical ? h : w) + 3) / 4;
    const int qp = clampi(A.prm.qp[0], 0, 63);
    const int beta_off = A.prm.beta_offset_div2[0], tc_off = A.prm.tc_offset_div2[0];
    const int idx_b = clampi(qp + 2 * beta_off, 0, 63);
    const int beta = c_dbf_beta[idx_b] << (A.bd - 8);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n_edges * n_segs; idx += gridDim.x * blockDim.x) {
      const int e = idx / n_segs, s = idx % n_segs;
      const int pos = 4 * (e + 1), seg = 4 * s;
      const int x = kVertical ? pos : seg, y = kVertical ? seg : pos;
      const vvcg_dbk_cell& q = A.cells[(y / 4) * A.cols + x / 4];
      const vvcg_dbk_cell& p = kVertical ? A.cells[(y / 4) * A.cols + x / 4 - 1] : A.cells[(y / 4 - 1) * A.cols + x / 4];
      const uint32_t pid = p.tu_id, qid = q.tu_id;
      if (pid == VVCG_DBK_NO_TU || qid == VVCG_DBK_NO_TU || pid == qid) continue;
      const int bs = dbk_bs(p, q, A.prm);
      if (bs == 0) continue;
      const int idx_tc = clampi(qp + 2 * (bs - 1) + 2 * tc_off, 0, 65);
      const int tc = tc_for(idx_tc, A.bd);
      if (beta == 0 || tc == 0) continue;
      const int sp = kVertical ? p.tu_w : p.tu_h, sq = kVertical ? q.tu_w : q.tu_h;
      int len_p = 1, len_q = 1;  // luma_lens
      if (sp > 4 && sq > 4) {
        len_p = sp >= 32 ? 7 : 3;
        len_q = sq >= 32 ? 7 : 3;
      }
      // line i is the row (column) seg + i, clamped; k runs across the edge
      const int ext = kVertical ? w : h, lim = kVertical ? h : w;
      int ln[4][16];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int a = min(seg + i, lim - 1);
#pragma unroll
        for (int k = 0; k < 16; k++) {
          const int b = clampi(pos - 8 + k, 0, ext - 1);
          ln[i][k] = kVertical ? pl[(size_t)a * st + b] : pl[(size_t)b * st + a];
        }
      }
      LumaEdgeDec dec;
      if (!decide_luma(ln, beta, tc, len_p, len_q, !kVertical && (pos % A.ctu) == 0, &dec)) continue;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        if (dec.de == 3)
          long_tap_line(ln[i], dec.len_p, dec.len_q, tc, maxv);
        else
          short_line(ln[i], dec, tc, maxv);
      }
      // changed positions are 8 - len_p .. 7 + len_q
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int a = min(seg + i, lim - 1);
#pragma unroll
        for (int k = 1; k < 15; k++) {
          if (k < 8 - dec.len_p || k >= 8 + dec.len_q) continue;
          const int b = clampi(pos - 8 + k, 0, ext - 1);
          if (clampi(pos - 7 + k, 0, ext - 1) == b) continue;  // a later k writes this sample
          const uint16_t v = (uint16_t)clampi(ln[i][k], 0, maxv);
          if (kVertical)
            pl[(size_t)a * st + b] = v;
          else
            pl[(size_t)b * st + a] = v;
        }
      }
    }
  } else {
    const int w = A.cw, h = A.ch;
    // edges at 8, 16, .. below the extent; 2-line groups that fit whole
    const int n_edges = ((kVertical ? w : h) - 1) / 8, n_segs = (kVertical ? h : w) / 2;
    const int qp = clampi(A.prm.qp[comp], 0, 63);
    const int idx_b = clampi(qp + 2 * A.prm.beta_offset_div2[comp], 0, 63);
    const int idx_tc = clampi(qp + 2 + 2 * A.prm.tc_offset_div2[comp], 0, 65);  // bS 2
    const int beta = c_dbf_beta[idx_b] << (A.bd - 8);
    const int tc = tc_for(idx_tc, A.bd);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n_edges * n_segs; idx += gridDim.x * blockDim.x) {
      const int e = idx / n_segs, s = idx % n_segs;
      const int pos = 8 * (e + 1), seg = 2 * s;
      const int x = kVertical ? pos : seg, y = kVertical ? seg : pos;
      const vvcg_dbk_ccell& q = A.cc[(y / 2) * A.ccols + x / 2];
      const vvcg_dbk_ccell& p = kVertical ? A.cc[(y / 2) * A.ccols + x / 2 - 1] : A.cc[(y / 2 - 1) * A.ccols + x / 2];
      const uint32_t pid = comp == 1 ? p.tu_cb : p.tu_cr, qid = comp == 1 ? q.tu_cb : q.tu_cr;
      if (pid == VVCG_DBK_NO_TU || qid == VVCG_DBK_NO_TU || pid == qid) continue;
      const int sp = kVertical ? p.tu_w : p.tu_h, sq = kVertical ? q.tu_w : q.tu_h;
      int len_p = 1, len_q = 1;  // chroma_lens
      if (sp >= 8 && sq >= 8) {
        len_p = (!kVertical && (pos % (A.ctu / 2)) == 0) ? 1 : 3;
        len_q = 3;
      }
      const int ext = kVertical ? w : h, lim = kVertical ? h : w;
      int ln[2][8];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int a = min(seg + i, lim - 1);
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int b = clampi(pos - 4 + k, 0, ext - 1);
          ln[i][k] = kVertical ? pl[(size_t)a * st + b] : pl[(size_t)b * st + a];
        }
      }
      chroma_edge_lines(ln, 2, len_p, len_q, tc, beta, maxv);
      // positions 1..6 (p2..q2) may change; chroma edges are 8 samples apart
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int a = min(seg + i, lim - 1);
#pragma unroll
        for (int k = 1; k < 7; k++) {
          const int b = clampi(pos - 4 + k, 0, ext - 1);
          if (clampi(pos - 3 + k, 0, ext - 1) == b) continue;  // a later k writes this sample
          const uint16_t v = (uint16_t)clampi(ln[i][k], 0, maxv);
          if (kVertical)
            pl[(size_t)a * st + b] = v;
          else
            pl[(size_t)b * st + a] = v;
        }
      }
    }
  }
}

}  // namespace vvcg
