// In-loop filters of the frame path on 16-bit planes: deblocking (vertical
// edges, then horizontal edges), SAO and ALF. Each follows the reference
// function named beside it (crates/rustmpeg-video/src/vvc/filter.rs) and is
// bit-identical to it. Edge segments of one direction never read samples that
// another segment of the same direction writes (edges are at least 8 samples
// apart and a segment writes at most 7 samples on each side, reading 8), so
// each direction runs fully parallel and matches the reference's serial scan.
#pragma once
#include "tma.cuh"
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

__device__ __forceinline__ int tc_for(int idx, int bd) {
  return bd < 10 ? (c_dbf_tc[idx] + (1 << (9 - bd))) >> (10 - bd) : c_dbf_tc[idx] << (bd - 10);
}

struct LumaEdgeDec {
  int de, len_p, len_q;
  bool dep, deq;
};

#define LP(l, i) ((l)[7 - (i)])
#define LQ(l, j) ((l)[8 + (j)])

// filter.rs:282-305 luma_sample_decision
__device__ __forceinline__ bool luma_sample_dec(int p0, int p3, int q0, int q3, int dpq, int sp,
                                                int sq, int spq, bool lp, bool lq, int beta, int tc) {
  if (lp) sp = (sp + abs(p3 - p0) + 1) >> 1;
  if (lq) sq = (sq + abs(q3 - q0) + 1) >> 1;
  int t1 = (lp || lq) ? (3 * beta) >> 5 : beta >> 3;
  int t2 = (lp || lq) ? beta >> 4 : beta >> 2;
  return dpq < t2 && sp + sq < t1 && spq < ((5 * tc + 1) >> 1);
}

// filter.rs:311-468 decide_luma_edge
__device__ __forceinline__ bool decide_luma(const int (*ln)[16], int beta, int tc, int lpi, int lqi, bool ctb_hor,
                            LumaEdgeDec* e) {
  const int* l0 = ln[0];
  const int* l3 = ln[3];
  int dp0 = abs(LP(l0, 2) - 2 * LP(l0, 1) + LP(l0, 0)), dp3 = abs(LP(l3, 2) - 2 * LP(l3, 1) + LP(l3, 0));
  int dq0 = abs(LQ(l0, 2) - 2 * LQ(l0, 1) + LQ(l0, 0)), dq3 = abs(LQ(l3, 2) - 2 * LQ(l3, 1) + LQ(l3, 0));
  int dpq0 = dp0 + dq0, dpq3 = dp3 + dq3;
  int sp0 = abs(LP(l0, 3) - LP(l0, 0)), sp3 = abs(LP(l3, 3) - LP(l3, 0));
  int sq0 = abs(LQ(l0, 0) - LQ(l0, 3)), sq3 = abs(LQ(l3, 0) - LQ(l3, 3));
  int spq0 = abs(LP(l0, 0) - LQ(l0, 0)), spq3 = abs(LP(l3, 0) - LQ(l3, 0));
  int len_p = clampi(lpi, 1, 7), len_q = clampi(lqi, 1, 7);
  bool lp = len_p > 3 && !ctb_hor, lq = len_q > 3;
  if (lp || lq) {
    int dp0l = lp ? (dp0 + abs(LP(l0, 5) - 2 * LP(l0, 4) + LP(l0, 3)) + 1) >> 1 : dp0;
    int dp3l = lp ? (dp3 + abs(LP(l3, 5) - 2 * LP(l3, 4) + LP(l3, 3)) + 1) >> 1 : dp3;
    int dq0l = lq ? (dq0 + abs(LQ(l0, 5) - 2 * LQ(l0, 4) + LQ(l0, 3)) + 1) >> 1 : dq0;
    int dq3l = lq ? (dq3 + abs(LQ(l3, 5) - 2 * LQ(l3, 4) + LQ(l3, 3)) + 1) >> 1 : dq3;
    if (!lp) len_p = 3;
    if (!lq) len_q = 3;
    int sp0l = len_p == 7 ? sp0 + abs(LP(l0, 7) - LP(l0, 6) - LP(l0, 5) + LP(l0, 4)) : sp0;
    int sp3l = len_p == 7 ? sp3 + abs(LP(l3, 7) - LP(l3, 6) - LP(l3, 5) + LP(l3, 4)) : sp3;
    int sq0l = len_q == 7 ? sq0 + abs(LQ(l0, 4) - LQ(l0, 5) - LQ(l0, 6) + LQ(l0, 7)) : sq0;
    int sq3l = len_q == 7 ? sq3 + abs(LQ(l3, 4) - LQ(l3, 5) - LQ(l3, 6) + LQ(l3, 7)) : sq3;
    int d0l = dp0l + dq0l, d3l = dp3l + dq3l;
    if (d0l + d3l < beta) {
      // len_p / len_q are 3, 5 or 7 here
      auto at_p = [&](const int* l) { return len_p == 7 ? LP(l, 7) : len_p == 5 ? LP(l, 5) : LP(l, 3); };
      auto at_q = [&](const int* l) { return len_q == 7 ? LQ(l, 7) : len_q == 5 ? LQ(l, 5) : LQ(l, 3); };
      bool s0 = luma_sample_dec(lp ? at_p(l0) : 0, lp ? LP(l0, 3) : 0, lq ? at_q(l0) : 0,
                                lq ? LQ(l0, 3) : 0, 2 * d0l, sp0l, sq0l, spq0, lp, lq, beta, tc);
      bool s3 = luma_sample_dec(lp ? at_p(l3) : 0, lp ? LP(l3, 3) : 0, lq ? at_q(l3) : 0,
                                lq ? LQ(l3, 3) : 0, 2 * d3l, sp3l, sq3l, spq3, lp, lq, beta, tc);
      if (s0 && s3) {
        *e = LumaEdgeDec{3, len_p, len_q, true, true};
        return true;
      }
    }
  }
  int dp = dp0 + dp3, dq = dq0 + dq3;
  if (dpq0 + dpq3 >= beta) return false;
  bool s0 = false, s3 = false;
  if (len_p > 2 && len_q > 2) {
    s0 = luma_sample_dec(0, 0, 0, 0, 2 * dpq0, sp0, sq0, spq0, false, false, beta, tc);
    s3 = luma_sample_dec(0, 0, 0, 0, 2 * dpq3, sp3, sq3, spq3, false, false, beta, tc);
  }
  int de = 1;
  if (s0 && s3) {
    de = 2;
    len_p = 3;
    len_q = 3;
  }
  int thr = (beta + (beta >> 1)) >> 3;
  bool dep = len_p > 1 && len_q > 1 && dp < thr;
  bool deq = len_p > 1 && len_q > 1 && dq < thr;
  if (de == 1) {
    len_p = 1 + (dep ? 1 : 0);
    len_q = 1 + (deq ? 1 : 0);
  }
  *e = LumaEdgeDec{de, len_p, len_q, dep, deq};
  return true;
}

// filter.rs:477-582 long_tap_luma_line (in place on a 16-sample line)
__device__ __forceinline__ void long_tap_line(int* l, int np, int nq, int tc, int maxv) {
  int m[16];
#pragma unroll
  for (int i = 0; i < 16; i++) m[i] = l[i];
#define MP(i) m[7 - (i)]
#define MQ(j) m[8 + (j)]
  int rm;
  if (np == 5 && nq == 5)
    rm = (2 * (MP(0) + MQ(0) + MP(1) + MQ(1) + MP(2) + MQ(2)) + MP(3) + MQ(3) + MP(4) + MQ(4) + 8) >> 4;
  else if ((np == 7 && nq == 5) || (np == 5 && nq == 7))
    rm = (2 * (MP(0) + MQ(0) + MP(1) + MQ(1)) + MP(2) + MQ(2) + MP(3) + MQ(3) + MP(4) + MQ(4) +
          MP(5) + MQ(5) + 8) >> 4;
  else if ((np == 5 && nq == 3) || (np == 3 && nq == 5))
    rm = (MP(0) + MQ(0) + MP(1) + MQ(1) + MP(2) + MQ(2) + MP(3) + MQ(3) + 4) >> 3;
  else if (np == 7 && nq == 3)
    rm = (2 * (MP(0) + MQ(0)) + MQ(0) + 2 * (MQ(1) + MQ(2)) + MP(1) + MQ(1) + MP(2) + MP(3) + MP(4) +
          MP(5) + MP(6) + 8) >> 4;
  else if (np == 3 && nq == 7)
    rm = (2 * (MP(0) + MQ(0)) + MP(0) + 2 * (MP(1) + MP(2)) + MP(1) + MQ(1) + MQ(2) + MQ(3) + MQ(4) +
          MQ(5) + MQ(6) + 8) >> 4;
  else
    rm = (2 * (MP(0) + MQ(0)) + MP(1) + MQ(1) + MP(2) + MQ(2) + MP(3) + MQ(3) + MP(4) + MQ(4) +
          MP(5) + MQ(5) + MP(6) + MQ(6) + 8) >> 4;
  // lengths are 3, 5 or 7: every index below is a compile-time constant
  const int ref_p = np == 7 ? (MP(7) + MP(6) + 1) >> 1 : np == 5 ? (MP(5) + MP(4) + 1) >> 1 : (MP(3) + MP(2) + 1) >> 1;
  const int ref_q = nq == 7 ? (MQ(7) + MQ(6) + 1) >> 1 : nq == 5 ? (MQ(5) + MQ(4) + 1) >> 1 : (MQ(3) + MQ(2) + 1) >> 1;
  const int c7[7] = {59, 50, 41, 32, 23, 14, 5}, t7[7] = {6, 5, 4, 3, 2, 1, 1};
  const int c5[7] = {58, 45, 32, 19, 6, 0, 0}, t5[7] = {6, 5, 4, 3, 2, 0, 0};
  const int c3[7] = {53, 32, 11, 0, 0, 0, 0}, t3[7] = {6, 4, 2, 0, 0, 0, 0};
#pragma unroll
  for (int pos = 0; pos < 7; pos++) {
    if (pos < np) {
      int f = np == 7 ? c7[pos] : (np == 5 ? c5[pos] : c3[pos]);
      int t = np == 7 ? t7[pos] : (np == 5 ? t5[pos] : t3[pos]);
      int o = MP(pos), cv = (tc * t) >> 1;
      int it = (rm * f + ref_p * (64 - f) + 32) >> 6;
      l[7 - pos] = clampi(clampi(it, o - cv, o + cv), 0, maxv);
    }
    if (pos < nq) {
      int f = nq == 7 ? c7[pos] : (nq == 5 ? c5[pos] : c3[pos]);
      int t = nq == 7 ? t7[pos] : (nq == 5 ? t5[pos] : t3[pos]);
      int o = MQ(pos), cv = (tc * t) >> 1;
      int it = (rm * f + ref_q * (64 - f) + 32) >> 6;
      l[8 + pos] = clampi(clampi(it, o - cv, o + cv), 0, maxv);
    }
  }
#undef MP
#undef MQ
}

// filter.rs:586-631 short_filter_luma_line
__device__ __forceinline__ void short_line(int* l, const LumaEdgeDec& e, int tc, int maxv) {
  int m[16];
#pragma unroll
  for (int i = 0; i < 16; i++) m[i] = l[i];
  if (e.de == 2) {
    l[7] = clampi((LP(m, 2) + 2 * LP(m, 1) + 2 * LP(m, 0) + 2 * LQ(m, 0) + LQ(m, 1) + 4) >> 3,
                  LP(m, 0) - 3 * tc, LP(m, 0) + 3 * tc);
    l[6] = clampi((LP(m, 2) + LP(m, 1) + LP(m, 0) + LQ(m, 0) + 2) >> 2, LP(m, 1) - 2 * tc,
                  LP(m, 1) + 2 * tc);
    l[5] = clampi((2 * LP(m, 3) + 3 * LP(m, 2) + LP(m, 1) + LP(m, 0) + LQ(m, 0) + 4) >> 3,
                  LP(m, 2) - tc, LP(m, 2) + tc);
    l[8] = clampi((LP(m, 1) + 2 * LP(m, 0) + 2 * LQ(m, 0) + 2 * LQ(m, 1) + LQ(m, 2) + 4) >> 3,
                  LQ(m, 0) - 3 * tc, LQ(m, 0) + 3 * tc);
    l[9] = clampi((LP(m, 0) + LQ(m, 0) + LQ(m, 1) + LQ(m, 2) + 2) >> 2, LQ(m, 1) - 2 * tc,
                  LQ(m, 1) + 2 * tc);
    l[10] = clampi((LP(m, 0) + LQ(m, 0) + LQ(m, 1) + 3 * LQ(m, 2) + 2 * LQ(m, 3) + 4) >> 3,
                   LQ(m, 2) - tc, LQ(m, 2) + tc);
    return;
  }
  int delta = (9 * (LQ(m, 0) - LP(m, 0)) - 3 * (LQ(m, 1) - LP(m, 1)) + 8) >> 4;
  if (abs(delta) >= tc * 10) return;
  delta = clampi(delta, -tc, tc);
  l[7] = clampi(LP(m, 0) + delta, 0, maxv);
  l[8] = clampi(LQ(m, 0) - delta, 0, maxv);
  int tc2 = tc >> 1;
  if (e.dep) {
    int d = clampi((((LP(m, 2) + LP(m, 0) + 1) >> 1) - LP(m, 1) + delta) >> 1, -tc2, tc2);
    l[6] = clampi(LP(m, 1) + d, 0, maxv);
  }
  if (e.deq) {
    int d = clampi((((LQ(m, 2) + LQ(m, 0) + 1) >> 1) - LQ(m, 1) - delta) >> 1, -tc2, tc2);
    l[9] = clampi(LQ(m, 1) + d, 0, maxv);
  }
}

// Picture-level parameters of one deblocking pass over one plane.
struct DbfPass {
  uint16_t* plane;
  int32_t stride, w, h, bd;
  int32_t step, ctb, qp, bs, beta_off, tc_off;
  int32_t len_p, len_q;  // luma: max filter length; chroma: lengths from the lattice
  int32_t sub;           // chroma: SubHeightC (vertical pass) / SubWidthC (horizontal pass)
  int32_t n_edges, n_segs;
  // Per-edge boundary strength on a CTU lattice (step = the CTU size in this
  // plane) instead of `bs`: cells of the CTUs (cell_cols per row), the cbf
  // bit of this plane, and this plane's samples per CTU along an edge.
  const vvcg_ctu_motion* cells;
  int32_t cell_cols, comp, span;
};

// derive_boundary_strength (filter.rs:202-226) of a CTU edge of an inter
// picture (not intra, a transform edge) between CTU cells p and q, reading
// motion entry pk of p and qk of q (0 top-left, 1 top-right, 2 bottom-left).
__device__ __forceinline__ int ctu_edge_bs(const vvcg_ctu_motion& p, int pk, const vvcg_ctu_motion& q, int qk,
                                           int comp) {
  if (((p.cbf | q.cbf) >> comp) & 1) return 1;
  if (p.ref[pk] != q.ref[qk] || abs(p.mv[pk][0] - q.mv[qk][0]) >= 8 || abs(p.mv[pk][1] - q.mv[qk][1]) >= 8)
    return 1;
  return 0;
}

// Boundary strength of segment position `seg` on edge e of pass D: the
// pass's constant, or from the CTU cells either side of a CTU-lattice edge
// (slice.rs:2319-2334 for vertical, :2438-2452 for horizontal edges).
template <bool kVertical>
__device__ __forceinline__ int pass_bs(const DbfPass& D, int e, int seg) {
  if (!D.cells) return D.bs;
  const int along = seg / D.span;
  if (kVertical) {
    const vvcg_ctu_motion* row = D.cells + (size_t)along * D.cell_cols;
    return ctu_edge_bs(row[e], 1, row[e + 1], 0, D.comp);
  }
  return ctu_edge_bs(D.cells[(size_t)e * D.cell_cols + along], 2, D.cells[(size_t)(e + 1) * D.cell_cols + along], 0,
                     D.comp);
}

// deblock_luma_edge_bd (filter.rs:638-679) on the segment's 4 lines;
// vertical edges (filter.rs:2360-2390) or horizontal edges (:2392-2425) of
// deblock_luma_plane_16. One thread per 4-line segment.
template <bool kVertical>
__global__ void k_deblock_luma(const DbfPass* __restrict__ passes, int n_pass) {
  const DbfPass& D = passes[blockIdx.y];
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= D.n_edges * D.n_segs) return;
  int e = idx / D.n_segs, s = idx % D.n_segs;
  int pos = D.step * (e + 1);  // edge x (vertical) or y (horizontal)
  int seg = s * 4;
  int bd = D.bd, maxv = (1 << bd) - 1;
  int qp = D.qp;
  const int bs = pass_bs<kVertical>(D, e, seg);
  int idx_tc = clampi(qp + 2 * (bs - 1) + 2 * D.tc_off, 0, 65);
  int idx_b = clampi(qp + 2 * D.beta_off, 0, 63);
  int tc = tc_for(idx_tc, bd);
  int beta = c_dbf_beta[idx_b] << (bd - 8);
  if (bs == 0 || beta == 0 || tc == 0) return;
  int ln[4][16];
  uint16_t* pl = D.plane;
  const int st = D.stride;
  // vertical edges: one row of 16 samples is two 16-byte loads (pos - 8 is a
  // multiple of 8); horizontal edges: the 4 columns of a row are one 8-byte load
  if (kVertical) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint4* r = reinterpret_cast<const uint4*>(pl + (size_t)(seg + k) * st + pos - 8);
      const uint4 a = r[0], b = r[1];
      const uint32_t wv[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
      for (int i = 0; i < 8; i++) {
        ln[k][2 * i] = (int)(wv[i] & 0xFFFFu);
        ln[k][2 * i + 1] = (int)(wv[i] >> 16);
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const uint2 v = *reinterpret_cast<const uint2*>(pl + (size_t)(pos - 8 + i) * st + seg);
      ln[0][i] = (int)(v.x & 0xFFFFu);
      ln[1][i] = (int)(v.x >> 16);
      ln[2][i] = (int)(v.y & 0xFFFFu);
      ln[3][i] = (int)(v.y >> 16);
    }
  }
  bool ctb_hor = !kVertical && (pos % D.ctb) == 0;
  LumaEdgeDec dec;
  if (!decide_luma(ln, beta, tc, D.len_p, D.len_q, ctb_hor, &dec)) return;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (dec.de == 3)
      long_tap_line(ln[k], dec.len_p, dec.len_q, tc, maxv);
    else
      short_line(ln[k], dec, tc, maxv);
  }
  // positions 0 and 15 are never modified; rewriting them is safe because
  // edges of one pass are at least 16 samples apart on this path's lattice
  if (kVertical) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t wv[8];
#pragma unroll
      for (int i = 0; i < 8; i++)
        wv[i] = (uint32_t)clampi(ln[k][2 * i], 0, maxv) | ((uint32_t)clampi(ln[k][2 * i + 1], 0, maxv) << 16);
      uint4* r = reinterpret_cast<uint4*>(pl + (size_t)(seg + k) * st + pos - 8);
      r[0] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
      r[1] = make_uint4(wv[4], wv[5], wv[6], wv[7]);
    }
  } else {
#pragma unroll
    for (int i = 1; i < 15; i++) {
      uint2 v;
      v.x = (uint32_t)clampi(ln[0][i], 0, maxv) | ((uint32_t)clampi(ln[1][i], 0, maxv) << 16);
      v.y = (uint32_t)clampi(ln[2][i], 0, maxv) | ((uint32_t)clampi(ln[3][i], 0, maxv) << 16);
      *reinterpret_cast<uint2*>(pl + (size_t)(pos - 8 + i) * st + seg) = v;
    }
  }
}

// filter.rs:907-919 chroma_sample_decision
__device__ __forceinline__ bool chroma_dec(int p0, int p3, int q0, int q3, int dpq, int beta, int tc) {
  return dpq < (beta >> 2) && abs(p3 - p0) + abs(q0 - q3) < (beta >> 3) &&
         abs(p0 - q0) < ((5 * tc + 1) >> 1);
}

// The decision and line filters of deblock_chroma_edge (filter.rs:960-1007)
// on n lines of [p3 p2 p1 p0 q0 q1 q2 q3]; len_p / len_q are 1 or 3.
__device__ __forceinline__ void chroma_edge_lines(int (*ln)[8], int n, int len_p, int len_q, int tc, int beta,
                                                  int maxv) {
  if (len_q == 3) {
    int a[8], b[8];
    for (int i = 0; i < 8; i++) {
      a[i] = ln[0][i];
      b[i] = ln[n - 1][i];
    }
    if (len_p == 1) {
      a[0] = a[1] = a[2];
      b[0] = b[1] = b[2];
    }
    int dp0 = abs(a[1] - 2 * a[2] + a[3]), dp1 = abs(b[1] - 2 * b[2] + b[3]);
    int dq0 = abs(a[6] - 2 * a[5] + a[4]), dq1 = abs(b[6] - 2 * b[5] + b[4]);
    int dpq0 = dp0 + dq0, dpq1 = dp1 + dq1;
    bool strong = (dpq0 + dpq1) < beta && chroma_dec(a[3], a[0], a[4], a[7], 2 * dpq0, beta, tc) &&
                  chroma_dec(b[3], b[0], b[4], b[7], 2 * dpq1, beta, tc);
    if (!strong) {
      len_p = 1;
      len_q = 1;
    }
  }
  for (int k = 0; k < n; k++) {
    int* l = ln[k];
    int m[8];
    for (int i = 0; i < 8; i++) m[i] = l[i];
    auto cl = [&](int o, int v) { return clampi(clampi(v, o - tc, o + tc), 0, maxv); };
    if (len_p == 3 && len_q == 3) {
      l[1] = cl(m[1], (3 * m[0] + 2 * m[1] + m[2] + m[3] + m[4] + 4) >> 3);
      l[2] = cl(m[2], (2 * m[0] + m[1] + 2 * m[2] + m[3] + m[4] + m[5] + 4) >> 3);
      l[3] = cl(m[3], (m[0] + m[1] + m[2] + 2 * m[3] + m[4] + m[5] + m[6] + 4) >> 3);
      l[4] = cl(m[4], (m[1] + m[2] + m[3] + 2 * m[4] + m[5] + m[6] + m[7] + 4) >> 3);
      l[5] = cl(m[5], (m[2] + m[3] + m[4] + 2 * m[5] + m[6] + 2 * m[7] + 4) >> 3);
      l[6] = cl(m[6], (m[3] + m[4] + m[5] + 2 * m[6] + 3 * m[7] + 4) >> 3);
    } else if (len_p == 1 && len_q == 3) {
      l[3] = cl(m[3], (3 * m[2] + 2 * m[3] + m[4] + m[5] + m[6] + 4) >> 3);
      l[4] = cl(m[4], (2 * m[2] + m[3] + 2 * m[4] + m[5] + m[6] + m[7] + 4) >> 3);
      l[5] = cl(m[5], (m[2] + m[3] + m[4] + 2 * m[5] + m[6] + 2 * m[7] + 4) >> 3);
      l[6] = cl(m[6], (m[3] + m[4] + m[5] + 2 * m[6] + 3 * m[7] + 4) >> 3);
    } else {
      int delta = clampi((4 * (m[4] - m[3]) + m[2] - m[5] + 4) >> 3, -tc, tc);
      l[3] = clampi(m[3] + delta, 0, maxv);
      l[4] = clampi(m[4] - delta, 0, maxv);
    }
  }
}

// deblock_chroma_edge (filter.rs:935-1007) + the strong / p1q3 / weak line
// filters (:1010-1057), driven as in deblock_chroma_plane_16 (:2433-2527).
// One thread per 2- or 4-line group.
template <bool kVertical>
__global__ void k_deblock_chroma(const DbfPass* __restrict__ passes, int n_pass) {
  const DbfPass& D = passes[blockIdx.y];
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= D.n_edges * D.n_segs) return;
  const int e = idx / D.n_segs, s = idx % D.n_segs;
  const int pos = D.step * (e + 1);
  const int group = D.sub == 1 ? 4 : 2;
  const int seg = s * group;
  const int bd = D.bd, maxv = (1 << bd) - 1;
  const int bs = pass_bs<kVertical>(D, e, seg);
  if (bs == 0) return;
  int len_p = min(D.len_p, 3), len_q = min(D.len_q, 3);
  if (!kVertical && (pos % D.ctb) == 0) len_p = 1;  // upper chroma CTB boundary
  if (len_p == 1 && len_q == 1 && bs != 2) return;
  int idx_tc = clampi(D.qp + 2 * (bs - 1) + 2 * D.tc_off, 0, 65);
  int idx_b = clampi(D.qp + 2 * D.beta_off, 0, 63);
  int tc = tc_for(idx_tc, bd);
  int beta = c_dbf_beta[idx_b] << (bd - 8);
  int ln[4][8];
  uint16_t* pl = D.plane;
  const int st = D.stride;
  // vertical edges: a row of 8 samples is two 8-byte loads (pos - 4 is a
  // multiple of 4); horizontal edges: the group's columns of a row in one load
  if (kVertical) {
    for (int k = 0; k < group; k++) {
      const uint2* r = reinterpret_cast<const uint2*>(pl + (size_t)(seg + k) * st + pos - 4);
      const uint2 a = r[0], b = r[1];
      const uint32_t wv[4] = {a.x, a.y, b.x, b.y};
#pragma unroll
      for (int i = 0; i < 4; i++) {
        ln[k][2 * i] = (int)(wv[i] & 0xFFFFu);
        ln[k][2 * i + 1] = (int)(wv[i] >> 16);
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const uint16_t* rp = pl + (size_t)(pos - 4 + i) * st + seg;
      if (group == 4) {
        const uint2 v = *reinterpret_cast<const uint2*>(rp);
        ln[0][i] = (int)(v.x & 0xFFFFu);
        ln[1][i] = (int)(v.x >> 16);
        ln[2][i] = (int)(v.y & 0xFFFFu);
        ln[3][i] = (int)(v.y >> 16);
      } else {
        const uint32_t v = *reinterpret_cast<const uint32_t*>(rp);
        ln[0][i] = (int)(v & 0xFFFFu);
        ln[1][i] = (int)(v >> 16);
      }
    }
  }
  chroma_edge_lines(ln, group, len_p, len_q, tc, beta, maxv);
  // positions 0 and 7 are never modified; rewriting them is safe because
  // edges of one pass are at least 8 samples apart
  if (kVertical) {
    for (int k = 0; k < group; k++) {
      uint32_t wv[4];
#pragma unroll
      for (int i = 0; i < 4; i++)
        wv[i] = (uint32_t)clampi(ln[k][2 * i], 0, maxv) | ((uint32_t)clampi(ln[k][2 * i + 1], 0, maxv) << 16);
      uint2* r = reinterpret_cast<uint2*>(pl + (size_t)(seg + k) * st + pos - 4);
      r[0] = make_uint2(wv[0], wv[1]);
      r[1] = make_uint2(wv[2], wv[3]);
    }
  } else {
#pragma unroll
    for (int i = 1; i < 7; i++) {
      uint16_t* rp = pl + (size_t)(pos - 4 + i) * st + seg;
      const uint32_t v0 = (uint32_t)clampi(ln[0][i], 0, maxv) | ((uint32_t)clampi(ln[1][i], 0, maxv) << 16);
      if (group == 4)
        *reinterpret_cast<uint2*>(rp) =
            make_uint2(v0, (uint32_t)clampi(ln[2][i], 0, maxv) | ((uint32_t)clampi(ln[3][i], 0, maxv) << 16));
      else
        *reinterpret_cast<uint32_t*>(rp) = v0;
    }
  }
}

// One SAO pass over one plane of one picture.
struct SaoPass {
  const uint16_t* src;
  uint16_t* dst;
  const vvcg_ctu_filter* ctus;
  int32_t stride, w, h, bd, comp;
  int32_t ctu_w_log2, ctu_h_log2;  // CTU size in this plane's samples (powers of 2)
  int32_t ctu_cols;                // CTUs per row
  uint32_t cols_magic;             // ceil(2^32 / ctu_cols): ctu / ctu_cols = umulhi(ctu, magic)
};

// apply_sao_region_16 (filter.rs:1880-1947), every sample of the plane; the
// CTU containing a sample supplies its parameters and unmodified samples are
// copied (the reference filters a copy in place). For edge class 3 the
// reference pairs the neighbour offset (1, -1) with a bounds test for (1, 1),
// so on the first and last rows it indexes row -1 / row h and panics; here
// such a sample raises kStatusSaoAbort and nothing outside the plane is read.
// One thread per 4 consecutive samples of a row (plane widths are multiples of
// 16 on this path, CTU widths multiples of 4): 8-byte loads and stores, the
// two outer neighbours of edge classes as single loads.
__device__ __forceinline__ void unpack4(uint2 v, int* o) {
  o[0] = (int)(v.x & 0xFFFFu);
  o[1] = (int)(v.x >> 16);
  o[2] = (int)(v.y & 0xFFFFu);
  o[3] = (int)(v.y >> 16);
}

// Work split: each warp takes one CTU and a group of its rows, lanes on 4
// consecutive samples of a row (a CTU row of ctu_w samples is ctu_w / 4
// lanes), so the CTU's parameters and the branch on its type are uniform
// across the warp. Coded sizes are CTU multiples: no partial CTUs.
// Grid: (ceil(items / 8), passes) with 8 warps per CTA; item = CTU x group.
__global__ void __launch_bounds__(256) k_sao(const SaoPass* __restrict__ passes, uint32_t* status) {
  const SaoPass& S = passes[blockIdx.y];
  const int lane = threadIdx.x & 31;
  // CTU sizes are powers of two: shifts and masks only (a CTU row is at
  // least 4 and at most 32 lanes), and one multiply-high for the CTU row
  const int tpr_log2 = max(0, S.ctu_w_log2 - 2);       // lanes per CTU row (log2)
  const int rpw_log2 = 5 - tpr_log2;                   // CTU rows per warp (log2)
  const int ctu_h = 1 << S.ctu_h_log2;
  const int groups_log2 = max(0, S.ctu_h_log2 - rpw_log2);
  const int n_ctu = S.ctu_cols * ((S.h + ctu_h - 1) >> S.ctu_h_log2);
  const int item = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (item >= (n_ctu << groups_log2)) return;
  const int ctu = item >> groups_log2, grp = item & ((1 << groups_log2) - 1);
  const int cyi = (int)__umulhi((uint32_t)ctu, S.cols_magic), cxi = ctu - cyi * S.ctu_cols;
  const int cxs = cxi << S.ctu_w_log2, cys = cyi << S.ctu_h_log2;
  const int x = cxs + ((lane & ((1 << tpr_log2) - 1)) << 2);
  const int y = cys + (grp << rpw_log2) + (lane >> tpr_log2);
  if (x >= S.w || y >= S.h || y >= cys + ctu_h) return;
  const int st = S.stride, w = S.w, h = S.h;
  const uint16_t* src = S.src;
  int c[4];
  unpack4(*reinterpret_cast<const uint2*>(src + (size_t)y * st + x), c);
  const vvcg_sao sp = S.ctus[ctu].sao[S.comp];
  const int maxv = (1 << S.bd) - 1;
  int out[4] = {c[0], c[1], c[2], c[3]};
  if (sp.type == 1) {
    const int o0 = sp.offsets[0], o1 = sp.offsets[1], o2 = sp.offsets[2], o3 = sp.offsets[3];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int band = ((uint8_t)((uint8_t)(c[i] >> (S.bd - 5)) - sp.band_or_class)) & 31;
      const int off = band == 0 ? o0 : band == 1 ? o1 : band == 2 ? o2 : o3;
      if (band < 4) out[i] = clampi(c[i] + off, 0, maxv);
    }
  } else if (sp.type == 2) {
    const int cls = sp.band_or_class & 3;
    const int dx = cls == 1 ? 0 : 1, dy = cls == 0 ? 0 : (cls == 3 ? -1 : 1);
    // neighbours a (at -dx, -dy) and b (at +dx, +dy): a[k] / b[k] hold columns x + k - 1
    int a[6], b[6];
    const int ya = y - dy, yb = y + dy;
    const bool ra = ya >= 0 && ya < h, rb = yb >= 0 && yb < h;
#pragma unroll
    for (int i = 0; i < 6; i++) a[i] = b[i] = 0;
    if (ra) {
      const uint16_t* r = src + (size_t)ya * st;
      unpack4(*reinterpret_cast<const uint2*>(r + x), a + 1);
      if (dx && x > 0) a[0] = r[x - 1];
    }
    if (rb) {
      const uint16_t* r = src + (size_t)yb * st;
      unpack4(*reinterpret_cast<const uint2*>(r + x), b + 1);
      if (dx && x + 4 < w) b[5] = r[x + 4];
    }
    const int o0 = sp.offsets[0], o1 = sp.offsets[1], o2 = sp.offsets[2], o3 = sp.offsets[3];
    bool abort = false;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int xi = x + i;
      const bool xin = !(xi - dx < 0 || xi + dx >= w);
      if (dy == -1 && xin && (y == 0 || y == h - 1)) {
        abort = true;
      } else if (xin && ra && rb) {
        const int av = dx ? a[i] : a[i + 1], bv = dx ? b[i + 2] : b[i + 1];
        const int ei = 2 + ((c[i] > av) - (c[i] < av)) + ((c[i] > bv) - (c[i] < bv));
        const int off = ei == 0 ? o0 : ei == 1 ? o1 : ei == 3 ? o2 : ei == 4 ? o3 : 0;
        out[i] = clampi(c[i] + off, 0, maxv);
      }
    }
    if (abort) atomicOr(status, kStatusSaoAbort);
  }
  *reinterpret_cast<uint2*>(S.dst + (size_t)y * st + x) =
      make_uint2((uint32_t)out[0] | ((uint32_t)out[1] << 16), (uint32_t)out[2] | ((uint32_t)out[3] << 16));
}

// SAO of one plane as the general decoder applies it:
// apply_sao_region_bounded_16 (filter.rs:1954-2033) per CTU, driven by
// apply_sao (decode_general.rs:5189-5223). CTU regions are cropped to the
// visible size, edge class 3 pairs (-1, 1) with (1, -1), and a sample whose
// edge-offset neighbour lies outside the visible picture is unchanged.
// Thread per sample; dst receives every sample of the plane.
struct SaoBoundedPass {
  const uint16_t* src;
  uint16_t* dst;
  const vvcg_sao* params;  // one per CTU, ctu_cols per row
  int32_t stride, w, h, vis_w, vis_h, bd, ctu, ctu_cols;
};

__global__ void __launch_bounds__(256) k_sao_bounded(SaoBoundedPass S) {
  const int bd = clampi(S.bd, 8, 12), maxv = (1 << bd) - 1;
  const int bw = min(S.vis_w, S.w), bh = min(S.vis_h, S.h);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (uint64_t)S.w * S.h;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / S.w), x = (int)(i % S.w);
    const int c = S.src[(size_t)y * S.stride + x];
    int out = c;
    if (x < S.vis_w && y < S.vis_h) {
      const vvcg_sao sp = S.params[(y / S.ctu) * S.ctu_cols + x / S.ctu];
      if (sp.type == 1) {
        const int band = ((uint8_t)((uint8_t)(c >> (bd - 5)) - sp.band_or_class)) & 31;
        if (band < 4) {
          const int off = band == 0 ? sp.offsets[0] : band == 1 ? sp.offsets[1] : band == 2 ? sp.offsets[2] : sp.offsets[3];
          out = clampi(c + off, 0, maxv);
        }
      } else if (sp.type == 2) {
        const int cls = sp.band_or_class & 3;
        const int dx = cls == 1 ? 0 : (cls == 3 ? -1 : 1), dy = cls == 0 ? 0 : 1;
        const int ax = x - dx, ay = y - dy, bx = x + dx, by = y + dy;
        if (!(ax < 0 || ay < 0 || ax >= bw || ay >= bh || bx < 0 || by < 0 || bx >= bw || by >= bh)) {
          const int a = S.src[(size_t)ay * S.stride + ax], b = S.src[(size_t)by * S.stride + bx];
          const int ei = 2 + ((c > a) - (c < a)) + ((c > b) - (c < b));
          const int off = ei == 0 ? sp.offsets[0] : ei == 1 ? sp.offsets[1] : ei == 3 ? sp.offsets[2]
                          : ei == 4 ? sp.offsets[3] : 0;
          out = clampi(c + off, 0, maxv);
        }
      }
    }
    S.dst[(size_t)y * S.stride + x] = (uint16_t)out;
  }
}

// One luma ALF pass (whole plane, apply_alf_luma_plane_16 of filter.rs:2045-2124).
struct AlfPass {
  const uint16_t* src;
  uint16_t* dst;
  const vvcg_alf_aps* aps;  // NULL = fixed filter of each class
  int32_t stride, w, h, bd;
};

constexpr int kAlfTw = 64, kAlfTh = 16, kAlfHalo = 4;
constexpr int kAlfBlocks = (kAlfTw / 4) * (kAlfTh / 4);
constexpr int kAlfW = kAlfTw + 2 * kAlfHalo, kAlfH = kAlfTh + 2 * kAlfHalo;  // staged tile with its halo

// Per-tile filter state of the luma ALF: each 4x4 block's transposed
// coefficients and clip values, and whether the reference aborts on it.
struct AlfTileWs {
  int16_t fc[kAlfBlocks][12];
  int16_t fcl[kAlfBlocks][12];
  uint8_t abort[kAlfBlocks];
};

// classify_alf_4x4_16 (filter.rs:2126-2182) of the tile's 4x4 blocks and the
// filter each block uses, for a 256-thread CTA: four threads per block, each
// summing one of the four gradient directions over the block's 3x3
// subsampled positions; the group then shares the sums and every thread
// forms three of the block's twelve coefficient / clip pairs. `t` is the
// staged tile (kAlfH x kAlfW, output (x0, y0) at (kAlfHalo, kAlfHalo),
// positions outside the plane holding the clamped samples). Not inlined:
// inlined, it raised the filtering kernels from 40 to 73 registers.
__device__ __noinline__ void alf_classify_tile(const uint16_t (&t)[kAlfH][kAlfW], int x0, int y0, int w, int h, int bd,
                                                  const vvcg_alf_aps* aps_p, AlfTileWs& ws) {
  const int b = threadIdx.x >> 2, q = threadIdx.x & 3;
  const int bxi = b % (kAlfTw / 4), byi = b / (kAlfTw / 4);
  const int bx = x0 + bxi * 4, by = y0 + byi * 4;
  // direction q: 0 horizontal, 1 vertical, 2 the 135-degree diagonal, 3 the 45-degree one
  const int ax = q == 1 ? 0 : (q == 3 ? 1 : -1), ay = q == 0 ? 0 : -1;
  int sum = 0;
  for (int dy = 0; dy <= 4; dy += 2)
    for (int dx = 0; dx <= 4; dx += 2) {
      const int tx = bxi * 4 + dx + kAlfHalo, ty = byi * 4 + dy + kAlfHalo;
      sum += abs(((int)t[ty][tx] << 1) - (int)t[ty + ay][tx + ax] - (int)t[ty - ay][tx - ax]);
    }
  const int base = threadIdx.x & ~3 & 31;
  const int sh = __shfl_sync(0xffffffffu, sum, base), sv = __shfl_sync(0xffffffffu, sum, base + 1);
  const int d0 = __shfl_sync(0xffffffffu, sum, base + 2), d1 = __shfl_sync(0xffffffffu, sum, base + 3);
  int cls = 0, tr = 0;
  if (bx < w && by < h) {
    long long act = ((long long)(sh + sv) * 64) >> (bd + 4);
    // activity quantiser {0, 1, 2 x5, 3 x8, 4} of filter.rs:2163
    const int ac = (int)(act < 0 ? 0 : (act > 15 ? 15 : act));
    const int q_act = ac == 0 ? 0 : ac == 1 ? 1 : ac <= 6 ? 2 : ac <= 14 ? 3 : 4;
    int hv1, hv0, dhv, dd1, dd0, ddd;
    if (sv > sh) { hv1 = sv; hv0 = sh; dhv = 1; } else { hv1 = sh; hv0 = sv; dhv = 3; }
    if (d0 > d1) { dd1 = d0; dd0 = d1; ddd = 0; } else { dd1 = d1; dd0 = d0; ddd = 2; }
    int h1, h0, mdir, sdir;
    if ((long long)dd1 * hv0 > (long long)hv1 * dd0) { h1 = dd1; h0 = dd0; mdir = ddd; sdir = dhv; }
    else { h1 = hv1; h0 = hv0; mdir = dhv; sdir = ddd; }
    int ds = 0;
    if (h1 > 2 * h0) ds = (h1 * 2 > 9 * h0) ? 2 : 1;
    // transpose index {0, 1, 0, 2, 2, 3, 1, 3}[mdir * 2 + sdir / 2], 2 bits each
    tr = (0xDE84 >> (2 * (mdir * 2 + (sdir >> 1)))) & 3;
    cls = q_act;
    if (ds) cls += (((mdir & 1) << 1) + ds - 1 + 1) * 5;
    cls = min(cls, 24);
  }
  // filter of the class: APS filter (coeff_delta_idx) or the fixed filter
  // (the reference indexes a [16][25] table by class and aborts for >= 16)
  const int* ct = bd >= 12 ? c_alf_clip[2] : (bd >= 10 ? c_alf_clip[1] : c_alf_clip[0]);
  const bool aps = aps_p && aps_p->num_luma_filters > 0;
  const int filt = aps ? min((int)aps_p->coeff_delta_idx[cls], (int)aps_p->num_luma_filters - 1) : 0;
  const bool abort = !aps && cls >= 16;
  const bool use_clip = aps_p && aps_p->luma_clip && filt < (int)aps_p->num_luma_filters;
  const int fixed = abort ? 0 : c_alf_class_to_filter[cls * 25];
#pragma unroll
  for (int k = 3 * q; k < 3 * q + 3; k++) {
    const int p = c_alf_transpose_perm[(tr & 3) * 12 + k];
    ws.fc[b][k] = (int16_t)(aps ? aps_p->coeff[filt][p] : (abort ? 0 : c_alf_fixed[fixed * 13 + p]));
    ws.fcl[b][k] = (int16_t)ct[(use_clip ? aps_p->clip_idx[filt][p] : 0) & 3];
  }
  if (q == 0) ws.abort[b] = abort ? 1 : 0;
}

// The 7x7 diamond of four horizontally adjacent outputs (row ty, columns
// tx0..tx0+3, tx0 a multiple of 4) with every coefficient in a signed byte.
// Each row of the diamond is read once as 8-byte words (columns tx0-4 ..
// tx0+7); for each output and coefficient the two symmetric samples are
// packed into one register (byte permute), their differences to the centre
// clipped as two 16-bit lanes (vmaxs2 / vmins2) and both multiplied by the
// coefficient and summed by one dp2a. The sums are exact integers, equal to
// the scalar loop's: sum_k f_k * (clip(p0 - c) + clip(p1 - c)).
__device__ __forceinline__ void alf_filter4_packed(const uint16_t (&t)[kAlfH][kAlfW], int tx0, int ty,
                                                   const int (&fc)[12], const int (&fcl)[12], int maxv, int (&out)[4]) {
  // (column, row) offset of the first sample of each coefficient's pair; the
  // second is its mirror (filter.rs:2045 apply_alf_luma_plane_16 order)
  constexpr int kAx[12] = {0, 1, 0, -1, 2, 1, 0, -1, -2, 3, 2, 1};
  constexpr int kAy[12] = {3, 2, 2, 2, 1, 1, 1, 1, 1, 0, 0, 0};
  uint32_t R[7][6];  // R[dy + 3][w]: samples tx0 - 4 + 2w (low half) and tx0 - 3 + 2w (high half)
#pragma unroll
  for (int dy = -3; dy <= 3; dy++) {
    const uint2* row = reinterpret_cast<const uint2*>(&t[ty + dy][tx0 - 4]);
#pragma unroll
    for (int g = 0; g < 3; g++) {
      const uint2 v = row[g];
      R[dy + 3][2 * g] = v.x;
      R[dy + 3][2 * g + 1] = v.y;
    }
  }
  uint32_t pcl[12], ncl[12], cb[6];
#pragma unroll
  for (int k = 0; k < 12; k++) {
    pcl[k] = ((uint32_t)fcl[k] & 0xFFFFu) * 0x10001u;
    ncl[k] = ((uint32_t)(-fcl[k]) & 0xFFFFu) * 0x10001u;
  }
#pragma unroll
  for (int m = 0; m < 6; m++)
    cb[m] = ((uint32_t)(uint8_t)fc[2 * m] * 0x0101u) | (((uint32_t)(uint8_t)fc[2 * m + 1] * 0x0101u) << 16);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int jc = i + 4;  // the centre's column index within R's 12 samples
    const uint32_t hc = 2 * (jc & 1);
    const uint32_t cc = __byte_perm(R[3][jc >> 1], 0, hc | ((hc + 1) << 4) | (hc << 8) | ((hc + 1) << 12));
    int s = 0;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const int ja = jc + kAx[k], jb = jc - kAx[k];
      const uint32_t ha = 2 * (ja & 1), hb = 2 * (jb & 1) + 4;
      const uint32_t pair = __byte_perm(R[3 + kAy[k]][ja >> 1], R[3 - kAy[k]][jb >> 1],
                                        ha | ((ha + 1) << 4) | (hb << 8) | ((hb + 1) << 12));
      const uint32_t d = __vmins2(__vmaxs2(__vsub2(pair, cc), ncl[k]), pcl[k]);
      s = (k & 1) ? __dp2a_hi((int)d, (int)cb[k >> 1], s) : __dp2a_lo((int)d, (int)cb[k >> 1], s);
    }
    const int c = (int)(cc & 0xFFFFu);
    out[i] = clampi(c + ((s + 64) >> 7), 0, maxv);
  }
}

// The 7x7 diamond (apply_alf_luma_plane_16, filter.rs:2045-2124) on the
// staged tile after alf_classify_tile: each of the 256 threads filters one
// 4-sample row of a block and stores it to dst.
__device__ __forceinline__ void alf_filter_tile(const uint16_t (&t)[kAlfH][kAlfW], int x0, int y0, int w, int h, int bd,
                                                const AlfTileWs& ws, uint16_t* dst, int stride, uint32_t* status) {
  auto g = [&](int tx, int ty) -> int { return t[ty][tx]; };
  const int b = threadIdx.x >> 2, r = threadIdx.x & 3;
  const int bxi = b % (kAlfTw / 4), byi = b / (kAlfTw / 4);
  const int x = x0 + bxi * 4, y = y0 + byi * 4 + r;
  if (x >= w || y >= h) return;
  const int tx0 = bxi * 4 + kAlfHalo, ty = byi * 4 + r + kAlfHalo;
  int out[4];
  if (ws.abort[b]) {
    atomicOr(status, kStatusAlfAbort);
    for (int i = 0; i < 4; i++) out[i] = g(tx0 + i, ty);
  } else {
    int fc[12], fcl[12];
#pragma unroll
    for (int k = 0; k < 12; k++) {
      fc[k] = ws.fc[b][k];
      fcl[k] = ws.fcl[b][k];
    }
    const int maxv = (1 << bd) - 1;
    bool narrow = true;  // every coefficient fits a signed byte (the packed path's dp2a operand)
#pragma unroll
    for (int k = 0; k < 12; k++) narrow &= fc[k] >= -128 && fc[k] <= 127;
    if (narrow) {
      alf_filter4_packed(t, tx0, ty, fc, fcl, maxv, out);
    } else {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int tx = tx0 + i;
      const int c = g(tx, ty);
      auto ca = [&](int cv, int p0, int p1) { return clampi(p0 - c, -cv, cv) + clampi(p1 - c, -cv, cv); };
      int s = 0;
      s += fc[0] * ca(fcl[0], g(tx, ty + 3), g(tx, ty - 3));
      s += fc[1] * ca(fcl[1], g(tx + 1, ty + 2), g(tx - 1, ty - 2));
      s += fc[2] * ca(fcl[2], g(tx, ty + 2), g(tx, ty - 2));
      s += fc[3] * ca(fcl[3], g(tx - 1, ty + 2), g(tx + 1, ty - 2));
      s += fc[4] * ca(fcl[4], g(tx + 2, ty + 1), g(tx - 2, ty - 1));
      s += fc[5] * ca(fcl[5], g(tx + 1, ty + 1), g(tx - 1, ty - 1));
      s += fc[6] * ca(fcl[6], g(tx, ty + 1), g(tx, ty - 1));
      s += fc[7] * ca(fcl[7], g(tx - 1, ty + 1), g(tx + 1, ty - 1));
      s += fc[8] * ca(fcl[8], g(tx - 2, ty + 1), g(tx + 2, ty - 1));
      s += fc[9] * ca(fcl[9], g(tx + 3, ty), g(tx - 3, ty));
      s += fc[10] * ca(fcl[10], g(tx + 2, ty), g(tx - 2, ty));
      s += fc[11] * ca(fcl[11], g(tx + 1, ty), g(tx - 1, ty));
      out[i] = clampi(c + ((s + 64) >> 7), 0, maxv);
    }
    }
  }
  *reinterpret_cast<uint2*>(dst + (size_t)y * stride + x) =
      make_uint2((uint32_t)out[0] | ((uint32_t)out[1] << 16), (uint32_t)out[2] | ((uint32_t)out[3] << 16));
}

// Tile of 64x16 outputs: the tile plus a 4-sample halo (coordinates clamped
// to the plane, as the reference's get_p does, so reads inside the staged
// tile need no further clamping) is staged in shared memory; a tile whose
// halo lies inside the plane needs no clamping and is staged with 8-byte
// loads. Then the blocks are classified and filtered (alf_classify_tile,
// alf_filter_tile).
__global__ void __launch_bounds__(256, 5) k_alf_luma(const AlfPass* __restrict__ passes, uint32_t* status) {
  const AlfPass& A = passes[blockIdx.z];
  __shared__ __align__(16) uint16_t t[kAlfH][kAlfW];
  __shared__ AlfTileWs ws;
  const int x0 = blockIdx.x * kAlfTw, y0 = blockIdx.y * kAlfTh;
  if (x0 >= A.w || y0 >= A.h) return;
  static_assert(kAlfW % 4 == 0 && kAlfHalo % 4 == 0 && kAlfTw % 4 == 0, "8-byte staging");
  const bool inner = x0 >= kAlfHalo && y0 >= kAlfHalo && x0 + kAlfTw + kAlfHalo <= A.w &&
                     y0 + kAlfTh + kAlfHalo <= A.h && (A.stride & 3) == 0 &&
                     (reinterpret_cast<uintptr_t>(A.src) & 7) == 0;
  if (inner) {  // no clamping: 4 samples per 8-byte load
    const uint16_t* base = A.src + (size_t)(y0 - kAlfHalo) * A.stride + (x0 - kAlfHalo);
    for (int i = threadIdx.x; i < (kAlfW / 4) * kAlfH; i += blockDim.x) {
      const int ty = i / (kAlfW / 4), q = i - ty * (kAlfW / 4);
      *reinterpret_cast<uint2*>(&t[ty][4 * q]) = *reinterpret_cast<const uint2*>(base + (size_t)ty * A.stride + 4 * q);
    }
  } else {
    for (int i = threadIdx.x; i < kAlfW * kAlfH; i += blockDim.x) {
      int ty = i / kAlfW, tx = i % kAlfW;
      int gx = clampi(x0 + tx - kAlfHalo, 0, A.w - 1), gy = clampi(y0 + ty - kAlfHalo, 0, A.h - 1);
      t[ty][tx] = A.src[(size_t)gy * A.stride + gx];
    }
  }
  __syncthreads();
  alf_classify_tile(t, x0, y0, A.w, A.h, A.bd, A.aps, ws);
  __syncthreads();
  alf_filter_tile(t, x0, y0, A.w, A.h, A.bd, ws, A.dst, A.stride, status);
}

// ---------------------------------------------------------------------------
// SAO then ALF of a luma plane in one pass per 64x16 tile (the frame path's
// order, slice.rs:5022-5069: apply_sao_region_16 per CTU into a copy, then
// apply_alf_luma_plane_16 over the whole SAO output). The deblocked samples
// of the tile and a halo of 5 (SAO's neighbour plus ALF's 4) are staged in
// shared memory, by one TMA box load for tiles whose staged region lies
// inside the plane, else by clamped plain loads; SAO is evaluated for the
// tile and ALF's 4-sample halo into a second shared tile (positions outside
// the plane take the SAO output of the clamped position, which is what the
// reference's clamped ALF reads see), and ALF filters from there. The SAO
// output never goes to memory: luma moves 2 B in and 2 B out per sample
// instead of 4 B each way for SAO and ALF separately.
// ---------------------------------------------------------------------------
struct SaoAlfPass {
  const uint16_t* src;         // deblocked luma
  uint16_t* dst;               // SAO + ALF output
  const vvcg_ctu_filter* ctus;  // per-CTU SAO parameters (component 0)
  const vvcg_alf_aps* aps;      // NULL = fixed filter of each class
  const CUtensorMap* tmap;      // src as a tensor map with a kSaStW x kSaStH box; NULL = plain loads
  int32_t stride, w, h, bd, ctu_log2, ctu_cols;
};

constexpr int kSaStX = 8, kSaStY = 5;                       // staged origin: (x0 - 8, y0 - 5)
constexpr int kSaStW = kAlfTw + 16, kSaStH = kAlfTh + 10;   // 80 x 26 samples (x 16-byte aligned)
constexpr uint32_t kSaStBytes = kSaStW * kSaStH * 2;

// SAO output of the deblocked sample at plane position (gx, gy), from the
// staged tile `d` whose element [0][0] is plane position (ox, oy); same
// rules as k_sao (apply_sao_region_16, filter.rs:1880-1947).
__device__ __forceinline__ int sao_at(const uint16_t (*d)[kSaStW], int ox, int oy, int gx, int gy,
                                      const SaoAlfPass& S, bool& abort) {
  const int c = d[gy - oy][gx - ox];
  const vvcg_sao sp = S.ctus[(gy >> S.ctu_log2) * S.ctu_cols + (gx >> S.ctu_log2)].sao[0];
  if (sp.type == 1) {
    const int band = ((uint8_t)((uint8_t)(c >> (S.bd - 5)) - sp.band_or_class)) & 31;
    if (band < 4) {
      const int off = band == 0 ? sp.offsets[0] : band == 1 ? sp.offsets[1] : band == 2 ? sp.offsets[2] : sp.offsets[3];
      return clampi(c + off, 0, (1 << S.bd) - 1);
    }
  } else if (sp.type == 2) {
    const int cls = sp.band_or_class & 3;
    const int dx = cls == 1 ? 0 : 1, dy = cls == 0 ? 0 : (cls == 3 ? -1 : 1);
    const bool xin = !(gx - dx < 0 || gx + dx >= S.w);
    const int ya = gy - dy, yb = gy + dy;
    if (dy == -1 && xin && (gy == 0 || gy == S.h - 1)) {
      abort = true;
    } else if (xin && ya >= 0 && ya < S.h && yb >= 0 && yb < S.h) {
      const int av = d[ya - oy][gx - dx - ox], bv = d[yb - oy][gx + dx - ox];
      const int ei = 2 + ((c > av) - (c < av)) + ((c > bv) - (c < bv));
      const int off = ei == 0 ? sp.offsets[0] : ei == 1 ? sp.offsets[1] : ei == 3 ? sp.offsets[2]
                      : ei == 4 ? sp.offsets[3] : 0;
      return clampi(c + off, 0, (1 << S.bd) - 1);
    }
  }
  return c;
}

__global__ void __launch_bounds__(256, 5) k_sao_alf_luma(const SaoAlfPass* __restrict__ passes, uint32_t spin_limit,
                                                      uint32_t* status) {
  const SaoAlfPass& S = passes[blockIdx.z];
  __shared__ __align__(128) uint16_t d[kSaStH][kSaStW];
  __shared__ __align__(16) uint16_t t[kAlfH][kAlfW];
  __shared__ AlfTileWs ws;
  __shared__ __align__(8) uint64_t mbar;
  const int x0 = blockIdx.x * kAlfTw, y0 = blockIdx.y * kAlfTh;
  if (x0 >= S.w || y0 >= S.h) return;
  const int ox = x0 - kSaStX, oy = y0 - kSaStY;
  const bool boxed = S.tmap && ox >= 0 && oy >= 0 && ox + kSaStW <= S.w && oy + kSaStH <= S.h;
  if (boxed) {
    if (threadIdx.x == 0) {
      mbar_init(&mbar, 1);
      mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      tma_acquire_map(S.tmap);
      mbar_expect_tx(&mbar, kSaStBytes);
      tma_load_2d(&d[0][0], S.tmap, ox, oy, &mbar);
    }
    // bounded wait; a copy that never lands voids the batch (status) and the
    // wait goes on, again bounded, so the CTA does not leave with it in flight
    if (!mbar_wait(&mbar, 0, spin_limit)) {
      atomicOr(status, kStatusTimeout);
      mbar_wait(&mbar, 0, spin_limit);
    }
  } else {
    for (int i = threadIdx.x; i < kSaStW * kSaStH; i += blockDim.x) {
      const int ty = i / kSaStW, tx = i - ty * kSaStW;
      d[ty][tx] = S.src[(size_t)clampi(oy + ty, 0, S.h - 1) * S.stride + clampi(ox + tx, 0, S.w - 1)];
    }
    __syncthreads();
  }
  // SAO of the tile and ALF's halo
  bool abort = false;
  if (boxed) {
    // The staged region lies inside the plane with a margin, so every
    // position and its edge-offset neighbours are in the picture and none is
    // on the first or last row: 4 samples per thread, one CTU's parameters
    // each (CTU widths are multiples of 4).
    const int maxv = (1 << S.bd) - 1;
    for (int i = threadIdx.x; i < (kAlfW / 4) * kAlfH; i += blockDim.x) {
      const int ty = i / (kAlfW / 4), q = i - ty * (kAlfW / 4);
      const int gx = x0 - kAlfHalo + 4 * q, gy = y0 - kAlfHalo + ty;
      const int dx0 = gx - ox, dy0 = gy - oy;
      int c[4];
      unpack4(*reinterpret_cast<const uint2*>(&d[dy0][dx0]), c);
      int out[4] = {c[0], c[1], c[2], c[3]};
      const vvcg_sao sp = S.ctus[(gy >> S.ctu_log2) * S.ctu_cols + (gx >> S.ctu_log2)].sao[0];
      const int o0 = sp.offsets[0], o1 = sp.offsets[1], o2 = sp.offsets[2], o3 = sp.offsets[3];
      if (sp.type == 1) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const int band = ((uint8_t)((uint8_t)(c[k] >> (S.bd - 5)) - sp.band_or_class)) & 31;
          const int off = band == 0 ? o0 : band == 1 ? o1 : band == 2 ? o2 : o3;
          if (band < 4) out[k] = clampi(c[k] + off, 0, maxv);
        }
      } else if (sp.type == 2) {
        const int cls = sp.band_or_class & 3;
        const int dx = cls == 1 ? 0 : 1, dy = cls == 0 ? 0 : (cls == 3 ? -1 : 1);
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const int av = d[dy0 - dy][dx0 + k - dx], bv = d[dy0 + dy][dx0 + k + dx];
          const int ei = 2 + ((c[k] > av) - (c[k] < av)) + ((c[k] > bv) - (c[k] < bv));
          const int off = ei == 0 ? o0 : ei == 1 ? o1 : ei == 3 ? o2 : ei == 4 ? o3 : 0;
          out[k] = clampi(c[k] + off, 0, maxv);
        }
      }
      *reinterpret_cast<uint2*>(&t[ty][4 * q]) =
          make_uint2((uint32_t)out[0] | ((uint32_t)out[1] << 16), (uint32_t)out[2] | ((uint32_t)out[3] << 16));
    }
  } else {
    // at clamped plane positions, with the picture-edge rules
    for (int i = threadIdx.x; i < kAlfW * kAlfH; i += blockDim.x) {
      const int ty = i / kAlfW, tx = i - ty * kAlfW;
      const int gx = clampi(x0 - kAlfHalo + tx, 0, S.w - 1), gy = clampi(y0 - kAlfHalo + ty, 0, S.h - 1);
      t[ty][tx] = (uint16_t)sao_at(d, ox, oy, gx, gy, S, abort);
    }
  }
  if (abort) atomicOr(status, kStatusSaoAbort);
  __syncthreads();
  alf_classify_tile(t, x0, y0, S.w, S.h, S.bd, S.aps, ws);
  __syncthreads();
  alf_filter_tile(t, x0, y0, S.w, S.h, S.bd, ws, S.dst, S.stride, status);
}

#undef LP
#undef LQ

}  // namespace vvcg
