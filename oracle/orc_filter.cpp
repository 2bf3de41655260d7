// CPU oracle (test infrastructure only; see oracle.h): deblocking, SAO and ALF
// on 16-bit sample planes. Restates crates/rustmpeg-video/src/vvc/filter.rs of
// the reference, including its VTM-following long-tap rule (filter.rs:473-476).
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../rustmpeg-next_b200/csrc/vvc_tables.h"
#include "oracle.h"

namespace orc {
using namespace vvc_tables;

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------- luma DBF ---

// filter.rs:240-248 luma_filter_length
static int luma_filter_length(int size) { return size <= 4 ? 1 : (size >= 32 ? 7 : 3); }

struct LumaEdge {
  int de;
  bool dep, deq;
  int len_p, len_q, tc;
};

static inline int P(const int* l, int i) { return l[7 - i]; }
static inline int Q(const int* l, int j) { return l[8 + j]; }

// filter.rs:282-305 luma_sample_decision
static bool luma_sample_decision(int p0, int p3, int q0, int q3, int dpq, int sp, int sq, int spq,
                                 bool lp, bool lq, int beta, int tc) {
  if (lp) sp = (sp + std::abs(p3 - p0) + 1) >> 1;
  if (lq) sq = (sq + std::abs(q3 - q0) + 1) >> 1;
  int t1, t2;
  if (lp || lq) {
    t1 = (3 * beta) >> 5;
    t2 = beta >> 4;
  } else {
    t1 = beta >> 3;
    t2 = beta >> 2;
  }
  return dpq < t2 && sp + sq < t1 && spq < ((5 * tc + 1) >> 1);
}

// filter.rs:311-468 decide_luma_edge; returns false for "no filtering"
static bool decide_luma_edge(int lines[4][16], int beta, int tc, int len_p_in, int len_q_in,
                             bool at_ctb_hor, LumaEdge* e) {
  const int* l0 = lines[0];
  const int* l3 = lines[3];
  int dp0 = std::abs(P(l0, 2) - 2 * P(l0, 1) + P(l0, 0));
  int dp3 = std::abs(P(l3, 2) - 2 * P(l3, 1) + P(l3, 0));
  int dq0 = std::abs(Q(l0, 2) - 2 * Q(l0, 1) + Q(l0, 0));
  int dq3 = std::abs(Q(l3, 2) - 2 * Q(l3, 1) + Q(l3, 0));
  int dpq0 = dp0 + dq0, dpq3 = dp3 + dq3;
  int sp0 = std::abs(P(l0, 3) - P(l0, 0)), sp3 = std::abs(P(l3, 3) - P(l3, 0));
  int sq0 = std::abs(Q(l0, 0) - Q(l0, 3)), sq3 = std::abs(Q(l3, 0) - Q(l3, 3));
  int spq0 = std::abs(P(l0, 0) - Q(l0, 0)), spq3 = std::abs(P(l3, 0) - Q(l3, 0));
  int len_p = clampi(len_p_in, 1, 7), len_q = clampi(len_q_in, 1, 7);
  bool lp = len_p > 3 && !at_ctb_hor;
  bool lq = len_q > 3;
  if (lp || lq) {
    int dp0l = lp ? (dp0 + std::abs(P(l0, 5) - 2 * P(l0, 4) + P(l0, 3)) + 1) >> 1 : dp0;
    int dp3l = lp ? (dp3 + std::abs(P(l3, 5) - 2 * P(l3, 4) + P(l3, 3)) + 1) >> 1 : dp3;
    int dq0l = lq ? (dq0 + std::abs(Q(l0, 5) - 2 * Q(l0, 4) + Q(l0, 3)) + 1) >> 1 : dq0;
    int dq3l = lq ? (dq3 + std::abs(Q(l3, 5) - 2 * Q(l3, 4) + Q(l3, 3)) + 1) >> 1 : dq3;
    if (!lp) len_p = 3;
    if (!lq) len_q = 3;
    int sp0l = len_p == 7 ? sp0 + std::abs(P(l0, 7) - P(l0, 6) - P(l0, 5) + P(l0, 4)) : sp0;
    int sp3l = len_p == 7 ? sp3 + std::abs(P(l3, 7) - P(l3, 6) - P(l3, 5) + P(l3, 4)) : sp3;
    int sq0l = len_q == 7 ? sq0 + std::abs(Q(l0, 4) - Q(l0, 5) - Q(l0, 6) + Q(l0, 7)) : sq0;
    int sq3l = len_q == 7 ? sq3 + std::abs(Q(l3, 4) - Q(l3, 5) - Q(l3, 6) + Q(l3, 7)) : sq3;
    int d0l = dp0l + dq0l, d3l = dp3l + dq3l;
    if (d0l + d3l < beta) {
      bool s0 = luma_sample_decision(lp ? P(l0, len_p) : 0, lp ? P(l0, 3) : 0,
                                     lq ? Q(l0, len_q) : 0, lq ? Q(l0, 3) : 0, 2 * d0l, sp0l, sq0l,
                                     spq0, lp, lq, beta, tc);
      bool s3 = luma_sample_decision(lp ? P(l3, len_p) : 0, lp ? P(l3, 3) : 0,
                                     lq ? Q(l3, len_q) : 0, lq ? Q(l3, 3) : 0, 2 * d3l, sp3l, sq3l,
                                     spq3, lp, lq, beta, tc);
      if (s0 && s3) {
        *e = LumaEdge{3, true, true, len_p, len_q, tc};
        return true;
      }
    }
  }
  int dp = dp0 + dp3, dq = dq0 + dq3;
  if (dpq0 + dpq3 >= beta) return false;
  bool s0 = false, s3 = false;
  if (len_p > 2 && len_q > 2) {
    s0 = luma_sample_decision(0, 0, 0, 0, 2 * dpq0, sp0, sq0, spq0, false, false, beta, tc);
    s3 = luma_sample_decision(0, 0, 0, 0, 2 * dpq3, sp3, sq3, spq3, false, false, beta, tc);
  }
  int de = 1;
  if (s0 && s3) {
    de = 2;
    len_p = 3;
    len_q = 3;
  }
  int side_thr = (beta + (beta >> 1)) >> 3;
  bool dep = len_p > 1 && len_q > 1 && dp < side_thr;
  bool deq = len_p > 1 && len_q > 1 && dq < side_thr;
  if (de == 1) {
    len_p = 1 + (dep ? 1 : 0);
    len_q = 1 + (deq ? 1 : 0);
  }
  *e = LumaEdge{de, dep, deq, len_p, len_q, tc};
  return true;
}

// filter.rs:477-582 long_tap_luma_line
static void long_tap_luma_line(int* line, int len_p, int len_q, int tc, int max_val) {
  int m[16];
  memcpy(m, line, sizeof(m));
  auto p = [&](int i) { return m[7 - i]; };
  auto q = [&](int j) { return m[8 + j]; };
  int np = std::min(len_p, 7), nq = std::min(len_q, 7);
  int rm;
  if (np == 5 && nq == 5) {
    rm = (2 * (p(0) + q(0) + p(1) + q(1) + p(2) + q(2)) + p(3) + q(3) + p(4) + q(4) + 8) >> 4;
  } else if ((np == 7 && nq == 5) || (np == 5 && nq == 7)) {
    rm = (2 * (p(0) + q(0) + p(1) + q(1)) + p(2) + q(2) + p(3) + q(3) + p(4) + q(4) + p(5) + q(5) +
          8) >> 4;
  } else if ((np == 5 && nq == 3) || (np == 3 && nq == 5)) {
    rm = (p(0) + q(0) + p(1) + q(1) + p(2) + q(2) + p(3) + q(3) + 4) >> 3;
  } else if (np == 7 && nq == 3) {
    rm = (2 * (p(0) + q(0)) + q(0) + 2 * (q(1) + q(2)) + p(1) + q(1) + p(2) + p(3) + p(4) + p(5) +
          p(6) + 8) >> 4;
  } else if (np == 3 && nq == 7) {
    rm = (2 * (p(0) + q(0)) + p(0) + 2 * (p(1) + p(2)) + p(1) + q(1) + q(2) + q(3) + q(4) + q(5) +
          q(6) + 8) >> 4;
  } else {
    rm = (2 * (p(0) + q(0)) + p(1) + q(1) + p(2) + q(2) + p(3) + q(3) + p(4) + q(4) + p(5) + q(5) +
          p(6) + q(6) + 8) >> 4;
  }
  int ref_p = (p(np) + p(np - 1) + 1) >> 1;
  int ref_q = (q(nq) + q(nq - 1) + 1) >> 1;
  static const int c7[7] = {59, 50, 41, 32, 23, 14, 5}, t7[7] = {6, 5, 4, 3, 2, 1, 1};
  static const int c5[5] = {58, 45, 32, 19, 6}, t5[5] = {6, 5, 4, 3, 2};
  static const int c3[3] = {53, 32, 11}, t3[3] = {6, 4, 2};
  auto co = [&](int n) { return n == 7 ? c7 : (n == 5 ? c5 : c3); };
  auto tm = [&](int n) { return n == 7 ? t7 : (n == 5 ? t5 : t3); };
  auto cnt = [&](int n) { return n == 7 ? 7 : (n == 5 ? 5 : 3); };
  const int *cp = co(np), *tp = tm(np), *cq = co(nq), *tq = tm(nq);
  for (int pos = 0; pos < cnt(np); pos++) {
    int orig = p(pos), cval = (tc * tp[pos]) >> 1;
    int it = (rm * cp[pos] + ref_p * (64 - cp[pos]) + 32) >> 6;
    line[7 - pos] = clampi(clampi(it, orig - cval, orig + cval), 0, max_val);
  }
  for (int pos = 0; pos < cnt(nq); pos++) {
    int orig = q(pos), cval = (tc * tq[pos]) >> 1;
    int it = (rm * cq[pos] + ref_q * (64 - cq[pos]) + 32) >> 6;
    line[8 + pos] = clampi(clampi(it, orig - cval, orig + cval), 0, max_val);
  }
}

// filter.rs:586-631 short_filter_luma_line
static void short_filter_luma_line(int* line, const LumaEdge& e, int max_val) {
  int m[16];
  memcpy(m, line, sizeof(m));
  int tc = e.tc;
  if (e.de == 2) {
    line[7] = clampi((P(m, 2) + 2 * P(m, 1) + 2 * P(m, 0) + 2 * Q(m, 0) + Q(m, 1) + 4) >> 3,
                     P(m, 0) - 3 * tc, P(m, 0) + 3 * tc);
    line[6] = clampi((P(m, 2) + P(m, 1) + P(m, 0) + Q(m, 0) + 2) >> 2, P(m, 1) - 2 * tc,
                     P(m, 1) + 2 * tc);
    line[5] = clampi((2 * P(m, 3) + 3 * P(m, 2) + P(m, 1) + P(m, 0) + Q(m, 0) + 4) >> 3,
                     P(m, 2) - tc, P(m, 2) + tc);
    line[8] = clampi((P(m, 1) + 2 * P(m, 0) + 2 * Q(m, 0) + 2 * Q(m, 1) + Q(m, 2) + 4) >> 3,
                     Q(m, 0) - 3 * tc, Q(m, 0) + 3 * tc);
    line[9] = clampi((P(m, 0) + Q(m, 0) + Q(m, 1) + Q(m, 2) + 2) >> 2, Q(m, 1) - 2 * tc,
                     Q(m, 1) + 2 * tc);
    line[10] = clampi((P(m, 0) + Q(m, 0) + Q(m, 1) + 3 * Q(m, 2) + 2 * Q(m, 3) + 4) >> 3,
                      Q(m, 2) - tc, Q(m, 2) + tc);
    return;
  }
  int delta = (9 * (Q(m, 0) - P(m, 0)) - 3 * (Q(m, 1) - P(m, 1)) + 8) >> 4;
  if (std::abs(delta) >= tc * 10) return;
  delta = clampi(delta, -tc, tc);
  line[7] = clampi(P(m, 0) + delta, 0, max_val);
  line[8] = clampi(Q(m, 0) - delta, 0, max_val);
  int tc2 = tc >> 1;
  if (e.dep) {
    int dp = clampi((((P(m, 2) + P(m, 0) + 1) >> 1) - P(m, 1) + delta) >> 1, -tc2, tc2);
    line[6] = clampi(P(m, 1) + dp, 0, max_val);
  }
  if (e.deq) {
    int dq = clampi((((Q(m, 2) + Q(m, 0) + 1) >> 1) - Q(m, 1) - delta) >> 1, -tc2, tc2);
    line[9] = clampi(Q(m, 1) + dq, 0, max_val);
  }
}

static int tc_for(int idx_tc, int bd) {
  return bd < 10 ? (kDbfTc[idx_tc] + (1 << (9 - bd))) >> (10 - bd) : kDbfTc[idx_tc] << (bd - 10);
}

// filter.rs:638-679 deblock_luma_edge_bd
static void deblock_luma_edge_bd(int lines[4][16], int qp_p, int qp_q, int bs, int beta_off,
                                 int tc_off, int bd, int len_p, int len_q, bool at_ctb_hor) {
  if (bs == 0) return;
  bd = clampi(bd, 8, 12);
  int max_val = (1 << bd) - 1;
  int qp = (qp_p + qp_q + 1) >> 1;
  int idx_tc = clampi(qp + 2 * (bs - 1) + 2 * tc_off, 0, 65);
  int idx_b = clampi(qp + 2 * beta_off, 0, 63);
  int tc = tc_for(idx_tc, bd);
  int beta = kDbfBeta[idx_b] << (bd - 8);
  if (beta == 0 || tc == 0) return;
  LumaEdge e;
  if (!decide_luma_edge(lines, beta, tc, len_p, len_q, at_ctb_hor, &e)) return;
  for (int k = 0; k < 4; k++) {
    if (e.de == 3)
      long_tap_luma_line(lines[k], e.len_p, e.len_q, e.tc, max_val);
    else
      short_filter_luma_line(lines[k], e, max_val);
  }
}

// filter.rs:2344-2427 deblock_luma_plane_16
void deblock_luma_plane_16(Plane16& p, int cu_step, int ctb_size, int qp, int bs, int beta_off,
                           int tc_off) {
  int step = std::max(cu_step, 8);
  int ctb = std::max(ctb_size, step);
  int max_len = luma_filter_length(step);
  int w = p.width, h = p.height;
  int bd = clampi(p.bd, 8, 12);
  int max_val = (1 << bd) - 1;
  int lines[4][16];
  for (int x = step; x + 8 <= w && x >= 8; x += step) {
    for (int y = 0; y + 4 <= h; y += 4) {
      for (int dy = 0; dy < 4; dy++)
        for (int k = 0; k < 16; k++) lines[dy][k] = p.get(x - 8 + k, y + dy);
      deblock_luma_edge_bd(lines, qp, qp, bs, beta_off, tc_off, bd, max_len, max_len, false);
      for (int dy = 0; dy < 4; dy++)
        for (int k = 0; k < 16; k++) p.set(x - 8 + k, y + dy, clampi(lines[dy][k], 0, max_val));
    }
  }
  for (int y = step; y + 8 <= h && y >= 8; y += step) {
    bool at_ctb = (y % ctb) == 0;
    for (int bx = 0; bx + 4 <= w; bx += 4) {
      for (int dx = 0; dx < 4; dx++)
        for (int k = 0; k < 16; k++) lines[dx][k] = p.get(bx + dx, y - 8 + k);
      deblock_luma_edge_bd(lines, qp, qp, bs, beta_off, tc_off, bd, max_len, max_len, at_ctb);
      for (int dx = 0; dx < 4; dx++)
        for (int k = 0; k < 16; k++) p.set(bx + dx, y - 8 + k, clampi(lines[dx][k], 0, max_val));
    }
  }
}

// -------------------------------------------------------------- chroma DBF ---

// filter.rs:901-903 chroma_filter_length
static int chroma_filter_length(int size) { return size >= 8 ? 3 : 1; }

// filter.rs:907-919 chroma_sample_decision
static bool chroma_sample_decision(int p0, int p3, int q0, int q3, int dpq, int beta, int tc) {
  return dpq < (beta >> 2) && std::abs(p3 - p0) + std::abs(q0 - q3) < (beta >> 3) &&
         std::abs(p0 - q0) < ((5 * tc + 1) >> 1);
}

// filter.rs:1010-1057 chroma_strong_line / chroma_weak_line_p1q3 / chroma_weak_line
static void chroma_strong_line(int* l, int tc, int mx) {
  int m[8];
  memcpy(m, l, sizeof(m));
  auto c = [&](int o, int v) { return clampi(clampi(v, o - tc, o + tc), 0, mx); };
  l[1] = c(m[1], (3 * m[0] + 2 * m[1] + m[2] + m[3] + m[4] + 4) >> 3);
  l[2] = c(m[2], (2 * m[0] + m[1] + 2 * m[2] + m[3] + m[4] + m[5] + 4) >> 3);
  l[3] = c(m[3], (m[0] + m[1] + m[2] + 2 * m[3] + m[4] + m[5] + m[6] + 4) >> 3);
  l[4] = c(m[4], (m[1] + m[2] + m[3] + 2 * m[4] + m[5] + m[6] + m[7] + 4) >> 3);
  l[5] = c(m[5], (m[2] + m[3] + m[4] + 2 * m[5] + m[6] + 2 * m[7] + 4) >> 3);
  l[6] = c(m[6], (m[3] + m[4] + m[5] + 2 * m[6] + 3 * m[7] + 4) >> 3);
}
static void chroma_weak_line_p1q3(int* l, int tc, int mx) {
  int m[8];
  memcpy(m, l, sizeof(m));
  auto c = [&](int o, int v) { return clampi(clampi(v, o - tc, o + tc), 0, mx); };
  l[3] = c(m[3], (3 * m[2] + 2 * m[3] + m[4] + m[5] + m[6] + 4) >> 3);
  l[4] = c(m[4], (2 * m[2] + m[3] + 2 * m[4] + m[5] + m[6] + m[7] + 4) >> 3);
  l[5] = c(m[5], (m[2] + m[3] + m[4] + 2 * m[5] + m[6] + 2 * m[7] + 4) >> 3);
  l[6] = c(m[6], (m[3] + m[4] + m[5] + 2 * m[6] + 3 * m[7] + 4) >> 3);
}
static void chroma_weak_line(int* l, int tc, int mx) {
  int p1 = l[2], p0 = l[3], q0 = l[4], q1 = l[5];
  int delta = clampi((4 * (q0 - p0) + p1 - q1 + 4) >> 3, -tc, tc);
  l[3] = clampi(p0 + delta, 0, mx);
  l[4] = clampi(q0 - delta, 0, mx);
}

// filter.rs:935-1007 deblock_chroma_edge
static void deblock_chroma_edge(int lines[4][8], int n, int qp_c, int bs, int beta_off, int tc_off,
                                int max_len_p, int max_len_q, int bd) {
  if (bs == 0 || !(n == 2 || n == 4)) return;
  int len_p = std::min(max_len_p, 3), len_q = std::min(max_len_q, 3);
  if (len_p == 1 && len_q == 1 && bs != 2) return;
  bd = clampi(bd, 8, 12);
  int mx = (1 << bd) - 1;
  int idx_tc = clampi(qp_c + 2 * (bs - 1) + 2 * tc_off, 0, 65);
  int idx_b = clampi(qp_c + 2 * beta_off, 0, 63);
  int tc = tc_for(idx_tc, bd);
  int beta = kDbfBeta[idx_b] << (bd - 8);
  int n1 = n - 1;
  if (len_q == 3) {
    int l0[8], l1[8];
    memcpy(l0, lines[0], sizeof(l0));
    memcpy(l1, lines[n1], sizeof(l1));
    if (len_p == 1) {
      l0[0] = l0[2];
      l0[1] = l0[2];
      l1[0] = l1[2];
      l1[1] = l1[2];
    }
    int dp0 = std::abs(l0[1] - 2 * l0[2] + l0[3]), dp1 = std::abs(l1[1] - 2 * l1[2] + l1[3]);
    int dq0 = std::abs(l0[6] - 2 * l0[5] + l0[4]), dq1 = std::abs(l1[6] - 2 * l1[5] + l1[4]);
    int dpq0 = dp0 + dq0, dpq1 = dp1 + dq1;
    bool strong = (dpq0 + dpq1) < beta &&
                  chroma_sample_decision(l0[3], l0[0], l0[4], l0[7], 2 * dpq0, beta, tc) &&
                  chroma_sample_decision(l1[3], l1[0], l1[4], l1[7], 2 * dpq1, beta, tc);
    if (!strong) {
      len_p = 1;
      len_q = 1;
    }
  }
  for (int k = 0; k < n; k++) {
    if (len_p == 3 && len_q == 3)
      chroma_strong_line(lines[k], tc, mx);
    else if (len_p == 1 && len_q == 3)
      chroma_weak_line_p1q3(lines[k], tc, mx);
    else
      chroma_weak_line(lines[k], tc, mx);
  }
}

// filter.rs:2433-2527 deblock_chroma_plane_16
void deblock_chroma_plane_16(Plane16& p, int cu_step, int ctb_height_c, int qp_c, int bs,
                             int beta_off, int tc_off, int sub_w, int sub_h) {
  if (bs == 0 || p.width == 0 || p.height == 0) return;
  int bd = clampi(p.bd, 8, 12);
  int mx = (1 << bd) - 1;
  int step = std::max(cu_step, 8);
  int ctb = std::max(ctb_height_c, step);
  int len = chroma_filter_length(step);
  int w = p.width, h = p.height;
  int gv = sub_h == 1 ? 4 : 2;
  int gh = sub_w == 1 ? 4 : 2;
  int lines[4][8];
  for (int x = step; x >= 4 && x + 4 <= w; x += step) {
    for (int y = 0; y + gv <= h; y += gv) {
      for (int k = 0; k < gv; k++)
        for (int i = 0; i < 8; i++) lines[k][i] = p.get(x - 4 + i, y + k);
      deblock_chroma_edge(lines, gv, qp_c, bs, beta_off, tc_off, len, len, bd);
      for (int k = 0; k < gv; k++)
        for (int i = 0; i < 8; i++) p.set(x - 4 + i, y + k, clampi(lines[k][i], 0, mx));
    }
  }
  for (int y = step; y >= 4 && y + 4 <= h; y += step) {
    int lp = (y % ctb) == 0 ? 1 : len, lq = len;
    for (int bx = 0; bx + gh <= w; bx += gh) {
      for (int k = 0; k < gh; k++)
        for (int i = 0; i < 8; i++) lines[k][i] = p.get(bx + k, y - 4 + i);
      deblock_chroma_edge(lines, gh, qp_c, bs, beta_off, tc_off, lp, lq, bd);
      for (int k = 0; k < gh; k++)
        for (int i = 0; i < 8; i++) p.set(bx + k, y - 4 + i, clampi(lines[k][i], 0, mx));
    }
  }
}

// ------------------------------------------------ general-decoder DBF ---

// decode_general.rs:4916-4925 luma_lens
void dbk_luma_lens(int size_p, int size_q, int* lp, int* lq) {
  if (size_p <= 4 || size_q <= 4) {
    *lp = *lq = 1;
    return;
  }
  *lp = size_p >= 32 ? 7 : 3;
  *lq = size_q >= 32 ? 7 : 3;
}

// decode_general.rs:4929-4935 chroma_lens
void dbk_chroma_lens(int size_p, int size_q, bool ctb_boundary, int* lp, int* lq) {
  if (size_p >= 8 && size_q >= 8) {
    *lp = ctb_boundary ? 1 : 3;
    *lq = 3;
  } else {
    *lp = *lq = 1;
  }
}

// filter.rs:202-226 derive_boundary_strength
int dbk_boundary_strength(bool p_intra, bool q_intra, bool p_cbf, bool q_cbf, bool tu_edge, int pmv_h,
                          int pmv_v, int qmv_h, int qmv_v, int pref, int qref) {
  if (p_intra || q_intra) return 2;
  if (tu_edge && (p_cbf || q_cbf)) return 1;
  if (pref != qref || std::abs(pmv_h - qmv_h) >= 8 || std::abs(pmv_v - qmv_v) >= 8) return 1;
  return 0;
}

// slice.rs:2291-2554 apply_inter_loop_filters, its deblocking part: CTU
// boundaries of an 8-bit 4:2:0 inter picture, vertical then horizontal, with
// a per-edge bS from the two CTUs' cbf and motion (8-bit samples in 16-bit
// planes; the reference clamps to 0..255).
void inter_ctu_deblock(uint16_t* const planes[3], const int stride[3], int w, int h, int ctu, int qp,
                       const vvcg_ctu_motion* cells) {
  const int grid_w = w / ctu, grid_h = h / ctu;
  const int cw = ctu / 2;
  const int cwid = (w + 1) / 2, chei = (h + 1) / 2;
  const int chroma_qp = clampi(derived_chroma_qp(qp), 0, 63);
  const int luma_max_len = luma_filter_length(std::min(ctu, 32));
  const int chroma_len = chroma_filter_length(cw);
  auto Y = [&](int x, int y) -> uint16_t& { return planes[0][(size_t)y * stride[0] + x]; };
  auto bs_of = [&](const vvcg_ctu_motion& p, int pk, const vvcg_ctu_motion& q, int qk, int comp) {
    return dbk_boundary_strength(false, false, (p.cbf >> comp) & 1, (q.cbf >> comp) & 1, true, p.mv[pk][0],
                                 p.mv[pk][1], q.mv[qk][0], q.mv[qk][1], p.ref[pk], q.ref[qk]);
  };
  // filter.rs:1069-1112 deblock_chroma_edge_region at bit depth 8
  auto chroma_region = [&](int comp, bool vertical, int edge, int start, int end, int bs, int lp, int lq) {
    uint16_t* pl = planes[comp];
    const int st = stride[comp];
    const int limit = vertical ? cwid : chei;
    if (edge < 4 || edge + 4 > limit) return;
    for (int pos = start; pos + 2 <= end; pos += 2) {
      int lines[4][8];
      for (int k = 0; k < 2; k++)
        for (int i = 0; i < 8; i++) {
          const int d = edge - 4 + i;
          lines[k][i] = vertical ? pl[(size_t)(pos + k) * st + d] : pl[(size_t)d * st + pos + k];
        }
      deblock_chroma_edge(lines, 2, chroma_qp, bs, 0, 0, lp, lq, 8);
      for (int k = 0; k < 2; k++)
        for (int i = 0; i < 8; i++) {
          const int d = edge - 4 + i;
          const uint16_t v = (uint16_t)clampi(lines[k][i], 0, 255);
          if (vertical)
            pl[(size_t)(pos + k) * st + d] = v;
          else
            pl[(size_t)d * st + pos + k] = v;
        }
    }
  };
  int lines[4][16];
  // 1. vertical CTU boundaries
  for (int gx = 1; gx < grid_w; gx++) {
    const int x = gx * ctu, cx = gx * cw;
    for (int gy = 0; gy < grid_h; gy++) {
      const vvcg_ctu_motion& P = cells[gy * grid_w + gx - 1];
      const vvcg_ctu_motion& Q = cells[gy * grid_w + gx];
      const int bs_y = bs_of(P, 1, Q, 0, 0);
      if (bs_y > 0 && x >= 8 && x + 8 <= w) {
        const int y_end = std::min((gy + 1) * ctu, h);
        for (int y = gy * ctu; y + 4 <= y_end; y += 4) {
          for (int dy = 0; dy < 4; dy++)
            for (int k = 0; k < 16; k++) lines[dy][k] = Y(x - 8 + k, y + dy);
          deblock_luma_edge_bd(lines, qp, qp, bs_y, 0, 0, 8, luma_max_len, luma_max_len, false);
          for (int dy = 0; dy < 4; dy++)
            for (int k = 0; k < 16; k++) Y(x - 8 + k, y + dy) = (uint16_t)clampi(lines[dy][k], 0, 255);
        }
      }
      for (int c = 1; c <= 2; c++) {
        const int bs = bs_of(P, 1, Q, 0, c);
        if (bs > 0) chroma_region(c, true, cx, gy * cw, std::min((gy + 1) * cw, chei), bs, chroma_len, chroma_len);
      }
    }
  }
  // 2. horizontal CTU boundaries
  for (int gy = 1; gy < grid_h; gy++) {
    const int y = gy * ctu, cy = gy * cw;
    for (int gx = 0; gx < grid_w; gx++) {
      const vvcg_ctu_motion& P = cells[(gy - 1) * grid_w + gx];
      const vvcg_ctu_motion& Q = cells[gy * grid_w + gx];
      const int bs_y = bs_of(P, 2, Q, 0, 0);
      if (bs_y > 0 && y >= 8 && y + 8 <= h) {
        const int x_end = std::min((gx + 1) * ctu, w);
        for (int bx = gx * ctu; bx + 4 <= x_end; bx += 4) {
          for (int dx = 0; dx < 4; dx++)
            for (int k = 0; k < 16; k++) lines[dx][k] = Y(bx + dx, y - 8 + k);
          deblock_luma_edge_bd(lines, qp, qp, bs_y, 0, 0, 8, luma_max_len, luma_max_len, true);
          for (int dx = 0; dx < 4; dx++)
            for (int k = 0; k < 16; k++) Y(bx + dx, y - 8 + k) = (uint16_t)clampi(lines[dx][k], 0, 255);
        }
      }
      for (int c = 1; c <= 2; c++) {
        const int bs = bs_of(P, 2, Q, 0, c);
        if (bs > 0) chroma_region(c, false, cy, gx * cw, std::min((gx + 1) * cw, cwid), bs, 1, chroma_len);
      }
    }
  }
}

namespace {

struct GenDbk {
  const vvcg_dbk_cell* cells;
  int cols, rows;
  const vvcg_dbk_params* prm;
  // Gen::lcell (decode_general.rs:463-469): None outside the grid or when invalid
  const vvcg_dbk_cell* lcell(int x, int y) const {
    if (x < 0 || y < 0 || x / 4 >= cols || y / 4 >= rows) return nullptr;
    const vvcg_dbk_cell* c = &cells[(y / 4) * cols + x / 4];
    return (c->flags & VVCG_DBK_CODED) ? c : nullptr;
  }
  // the `field` closure of deblock_bs: motion of the first list in use, POC via
  // Gen::ref_poc (decode_general.rs:497-504) with unwrap_or(0)
  void field(const vvcg_dbk_cell* c, int* mh, int* mv, int* poc) const {
    *mh = *mv = *poc = 0;
    if (!c) return;
    for (int l = 0; l < 2; l++) {
      if (c->ref_idx[l] >= 0) {
        *mh = c->mv[l][0];
        *mv = c->mv[l][1];
        int idx = c->ref_idx[l];
        *poc = idx < prm->num_ref[l] && idx < 16 ? prm->ref_poc[l][idx] : 0;
        return;
      }
    }
  }
  bool cbf(int x, int y) const {
    if (x / 4 < cols && y / 4 < rows) return (cells[(y / 4) * cols + x / 4].flags & VVCG_DBK_CBF) != 0;
    return false;
  }
  // decode_general.rs:4939-4975 deblock_bs
  int bs(int x, int y, bool vertical) const {
    const vvcg_dbk_cell* p = vertical ? lcell(x - 1, y) : lcell(x, y - 1);
    const vvcg_dbk_cell* q = lcell(x, y);
    bool pi = p && (p->flags & VVCG_DBK_INTRA), qi = q && (q->flags & VVCG_DBK_INTRA);
    if (pi || qi) return 2;
    int ph, pv, pr, qh, qv, qr;
    field(p, &ph, &pv, &pr);
    field(q, &qh, &qv, &qr);
    bool pc = vertical ? cbf(x - 1, y) : cbf(x, y - 1), qc = cbf(x, y);
    return dbk_boundary_strength(pi, qi, pc, qc, true, ph, pv, qh, qv, pr, qr);
  }
};

}  // namespace

// decode_general.rs:4977-5187 apply_deblock: luma vertical then horizontal
// edges on the 4-sample grid, then per chroma component vertical and
// horizontal edges on the 8-sample grid in 2-line groups. Each segment is
// gathered with clamped coordinates, filtered, and written back sample by
// sample in gather order, as the reference does.
void deblock_general(uint16_t* const planes[3], const int stride[3], int vis_w, int vis_h, int bd, int ctu,
                     const vvcg_dbk_cell* cells, int cols, int rows, const vvcg_dbk_ccell* cc, int ccols,
                     int crows, const vvcg_dbk_params& prm) {
  const int max_val = (1 << bd) - 1;
  const int qp_y = clampi(prm.qp[0], 0, 63);
  GenDbk g{cells, cols, rows, &prm};
  const int w = vis_w, h = vis_h;
  uint16_t* Y = planes[0];
  const int sy = stride[0];
  auto id = [&](int cx, int cy) { return cells[cy * cols + cx].tu_id; };
  int lines[4][16];
  for (int x = 4; x < w; x += 4) {
    for (int y = 0; y < h; y += 4) {
      uint32_t a = id(x / 4 - 1, y / 4), b = id(x / 4, y / 4);
      if (a == VVCG_DBK_NO_TU || b == VVCG_DBK_NO_TU || a == b) continue;
      int lp, lq;
      dbk_luma_lens(cells[(y / 4) * cols + x / 4 - 1].tu_w, cells[(y / 4) * cols + x / 4].tu_w, &lp, &lq);
      for (int i = 0; i < 4; i++) {
        int yy = std::min(y + i, h - 1);
        for (int k = 0; k < 16; k++) lines[i][k] = Y[yy * sy + clampi(x - 8 + k, 0, w - 1)];
      }
      deblock_luma_edge_bd(lines, qp_y, qp_y, g.bs(x, y, true), prm.beta_offset_div2[0], prm.tc_offset_div2[0],
                           bd, lp, lq, false);
      for (int i = 0; i < 4; i++) {
        int yy = std::min(y + i, h - 1);
        for (int k = 0; k < 16; k++) Y[yy * sy + clampi(x - 8 + k, 0, w - 1)] = (uint16_t)clampi(lines[i][k], 0, max_val);
      }
    }
  }
  for (int y = 4; y < h; y += 4) {
    for (int x = 0; x < w; x += 4) {
      uint32_t a = id(x / 4, y / 4 - 1), b = id(x / 4, y / 4);
      if (a == VVCG_DBK_NO_TU || b == VVCG_DBK_NO_TU || a == b) continue;
      int lp, lq;
      dbk_luma_lens(cells[(y / 4 - 1) * cols + x / 4].tu_h, cells[(y / 4) * cols + x / 4].tu_h, &lp, &lq);
      for (int i = 0; i < 4; i++) {
        int xx = std::min(x + i, w - 1);
        for (int k = 0; k < 16; k++) lines[i][k] = Y[clampi(y - 8 + k, 0, h - 1) * sy + xx];
      }
      deblock_luma_edge_bd(lines, qp_y, qp_y, g.bs(x, y, false), prm.beta_offset_div2[0], prm.tc_offset_div2[0],
                           bd, lp, lq, y % ctu == 0);
      for (int i = 0; i < 4; i++) {
        int xx = std::min(x + i, w - 1);
        for (int k = 0; k < 16; k++) Y[clampi(y - 8 + k, 0, h - 1) * sy + xx] = (uint16_t)clampi(lines[i][k], 0, max_val);
      }
    }
  }
  const int cw = (vis_w + 1) / 2, ch = (vis_h + 1) / 2;
  int cl[4][8];
  for (int comp = 1; comp < 3; comp++) {
    uint16_t* P = planes[comp];
    const int sc = stride[comp];
    const int qp = clampi(prm.qp[comp], 0, 63);
    const int bo = prm.beta_offset_div2[comp], to = prm.tc_offset_div2[comp];
    auto cid = [&](int cx, int cy) { return comp == 1 ? cc[cy * ccols + cx].tu_cb : cc[cy * ccols + cx].tu_cr; };
    for (int x = 8; x < cw; x += 8) {
      for (int y = 0; y + 2 <= ch; y += 2) {
        uint32_t a = cid(x / 2 - 1, y / 2), b = cid(x / 2, y / 2);
        if (a == VVCG_DBK_NO_TU || b == VVCG_DBK_NO_TU || a == b) continue;
        int lp, lq;
        dbk_chroma_lens(cc[(y / 2) * ccols + x / 2 - 1].tu_w, cc[(y / 2) * ccols + x / 2].tu_w, false, &lp, &lq);
        for (int i = 0; i < 2; i++) {
          int yy = std::min(y + i, ch - 1);
          for (int k = 0; k < 8; k++) cl[i][k] = P[yy * sc + clampi(x - 4 + k, 0, cw - 1)];
        }
        deblock_chroma_edge(cl, 2, qp, 2, bo, to, lp, lq, bd);
        for (int i = 0; i < 2; i++) {
          int yy = std::min(y + i, ch - 1);
          for (int k = 0; k < 8; k++) P[yy * sc + clampi(x - 4 + k, 0, cw - 1)] = (uint16_t)clampi(cl[i][k], 0, max_val);
        }
      }
    }
    for (int y = 8; y < ch; y += 8) {
      for (int x = 0; x + 2 <= cw; x += 2) {
        uint32_t a = cid(x / 2, y / 2 - 1), b = cid(x / 2, y / 2);
        if (a == VVCG_DBK_NO_TU || b == VVCG_DBK_NO_TU || a == b) continue;
        int lp, lq;
        dbk_chroma_lens(cc[(y / 2 - 1) * ccols + x / 2].tu_h, cc[(y / 2) * ccols + x / 2].tu_h, y % (ctu / 2) == 0,
                        &lp, &lq);
        for (int i = 0; i < 2; i++) {
          int xx = std::min(x + i, cw - 1);
          for (int k = 0; k < 8; k++) cl[i][k] = P[clampi(y - 4 + k, 0, ch - 1) * sc + xx];
        }
        deblock_chroma_edge(cl, 2, qp, 2, bo, to, lp, lq, bd);
        for (int i = 0; i < 2; i++) {
          int xx = std::min(x + i, cw - 1);
          for (int k = 0; k < 8; k++) P[clampi(y - 4 + k, 0, ch - 1) * sc + xx] = (uint16_t)clampi(cl[i][k], 0, max_val);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------- SAO ---

// filter.rs:1880-1947 apply_sao_region_16. For edge class 3 the reference uses
// the neighbour offset (1, -1) with a bounds test written for (1, 1): on the
// first and last picture rows it indexes row -1 / row height, which panics
// (slice index out of bounds). This restatement returns -1 before writing
// anything in that case.
int apply_sao_region_16(const Plane16& src, Plane16& dst, int bx, int by, int w, int h,
                        const Sao& sao) {
  if (sao.type == 2 && (sao.band_pos_or_class & 3) == 3 && src.width >= 3) {
    int hl_ = std::min(by + h, src.height);
    if ((by == 0 && hl_ > 0) || (hl_ == src.height && by < hl_)) {
      int xl = std::max(bx, 1), xr = std::min(bx + w, src.width) - 1;  // x in [1, width-2]
      if (xl <= std::min(xr, src.width - 2)) return -1;
    }
  }
  int bd = clampi(src.bd, 8, 12);
  int mx = (1 << bd) - 1;
  int band_shift = bd - 5;
  int wl = std::min(bx + w, src.width), hl = std::min(by + h, src.height);
  if (sao.type == 1) {
    for (int y = by; y < hl; y++)
      for (int x = bx; x < wl; x++) {
        int s = src.get(x, y);
        int band = ((uint8_t)((uint8_t)(s >> band_shift) - (uint8_t)sao.band_pos_or_class)) & 31;
        if (band < 4) dst.set(x, y, clampi(s + sao.offsets[band], 0, mx));
      }
  } else if (sao.type == 2) {
    int dx, dy;
    switch (sao.band_pos_or_class & 3) {
      case 0: dx = 1; dy = 0; break;
      case 1: dx = 0; dy = 1; break;
      case 2: dx = 1; dy = 1; break;
      default: dx = 1; dy = -1; break;
    }
    for (int y = by; y < hl; y++)
      for (int x = bx; x < wl; x++) {
        if (x - dx < 0 || x + dx >= src.width || y - dy < 0 || y + dy >= src.height) continue;
        int c = src.get(x, y);
        int a = src.get(x - dx, y - dy);
        int b = src.get(x + dx, y + dy);
        int ei = 2 + ((c > a) - (c < a)) + ((c > b) - (c < b));
        int off = ei == 0 ? sao.offsets[0]
                          : ei == 1 ? sao.offsets[1] : ei == 3 ? sao.offsets[2]
                                                               : ei == 4 ? sao.offsets[3] : 0;
        dst.set(x, y, clampi(c + off, 0, mx));
      }
  }
  return 0;
}

// ---------------------------------------------------------------------- ALF ---

// filter.rs:2126-2182 classify_alf_4x4_16
void classify_alf_4x4_16(const Plane16& p, int bx, int by, int* class_idx, int* transpose_idx) {
  static const int TH[16] = {0, 1, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 4};
  auto g = [&](int x, int y) {
    return (int)p.get(clampi(x, 0, p.width - 1), clampi(y, 0, p.height - 1));
  };
  int sh = 0, sv = 0, d0 = 0, d1 = 0;
  for (int dy = -1; dy < 5; dy++)
    for (int dx = -1; dx < 5; dx++) {
      if ((dy & 1) != 0 || (dx & 1) != 0) continue;
      int x = bx + dx, y = by + dy;
      int c2 = g(x, y) << 1;
      sh += std::abs(c2 - g(x - 1, y) - g(x + 1, y));
      sv += std::abs(c2 - g(x, y - 1) - g(x, y + 1));
      d0 += std::abs(c2 - g(x - 1, y - 1) - g(x + 1, y + 1));
      d1 += std::abs(c2 - g(x + 1, y - 1) - g(x - 1, y + 1));
    }
  int temp_act = sh + sv;
  int shift = clampi(p.bd, 8, 12) + 4;
  int64_t act = ((int64_t)temp_act * 64) >> shift;
  int activity = (int)std::min<int64_t>(15, std::max<int64_t>(0, act));
  int q_act = TH[activity];
  int hv1, hv0, dir_hv, dd1, dd0, dir_d;
  if (sv > sh) {
    hv1 = sv; hv0 = sh; dir_hv = 1;
  } else {
    hv1 = sh; hv0 = sv; dir_hv = 3;
  }
  if (d0 > d1) {
    dd1 = d0; dd0 = d1; dir_d = 0;
  } else {
    dd1 = d1; dd0 = d0; dir_d = 2;
  }
  int hvd1, hvd0, main_dir, sec_dir;
  if ((int64_t)dd1 * hv0 > (int64_t)hv1 * dd0) {
    hvd1 = dd1; hvd0 = dd0; main_dir = dir_d; sec_dir = dir_hv;
  } else {
    hvd1 = hv1; hvd0 = hv0; main_dir = dir_hv; sec_dir = dir_d;
  }
  int ds = 0;
  if (hvd1 > 2 * hvd0) ds = (hvd1 * 2 > 9 * hvd0) ? 2 : 1;
  static const int TT[8] = {0, 1, 0, 2, 2, 3, 1, 3};
  *transpose_idx = TT[main_dir * 2 + (sec_dir >> 1)];
  int ci = q_act;
  if (ds != 0) ci += (((main_dir & 1) << 1) + ds - 1 + 1) * 5;
  *class_idx = std::min(ci, 24);
}

static inline int clip_alf(int cv, int curr, int p0, int p1) {  // filter.rs:1693-1695
  return clampi(p0 - curr, -cv, cv) + clampi(p1 - curr, -cv, cv);
}

// filter.rs:2045-2124 apply_alf_luma_plane_16. With no APS luma filters the
// reference reads ALF_CLASS_TO_FILTER_MAPPING[class_idx][0] from a [16][25]
// table, which panics (index out of bounds) for class_idx >= 16; this
// restatement reports that case by returning early with *status = -1.
int g_alf_status = 0;

void apply_alf_luma_plane_16(Plane16& p, const AlfAps& aps) {
  g_alf_status = 0;
  int bd = clampi(p.bd, 8, 12);
  int mx = (1 << bd) - 1;
  const int* ct = bd >= 12 ? kAlfClip[2] : (bd >= 10 ? kAlfClip[1] : kAlfClip[0]);
  std::vector<uint16_t> copy(p.data, p.data + (size_t)p.width * p.height);
  Plane16 src{copy.data(), p.width, p.height, p.bd};
  auto g = [&](int x, int y) {
    return (int)src.get(clampi(x, 0, src.width - 1), clampi(y, 0, src.height - 1));
  };
  for (int by = 0; by < p.height; by += 4)
    for (int bx = 0; bx < p.width; bx += 4) {
      int cls, tr;
      classify_alf_4x4_16(src, bx, by, &cls, &tr);
      int filt = 0;
      int base_c[12];
      uint8_t base_clip[12] = {0};
      if (aps.num_luma_filters > 0) {
        filt = std::min((int)aps.coeff_delta_idx[cls], aps.num_luma_filters - 1);
        for (int k = 0; k < 12; k++) base_c[k] = aps.coeff[filt][k];
      } else {
        if (cls >= 16) {
          g_alf_status = -1;
          return;
        }
        int fixed = kAlfClassToFilter[cls * 25 + 0];
        for (int k = 0; k < 12; k++) base_c[k] = kAlfFixedCoeff[fixed * 13 + k];
      }
      if (aps.luma_clip && filt < std::max(aps.num_luma_filters, 0))
        for (int k = 0; k < 12; k++) base_clip[k] = aps.clip_idx[filt][k];
      const uint8_t* perm = &kAlfTransposePerm[(tr & 3) * 12];
      int fc[12], fcl[12];
      for (int k = 0; k < 12; k++) {
        fc[k] = base_c[perm[k]];
        fcl[k] = ct[base_clip[perm[k]] & 3];
      }
      int he = std::min(by + 4, p.height), we = std::min(bx + 4, p.width);
      for (int y = by; y < he; y++)
        for (int x = bx; x < we; x++) {
          int c = g(x, y);
          int s = 0;
          s += fc[0] * clip_alf(fcl[0], c, g(x, y + 3), g(x, y - 3));
          s += fc[1] * clip_alf(fcl[1], c, g(x + 1, y + 2), g(x - 1, y - 2));
          s += fc[2] * clip_alf(fcl[2], c, g(x, y + 2), g(x, y - 2));
          s += fc[3] * clip_alf(fcl[3], c, g(x - 1, y + 2), g(x + 1, y - 2));
          s += fc[4] * clip_alf(fcl[4], c, g(x + 2, y + 1), g(x - 2, y - 1));
          s += fc[5] * clip_alf(fcl[5], c, g(x + 1, y + 1), g(x - 1, y - 1));
          s += fc[6] * clip_alf(fcl[6], c, g(x, y + 1), g(x, y - 1));
          s += fc[7] * clip_alf(fcl[7], c, g(x - 1, y + 1), g(x + 1, y - 1));
          s += fc[8] * clip_alf(fcl[8], c, g(x - 2, y + 1), g(x + 2, y - 1));
          s += fc[9] * clip_alf(fcl[9], c, g(x + 3, y), g(x - 3, y));
          s += fc[10] * clip_alf(fcl[10], c, g(x + 2, y), g(x - 2, y));
          s += fc[11] * clip_alf(fcl[11], c, g(x + 1, y), g(x - 1, y));
          p.set(x, y, clampi(c + ((s + 64) >> 7), 0, mx));
        }
    }
}

}  // namespace orc

namespace orc {

// filter.rs:1954-2033 apply_sao_region_bounded_16, driven per CTU as
// decode_general.rs:5189-5223 apply_sao does for one plane: CTU regions
// cropped to the visible size; edge-offset neighbours outside the visible
// picture leave the sample unchanged. `params` holds one Sao per CTU,
// ctu_cols per row. Writes dst (a copy of src outside the changed samples).
void sao_plane_bounded_16(const uint16_t* src, uint16_t* dst, int stride, int pw, int ph, int vis_w, int vis_h,
                          int bd, int ctu, int ctu_cols, const Sao* params) {
  for (int y = 0; y < ph; y++)
    for (int x = 0; x < pw; x++) dst[y * stride + x] = src[y * stride + x];
  bd = std::min(12, std::max(8, bd));
  const int max_val = (1 << bd) - 1, band_shift = bd - 5;
  const int bw = std::min(vis_w, pw), bh = std::min(vis_h, ph);
  for (int gy = 0; gy * ctu < vis_h; gy++)
    for (int gx = 0; gx * ctu < vis_w; gx++) {
      const Sao& s = params[gy * ctu_cols + gx];
      const int x0 = gx * ctu, y0 = gy * ctu;
      const int w_lim = std::min(x0 + std::min(ctu, vis_w - x0), pw), h_lim = std::min(y0 + std::min(ctu, vis_h - y0), ph);
      if (s.type == 1) {
        for (int y = y0; y < h_lim; y++)
          for (int x = x0; x < w_lim; x++) {
            const int c = src[y * stride + x];
            const int band = (uint8_t)((uint8_t)(c >> band_shift) - (uint8_t)s.band_pos_or_class) & 31;
            if (band < 4) dst[y * stride + x] = (uint16_t)std::min(max_val, std::max(0, c + s.offsets[band]));
          }
      } else if (s.type == 2) {
        int dx, dy;
        switch (s.band_pos_or_class & 3) {
          case 0: dx = 1; dy = 0; break;
          case 1: dx = 0; dy = 1; break;
          case 2: dx = 1; dy = 1; break;
          default: dx = -1; dy = 1; break;
        }
        for (int y = y0; y < h_lim; y++)
          for (int x = x0; x < w_lim; x++) {
            const int ax = x - dx, ay = y - dy, bxn = x + dx, byn = y + dy;
            if (ax < 0 || ay < 0 || ax >= bw || ay >= bh || bxn < 0 || byn < 0 || bxn >= bw || byn >= bh) continue;
            const int c = src[y * stride + x], a = src[ay * stride + ax], b = src[byn * stride + bxn];
            const int ei = 2 + ((c > a) - (c < a)) + ((c > b) - (c < b));
            const int off = ei == 0 ? s.offsets[0] : ei == 1 ? s.offsets[1] : ei == 3 ? s.offsets[2] : ei == 4 ? s.offsets[3] : 0;
            dst[y * stride + x] = (uint16_t)std::min(max_val, std::max(0, c + off));
          }
      }
    }
}

}  // namespace orc
