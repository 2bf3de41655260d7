// Host-side parse of the multi-tool stream's slice data (VvcMultiToolEncoder,
// mod.rs:1512-1720): its IDR pictures (decode_picture_multitool,
// slice.rs:3012-3190) into frame-path records, and its P pictures
// (decode_inter_picture, slice.rs:3552-3677) into vvcg_inter_cu records with
// the motion each coding unit ends up with. The motion derivation restates
// derive_merge_candidates (inter.rs:574-722), derive_amvp_candidates
// (inter.rs:814-884, quarter-sample precision), the HMVP table (inter.rs:527)
// and decode_mvd (slice.rs:1808-1834) for pictures whose coding units are
// whole 32 x 32 CTUs: the motion field is kept per CTU, which is what every
// 4x4 lookup of those functions reads there (a neighbour position lies in a
// CTU decoded before, or in none).
#pragma once
#include "cabac_parse.h"

namespace vvcg_parse {

// predict.rs:1455-1506 derive_intra_mpms (left / above < 0: absent, Planar)
inline void intra_mpms(int left, int above, uint8_t mpm[6]) {
  const int l = std::min(left < 0 ? 0 : left, 66), a = std::min(above < 0 ? 0 : above, 66);
  auto wrap = [](int m) { return (uint8_t)(((m + 62) & 63) + 2); };
  const int lo = std::min(l, a), hi = std::max(l, a);
  mpm[0] = 0;
  if (hi < 2) {
    memcpy(mpm, kMpmNoNeighbours, 6);
    return;
  }
  if (l == a || lo < 2) {
    const uint8_t r[5] = {(uint8_t)hi, wrap(hi - 1), wrap(hi + 1), wrap(hi - 2), wrap(hi + 2)};
    memcpy(mpm + 1, r, 5);
    return;
  }
  mpm[1] = (uint8_t)l;
  mpm[2] = (uint8_t)a;
  const int d = hi - lo;
  if (d == 1) {
    mpm[3] = wrap(lo - 1), mpm[4] = wrap(hi + 1), mpm[5] = wrap(lo - 2);
  } else if (d >= 62) {
    mpm[3] = wrap(lo + 1), mpm[4] = wrap(hi - 1), mpm[5] = wrap(lo + 2);
  } else if (d == 2) {
    mpm[3] = wrap(lo + 1), mpm[4] = wrap(lo - 1), mpm[5] = wrap(hi + 1);
  } else {
    mpm[3] = wrap(lo - 1), mpm[4] = wrap(lo + 1), mpm[5] = wrap(hi - 1);
  }
}

// slice.rs:1691-1717 decode_full_luma_intra_mode (no MRL, no ISP) with
// resolve_non_mpm_luma_mode (predict.rs:1512-1522)
inline int decode_full_luma_mode(Reader& r, Models& m, const uint8_t mpm[6]) {
  if (r.bin(m[kCtxIntraLumaMpmFlag])) {
    if (!r.bin(m[kCtxIntraLumaPlanarFlag + 1])) return mpm[0];
    return mpm[std::min(5u, r.unary_max(4) + 1)];
  }
  uint8_t sorted[6];
  memcpy(sorted, mpm, 6);
  std::sort(sorted, sorted + 6);
  int mode = (int)r.trunc_bin(61);
  for (int k = 0; k < 6; k++)
    if (mode >= sorted[k]) mode++;
  return mode;
}

// slice.rs:1756-1780 decode_chroma_intra_mode without CCLM
inline int decode_chroma_mode(Reader& r, Models& m, int luma) {
  if (!r.bin(m[kCtxIntraChromaPredMode])) return luma;
  static const int kCand[4] = {0, 50, 18, 1};
  const int c = kCand[std::min(3u, r.bypass_bins(2))];
  return c == luma ? 66 : c;
}

// A coded TB: transform_skip_flag, then residual_ts_coding or residual_coding.
inline int parse_tb(Reader& r, Models& m, const Scan& s, int32_t* c, bool luma, bool dq, bool sdh, bool* ts) {
  *ts = r.bin(m[kCtxTransformSkipFlag + (luma ? 0 : 1)]);
  if (*ts) {
    decode_ts_residual(r, m, s, c);
    return kOk;
  }
  return decode_residual(r, m, s, c, luma, dq, sdh);
}

// A TB's levels into the sink; its level_off (absolute) or an error.
inline int sink_tb(LevelSink& sink, const int32_t* c, int n, int64_t level_base, int32_t* off) {
  const int64_t o = sink.put(c, n);
  if (o < 0 || level_base + o > INT32_MAX) return kTruncated;
  *off = (int32_t)(level_base + o);
  return kOk;
}

// decode_picture_multitool's parse (slice.rs:3040-3190) of one IDR picture
// with every optional tool but dep_quant / sign_data_hiding off: per 32 x 32
// coding unit in raster order the luma mode against the MPM list of the left
// neighbour's mode (the above neighbour is never in the same CTU), the chroma
// mode, cbf_cb / cbf_cr / cbf_y, each coded TB's transform_skip_flag and
// residual; then end_of_slice_one_bit and the alignment.
inline int parse_mt_idr_picture(const uint8_t* data, size_t size, int qp, int width, int height, bool dq, bool sdh,
                                vvcg_cu_rec* cus, LevelSink& sink, int64_t level_base) {
  thread_local const Scan luma_scan = make_scan(32, 32), chroma_scan = make_scan(16, 16);
  Reader r;
  r.start(data, size);
  Models m;
  m.init_i_slice(qp);
  int32_t coef[3][1024];
  const int gw = width / 32, gh = height / 32;
  for (int k = 0; k < gw * gh; k++) {
    uint8_t mpm[6];
    intra_mpms(k % gw ? cus[k - 1].luma_mode : -1, -1, mpm);
    const int mode = decode_full_luma_mode(r, m, mpm);
    const int cmode = decode_chroma_mode(r, m, mode);
    const bool cbf_cb = r.bin(m[kCtxQtCbfCb]);
    const bool cbf_cr = r.bin(m[kCtxQtCbfCr + (cbf_cb ? 1 : 0)]);
    const bool cbf_y = r.bin(m[kCtxQtCbfY]);
    const bool cbf[3] = {cbf_y, cbf_cb, cbf_cr};
    vvcg_cu_rec& rec = cus[k];
    rec.luma_mode = (uint8_t)mode;
    rec.chroma_mode = (uint8_t)cmode;
    rec.cbf = (uint8_t)((cbf_y ? 1 : 0) | (cbf_cb ? 2 : 0) | (cbf_cr ? 4 : 0));
    rec.tu_tools = 0;
    for (int c = 0; c < 3; c++) {
      rec.level_off[c] = -1;
      if (!cbf[c]) continue;
      bool ts;
      int e = parse_tb(r, m, c ? chroma_scan : luma_scan, coef[c], c == 0, dq, sdh, &ts);
      if (e) return e;
      if (ts) rec.tu_tools |= (uint8_t)(1u << c);
      if ((e = sink_tb(sink, coef[c], c ? 256 : 1024, level_base, &rec.level_off[c]))) return e;
    }
  }
  if (!r.terminate() || !r.aligned_end()) return kBadEnd;
  return kOk;
}

// ------------------------------------------------------ motion of P CUs --
struct Motion {
  int32_t mv[2][2];
  int8_t ref[2];
  uint8_t dir, bcw;
  bool alt;
  bool same_fields(const Motion& o) const {
    return ref[0] == o.ref[0] && ref[1] == o.ref[1] && mv[0][0] == o.mv[0][0] && mv[0][1] == o.mv[0][1] &&
           mv[1][0] == o.mv[1][0] && mv[1][1] == o.mv[1][1];
  }
};

inline Motion zero_l0() {
  Motion z{};
  z.ref[0] = 0;
  z.ref[1] = -1;
  z.dir = 1;
  z.bcw = 2;
  return z;
}

// inter.rs:170-183 Mv::shr_round: symmetric rounding shift
inline int32_t mv_shr_round(int32_t v, int s) { return s ? (v + (1 << (s - 1)) + (v >= 0 ? -1 : 0)) >> s : v; }

// Motion of the CTUs decoded so far (a CTU-sized coding unit covers every
// 4x4 cell of its CTU) and the HMVP list of the current CTU row.
struct MotionField {
  int cols = 0, rows = 0;
  std::vector<Motion> at;
  std::vector<char> have;
  Motion hmvp[5];
  int n_hmvp = 0;
  void reset(int c, int r) {
    cols = c;
    rows = r;
    at.assign((size_t)c * r, Motion{});
    have.assign((size_t)c * r, 0);
    n_hmvp = 0;
  }
  // MotionFieldGrid::get_at_luma for CTU-sized coding units of 32
  const Motion* get(int x, int y) const {
    if (x < 0 || y < 0) return nullptr;
    const int cx = x >> 5, cy = y >> 5;
    if (cx >= cols || cy >= rows || !have[(size_t)cy * cols + cx]) return nullptr;
    return &at[(size_t)cy * cols + cx];
  }
  void set(int cx, int cy, const Motion& mo) {
    at[(size_t)cy * cols + cx] = mo;
    have[(size_t)cy * cols + cx] = 1;
  }
  // HmvpTable::push: an identical entry moves to the newest end
  void push_hmvp(const Motion& mo) {
    int i = 0;
    while (i < n_hmvp && !(hmvp[i].same_fields(mo) && hmvp[i].dir == mo.dir)) i++;
    if (i == n_hmvp && n_hmvp == 5) i = 0;  // drop the oldest
    if (i < n_hmvp) {
      for (int k = i; k + 1 < n_hmvp; k++) hmvp[k] = hmvp[k + 1];
      n_hmvp--;
    }
    hmvp[n_hmvp++] = mo;
  }
};

// derive_merge_candidates(grid, hmvp, None, bx, by, 32, 32, false, 6)[0]:
// the first of B1, A1, B0, A0, B2 (each pruned against the ones the
// reference compares it with), the newest HMVP entry, the pairwise average
// (never first) and the zero candidate.
inline Motion merge_candidate0(const MotionField& f, int bx, int by) {
  const Motion* b1 = by > 0 ? f.get(bx + 31, by - 1) : nullptr;
  const Motion* a1 = bx > 0 ? f.get(bx - 1, by + 31) : nullptr;
  const Motion* b0 = by > 0 ? f.get(bx + 32, by - 1) : nullptr;
  const Motion* a0 = bx > 0 ? f.get(bx - 1, by + 32) : nullptr;
  const Motion* b2 = (bx > 0 && by > 0) ? f.get(bx - 1, by - 1) : nullptr;
  if (b1) return *b1;
  if (a1) return *a1;
  if (b0) return *b0;  // B1 is absent here, so nothing prunes B0
  if (a0) return *a0;  // A1 is absent here
  if (b2) return *b2;
  if (f.n_hmvp) return f.hmvp[f.n_hmvp - 1];  // A1 and B1 absent: no duplicate check applies
  return zero_l0();
}

// derive_amvp_candidates(grid, hmvp, bx, by, 32, 32, 0, 0, QuarterPel)
inline void amvp_l0(const MotionField& f, int bx, int by, int32_t out[2][2]) {
  auto rnd = [](const int32_t* mv, int32_t* o) {
    for (int k = 0; k < 2; k++) o[k] = std::min(131071, std::max(-131072, mv_shr_round(mv[k], 2) * 4));
  };
  int32_t c[2][2];
  int n = 0;
  if (bx > 0) {
    const int pos[2][2] = {{bx - 1, by + 32}, {bx - 1, by + 31}};
    for (const auto& p : pos) {
      const Motion* mi = f.get(p[0], p[1]);
      if (mi && mi->ref[0] == 0) {
        rnd(mi->mv[0], c[n++]);
        break;
      }
    }
  }
  if (by > 0) {
    int pos[3][2] = {{bx + 32, by - 1}, {bx + 31, by - 1}, {bx - 1, by - 1}};
    for (int i = 0; i < (bx > 0 ? 3 : 2); i++) {
      const Motion* mi = f.get(pos[i][0], pos[i][1]);
      if (mi && mi->ref[0] == 0) {
        int32_t v[2];
        rnd(mi->mv[0], v);
        if (n == 0 || c[0][0] != v[0] || c[0][1] != v[1]) {
          c[n][0] = v[0];
          c[n][1] = v[1];
          n++;
        }
        break;
      }
    }
  }
  for (int i = f.n_hmvp - 1; i >= 0 && n < 2; i--) {
    if (f.hmvp[i].ref[0] != 0) continue;
    int32_t v[2];
    rnd(f.hmvp[i].mv[0], v);
    bool dup = false;
    for (int k = 0; k < n; k++) dup |= c[k][0] == v[0] && c[k][1] == v[1];
    if (!dup) {
      c[n][0] = v[0];
      c[n][1] = v[1];
      n++;
    }
  }
  for (; n < 2; n++) c[n][0] = c[n][1] = 0;
  memcpy(out, c, sizeof(c));
}

// slice.rs:1808-1834 decode_mvd
inline void decode_mvd(Reader& r, Models& m, int32_t mvd[2]) {
  bool gt0[2], gt1[2] = {false, false};
  for (int i = 0; i < 2; i++) gt0[i] = r.bin(m[kCtxMvd]);
  for (int i = 0; i < 2; i++)
    if (gt0[i]) gt1[i] = r.bin(m[kCtxMvd + 1]);
  for (int i = 0; i < 2; i++) {
    mvd[i] = 0;
    if (!gt0[i]) continue;
    const int32_t a = gt1[i] ? (int32_t)r.rem_abs(1, 0, 17) + 2 : 1;
    mvd[i] = r.bypass() ? -a : a;
  }
}

// decode_inter_picture's parse (slice.rs:3591-3677, P slice, SAO / ALF /
// joint Cb-Cr off) of one P picture with 32 x 32 CTUs: per CTU the skip flag
// (context from the left / above CTUs' skip flags); unless skipped
// pred_mode_flag (an intra coding unit is an error, as in the reference),
// general_merge_flag, and for AMVP the mvd, mvp_l0_flag and rqt_root_cbf;
// the motion (merge candidate 0, or the AMVP predictor plus the difference)
// into the CTU motion field and the HMVP list; then when a residual is
// coded the cbfs (tu_y_coded_flag inferred 1 when both chroma cbfs are 0)
// and each coded TB's transform_skip_flag and residual.
inline int parse_mt_p_picture(const uint8_t* data, size_t size, int qp, int width, int height, bool dq, bool sdh,
                              vvcg_inter_cu* cus, LevelSink& sink, int64_t level_base) {
  thread_local const Scan luma_scan = make_scan(32, 32), chroma_scan = make_scan(16, 16);
  thread_local MotionField field;
  Reader r;
  r.start(data, size);
  Models m;
  m.init(qp, kCtxInitP);
  int32_t coef[3][1024];
  const int gw = width / 32, gh = height / 32;
  field.reset(gw, gh);
  std::vector<char> skip((size_t)gw * gh, 0);
  for (int gy = 0; gy < gh; gy++) {
    field.n_hmvp = 0;
    for (int gx = 0; gx < gw; gx++) {
      const int k = gy * gw + gx, bx = gx * 32, by = gy * 32;
      vvcg_inter_cu& rec = cus[k];
      memset(&rec, 0, sizeof(rec));
      const int sctx = kCtxSkipFlag + (gx > 0 && skip[k - 1] ? 1 : 0) + (gy > 0 && skip[k - gw] ? 1 : 0);
      const bool cu_skip = r.bin(m[sctx]);
      skip[k] = cu_skip;
      Motion mo;
      bool any_cbf = false;
      if (cu_skip) {
        mo = merge_candidate0(field, bx, by);
        rec.flags = VVCG_INTER_CU_SKIP | VVCG_INTER_CU_MERGE;
      } else {
        if (r.bin(m[kCtxPredMode])) return kIntraInP;
        const bool merge = r.bin(m[kCtxMergeFlag]);
        if (merge) {
          mo = merge_candidate0(field, bx, by);
          rec.flags = VVCG_INTER_CU_MERGE;
        } else {
          decode_mvd(r, m, rec.mvd);
          rec.mvp_idx = r.bin(m[kCtxMvpIdx]) ? 1 : 0;
          int32_t mvp[2][2];
          amvp_l0(field, bx, by, mvp);
          mo = zero_l0();
          mo.mv[0][0] = mvp[rec.mvp_idx][0] + rec.mvd[0];
          mo.mv[0][1] = mvp[rec.mvp_idx][1] + rec.mvd[1];
        }
        any_cbf = merge || r.bin(m[kCtxQtRootCbf]);
      }
      field.set(gx, gy, mo);
      field.push_hmvp(mo);
      memcpy(rec.mv, mo.mv, sizeof(rec.mv));
      rec.ref_idx[0] = mo.ref[0];
      rec.ref_idx[1] = mo.ref[1];
      rec.inter_dir = mo.dir;
      rec.bcw_idx = mo.bcw;
      if (mo.alt) rec.flags |= VVCG_INTER_CU_ALT_HPEL;
      rec.level_off[0] = rec.level_off[1] = rec.level_off[2] = -1;
      if (!any_cbf) continue;
      const bool cbf_cb = r.bin(m[kCtxQtCbfCb]);
      const bool cbf_cr = r.bin(m[kCtxQtCbfCr + (cbf_cb ? 1 : 0)]);
      const bool cbf_y = (cbf_cb || cbf_cr) ? r.bin(m[kCtxQtCbfY]) : true;
      const bool cbf[3] = {cbf_y, cbf_cb, cbf_cr};
      rec.cbf = (uint8_t)((cbf_y ? 1 : 0) | (cbf_cb ? 2 : 0) | (cbf_cr ? 4 : 0));
      for (int c = 0; c < 3; c++) {
        if (!cbf[c]) continue;
        bool ts;
        int e = parse_tb(r, m, c ? chroma_scan : luma_scan, coef[c], c == 0, dq, sdh, &ts);
        if (e) return e;
        if (ts) rec.tu_tools |= (uint8_t)(1u << c);
        if ((e = sink_tb(sink, coef[c], c ? 256 : 1024, level_base, &rec.level_off[c]))) return e;
      }
    }
  }
  if (!r.terminate() || !r.aligned_end()) return kBadEnd;
  return kOk;
}

}  // namespace vvcg_parse
