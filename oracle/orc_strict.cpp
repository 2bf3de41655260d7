// CPU oracle (test infrastructure only; see oracle.h): the strict 8-bit 4:2:0
// intra profile of the reference encoder and decoder
// (crates/rustmpeg-video/src/vvc/slice.rs):
//   encode_picture            slice.rs:325-455  decisions and reconstruction of
//                                               one IDR picture (the CABAC
//                                               writes are not restated)
//   decode_picture            slice.rs:458-627  reconstruction from the parsed
//                                               syntax
//   encode_chroma             slice.rs:771-808
//   encode_luma               slice.rs:810-874  (orc_luma_tx_search, orc_tu.cpp)
//   plan_primary / _ts        slice.rs:694-766
//   reconstruct_block         slice.rs:1050-1097
//   CuConstraints, scan_pos_last, max_lfnst_pos, violates_mts_constraint,
//   lfnst_syntax_present, mts_syntax_present        slice.rs:920-992
//   choose_intra_mode         predict.rs:2706-2733 (Planar wins ties)
//
// Both functions walk the tb x tb coding units (tb = min(CTU, 32)) in raster
// order of the tb grid, as the reference does. The records are what the
// decoder parses: luma and chroma modes, cbf, the transform-skip flags of the
// coded TBs, and the mts_idx / lfnst_idx values decode_picture reads (zero
// where their syntax is absent), in vvcg_cu_rec with VVCG_TOOL_TU_TOOLS; the
// levels of each coded TB are dense raster int16.
#include <string.h>

#include <algorithm>
#include <vector>

#include "oracle.h"

extern "C" int orc_luma_tx_search(int n, const int32_t* pred, const int32_t* src, int qp, int mode, int use_ts,
                                  int chroma_can_lfnst, int16_t* levels, int16_t* samples, uint64_t* sse_out);

namespace orc {
namespace {

const int PLANAR = 0, DC = 1;

struct Plane8w {  // writable 8-bit plane, stride = width
  std::vector<uint8_t> d;
  int w = 0, h = 0;
  Plane8 view() const { return Plane8{d.data(), w, h}; }
};

// slice.rs:920-925 scan_pos_last over CoeffScan(w, h)
int scan_pos_last(const int32_t* lv, int w, int h) {
  std::vector<int32_t> scan(w * h);
  const int ns = coeff_scan_raster(w, h, scan.data());
  for (int s = ns - 1; s >= 0; s--)
    if (lv[scan[s]] != 0) return s;
  return -1;
}

// slice.rs:927-934 max_lfnst_pos
int max_lfnst_pos(int w, int h) { return ((w == 4 && h == 4) || (w == 8 && h == 8)) ? 7 : 15; }

// slice.rs:937-948 violates_mts_constraint
bool violates_mts_constraint(const int32_t* lv, int size) {
  for (int i = 0; i < size * size; i++)
    if (lv[i] != 0 && ((i % size) / 4 > 3 || (i / size) / 4 > 3)) return true;
  return false;
}

// slice.rs:951-979 CuConstraints
struct CuConstraints {
  bool violates_lfnst[2] = {false, false};
  bool lfnst_last_scan_pos = false, violates_mts = false, mts_last_scan_pos = false;
  void update(const int32_t* lv, int size, bool is_luma, bool ts) {
    const int last = scan_pos_last(lv, size, size);
    if (last < 0 || ts) return;
    if (size >= 4) {
      violates_lfnst[is_luma ? 0 : 1] |= last > max_lfnst_pos(size, size);
      lfnst_last_scan_pos |= last >= 1;
    }
    if (is_luma) {
      mts_last_scan_pos |= last >= 1;
      violates_mts |= violates_mts_constraint(lv, size);
    }
  }
};

// slice.rs:981-992
bool lfnst_syntax_present(const CuConstraints& c, bool any_ts) {
  return !any_ts && c.lfnst_last_scan_pos && !c.violates_lfnst[0] && !c.violates_lfnst[1];
}
bool mts_syntax_present(const CuConstraints& c, bool luma_ts, int lfnst_idx) {
  return !luma_ts && !c.violates_mts && c.mts_last_scan_pos && lfnst_idx == 0;
}

// slice.rs:647-656 mts_types
void mts_types(int idx, int* th, int* tv) {
  static const int T[5][2] = {{kDct2, kDct2}, {kDst7, kDst7}, {kDct8, kDst7}, {kDst7, kDct8}, {kDct8, kDct8}};
  *th = T[idx][0];
  *tv = T[idx][1];
}

// A component plan (slice.rs:631-645 BlockPlan): levels, cbf, samples.
struct Plan {
  std::vector<int32_t> levels, samples;
  bool cbf = false, ts = false;
  int mts = 0, lfnst = 0;
};

// slice.rs:694-713 plan_transform_skip
Plan plan_ts(const std::vector<int32_t>& pred, const std::vector<int32_t>& res, int n, int qp) {
  Plan p;
  p.ts = true;
  p.levels.resize(n * n);
  p.samples.resize(n * n);
  for (int i = 0; i < n * n; i++) {
    p.levels[i] = quantize_ts(res[i], qp);
    p.cbf |= p.levels[i] != 0;
    p.samples[i] = std::min(255, std::max(0, pred[i] + dequantize_ts(p.levels[i], qp)));
  }
  return p;
}

// slice.rs:718-766 plan_primary with DCT-2 and no LFNST (the chroma plan;
// DCT-2 at 16 or 32 has no zero-out here, slice.rs:659-670)
Plan plan_dct2(const std::vector<int32_t>& pred, const std::vector<int32_t>& res, int n, int qp) {
  Plan p;
  std::vector<int32_t> co(n * n), deq(n * n), rec(n * n);
  forward_transform_rect_bd(n, n, res.data(), kDct2, kDct2, 0, 0, 8, co.data());
  p.levels.assign(n * n, 0);
  quantize_rect_bd(n, n, co.data(), qp, 8, true, p.levels.data());
  for (int v : p.levels) p.cbf |= v != 0;
  dequantize_rect_bd(n, n, p.levels.data(), qp, 8, deq.data());
  inverse_transform_rect_bd(n, n, deq.data(), kDct2, kDct2, 0, 0, 8, rec.data());
  p.samples.resize(n * n);
  for (int i = 0; i < n * n; i++) p.samples[i] = std::min(255, std::max(0, pred[i] + rec[i]));
  return p;
}

std::vector<int32_t> predict(const Plane8w& r, int bx, int by, int n, bool is_luma, int mode) {
  std::vector<int32_t> p(n * n);
  predict_block_8(r.view(), bx, by, n, n, is_luma, mode, p.data());
  return p;
}

std::vector<int32_t> block_of(const uint8_t* plane, int stride, int bx, int by, int n) {
  std::vector<int32_t> b(n * n);
  for (int y = 0; y < n; y++)
    for (int x = 0; x < n; x++) b[y * n + x] = plane[(size_t)(by + y) * stride + bx + x];
  return b;
}

void store(Plane8w& r, int bx, int by, int n, const std::vector<int32_t>& s) {
  for (int y = 0; y < n; y++)
    for (int x = 0; x < n; x++) r.d[(size_t)(by + y) * r.w + bx + x] = (uint8_t)s[y * n + x];
}

// predict.rs:2706-2733 choose_intra_mode: DC only on a strictly lower SAD
int choose_intra_mode(const Plane8w& recon, const uint8_t* src, int bx, int by, int n) {
  auto sad = [&](int mode) {
    std::vector<int32_t> p = predict(recon, bx, by, n, true, mode);
    uint64_t s = 0;
    for (int y = 0; y < n; y++)
      for (int x = 0; x < n; x++) s += (uint64_t)std::abs((int)src[(size_t)(by + y) * recon.w + bx + x] - p[y * n + x]);
    return s;
  };
  return sad(DC) < sad(PLANAR) ? DC : PLANAR;
}

int luma_qp_of(int qp) { return std::max(qp, 4); }
int chroma_qp_of(int qp) { return std::max(std::min(std::max(derived_chroma_qp(qp), 0), 63), 4); }

// slice.rs:1050-1097 reconstruct_block
int reconstruct_block(Plane8w& recon, int bx, int by, int n, bool is_luma, int qp, const int32_t* lv, int mode,
                      bool ts, int mts, int lfnst) {
  std::vector<int32_t> pred = predict(recon, bx, by, n, is_luma, mode), res(n * n, 0);
  if (ts) {
    for (int i = 0; i < n * n; i++) res[i] = dequantize_ts(lv[i], qp);
  } else {
    int th, tv, sw, sh;
    mts_types(mts, &th, &tv);
    if (lfnst > 0) {  // slice.rs:674-682 lfnst_skips
      sw = n >= 8 ? n - 8 : 0;
      sh = n >= 8 ? n - 8 : 0;
    } else {  // slice.rs:659-670 primary_skips
      sw = (n == 32 && th != kDct2) ? 16 : 0;
      sh = (n == 32 && tv != kDct2) ? 16 : 0;
    }
    std::vector<int32_t> deq(n * n);
    if (dequantize_rect_bd(n, n, lv, qp, 8, deq.data())) return -1;
    if (lfnst > 0 && inverse_lfnst_rect(deq.data(), n, n, lfnst, mode)) return -2;
    if (inverse_transform_rect_bd(n, n, deq.data(), th, tv, sw, sh, 8, res.data())) return -3;
  }
  for (int y = 0; y < n; y++)
    for (int x = 0; x < n; x++)
      recon.d[(size_t)(by + y) * recon.w + bx + x] = (uint8_t)std::min(255, std::max(0, pred[y * n + x] + res[y * n + x]));
  return 0;
}

}  // namespace

int strict_encode(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h, int qp, int ctu_log2,
                  vvcg_cu_rec* cus, int16_t* levels, uint64_t* num_levels, uint8_t* ry, uint8_t* ru, uint8_t* rv) {
  // encode_picture steps columns by tb and rows by the CTU size
  // (slice.rs:342-452), which codes every CU only at CTU 32
  if (ctu_log2 != 5 || w < 32 || h < 32 || w % 32 || h % 32 || qp < 0 || qp > 63) return -1;
  const int tb = 32, cw = tb / 2, pw = w, cwp = w / 2;
  const int lqp = luma_qp_of(qp), cqp = chroma_qp_of(qp);
  const bool luma_ts = lqp == 4, chroma_ts = cqp == 4;  // slice.rs:339-340
  // the reconstruction starts as a copy of the source (Planes::from_frame)
  Plane8w R[3];
  R[0].d.assign(y, y + (size_t)w * h);
  R[0].w = w, R[0].h = h;
  R[1].d.assign(u, u + (size_t)cwp * (h / 2));
  R[2].d.assign(v, v + (size_t)cwp * (h / 2));
  R[1].w = R[2].w = cwp;
  R[1].h = R[2].h = h / 2;
  const uint8_t* S[3] = {y, u, v};
  uint64_t at = 0;
  int k = 0;
  for (int by = 0; by < h; by += tb)
    for (int bx = 0; bx < w; bx += tb, k++) {
      const int cx = bx / 2, cy = by / 2;
      const int mode = choose_intra_mode(R[0], y, bx, by, tb);
      // encode_chroma (slice.rs:771-808): DCT-2, or transform skip at QP 4
      Plan ch[2];
      for (int c = 1; c <= 2; c++) {
        std::vector<int32_t> pred = predict(R[c], cx, cy, cw, false, mode), res(cw * cw);
        std::vector<int32_t> src = block_of(S[c], cwp, cx, cy, cw);
        for (int i = 0; i < cw * cw; i++) res[i] = src[i] - pred[i];
        ch[c - 1] = chroma_ts ? plan_ts(pred, res, cw, cqp) : plan_dct2(pred, res, cw, cqp);
      }
      CuConstraints cc;
      for (int c = 0; c < 2; c++)
        if (ch[c].cbf) cc.update(ch[c].levels.data(), cw, false, ch[c].ts);
      // encode_luma (slice.rs:810-874)
      Plan L;
      {
        std::vector<int32_t> pred = predict(R[0], bx, by, tb, true, mode);
        std::vector<int32_t> src = block_of(y, pw, bx, by, tb);
        std::vector<int16_t> lv(tb * tb), sm(tb * tb);
        uint64_t sse = 0;
        const int r = orc_luma_tx_search(tb, pred.data(), src.data(), lqp, mode, luma_ts, !cc.violates_lfnst[1],
                                         lv.data(), sm.data(), &sse);
        L.cbf = r & 1;
        L.ts = (r >> 1) & 1;
        L.lfnst = (r >> 4) & 0xF;
        L.mts = (r >> 8) & 0xF;
        L.levels.assign(lv.begin(), lv.end());
        L.samples.assign(sm.begin(), sm.end());
      }
      store(R[0], bx, by, tb, L.samples);
      store(R[1], cx, cy, cw, ch[0].samples);
      store(R[2], cx, cy, cw, ch[1].samples);
      // the syntax decode_picture reads back (slice.rs:545-572)
      CuConstraints con;
      if (L.cbf) con.update(L.levels.data(), tb, true, L.ts);
      for (int c = 0; c < 2; c++)
        if (ch[c].cbf) con.update(ch[c].levels.data(), cw, false, ch[c].ts);
      const bool any_ts = (L.cbf && L.ts) || (ch[0].cbf && ch[0].ts) || (ch[1].cbf && ch[1].ts);
      const int lfnst = lfnst_syntax_present(con, any_ts) ? L.lfnst : 0;
      const int mts = mts_syntax_present(con, any_ts && L.ts, lfnst) ? L.mts : 0;
      vvcg_cu_rec& rec = cus[k];
      memset(&rec, 0, sizeof(rec));
      rec.luma_mode = rec.chroma_mode = (uint8_t)mode;  // chroma DM
      const Plan* P[3] = {&L, &ch[0], &ch[1]};
      const int n[3] = {tb * tb, cw * cw, cw * cw};
      uint32_t tools = (uint32_t)(mts << VVCG_CU_MTS_SHIFT) | (uint32_t)(lfnst << VVCG_CU_LFNST_SHIFT);
      for (int c = 0; c < 3; c++) {
        rec.level_off[c] = -1;
        if (!P[c]->cbf) continue;
        rec.cbf |= (uint8_t)(1 << c);
        if (P[c]->ts) tools |= 1u << c;
        rec.level_off[c] = (int32_t)at;
        for (int i = 0; i < n[c]; i++) levels[at + i] = (int16_t)P[c]->levels[i];
        at += n[c];
      }
      rec.tu_tools = (uint8_t)tools;
    }
  *num_levels = at;
  memcpy(ry, R[0].d.data(), R[0].d.size());
  memcpy(ru, R[1].d.data(), R[1].d.size());
  memcpy(rv, R[2].d.data(), R[2].d.size());
  return 0;
}

int strict_decode(const vvcg_cu_rec* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                  int ctu_log2, uint8_t* ry, uint8_t* ru, uint8_t* rv) {
  if (ctu_log2 < 5 || ctu_log2 > 7 || w % (1 << ctu_log2) || h % (1 << ctu_log2) || !w || !h) return -1;
  const int tb = std::min(1 << ctu_log2, 32), cw = tb / 2;  // decode_picture's ctu.min(32)
  const int lqp = luma_qp_of(qp), cqp = chroma_qp_of(qp);
  Plane8w R[3];
  R[0].d.assign((size_t)w * h, 0);
  R[0].w = w, R[0].h = h;
  for (int c = 1; c <= 2; c++) {
    R[c].d.assign((size_t)(w / 2) * (h / 2), 0);
    R[c].w = w / 2;
    R[c].h = h / 2;
  }
  int k = 0;
  for (int by = 0; by < h; by += tb)
    for (int bx = 0; bx < w; bx += tb, k++) {
      const vvcg_cu_rec& r = cus[k];
      const uint32_t t = r.tu_tools;
      const int mts = (t >> VVCG_CU_MTS_SHIFT) & 7, lfnst = t >> VVCG_CU_LFNST_SHIFT;
      if (r.luma_mode > 66 || r.chroma_mode > 66 || mts > 4 || lfnst > 2 || (mts && lfnst)) return -2;
      const int n[3] = {tb * tb, cw * cw, cw * cw};
      std::vector<int32_t> lv[3];
      for (int c = 0; c < 3; c++) {
        lv[c].assign(n[c], 0);
        if (!((r.cbf >> c) & 1) || r.level_off[c] < 0) continue;
        if ((uint64_t)r.level_off[c] + n[c] > num_levels) return -3;
        for (int i = 0; i < n[c]; i++) lv[c][i] = levels[r.level_off[c] + i];
      }
      const bool ts_y = (r.cbf & 1) && (t & VVCG_CU_TS_Y);
      if (ts_y && (mts || lfnst)) return -2;
      int rc = reconstruct_block(R[0], bx, by, tb, true, lqp, lv[0].data(), r.luma_mode, ts_y, mts, lfnst);
      for (int c = 1; c <= 2 && !rc; c++)
        rc = reconstruct_block(R[c], bx / 2, by / 2, cw, false, cqp, lv[c].data(), r.chroma_mode,
                               ((r.cbf >> c) & 1) && ((t >> c) & 1), 0, 0);
      if (rc) return -4;
    }
  memcpy(ry, R[0].d.data(), R[0].d.size());
  memcpy(ru, R[1].d.data(), R[1].d.size());
  memcpy(rv, R[2].d.data(), R[2].d.size());
  return 0;
}

}  // namespace orc
