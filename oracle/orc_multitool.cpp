// CPU oracle (test infrastructure only; see oracle.h): the multi-tool 8-bit
// 4:2:0 stream of the reference (VvcMultiToolEncoder, mod.rs:1512-1720): its
// IDR picture and its P pictures, decisions and reconstruction (the CABAC
// writes are in orc_cabac.cpp). Restated from
// crates/rustmpeg-video/src/vvc/:
//   derive_intra_mpms           predict.rs:1455-1506
//   encode_picture_multitool    slice.rs:2575-2970 (options: dep_quant,
//                               sign_data_hiding, full_intra_modes,
//                               enable_deblock; the other tools are not
//                               restated and rejected)
//   decode_picture_multitool    slice.rs:3012-3300 (reconstruction)
//   encode_component_full       slice.rs:1836-1918
//   reconstruct_component_full  slice.rs:1920-1990
//   encode_inter_picture        slice.rs:3307-3549 (P slices)
//   decode_inter_picture        slice.rs:3552-3835 (reconstruction and the
//                               motion derivation of merge / AMVP CUs)
//   MotionFieldGrid, HmvpTable  inter.rs:311-369, :527-560
//   derive_merge_candidates     inter.rs:574-722
//   derive_amvp_candidates      inter.rs:814-884 (quarter-sample AMVR)
//   predict_inter_pu            inter.rs:1734-1848 (without DMVR / BDOF,
//                               which the P-slice decoder leaves off)
// Multi-tool records use vvcg_cu_rec (VVCG_TOOL_TU_TOOLS: transform-skip
// flags only); inter records use vvcg_inter_cu; levels are dense raster int16.
#include <string.h>

#include <algorithm>
#include <vector>

#include "oracle.h"

namespace orc {
namespace {

int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

struct Plane8w {  // writable 8-bit plane, stride = width
  std::vector<uint8_t> d;
  int w = 0, h = 0;
  Plane8 view() const { return Plane8{d.data(), w, h}; }
  void assign(const uint8_t* src, int ww, int hh) {
    w = ww;
    h = hh;
    if (src)
      d.assign(src, src + (size_t)ww * hh);
    else
      d.assign((size_t)ww * hh, 0);
  }
};

int luma_qp_of(int qp) { return std::max(qp, 4); }
int chroma_qp_of(int qp) { return std::max(clampi(derived_chroma_qp(qp), 0, 63), 4); }

std::vector<int32_t> scan_raster_of(int w, int h) {
  std::vector<int32_t> s(w * h);
  coeff_scan_raster(w, h, s.data());
  return s;
}

// slice.rs:1836-1918 encode_component_full: residual, DCT-2 (no extra
// zero-out at 16 / 32) or transform skip, quantisation (the intra rounding
// offset on every picture, as the reference passes is_intra = true), and the
// reconstruction.
struct Coded {
  std::vector<int32_t> levels;
  std::vector<uint8_t> recon;
  bool cbf = false;
};

int encode_component_full(const std::vector<int32_t>& pred, const uint8_t* src, int stride, int bx, int by, int w,
                          int h, int qp, bool ts, bool dq, Coded* out) {
  std::vector<int32_t> res(w * h);
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) res[y * w + x] = (int)src[(size_t)(by + y) * stride + bx + x] - pred[y * w + x];
  out->levels.assign(w * h, 0);
  out->recon.assign(w * h, 0);
  out->cbf = false;
  if (ts) {
    for (int i = 0; i < w * h; i++) {
      out->levels[i] = quantize_ts(res[i], qp);
      out->cbf |= out->levels[i] != 0;
    }
    for (int i = 0; i < w * h; i++)
      out->recon[i] = (uint8_t)clampi(pred[i] + (out->cbf ? dequantize_ts(out->levels[i], qp) : 0), 0, 255);
    return 0;
  }
  std::vector<int32_t> co(w * h), deq(w * h), inv(w * h);
  if (forward_transform_rect_bd(w, h, res.data(), kDct2, kDct2, 0, 0, 8, co.data())) return -1;
  const std::vector<int32_t> scan = scan_raster_of(w, h);
  if (dq) {
    if (quantize_dep_quant_bd(w, h, co.data(), scan.data(), qp, 8, out->levels.data())) return -1;
  } else if (quantize_rect_bd(w, h, co.data(), qp, 8, true, out->levels.data())) {
    return -1;
  }
  for (int v : out->levels) out->cbf |= v != 0;
  if (!out->cbf) {
    for (int i = 0; i < w * h; i++) out->recon[i] = (uint8_t)clampi(pred[i], 0, 255);
    return 0;
  }
  if (dq ? dequantize_dep_quant_bd(w, h, out->levels.data(), scan.data(), qp, 8, deq.data())
         : dequantize_rect_bd(w, h, out->levels.data(), qp, 8, deq.data()))
    return -1;
  if (inverse_transform_rect_bd(w, h, deq.data(), kDct2, kDct2, 0, 0, 8, inv.data())) return -1;
  for (int i = 0; i < w * h; i++) out->recon[i] = (uint8_t)clampi(pred[i] + inv[i], 0, 255);
  return 0;
}

// slice.rs:1920-1990 reconstruct_component_full
int reconstruct_component_full(Plane8w& recon, const std::vector<int32_t>& pred, int bx, int by, int w, int h, int qp,
                               const int32_t* levels, bool cbf, bool ts, bool dq) {
  std::vector<int32_t> add(w * h, 0);
  if (cbf && ts) {
    for (int i = 0; i < w * h; i++) add[i] = dequantize_ts(levels[i], qp);
  } else if (cbf) {
    std::vector<int32_t> deq(w * h);
    const std::vector<int32_t> scan = scan_raster_of(w, h);
    if (dq ? dequantize_dep_quant_bd(w, h, levels, scan.data(), qp, 8, deq.data())
           : dequantize_rect_bd(w, h, levels, qp, 8, deq.data()))
      return -1;
    if (inverse_transform_rect_bd(w, h, deq.data(), kDct2, kDct2, 0, 0, 8, add.data())) return -1;
  }
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++)
      recon.d[(size_t)(by + y) * recon.w + bx + x] = (uint8_t)clampi(pred[y * w + x] + add[y * w + x], 0, 255);
  return 0;
}

void store(Plane8w& r, int bx, int by, int w, int h, const std::vector<uint8_t>& s) {
  for (int y = 0; y < h; y++) memcpy(&r.d[(size_t)(by + y) * r.w + bx], &s[(size_t)y * w], w);
}

std::vector<int32_t> predict(const Plane8w& r, int bx, int by, int n, bool is_luma, int mode) {
  std::vector<int32_t> p(n * n);
  predict_block_8(r.view(), bx, by, n, n, is_luma, mode, p.data());
  return p;
}

// predict.rs:2706-2733 choose_intra_mode (Planar wins ties)
int choose_planar_dc(const Plane8w& recon, const uint8_t* src, int bx, int by, int n) {
  auto sad = [&](int mode) {
    std::vector<int32_t> p = predict(recon, bx, by, n, true, mode);
    uint64_t s = 0;
    for (int y = 0; y < n; y++)
      for (int x = 0; x < n; x++) s += (uint64_t)std::abs((int)src[(size_t)(by + y) * recon.w + bx + x] - p[y * n + x]);
    return s;
  };
  return sad(1) < sad(0) ? 1 : 0;
}

std::vector<int32_t> levels_of(const vvcg_cu_rec& r, const int16_t* levels, uint64_t num, int c, int n, bool* ok) {
  std::vector<int32_t> v(n, 0);
  if (!((r.cbf >> c) & 1)) return v;
  if (r.level_off[c] < 0 || (uint64_t)r.level_off[c] + n > num) {
    *ok = false;
    return v;
  }
  for (int i = 0; i < n; i++) v[i] = levels[r.level_off[c] + i];
  return v;
}

// ------------------------------------------------------------ motion --------
struct MvF {
  int mv[2] = {0, 0};
  int ref = -1;
  bool operator==(const MvF& o) const { return mv[0] == o.mv[0] && mv[1] == o.mv[1] && ref == o.ref; }
  bool operator!=(const MvF& o) const { return !(*this == o); }
};

struct Cand {
  int dir = 1;
  MvF f[2];
  int bcw = 2;
  bool alt = false;
  bool same_fields(const Cand& o) const { return f[0] == o.f[0] && f[1] == o.f[1]; }
};

// inter.rs:311-369 MotionFieldGrid: one entry per 4x4 luma block
struct MotionGrid {
  int cols, rows;
  std::vector<char> has;
  std::vector<Cand> c;
  MotionGrid(int w, int h) : cols((w + 3) / 4), rows((h + 3) / 4), has(cols * rows, 0), c(cols * rows) {}
  bool get(int x, int y, Cand* out) const {
    const int gx = x >> 2, gy = y >> 2;
    if (gx < cols && gy < rows && has[gy * cols + gx]) {
      *out = c[gy * cols + gx];
      return true;
    }
    return false;
  }
  void fill(int bx, int by, int w, int h, const Cand& v) {
    const int x1 = std::min((bx + w + 3) / 4, cols), y1 = std::min((by + h + 3) / 4, rows);
    for (int gy = by >> 2; gy < y1; gy++)
      for (int gx = bx >> 2; gx < x1; gx++) {
        has[gy * cols + gx] = 1;
        c[gy * cols + gx] = v;
      }
  }
};

// inter.rs:527-560 HmvpTable (5 entries, identical-candidate pruning)
struct Hmvp {
  std::vector<Cand> c;
  void push(const Cand& v) {
    for (size_t i = 0; i < c.size(); i++)
      if (c[i].same_fields(v) && c[i].dir == v.dir) {
        c.erase(c.begin() + (long)i);
        c.push_back(v);
        return;
      }
    if (c.size() >= 5) c.erase(c.begin());
    c.push_back(v);
  }
};

// inter.rs:170-183 Mv::shr_round
int shr_round(int v, int shift) {
  if (shift == 0) return v;
  return (v + (1 << (shift - 1)) + ((~v) >> 31)) >> shift;
}

// inter.rs:574-722 derive_merge_candidates (no collocated candidate)
std::vector<Cand> merge_candidates(const MotionGrid& g, const Hmvp& hm, int bx, int by, int w, int h, bool is_b,
                                   int max_num) {
  const size_t maxc = (size_t)clampi(max_num, 1, 6);
  std::vector<Cand> list;
  Cand b1, a1, b0, a0, b2;
  const bool hb1 = by > 0 && g.get(bx + w - 1, by - 1, &b1);
  const bool ha1 = bx > 0 && g.get(bx - 1, by + h - 1, &a1);
  const bool hb0 = by > 0 && g.get(bx + w, by - 1, &b0);
  const bool ha0 = bx > 0 && g.get(bx - 1, by + h, &a0);
  const bool hb2 = bx > 0 && by > 0 && g.get(bx - 1, by - 1, &b2);
  if (hb1) list.push_back(b1);
  if (list.size() < maxc && ha1 && (!hb1 || !b1.same_fields(a1))) list.push_back(a1);
  if (list.size() < maxc && hb0 && (!hb1 || !b1.same_fields(b0))) list.push_back(b0);
  if (list.size() < maxc && ha0 && (!ha1 || !a1.same_fields(a0))) list.push_back(a0);
  if (list.size() < 4 && list.size() < maxc && hb2 && (!ha1 || !a1.same_fields(b2)) &&
      (!hb1 || !b1.same_fields(b2)))
    list.push_back(b2);
  for (int i = (int)hm.c.size() - 1; i >= 0; i--) {
    if (list.size() >= maxc - 1) break;
    const Cand& hc = hm.c[i];
    const bool dup_a1 = ha1 && a1.same_fields(hc), dup_b1 = hb1 && b1.same_fields(hc);
    if (!dup_a1 && !dup_b1) list.push_back(hc);
  }
  if (list.size() >= 2 && list.size() < maxc) {
    const Cand c0 = list[0], c1 = list[1];
    Cand avg;
    avg.dir = 0;
    avg.f[0] = avg.f[1] = MvF();
    avg.bcw = 2;
    avg.alt = c0.alt && c1.alt;
    for (int l = 0; l < (is_b ? 2 : 1); l++) {
      const MvF f0 = c0.f[l], f1 = c1.f[l];
      if (f0.ref >= 0 && f1.ref >= 0) {
        avg.f[l].mv[0] = shr_round(f0.mv[0] + f1.mv[0], 1);
        avg.f[l].mv[1] = shr_round(f0.mv[1] + f1.mv[1], 1);
        avg.f[l].ref = f0.ref;
        avg.dir |= l + 1;
      } else if (f0.ref >= 0) {
        avg.f[l] = f0;
        avg.dir |= l + 1;
      } else if (f1.ref >= 0) {
        avg.f[l] = f1;
        avg.dir |= l + 1;
      }
    }
    if (avg.dir != 0) list.push_back(avg);
  }
  while (list.size() < maxc) {  // zero candidates with ref_idx min(zero_idx, 0) = 0
    Cand z;
    z.dir = is_b ? 3 : 1;
    z.f[0].ref = 0;
    if (is_b) z.f[1].ref = 0;
    list.push_back(z);
  }
  return list;
}

const int kMvMin = -131072, kMvMax = 131071;

// inter.rs:814-884 derive_amvp_candidates (AmvrPrecision::QuarterPel)
void amvp_candidates(const MotionGrid& g, const Hmvp& hm, int bx, int by, int w, int h, int list, int ref_idx,
                     int out[2][2]) {
  const int shift = 2;
  auto round_mv = [&](const int* mv, int* o) {
    for (int k = 0; k < 2; k++) o[k] = clampi(shr_round(mv[k], shift) * (1 << shift), kMvMin, kMvMax);
  };
  std::vector<std::pair<int, int>> cands;
  auto contains = [&](int x, int y) {
    for (auto& c : cands)
      if (c.first == x && c.second == y) return true;
    return false;
  };
  Cand mi;
  if (bx > 0) {
    const int pos[2][2] = {{bx - 1, by + h}, {bx - 1, by + h - 1}};
    for (auto& p : pos)
      if (g.get(p[0], p[1], &mi) && mi.f[list].ref == ref_idx) {
        int r[2];
        round_mv(mi.f[list].mv, r);
        cands.push_back({r[0], r[1]});
        break;
      }
  }
  if (by > 0) {
    std::vector<std::pair<int, int>> above = {{bx + w, by - 1}, {bx + w - 1, by - 1}};
    if (bx > 0) above.push_back({bx - 1, by - 1});
    for (auto& p : above)
      if (g.get(p.first, p.second, &mi) && mi.f[list].ref == ref_idx) {
        int r[2];
        round_mv(mi.f[list].mv, r);
        if (cands.empty() || cands[0].first != r[0] || cands[0].second != r[1]) cands.push_back({r[0], r[1]});
        break;
      }
  }
  if (cands.size() < 2)
    for (int i = (int)hm.c.size() - 1; i >= 0; i--)
      if (hm.c[i].f[list].ref == ref_idx) {
        int r[2];
        round_mv(hm.c[i].f[list].mv, r);
        if (!contains(r[0], r[1])) {
          cands.push_back({r[0], r[1]});
          if (cands.size() == 2) break;
        }
      }
  while (cands.size() < 2) cands.push_back({0, 0});
  for (int k = 0; k < 2; k++) {
    out[k][0] = cands[k].first;
    out[k][1] = cands[k].second;
  }
}

struct RefPic {
  const uint8_t* p[3];
};

// inter.rs:1734-1848 predict_inter_pu on 8-bit 4:2:0 references (BDOF and
// DMVR off); predictions are 8-bit samples in int32.
void predict_inter_pu(const Cand& cand, const RefPic* l0, int n0, const RefPic* l1, int n1, int pw, int ph, int bx,
                      int by, int w, int h, std::vector<int32_t> pred[3]) {
  const int cw = w / 2, ch = h / 2, cx = bx / 2, cy = by / 2, cpw = pw / 2, cph = ph / 2;
  const bool has0 = (cand.dir & 1) && cand.f[0].ref >= 0 && n0 > 0;
  const bool has1 = (cand.dir & 2) && cand.f[1].ref >= 0 && n1 > 0;
  pred[0].assign(w * h, 128);
  pred[1].assign(cw * ch, 128);
  pred[2].assign(cw * ch, 128);
  if (has0 && has1) {
    const RefPic& r0 = l0[std::min(cand.f[0].ref, n0 - 1)];
    const RefPic& r1 = l1[std::min(cand.f[1].ref, n1 - 1)];
    std::vector<int32_t> a(w * h), b(w * h);
    interpolate_luma_block_8(r0.p[0], pw, ph, pw, bx, by, w, h, cand.f[0].mv[0], cand.f[0].mv[1], true, cand.alt,
                             false, a.data());
    interpolate_luma_block_8(r1.p[0], pw, ph, pw, bx, by, w, h, cand.f[1].mv[0], cand.f[1].mv[1], true, cand.alt,
                             false, b.data());
    weighted_average_bi_8(a.data(), b.data(), w * h, cand.bcw, pred[0].data());
    for (int c = 1; c < 3; c++) {
      std::vector<int32_t> u(cw * ch), v(cw * ch);
      interpolate_chroma_block_420_8(r0.p[c], cpw, cph, cpw, cx, cy, cw, ch, cand.f[0].mv[0], cand.f[0].mv[1], true,
                                     u.data());
      interpolate_chroma_block_420_8(r1.p[c], cpw, cph, cpw, cx, cy, cw, ch, cand.f[1].mv[0], cand.f[1].mv[1], true,
                                     v.data());
      weighted_average_bi_8(u.data(), v.data(), cw * ch, cand.bcw, pred[c].data());
    }
  } else if (has0 || has1) {
    const int l = has0 ? 0 : 1;
    const RefPic& r = has0 ? l0[std::min(cand.f[0].ref, n0 - 1)] : l1[std::min(cand.f[1].ref, n1 - 1)];
    interpolate_luma_block_8(r.p[0], pw, ph, pw, bx, by, w, h, cand.f[l].mv[0], cand.f[l].mv[1], false, cand.alt,
                             false, pred[0].data());
    for (int c = 1; c < 3; c++)
      interpolate_chroma_block_420_8(r.p[c], cpw, cph, cpw, cx, cy, cw, ch, cand.f[l].mv[0], cand.f[l].mv[1], false,
                                     pred[c].data());
  }
}

Cand cand_of(const vvcg_inter_cu& r) {
  Cand c;
  c.dir = r.inter_dir;
  for (int l = 0; l < 2; l++) {
    c.f[l].mv[0] = r.mv[l][0];
    c.f[l].mv[1] = r.mv[l][1];
    c.f[l].ref = r.ref_idx[l];
  }
  c.bcw = r.bcw_idx;
  c.alt = (r.flags & VVCG_INTER_CU_ALT_HPEL) != 0;
  return c;
}

void put_cand(const Cand& c, vvcg_inter_cu* r) {
  r->inter_dir = (uint8_t)c.dir;
  for (int l = 0; l < 2; l++) {
    r->mv[l][0] = c.f[l].mv[0];
    r->mv[l][1] = c.f[l].mv[1];
    r->ref_idx[l] = (int8_t)c.f[l].ref;
  }
  r->bcw_idx = (uint8_t)c.bcw;
  r->flags = (uint8_t)((r->flags & ~VVCG_INTER_CU_ALT_HPEL) | (c.alt ? VVCG_INTER_CU_ALT_HPEL : 0));
}

// slice.rs:2188-2224 apply_loop_filters_with_ctu_params, its deblocking
// (SAO / ALF are off in the options restated here): deblock_luma_plane at
// SliceQpY with bS 2 on the min(CTU, 32) grid and deblock_chroma_plane at
// derived_chroma_qp on the CTU / 2 grid. The 8-bit drivers run the same edge
// filters as the 16-bit ones with bit depth 8 (filter.rs:689-712, :935,
// :1132), so the 16-bit restatement runs on a 16-bit copy.
void deblock_intra_picture(Plane8w R[3], int qp, int ctu) {
  std::vector<uint16_t> p16[3];
  for (int c = 0; c < 3; c++) p16[c].assign(R[c].d.begin(), R[c].d.end());
  Plane16 y{p16[0].data(), R[0].w, R[0].h, 8}, u{p16[1].data(), R[1].w, R[1].h, 8}, v{p16[2].data(), R[2].w, R[2].h, 8};
  deblock_luma_plane_16(y, std::min(ctu, 32), ctu, qp, 2, 0, 0);
  const int cqp = clampi(derived_chroma_qp(qp), 0, 63);
  deblock_chroma_plane_16(u, ctu / 2, ctu / 2, cqp, 2, 0, 0, 2, 2);
  deblock_chroma_plane_16(v, ctu / 2, ctu / 2, cqp, 2, 0, 0, 2, 2);
  for (int c = 0; c < 3; c++)
    for (size_t i = 0; i < p16[c].size(); i++) R[c].d[i] = (uint8_t)p16[c][i];
}

bool planes_ok(int w, int h, int ctu_log2) {
  const int ctu = 1 << ctu_log2;
  return ctu_log2 >= 5 && ctu_log2 <= 7 && w >= ctu && h >= ctu && w % ctu == 0 && h % ctu == 0;
}

}  // namespace

// predict.rs:1455-1506 derive_intra_mpms; left / above < 0 when absent.
void derive_intra_mpms(int left_dir, int above_dir, uint8_t mpm[6]) {
  const int left = std::min(left_dir < 0 ? 0 : left_dir, 66), above = std::min(above_dir < 0 ? 0 : above_dir, 66);
  auto wrap = [](int m) { return (uint8_t)(((m - 2 + 64) % 64) + 2); };
  const int num = left == above ? 1 : 2, mn = std::min(left, above), mx = std::max(left, above);
  mpm[0] = 0;
  if (mx < 2) {
    const uint8_t d[5] = {1, 50, 18, 46, 54};
    memcpy(mpm + 1, d, 5);
  } else if (num == 1 || mn < 2) {
    mpm[1] = (uint8_t)mx;
    mpm[2] = wrap(mx - 1);
    mpm[3] = wrap(mx + 1);
    mpm[4] = wrap(mx - 2);
    mpm[5] = wrap(mx + 2);
  } else {
    mpm[1] = (uint8_t)left;
    mpm[2] = (uint8_t)above;
    if (mx - mn == 1) {
      mpm[3] = wrap(mn - 1);
      mpm[4] = wrap(mx + 1);
      mpm[5] = wrap(mn - 2);
    } else if (mx - mn >= 62) {
      mpm[3] = wrap(mn + 1);
      mpm[4] = wrap(mx - 1);
      mpm[5] = wrap(mn + 2);
    } else if (mx - mn == 2) {
      mpm[3] = wrap(mn + 1);
      mpm[4] = wrap(mn - 1);
      mpm[5] = wrap(mx + 1);
    } else {
      mpm[3] = wrap(mn - 1);
      mpm[4] = wrap(mn + 1);
      mpm[5] = wrap(mx - 1);
    }
  }
}

int mt_encode(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h, int qp, int ctu_log2,
              uint32_t opts, vvcg_cu_rec* cus, int16_t* levels, uint64_t* num_levels, uint8_t* ry, uint8_t* ru,
              uint8_t* rv) {
  if (!planes_ok(w, h, ctu_log2) || qp < 0 || qp > 63) return -1;
  if (opts & ~(uint32_t)(VVCG_SLICE_DEP_QUANT | VVCG_SLICE_SIGN_HIDING | VVCG_SLICE_FULL_INTRA_MODES |
                         VVCG_SLICE_DEBLOCK))
    return -1;
  const bool dq = opts & VVCG_SLICE_DEP_QUANT;
  const int tb = std::min(1 << ctu_log2, 32), cw = tb / 2;
  const int lqp = luma_qp_of(qp), cqp = chroma_qp_of(qp);
  const bool luma_ts = lqp == 4 && !dq, chroma_ts = cqp == 4 && !dq;  // slice.rs:2592-2593
  Plane8w R[3];  // the reconstruction starts as a copy of the source
  R[0].assign(y, w, h);
  R[1].assign(u, w / 2, h / 2);
  R[2].assign(v, w / 2, h / 2);
  const uint8_t* S[3] = {y, u, v};
  const int gw = w / tb, gh = h / tb;
  std::vector<uint8_t> mode_grid(gw * gh, 0);
  uint64_t at = 0;
  for (int gy = 0; gy < gh; gy++)
    for (int gx = 0; gx < gw; gx++) {
      const int k = gy * gw + gx, bx = gx * tb, by = gy * tb, cx = bx / 2, cy = by / 2;
      // the above neighbour is never in the same CTU (the grid is the CTU grid)
      uint8_t mpm[6];
      derive_intra_mpms(gx > 0 ? mode_grid[k - 1] : -1, -1, mpm);
      int mode;
      if (opts & VVCG_SLICE_FULL_INTRA_MODES) {
        int best_mrl = 0;
        uint64_t sad = 0;
        luma_intra_search_8(R[0].view(), Plane8{y, w, h}, bx, by, tb, tb, mpm, false, false, tb, &mode, &best_mrl,
                            &sad);
      } else {
        mode = choose_planar_dc(R[0], y, bx, by, tb);
      }
      mode_grid[k] = (uint8_t)mode;
      Coded cy_, cu_[2];
      if (encode_component_full(predict(R[0], bx, by, tb, true, mode), y, w, bx, by, tb, tb, lqp, luma_ts, dq, &cy_))
        return -2;
      store(R[0], bx, by, tb, tb, cy_.recon);
      for (int c = 1; c <= 2; c++) {  // chroma DM
        if (encode_component_full(predict(R[c], cx, cy, cw, false, mode), S[c], w / 2, cx, cy, cw, cw, cqp, chroma_ts,
                                  dq, &cu_[c - 1]))
          return -2;
      }
      store(R[1], cx, cy, cw, cw, cu_[0].recon);
      store(R[2], cx, cy, cw, cw, cu_[1].recon);
      vvcg_cu_rec& rec = cus[k];
      memset(&rec, 0, sizeof(rec));
      rec.luma_mode = rec.chroma_mode = (uint8_t)mode;
      const Coded* P[3] = {&cy_, &cu_[0], &cu_[1]};
      const bool ts[3] = {luma_ts, chroma_ts, chroma_ts};
      uint32_t tools = 0;
      for (int c = 0; c < 3; c++) {
        rec.level_off[c] = -1;
        if (!P[c]->cbf) continue;
        rec.cbf |= (uint8_t)(1 << c);
        if (ts[c]) tools |= 1u << c;
        rec.level_off[c] = (int32_t)at;
        for (size_t i = 0; i < P[c]->levels.size(); i++) levels[at + i] = (int16_t)P[c]->levels[i];
        at += P[c]->levels.size();
      }
      rec.tu_tools = (uint8_t)tools;
    }
  if (opts & VVCG_SLICE_DEBLOCK) deblock_intra_picture(R, lqp, 1 << ctu_log2);
  *num_levels = at;
  memcpy(ry, R[0].d.data(), R[0].d.size());
  memcpy(ru, R[1].d.data(), R[1].d.size());
  memcpy(rv, R[2].d.data(), R[2].d.size());
  return 0;
}

int mt_decode(const vvcg_cu_rec* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp, int ctu_log2,
              uint32_t opts, uint8_t* ry, uint8_t* ru, uint8_t* rv) {
  if (!planes_ok(w, h, ctu_log2) || qp < 0 || qp > 63) return -1;
  const bool dq = opts & VVCG_SLICE_DEP_QUANT;
  const int tb = std::min(1 << ctu_log2, 32), cw = tb / 2;
  const int lqp = luma_qp_of(qp), cqp = chroma_qp_of(qp);
  Plane8w R[3];
  R[0].assign(nullptr, w, h);
  R[1].assign(nullptr, w / 2, h / 2);
  R[2].assign(nullptr, w / 2, h / 2);
  const int gw = w / tb, gh = h / tb;
  for (int k = 0; k < gw * gh; k++) {
    const vvcg_cu_rec& r = cus[k];
    const int bx = (k % gw) * tb, by = (k / gw) * tb;
    if (r.luma_mode > 66 || r.chroma_mode > 66 || (r.tu_tools >> 3)) return -2;
    bool ok = true;
    std::vector<int32_t> lv[3] = {levels_of(r, levels, num_levels, 0, tb * tb, &ok),
                                  levels_of(r, levels, num_levels, 1, cw * cw, &ok),
                                  levels_of(r, levels, num_levels, 2, cw * cw, &ok)};
    if (!ok) return -3;
    int rc = reconstruct_component_full(R[0], predict(R[0], bx, by, tb, true, r.luma_mode), bx, by, tb, tb, lqp,
                                        lv[0].data(), r.cbf & 1, (r.tu_tools & 1) != 0, dq);
    for (int c = 1; c <= 2 && !rc; c++)
      rc = reconstruct_component_full(R[c], predict(R[c], bx / 2, by / 2, cw, false, r.chroma_mode), bx / 2, by / 2,
                                      cw, cw, cqp, lv[c].data(), (r.cbf >> c) & 1, ((r.tu_tools >> c) & 1) != 0, dq);
    if (rc) return -4;
  }
  if (opts & VVCG_SLICE_DEBLOCK) deblock_intra_picture(R, lqp, 1 << ctu_log2);
  memcpy(ry, R[0].d.data(), R[0].d.size());
  memcpy(ru, R[1].d.data(), R[1].d.size());
  memcpy(rv, R[2].d.data(), R[2].d.size());
  return 0;
}

// encode_inter_picture (slice.rs:3307-3549) of a P picture: every CTU one
// coding unit coded with merge candidate 0 (skip when no residual remains),
// DCT-2 residuals at SliceQpY / the derived chroma QP (no transform skip),
// then the CTU-boundary deblocking when VVCG_SLICE_DEBLOCK is set.
// refs: num_refs pictures of L0, each three planes (w x h, w/2 x h/2).
int inter_encode(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h, int qp, int ctu_log2,
                 uint32_t opts, const uint8_t* const* refs, int num_refs, vvcg_inter_cu* cus, int16_t* levels,
                 uint64_t* num_levels, uint8_t* ry, uint8_t* ru, uint8_t* rv) {
  if (!planes_ok(w, h, ctu_log2) || ctu_log2 != 5 || qp < 0 || qp > 63 || num_refs < 1 || num_refs > 4) return -1;
  if (opts & ~(uint32_t)(VVCG_SLICE_DEP_QUANT | VVCG_SLICE_SIGN_HIDING | VVCG_SLICE_DEBLOCK |
                         VVCG_SLICE_FULL_INTRA_MODES))
    return -1;
  const bool dq = opts & VVCG_SLICE_DEP_QUANT;
  const int ctu = 32, cw = 16;
  const int lqp = luma_qp_of(qp), cqp = chroma_qp_of(qp);
  std::vector<RefPic> l0(num_refs);
  for (int i = 0; i < num_refs; i++) l0[i] = RefPic{{refs[3 * i], refs[3 * i + 1], refs[3 * i + 2]}};
  Plane8w R[3];
  R[0].assign(y, w, h);
  R[1].assign(u, w / 2, h / 2);
  R[2].assign(v, w / 2, h / 2);
  const uint8_t* S[3] = {y, u, v};
  MotionGrid grid(w, h);
  Hmvp hm;
  const int gw = w / ctu, gh = h / ctu;
  uint64_t at = 0;
  for (int gy = 0; gy < gh; gy++) {
    hm.c.clear();
    for (int gx = 0; gx < gw; gx++) {
      const int k = gy * gw + gx, bx = gx * ctu, by = gy * ctu;
      const Cand cand = merge_candidates(grid, hm, bx, by, ctu, ctu, false, 6)[0];
      std::vector<int32_t> pred[3];
      predict_inter_pu(cand, l0.data(), num_refs, nullptr, 0, w, h, bx, by, ctu, ctu, pred);
      Coded cc[3];
      for (int c = 0; c < 3; c++) {
        const int n = c ? cw : ctu, px = c ? bx / 2 : bx, py = c ? by / 2 : by;
        if (encode_component_full(pred[c], S[c], c ? w / 2 : w, px, py, n, n, c ? cqp : lqp, false, dq, &cc[c]))
          return -2;
        store(R[c], px, py, n, n, cc[c].recon);
      }
      grid.fill(bx, by, ctu, ctu, cand);
      hm.push(cand);
      vvcg_inter_cu& rec = cus[k];
      memset(&rec, 0, sizeof(rec));
      put_cand(cand, &rec);
      rec.flags |= VVCG_INTER_CU_MERGE;
      for (int c = 0; c < 3; c++) {
        rec.level_off[c] = -1;
        if (!cc[c].cbf) continue;
        rec.cbf |= (uint8_t)(1 << c);
        rec.level_off[c] = (int32_t)at;
        for (size_t i = 0; i < cc[c].levels.size(); i++) levels[at + i] = (int16_t)cc[c].levels[i];
        at += cc[c].levels.size();
      }
      if (!rec.cbf) rec.flags |= VVCG_INTER_CU_SKIP;
    }
  }
  if (opts & VVCG_SLICE_DEBLOCK) {
    std::vector<vvcg_ctu_motion> cells(gw * gh);
    inter_ctu_cells(cus, w, h, ctu, cells.data());
    std::vector<uint16_t> p16[3];
    for (int c = 0; c < 3; c++) p16[c].assign(R[c].d.begin(), R[c].d.end());
    uint16_t* const planes[3] = {p16[0].data(), p16[1].data(), p16[2].data()};
    const int stride[3] = {w, w / 2, w / 2};
    inter_ctu_deblock(planes, stride, w, h, ctu, qp, cells.data());
    for (int c = 0; c < 3; c++)
      for (size_t i = 0; i < p16[c].size(); i++) R[c].d[i] = (uint8_t)p16[c][i];
  }
  *num_levels = at;
  memcpy(ry, R[0].d.data(), R[0].d.size());
  memcpy(ru, R[1].d.data(), R[1].d.size());
  memcpy(rv, R[2].d.data(), R[2].d.size());
  return 0;
}

// decode_inter_picture's motion derivation (slice.rs:3617-3677): per CTU in
// raster order (HMVP reset per CTU row) merge candidate 0 for merge / skip
// records, or AMVP candidate mvp_idx of L0 reference 0 plus the coded mvd;
// writes the motion fields of each record.
int inter_resolve_motion(vvcg_inter_cu* cus, int w, int h, int ctu_log2) {
  if (!planes_ok(w, h, ctu_log2)) return -1;
  const int ctu = 1 << ctu_log2, gw = w / ctu, gh = h / ctu;
  MotionGrid grid(w, h);
  Hmvp hm;
  for (int gy = 0; gy < gh; gy++) {
    hm.c.clear();
    for (int gx = 0; gx < gw; gx++) {
      vvcg_inter_cu& r = cus[gy * gw + gx];
      const int bx = gx * ctu, by = gy * ctu;
      Cand c;
      if (r.flags & (VVCG_INTER_CU_MERGE | VVCG_INTER_CU_SKIP)) {
        c = merge_candidates(grid, hm, bx, by, ctu, ctu, false, 6)[0];
      } else {
        if (r.mvp_idx > 1) return -2;
        int mvp[2][2];
        amvp_candidates(grid, hm, bx, by, ctu, ctu, 0, 0, mvp);
        c = Cand();
        c.f[0].ref = 0;
        c.f[0].mv[0] = mvp[r.mvp_idx][0] + r.mvd[0];
        c.f[0].mv[1] = mvp[r.mvp_idx][1] + r.mvd[1];
      }
      grid.fill(bx, by, ctu, ctu, c);
      hm.push(c);
      put_cand(c, &r);
    }
  }
  return 0;
}

// decode_inter_picture's reconstruction (slice.rs:3680-3834) from records
// with their motion: the prediction, each component's residual, and the
// CTU-boundary deblocking when VVCG_SLICE_DEBLOCK is set.
int inter_decode(const vvcg_inter_cu* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                 int ctu_log2, uint32_t opts, const uint8_t* const* refs, int num_refs, uint8_t* ry, uint8_t* ru,
                 uint8_t* rv) {
  if (!planes_ok(w, h, ctu_log2) || ctu_log2 != 5 || qp < 0 || qp > 63 || num_refs < 1 || num_refs > 4) return -1;
  const bool dq = opts & VVCG_SLICE_DEP_QUANT;
  const int ctu = 32, cw = 16;
  const int lqp = luma_qp_of(qp), cqp = chroma_qp_of(qp);
  std::vector<RefPic> l0(num_refs);
  for (int i = 0; i < num_refs; i++) l0[i] = RefPic{{refs[3 * i], refs[3 * i + 1], refs[3 * i + 2]}};
  Plane8w R[3];
  R[0].assign(nullptr, w, h);
  R[1].assign(nullptr, w / 2, h / 2);
  R[2].assign(nullptr, w / 2, h / 2);
  const int gw = w / ctu, gh = h / ctu;
  for (int k = 0; k < gw * gh; k++) {
    const vvcg_inter_cu& r = cus[k];
    const int bx = (k % gw) * ctu, by = (k / gw) * ctu;
    if (r.inter_dir != 1 || r.ref_idx[0] < 0 || (r.tu_tools >> 3)) return -2;  // P slices: L0 only
    std::vector<int32_t> pred[3];
    predict_inter_pu(cand_of(r), l0.data(), num_refs, nullptr, 0, w, h, bx, by, ctu, ctu, pred);
    for (int c = 0; c < 3; c++) {
      const int n = c ? cw : ctu;
      std::vector<int32_t> lv(n * n, 0);
      const bool cbf = (r.cbf >> c) & 1;
      if (cbf) {
        if (r.level_off[c] < 0 || (uint64_t)r.level_off[c] + n * n > num_levels) return -3;
        for (int i = 0; i < n * n; i++) lv[i] = levels[r.level_off[c] + i];
      }
      if (reconstruct_component_full(R[c], pred[c], c ? bx / 2 : bx, c ? by / 2 : by, n, n, c ? cqp : lqp, lv.data(),
                                     cbf, ((r.tu_tools >> c) & 1) != 0, dq))
        return -4;
    }
  }
  if (opts & VVCG_SLICE_DEBLOCK) {
    std::vector<vvcg_ctu_motion> cells(gw * gh);
    inter_ctu_cells(cus, w, h, ctu, cells.data());
    std::vector<uint16_t> p16[3];
    for (int c = 0; c < 3; c++) p16[c].assign(R[c].d.begin(), R[c].d.end());
    uint16_t* const planes[3] = {p16[0].data(), p16[1].data(), p16[2].data()};
    const int stride[3] = {w, w / 2, w / 2};
    inter_ctu_deblock(planes, stride, w, h, ctu, qp, cells.data());
    for (int c = 0; c < 3; c++)
      for (size_t i = 0; i < p16[c].size(); i++) R[c].d[i] = (uint8_t)p16[c][i];
  }
  memcpy(ry, R[0].d.data(), R[0].d.size());
  memcpy(ru, R[1].d.data(), R[1].d.size());
  memcpy(rv, R[2].d.data(), R[2].d.size());
  return 0;
}

// The per-CTU motion and cbf cells the CTU-boundary deblocking reads
// (slice.rs:2319-2326, :2438-2444): with one coding unit per CTU, the
// top-left, top-right and bottom-left motion are the CTU's own.
void inter_ctu_cells(const vvcg_inter_cu* cus, int w, int h, int ctu, vvcg_ctu_motion* cells) {
  const int n = (w / ctu) * (h / ctu);
  for (int k = 0; k < n; k++) {
    vvcg_ctu_motion& m = cells[k];
    memset(&m, 0, sizeof(m));
    for (int j = 0; j < 3; j++) {
      m.mv[j][0] = cus[k].mv[0][0];
      m.mv[j][1] = cus[k].mv[0][1];
      m.ref[j] = cus[k].ref_idx[0];
    }
    m.cbf = cus[k].cbf;
  }
}

}  // namespace orc
