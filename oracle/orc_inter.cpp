// CPU oracle (test infrastructure only; see oracle.h): 8..12-bit motion
// compensation interpolation. Restates crates/rustmpeg-video/src/vvc/inter.rs
// (interpolate_luma_block_16, interpolate_chroma_block_format_16,
// weighted_average_bi_16) of the reference, including its uni-prediction
// second-stage shift `12 - bd` for 2-D fractional positions (inter.rs:2051,
// :2583), which differs from the 8-bit path's `6 + headroom`.
#include <algorithm>
#include <vector>

#include "../rustmpeg-next_b200/csrc/vvc_tables.h"
#include "oracle.h"

namespace orc {
using namespace vvc_tables;

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// inter.rs:2010-2134 interpolate_luma_block_16
void interpolate_luma_block_16(const Plane16& ref, int bx, int by, int w, int h, int mv_x, int mv_y,
                               bool bi, bool affine, bool alt_hpel, int32_t* out) {
  int dx = mv_x >> 4, dy = mv_y >> 4;
  int fx = mv_x & 15, fy = mv_y & 15;
  int bd = clampi(ref.bd, 8, 12);
  int mx = (1 << bd) - 1;
  auto g = [&](int x, int y) {
    return (int)ref.get(clampi(x, 0, ref.width - 1), clampi(y, 0, ref.height - 1));
  };
  auto filt = [&](int frac, int* f) {
    for (int k = 0; k < 8; k++) {
      if (affine)
        f[k] = kAffineTaps8[frac * 8 + k];
      else if (alt_hpel && frac == 8)
        f[k] = kLumaAltHpel[k];
      else
        f[k] = kLumaTaps8[frac * 8 + k];
    }
  };
  int head = std::max(14 - bd, 2);
  int shift1 = 6 - head;
  int shift2 = bi ? 6 : 12 - bd;
  // `1i32 << (shift2 - 1)` and `sum + add2` as the reference's release build
  // evaluates them: the shift count is masked to 5 bits (at 12 bit shift2 is 0,
  // giving 1 << 31) and the addition wraps.
  int add2 = bi ? 0 : (int)(1u << ((unsigned)(shift2 - 1) & 31));
  int offs = 1 << (bd + head - 1);
  if (fx == 0 && fy == 0) {
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++) {
        int s = g(bx + x + dx, by + y + dy);
        out[y * w + x] = bi ? (s << head) - offs : s;
      }
    return;
  }
  if (fy == 0) {
    int f[8];
    filt(fx, f);
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++) {
        int px = bx + x + dx, py = by + y + dy;
        int s = 0;
        for (int k = 0; k < 8; k++) s += f[k] * g(px + k - 3, py);
        out[y * w + x] = bi ? (s >> shift1) - offs : clampi((s + 32) >> 6, 0, mx);
      }
    return;
  }
  if (fx == 0) {
    int f[8];
    filt(fy, f);
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++) {
        int px = bx + x + dx, py = by + y + dy;
        int s = 0;
        for (int k = 0; k < 8; k++) s += f[k] * g(px, py + k - 3);
        out[y * w + x] = bi ? (s >> shift1) - offs : clampi((s + 32) >> 6, 0, mx);
      }
    return;
  }
  int fh[8], fv[8];
  filt(fx, fh);
  filt(fy, fv);
  int th = h + 7;
  std::vector<int> tmp((size_t)w * th);
  for (int ty = 0; ty < th; ty++) {
    int py = by + ty - 3 + dy;
    for (int x = 0; x < w; x++) {
      int px = bx + x + dx;
      int s = 0;
      for (int k = 0; k < 8; k++) s += fh[k] * g(px + k - 3, py);
      tmp[ty * w + x] = s >> shift1;
    }
  }
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      int s = 0;
      for (int k = 0; k < 8; k++) s += fv[k] * tmp[(y + k) * w + x];
      out[y * w + x] = bi ? (s >> shift2) - offs : clampi((int)((unsigned)s + (unsigned)add2) >> shift2, 0, mx);
    }
}

// inter.rs:2543-2672 interpolate_chroma_block_format_16 (cf: 1 = 4:2:0, 2 = 4:2:2, 3 = 4:4:4)
void interpolate_chroma_block_format_16(const Plane16& ref, int bxc, int byc, int cw, int ch,
                                        int mv_x, int mv_y, bool bi, int cf, int32_t* out) {
  if (cw == 0 || ch == 0 || cf == 0) return;
  int sub_w = (cf == 1 || cf == 2) ? 2 : 1;
  int sub_h = cf == 1 ? 2 : 1;
  int mvx32 = mv_x * (sub_w == 1 ? 2 : 1);
  int mvy32 = mv_y * (sub_h == 1 ? 2 : 1);
  int dx = mvx32 >> 5, dy = mvy32 >> 5;
  int fx = mvx32 & 31, fy = mvy32 & 31;
  int bd = clampi(ref.bd, 8, 12);
  int mx = (1 << bd) - 1;
  auto g = [&](int x, int y) {
    return (int)ref.get(clampi(x, 0, ref.width - 1), clampi(y, 0, ref.height - 1));
  };
  int head = std::max(14 - bd, 2);
  int shift1 = 6 - head;
  int shift2 = bi ? 6 : 12 - bd;
  // `1i32 << (shift2 - 1)` and `sum + add2` as the reference's release build
  // evaluates them: the shift count is masked to 5 bits (at 12 bit shift2 is 0,
  // giving 1 << 31) and the addition wraps.
  int add2 = bi ? 0 : (int)(1u << ((unsigned)(shift2 - 1) & 31));
  int offs = 1 << (bd + head - 1);
  if (fx == 0 && fy == 0) {
    for (int y = 0; y < ch; y++)
      for (int x = 0; x < cw; x++) {
        int s = g(bxc + x + dx, byc + y + dy);
        out[y * cw + x] = bi ? (s << head) - offs : s;
      }
    return;
  }
  const int8_t* fh = &kChromaTaps4[fx * 4];
  const int8_t* fv = &kChromaTaps4[fy * 4];
  if (fy == 0) {
    for (int y = 0; y < ch; y++)
      for (int x = 0; x < cw; x++) {
        int px = bxc + x + dx, py = byc + y + dy;
        int s = 0;
        for (int k = 0; k < 4; k++) s += fh[k] * g(px + k - 1, py);
        out[y * cw + x] = bi ? (s >> shift1) - offs : clampi((s + 32) >> 6, 0, mx);
      }
    return;
  }
  if (fx == 0) {
    for (int y = 0; y < ch; y++)
      for (int x = 0; x < cw; x++) {
        int px = bxc + x + dx, py = byc + y + dy;
        int s = 0;
        for (int k = 0; k < 4; k++) s += fv[k] * g(px, py + k - 1);
        out[y * cw + x] = bi ? (s >> shift1) - offs : clampi((s + 32) >> 6, 0, mx);
      }
    return;
  }
  int th = ch + 3;
  std::vector<int> tmp((size_t)cw * th);
  for (int ty = 0; ty < th; ty++) {
    int py = byc + ty - 1 + dy;
    for (int x = 0; x < cw; x++) {
      int px = bxc + x + dx;
      int s = 0;
      for (int k = 0; k < 4; k++) s += fh[k] * g(px + k - 1, py);
      tmp[ty * cw + x] = s >> shift1;
    }
  }
  for (int y = 0; y < ch; y++)
    for (int x = 0; x < cw; x++) {
      int s = 0;
      for (int k = 0; k < 4; k++) s += fv[k] * tmp[(y + k) * cw + x];
      out[y * cw + x] = bi ? (s >> shift2) - offs : clampi((int)((unsigned)s + (unsigned)add2) >> shift2, 0, mx);
    }
}

// inter.rs:896-1051 interpolate_luma_block (8-bit planes)
void interpolate_luma_block_8(const uint8_t* ref, int pw, int ph, int stride, int bx, int by, int w, int h,
                              int mv_x, int mv_y, bool bi, bool alt_hpel, bool affine, int32_t* out) {
  const int int_x = bx + (mv_x >> 4), int_y = by + (mv_y >> 4);
  const int fx = mv_x & 15, fy = mv_y & 15;
  const int head = 14 - 8, offs = 1 << 13;  // IF_INTERNAL_PREC - 8, IF_INTERNAL_OFFS
  auto g = [&](int x, int y) { return (int)ref[clampi(y, 0, ph - 1) * stride + clampi(x, 0, pw - 1)]; };
  auto coeffs = [&](int frac, int* c) {
    for (int k = 0; k < 8; k++)
      c[k] = affine ? kAffineTaps8[frac * 8 + k] : (alt_hpel && frac == 8) ? kLumaAltHpel[k] : kLumaTaps8[frac * 8 + k];
  };
  // tap k at position p + tap_start + k (affine: tap_start -2 and one more -1)
  const int tap0 = affine ? -2 - 1 : -3;
  if (fx == 0 && fy == 0) {
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++) {
        int s = g(int_x + x, int_y + y);
        out[y * w + x] = bi ? (s << head) - offs : s;
      }
    return;
  }
  if (fy == 0 || fx == 0) {
    int c[8];
    coeffs(fy == 0 ? fx : fy, c);
    const int shift = bi ? 6 - head : 6;
    const int offset = bi ? -offs << shift : 1 << (shift - 1);
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++) {
        int s = 0;
        for (int k = 0; k < 8; k++)
          s += (fy == 0 ? g(int_x + x + tap0 + k, int_y + y) : g(int_x + x, int_y + y + tap0 + k)) * c[k];
        int v = (s + offset) >> shift;
        out[y * w + x] = bi ? v : clampi(v, 0, 255);
      }
    return;
  }
  int cx[8], cy[8];
  coeffs(fx, cx);
  coeffs(fy, cy);
  const int eh = h + 7, shift1 = 6 - head, offset1 = -offs << shift1;
  std::vector<int> tmp((size_t)w * eh);
  for (int y = 0; y < eh; y++)
    for (int x = 0; x < w; x++) {
      int s = 0;
      for (int k = 0; k < 8; k++) s += g(int_x + x + tap0 + k, int_y - 3 + y) * cx[k];
      tmp[y * w + x] = (s + offset1) >> shift1;
    }
  const int shift2 = bi ? 6 : 6 + head;
  const int offset2 = bi ? 0 : (1 << (shift2 - 1)) + (offs << 6);
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      int s = 0;
      for (int k = 0; k < 8; k++) s += tmp[(y + k) * w + x] * cy[k];
      int v = (s + offset2) >> shift2;
      out[y * w + x] = bi ? v : clampi(v, 0, 255);
    }
}

// inter.rs:1056-1182 interpolate_chroma_block_420 (8-bit planes; MV in 1/16
// luma = 1/32 chroma units)
void interpolate_chroma_block_420_8(const uint8_t* ref, int pw, int ph, int stride, int cx, int cy, int cw,
                                    int ch, int mv_x, int mv_y, bool bi, int32_t* out) {
  const int int_x = cx + (mv_x >> 5), int_y = cy + (mv_y >> 5);
  const int fx = mv_x & 31, fy = mv_y & 31;
  const int head = 6, offs = 1 << 13;
  auto g = [&](int x, int y) { return (int)ref[clampi(y, 0, ph - 1) * stride + clampi(x, 0, pw - 1)]; };
  if (fx == 0 && fy == 0) {
    for (int y = 0; y < ch; y++)
      for (int x = 0; x < cw; x++) {
        int s = g(int_x + x, int_y + y);
        out[y * cw + x] = bi ? (s << head) - offs : s;
      }
    return;
  }
  if (fy == 0 || fx == 0) {
    const int8_t* c = &kChromaTaps4[(fy == 0 ? fx : fy) * 4];
    const int shift = bi ? 6 - head : 6;
    const int offset = bi ? -offs << shift : 1 << (shift - 1);
    for (int y = 0; y < ch; y++)
      for (int x = 0; x < cw; x++) {
        int s = 0;
        for (int k = 0; k < 4; k++)
          s += (fy == 0 ? g(int_x + x - 1 + k, int_y + y) : g(int_x + x, int_y + y - 1 + k)) * c[k];
        int v = (s + offset) >> shift;
        out[y * cw + x] = bi ? v : clampi(v, 0, 255);
      }
    return;
  }
  const int8_t* cxf = &kChromaTaps4[fx * 4];
  const int8_t* cyf = &kChromaTaps4[fy * 4];
  const int eh = ch + 3, shift1 = 6 - head, offset1 = -offs << shift1;
  std::vector<int> tmp((size_t)cw * eh);
  for (int y = 0; y < eh; y++)
    for (int x = 0; x < cw; x++) {
      int s = 0;
      for (int k = 0; k < 4; k++) s += g(int_x + x - 1 + k, int_y - 1 + y) * cxf[k];
      tmp[y * cw + x] = (s + offset1) >> shift1;
    }
  const int shift2 = bi ? 6 : 6 + head;
  const int offset2 = bi ? 0 : (1 << (shift2 - 1)) + (offs << 6);
  for (int y = 0; y < ch; y++)
    for (int x = 0; x < cw; x++) {
      int s = 0;
      for (int k = 0; k < 4; k++) s += tmp[(y + k) * cw + x] * cyf[k];
      int v = (s + offset2) >> shift2;
      out[y * cw + x] = bi ? v : clampi(v, 0, 255);
    }
}

// inter.rs:1189-1201 weighted_average_bi (8-bit output range)
void weighted_average_bi_8(const int32_t* p0, const int32_t* p1, int n, int bcw_idx, int32_t* out) {
  const int w1 = kBcwWeights[std::min(bcw_idx, 4)], w0 = 8 - w1;
  const int sn = 6 + 3, off = (1 << (sn - 1)) + ((1 << 13) << 3);
  for (int i = 0; i < n; i++) out[i] = clampi((p0[i] * w0 + p1[i] * w1 + off) >> sn, 0, 255);
}

// inter.rs:2676-2698 weighted_average_bi_16
void weighted_average_bi_16(const int32_t* p0, const int32_t* p1, int n, int bcw_idx, int bd,
                            uint16_t* out) {
  bd = clampi(bd, 8, 12);
  int mx = (1 << bd) - 1;
  int w1 = kBcwWeights[std::min(bcw_idx, 4)];
  int w0 = 8 - w1;
  int head = std::max(14 - bd, 2);
  int sn = head + 3;
  int io = 1 << (bd + head - 1);
  int off = (1 << (sn - 1)) + (io << 3);
  for (int i = 0; i < n; i++) out[i] = (uint16_t)clampi((p0[i] * w0 + p1[i] * w1 + off) >> sn, 0, mx);
}

// predict_inter_pu (inter.rs:1733-1847) luma part with BDOF and DMVR off, as
// estimate_inter_block calls it: bi-prediction = two 14-bit interpolations and
// weighted_average_bi; uni-prediction from the one usable list; 128 without.
static void predict_pu_luma_8(const uint8_t* const* l0, int n0, const uint8_t* const* l1, int n1, int pw, int ph,
                              int stride, const vvcg_mv_cand& c, int bx, int by, int w, int h, int32_t* out) {
  const bool has0 = (c.inter_dir & 1) && c.ref_idx[0] >= 0 && n0 > 0;
  const bool has1 = (c.inter_dir & 2) && c.ref_idx[1] >= 0 && n1 > 0;
  const bool alt = c.alt_hpel != 0;
  if (has0 && has1) {
    const uint8_t* r0 = l0[std::min((int)c.ref_idx[0], n0 - 1)];
    const uint8_t* r1 = l1[std::min((int)c.ref_idx[1], n1 - 1)];
    std::vector<int32_t> p0((size_t)w * h), p1((size_t)w * h);
    interpolate_luma_block_8(r0, pw, ph, stride, bx, by, w, h, c.mv[0][0], c.mv[0][1], true, alt, false, p0.data());
    interpolate_luma_block_8(r1, pw, ph, stride, bx, by, w, h, c.mv[1][0], c.mv[1][1], true, alt, false, p1.data());
    weighted_average_bi_8(p0.data(), p1.data(), w * h, c.bcw_idx, out);
  } else if (has0 || has1) {
    const int l = has0 ? 0 : 1;
    const uint8_t* r = has0 ? l0[std::min((int)c.ref_idx[0], n0 - 1)] : l1[std::min((int)c.ref_idx[1], n1 - 1)];
    interpolate_luma_block_8(r, pw, ph, stride, bx, by, w, h, c.mv[l][0], c.mv[l][1], false, alt, false, out);
  } else {
    for (int i = 0; i < w * h; i++) out[i] = 128;
  }
}

// estimate_inter_block (inter.rs:1866-2003): merge candidates by luma SAD
// (first lowest wins), then, with an L0 reference, the integer diamond search
// on L0 reference 0 from the AMVP predictor (at most max(range, 1) rounds of
// the four neighbours of the round's centre, stopping after a round without
// improvement) and the quarter-sample refinement around its result; the merge
// candidate wins ties with the searched vector.
void estimate_inter_block_8(const uint8_t* src, const uint8_t* const* l0, int n0, const uint8_t* const* l1, int n1,
                            int pw, int ph, int stride, const vvcg_mv_cand* cands, int ncand, int amvp_x, int amvp_y,
                            int bx, int by, int w, int h, int range, vvcg_me_res* res) {
  std::vector<int32_t> pred((size_t)w * h);
  auto sad_of = [&]() {
    uint64_t t = 0;
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++) t += (uint64_t)abs((int)src[(size_t)(by + y) * stride + bx + x] - pred[y * w + x]);
    return t;
  };
  vvcg_mv_cand best_merge{};
  best_merge.inter_dir = 1;  // InterMergeCand::default (inter.rs:297-306)
  best_merge.ref_idx[0] = 0;
  best_merge.ref_idx[1] = -1;
  best_merge.bcw_idx = 2;
  if (ncand > 0) best_merge = cands[0];
  uint64_t best_merge_sad = UINT64_MAX;
  int best_merge_idx = 0;
  for (int i = 0; i < ncand; i++) {
    predict_pu_luma_8(l0, n0, l1, n1, pw, ph, stride, cands[i], bx, by, w, h, pred.data());
    const uint64_t s = sad_of();
    if (s < best_merge_sad) {
      best_merge_sad = s;
      best_merge_idx = i;
      best_merge = cands[i];
    }
  }
  *res = vvcg_me_res{};
  res->cand = best_merge;
  res->is_merge = 1;
  res->merge_idx = (uint16_t)best_merge_idx;
  res->sad = best_merge_sad;
  if (n0 == 0) return;
  const uint8_t* r0 = l0[0];
  auto sad_at = [&](int mx, int my) {
    interpolate_luma_block_8(r0, pw, ph, stride, bx, by, w, h, mx, my, false, false, false, pred.data());
    return sad_of();
  };
  int bmx = (amvp_x >> 4) << 4, bmy = (amvp_y >> 4) << 4;
  uint64_t best = sad_at(bmx, bmy);
  static const int kDiamond[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
  for (int it = 0; it < std::max(range, 1); it++) {
    bool improved = false;
    const int cx = bmx >> 4, cy = bmy >> 4;
    for (int k = 0; k < 4; k++) {
      const int tx = (cx + kDiamond[k][0]) << 4, ty = (cy + kDiamond[k][1]) << 4;
      const uint64_t s = sad_at(tx, ty);
      if (s < best) {
        best = s;
        bmx = tx;
        bmy = ty;
        improved = true;
      }
    }
    if (!improved) break;
  }
  const int ix = bmx, iy = bmy;
  static const int kQuarter[4][2] = {{4, 0}, {-4, 0}, {0, 4}, {0, -4}};
  for (int k = 0; k < 4; k++) {
    const uint64_t s = sad_at(ix + kQuarter[k][0], iy + kQuarter[k][1]);
    if (s < best) {
      best = s;
      bmx = ix + kQuarter[k][0];
      bmy = iy + kQuarter[k][1];
    }
  }
  if (best_merge_sad <= best) return;
  vvcg_mv_cand c{};
  c.inter_dir = 1;
  c.mv[0][0] = bmx;
  c.mv[0][1] = bmy;
  c.ref_idx[0] = 0;
  c.ref_idx[1] = -1;
  c.bcw_idx = 2;
  res->cand = c;
  res->is_merge = 0;
  res->merge_idx = 0;
  res->sad = best;
}

}  // namespace orc
