// CPU oracle (test infrastructure only): the inter-prediction tools of the
// reference beyond plain motion compensation, restated from
// crates/rustmpeg-video/src/vvc/inter.rs:
//   apply_bdof_luma                      inter.rs:1218-1339
//   dmvr_subpel_1d / refine_dmvr_subblock inter.rs:1341-1471
//   is_subblock_vector_spread_over_limit inter.rs:1473-1495
//   derive_affine_subblock_mvs           inter.rs:1502-1579
//   apply_prof_4x4                       inter.rs:1581-1609
//   apply_ciip_blend                     inter.rs:1615-1630
//   derive_gpm_params_table / predict_gpm_block inter.rs:1641-1731
// The sample paths are the reference's 8-bit ones (outputs clamped to 255).
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "../rustmpeg-next_b200/csrc/vvc_tables.h"

using namespace vvc_tables;

namespace {

constexpr int kIfInternalPrec = 14, kIfInternalOffs = 1 << 13, kMvMin = -(1 << 17), kMvMax = (1 << 17) - 1;

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// inter.rs:1204-1211 right_shift_msb
int right_shift_msb(int numer, int denom) {
  if (denom <= 0) return 0;
  int log2_d = 31 - __builtin_clz((unsigned)denom);
  return numer >> log2_d;
}

// Mv::shr_round (inter.rs:183-195)
int shr_round(int v, int shift) {
  if (shift == 0) return v;
  const int offset = 1 << (shift - 1);
  const int neg_bias = (~v) >> 31;
  return (v + offset + neg_bias) >> shift;
}

}  // namespace

namespace orc {

// inter.rs:1218-1339 apply_bdof_luma: two 14-bit intermediate w x h luma
// predictions -> 8-bit samples.
void bdof_luma(const int32_t* pred0, const int32_t* pred1, int w, int h, int32_t* dst) {
  const int ew = w + 2, eh = h + 2;
  auto pad = [&](const int32_t* src) {
    std::vector<int> p(ew * eh, 0);
    for (int y = 0; y < h; y++) {
      const int sy = y + 1;
      p[sy * ew] = src[y * w];
      for (int x = 0; x < w; x++) p[sy * ew + x + 1] = src[y * w + x];
      p[sy * ew + w + 1] = src[y * w + w - 1];
    }
    for (int x = 0; x < ew; x++) {
      p[x] = p[ew + x];
      p[(h + 1) * ew + x] = p[h * ew + x];
    }
    return p;
  };
  const std::vector<int> p0 = pad(pred0), p1 = pad(pred1);
  auto grads = [&](const std::vector<int>& p, std::vector<int>& gx, std::vector<int>& gy) {
    gx.assign(ew * eh, 0);
    gy.assign(ew * eh, 0);
    for (int y = 1; y <= h; y++) {
      for (int x = 1; x <= w; x++) {
        const int i = y * ew + x;
        gx[i] = (p[i + 1] >> 6) - (p[i - 1] >> 6);
        gy[i] = (p[i + ew] >> 6) - (p[i - ew] >> 6);
      }
      gx[y * ew] = gx[y * ew + 1];
      gx[y * ew + w + 1] = gx[y * ew + w];
      gy[y * ew] = gy[y * ew + 1];
      gy[y * ew + w + 1] = gy[y * ew + w];
    }
    for (int x = 0; x < ew; x++) {
      gx[x] = gx[ew + x];
      gx[(h + 1) * ew + x] = gx[h * ew + x];
      gy[x] = gy[ew + x];
      gy[(h + 1) * ew + x] = gy[h * ew + x];
    }
  };
  std::vector<int> gx0, gy0, gx1, gy1;
  grads(p0, gx0, gy0);
  grads(p1, gx1, gy1);
  const int shift_num = kIfInternalPrec - 8 + 1;
  const int offset = (1 << (shift_num - 1)) + 2 * kIfInternalOffs;
  const int limit = 15;
  auto sgn = [](int s, int v) { return s < 0 ? -v : (s == 0 ? 0 : v); };
  for (int yu = 0; yu < (h >> 2); yu++)
    for (int xu = 0; xu < (w >> 2); xu++) {
      int sgx = 0, sgy = 0, sdx = 0, sdy = 0, sgygx = 0;
      for (int dy = 0; dy < 6; dy++)
        for (int dx = 0; dx < 6; dx++) {
          const int i = (yu * 4 + dy) * ew + xu * 4 + dx;
          const int tgx = (gx0[i] + gx1[i]) >> 1, tgy = (gy0[i] + gy1[i]) >> 1;
          const int tdi = (p1[i] >> 4) - (p0[i] >> 4);
          sgx += std::abs(tgx);
          sgy += std::abs(tgy);
          sdx += sgn(tgx, tdi);
          sdy += sgn(tgy, tdi);
          sgygx += sgn(tgy, tgx);
        }
      const int tmpx = sgx == 0 ? 0 : clampi(right_shift_msb(4 * sdx, sgx), -limit, limit);
      const int tmp_data = (sgygx * tmpx) >> 1;
      const int tmpy = sgy == 0 ? 0 : clampi(right_shift_msb(4 * sdy - tmp_data, sgy), -limit, limit);
      for (int dy = 0; dy < 4; dy++)
        for (int dx = 0; dx < 4; dx++) {
          const int y = yu * 4 + dy, x = xu * 4 + dx;
          const int i = (y + 1) * ew + x + 1;
          const int b = tmpx * (gx0[i] - gx1[i]) + tmpy * (gy0[i] - gy1[i]);
          dst[y * w + x] = clampi((p0[i] + p1[i] + b + offset) >> shift_num, 0, 255);
        }
    }
}

// inter.rs:1341-1363 dmvr_subpel_1d
static int dmvr_subpel_1d(int64_t s0, int64_t s1, int64_t s2) {
  const int64_t den = s1 + s2 - 2 * s0;
  if (den == 0) return 0;
  if (s1 != s0 && s2 != s0) {
    const int64_t num = ((s1 - s2) << 4) >> 1;
    int64_t rem = num < 0 ? -num : num;
    int q = 0;
    for (int i = 2; i >= 0; i--) {
      const int64_t div = den << i;
      if (rem >= div) {
        rem -= div;
        q += 1 << i;
      }
    }
    return num < 0 ? -q : q;
  }
  return s1 == s0 ? -8 : 8;
}

// inter.rs:1371-1471 refine_dmvr_subblock on 8-bit planes (w x h, stride):
// mv = [mv0 hor, mv0 ver, mv1 hor, mv1 ver] in and out.
void dmvr_refine(const uint8_t* ref0, const uint8_t* ref1, int pw, int ph, int stride, int bx, int by, int dx,
                 int dy, int32_t* mv) {
  auto sc = [&](const uint8_t* p, int x, int y) { return (int)p[(size_t)clampi(y, 0, ph - 1) * stride + clampi(x, 0, pw - 1)]; };
  auto pred = [&](const uint8_t* p, int mvh, int mvv, int ox, int oy, std::vector<int>& out) {
    const int ix = bx + (mvh >> 4) + ox, iy = by + (mvv >> 4) + oy;
    const int* wx = &kBilinear4[2 * (mvh & 15)];
    const int* wy = &kBilinear4[2 * (mvv & 15)];
    out.assign(dx * dy, 0);
    for (int y = 0; y < dy; y++)
      for (int x = 0; x < dx; x++) {
        const int px = ix + x, py = iy + y;
        const int h0 = (sc(p, px, py) * wx[0] + sc(p, px + 1, py) * wx[1] + 8) >> 4;
        const int h1 = (sc(p, px, py + 1) * wx[0] + sc(p, px + 1, py + 1) * wx[1] + 8) >> 4;
        out[y * dx + x] = (h0 * wy[0] + h1 * wy[1] + 8) >> 4;
      }
  };
  std::vector<int> a, b;
  auto cost = [&](int ox, int oy) {
    pred(ref0, mv[0], mv[1], ox, oy, a);
    pred(ref1, mv[2], mv[3], -ox, -oy, b);
    int64_t c = 0;
    for (int y = 0; y < dy; y += 2)
      for (int x = 0; x < dx; x++) c += std::abs(a[y * dx + x] - b[y * dx + x]);
    return c;
  };
  int64_t sads[5][5];
  for (auto& r : sads)
    for (auto& v : r) v = INT64_MAX / 4;
  int64_t min_cost = cost(0, 0);
  min_cost -= min_cost >> 2;
  sads[2][2] = min_cost;
  if (min_cost < (int64_t)dx * dy) return;
  int bix = 0, biy = 0;
  for (int oy = -2; oy <= 2; oy++)
    for (int ox = -2; ox <= 2; ox++) {
      if (ox == 0 && oy == 0) continue;
      const int64_t c = cost(ox, oy);
      sads[oy + 2][ox + 2] = c;
      if (c < min_cost) {
        min_cost = c;
        bix = ox;
        biy = oy;
      }
    }
  int dh = bix * 16, dv = biy * 16;
  if (std::abs(bix) < 2 && std::abs(biy) < 2) {
    const int ux = bix + 2, uy = biy + 2;
    dh += dmvr_subpel_1d(sads[uy][ux], sads[uy][ux - 1], sads[uy][ux + 1]);
    dv += dmvr_subpel_1d(sads[uy][ux], sads[uy - 1][ux], sads[uy + 1][ux]);
  }
  mv[0] = clampi(mv[0] + dh, kMvMin, kMvMax);
  mv[1] = clampi(mv[1] + dv, kMvMin, kMvMax);
  mv[2] = clampi(mv[2] - dh, kMvMin, kMvMax);
  mv[3] = clampi(mv[3] - dv, kMvMin, kMvMax);
}

// inter.rs:1473-1495 is_subblock_vector_spread_over_limit
static bool spread_over_limit(int a, int b, int c, int d, int pred_type) {
  const int s4 = 4 << 11, tap = 6;
  if (pred_type == 3) {
    const int max_w = std::max(std::max(0, 4 * a + s4), std::max(4 * c, 4 * a + 4 * c + s4));
    const int min_w = std::min(std::min(0, 4 * a + s4), std::min(4 * c, 4 * a + 4 * c + s4));
    const int max_h = std::max(std::max(0, 4 * b), std::max(4 * d + s4, 4 * b + 4 * d + s4));
    const int min_h = std::min(std::min(0, 4 * b), std::min(4 * d + s4, 4 * b + 4 * d + s4));
    const int rw = ((max_w - min_w) >> 11) + tap + 3, rh = ((max_h - min_h) >> 11) + tap + 3;
    return rw * rh > (tap + 9) * (tap + 9);
  }
  const int rw0 = (std::abs(4 * a + s4) >> 11) + tap + 3, rh0 = (std::abs(4 * b) >> 11) + tap + 3;
  if (rw0 * rh0 > (tap + 9) * (tap + 5)) return true;
  const int rw1 = (std::abs(4 * c) >> 11) + tap + 3, rh1 = (std::abs(4 * d + s4) >> 11) + tap + 3;
  return rw1 * rh1 > (tap + 5) * (tap + 9);
}

// inter.rs:1502-1579 derive_affine_subblock_mvs. cp: 3 control-point MVs
// (hor, ver); six_param; sub: (w/4 x h/4) x 2 outputs; prof_h / prof_v: 16
// each; returns enable_prof.
bool affine_mvs(const int32_t* cp, bool six_param, int w, int h, int inter_dir, int32_t* sub, int32_t* prof_h,
                int32_t* prof_v) {
  const int prec = 7;
  const int lw = __builtin_ctz((unsigned)w), lh = __builtin_ctz((unsigned)h);
  const int dhx = (cp[2] - cp[0]) << (prec - lw), dhy = (cp[3] - cp[1]) << (prec - lw);
  int dvx, dvy;
  if (six_param) {
    dvx = (cp[4] - cp[0]) << (prec - lh);
    dvy = (cp[5] - cp[1]) << (prec - lh);
  } else {
    dvx = -dhy;
    dvy = dhx;
  }
  const bool large = spread_over_limit(dhx, dhy, dvx, dvy, inter_dir);
  const bool prof = !large && (dhx || dhy || dvx || dvy);
  const int bh = cp[0] << prec, bv = cp[1] << prec;
  int k = 0;
  for (int sy = 0; sy < h / 4; sy++)
    for (int sx = 0; sx < w / 4; sx++) {
      const int wh = large ? (w >> 1) : 2 + sx * 4, wv = large ? (h >> 1) : 2 + sy * 4;
      sub[2 * k] = clampi(shr_round(bh + dhx * wh + dvx * wv, prec), kMvMin, kMvMax);
      sub[2 * k + 1] = clampi(shr_round(bv + dhy * wh + dvy * wv, prec), kMvMin, kMvMax);
      k++;
    }
  for (int i = 0; i < 16; i++) prof_h[i] = prof_v[i] = 0;
  if (prof) {
    const int lim = (1 << 5) - 1;
    for (int y = 0; y < 4; y++)
      for (int x = 0; x < 4; x++) {
        const int wx = 2 * x - 3, wy = 2 * y - 3;
        prof_h[y * 4 + x] = clampi(shr_round(wx * dhx + wy * dvx, 7), -lim, lim);
        prof_v[y * 4 + x] = clampi(shr_round(wx * dhy + wy * dvy, 7), -lim, lim);
      }
  }
  return prof;
}

// inter.rs:1581-1609 apply_prof_4x4
void prof_4x4(const int32_t* src6x6, const int32_t* dmv_x, const int32_t* dmv_y, bool bi, int32_t* out) {
  const int di_limit = 1 << 13, shift = kIfInternalPrec - 8, offset = (1 << (shift - 1)) + kIfInternalOffs;
  for (int y = 0; y < 4; y++)
    for (int x = 0; x < 4; x++) {
      const int c = (y + 1) * 6 + x + 1;
      const int gx = (src6x6[c + 1] >> 6) - (src6x6[c - 1] >> 6);
      const int gy = (src6x6[c + 6] >> 6) - (src6x6[c - 6] >> 6);
      const int i = y * 4 + x;
      const int di = clampi(dmv_x[i] * gx + dmv_y[i] * gy, -di_limit, di_limit - 1);
      const int v = src6x6[c] + di;
      out[i] = bi ? v : clampi((v + offset) >> shift, 0, 255);
    }
}

// inter.rs:1615-1630 apply_ciip_blend
void ciip_blend(const int32_t* inter, const int32_t* intra, int n, bool left_intra, bool above_intra, int32_t* out) {
  const int wi = 1 + (left_intra ? 1 : 0) + (above_intra ? 1 : 0);
  for (int i = 0; i < n; i++) out[i] = clampi(inter[i] + ((wi * (intra[i] - inter[i]) + 2) >> 2), 0, 255);
}

// inter.rs:1641-1731 derive_gpm_params_table + predict_gpm_block
void gpm_block(const int32_t* p0, const int32_t* p1, int w, int h, int split_dir, int scale_x, int scale_y,
               int32_t* out) {
  int ang[64] = {0}, dist[64] = {0}, m = 0;
  for (int a = 0; a < 32; a++)
    for (int d = 0; d < 4; d++) {
      const int mask = kGeoAngleToMask[a];
      if ((d == 0 && a >= 16) || ((d == 2 || d == 0) && (mask == 0 || mask == 5)) || mask == -1) continue;
      if (m < 64) {
        ang[m] = a;
        dist[m] = d;
        m++;
      }
    }
  const int angle = ang[split_dir & 63], distance = dist[split_dir & 63];
  const int lw = w << scale_x, lh = h << scale_y;
  int ox = -(lw >> 1), oy = -(lh >> 1);
  if (distance > 0) {
    const int am = angle % 16;
    if (am == 8 || (am != 0 && lh >= lw))
      oy += angle < 16 ? (distance * lh) >> 3 : -((distance * lh) >> 3);
    else
      ox += angle < 16 ? (distance * lw) >> 3 : -((distance * lw) >> 3);
  }
  const int dx = angle, dy = (dx + 8) % 32;
  for (int y = 0; y < h; y++) {
    const int ly = y << scale_y;
    const int lookup_y = (((ly + oy) << 1) + 1) * kGeoDis[dy];
    for (int x = 0; x < w; x++) {
      const int lx = x << scale_x;
      const int wi = (((lx + ox) << 1) + 1) * kGeoDis[dx] + lookup_y;
      const int w0 = clampi((32 + wi + 4) >> 3, 0, 8), w1 = 8 - w0;
      out[y * w + x] = clampi((w0 * p0[y * w + x] + w1 * p1[y * w + x] + 4) >> 3, 0, 255);
    }
  }
}

}  // namespace orc

extern "C" {

void orc_bdof(const int32_t* p0, const int32_t* p1, int w, int h, int32_t* dst) { orc::bdof_luma(p0, p1, w, h, dst); }
void orc_dmvr(const uint8_t* r0, const uint8_t* r1, int pw, int ph, int stride, int bx, int by, int dx, int dy,
              int32_t* mv) {
  orc::dmvr_refine(r0, r1, pw, ph, stride, bx, by, dx, dy, mv);
}
int orc_affine_mvs(const int32_t* cp, int six, int w, int h, int inter_dir, int32_t* sub, int32_t* ph, int32_t* pv) {
  return orc::affine_mvs(cp, six != 0, w, h, inter_dir, sub, ph, pv) ? 1 : 0;
}
void orc_prof(const int32_t* src, const int32_t* dx, const int32_t* dy, int bi, int32_t* out) {
  orc::prof_4x4(src, dx, dy, bi != 0, out);
}
void orc_ciip(const int32_t* inter, const int32_t* intra, int n, int left, int above, int32_t* out) {
  orc::ciip_blend(inter, intra, n, left != 0, above != 0, out);
}
void orc_gpm(const int32_t* p0, const int32_t* p1, int w, int h, int split, int sx, int sy, int32_t* out) {
  orc::gpm_block(p0, p1, w, h, split, sx, sy, out);
}

}  // extern "C"
