// CPU oracle (test infrastructure only; see oracle.h): ALF of the general
// decoding path. Restates crates/rustmpeg-video/src/vvc/:
//   apply_alf                              decode_general.rs:5225-5345
//   ccalf_block                            decode_general.rs:5348-5408
//   alf_luma_block                         decode_general.rs:5411-5565
//   alf_chroma_block                       decode_general.rs:5568-5660
//   derive_alf_class_4x4_vb_16 (+ _samples) filter.rs:1558-1691
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "../include/vvcg.h"
#include "../rustmpeg-next_b200/csrc/vvc_tables.h"
#include "oracle.h"

namespace orc {
using namespace vvc_tables;

namespace {

struct View {
  const uint16_t* p;
  int stride, lw, lh;  // clamp bounds: min(visible, plane)
  int get(int x, int y) const {
    x = std::min(std::max(x, 0), lw - 1);
    y = std::min(std::max(y, 0), lh - 1);
    return p[y * stride + x];
  }
};

const int* clip_table(int bd) { return bd >= 12 ? kAlfClip[2] : (bd >= 10 ? kAlfClip[1] : kAlfClip[0]); }

// filter.rs:1580-1691 derive_alf_class_4x4_vb_samples
void classify_vb(const View& v, int bx, int by, int vb_h, int vb_pos, int bd, int* cls, int* tr) {
  static const int TH[16] = {0, 1, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 4};
  static const int TT[8] = {0, 1, 0, 2, 2, 3, 1, 3};
  int sv = 0, sh = 0, d0 = 0, d1 = 0;
  const int row_vb = (vb_h > 0 && by % vb_h == vb_pos - 4) ? 1 : (vb_h > 0 && by % vb_h == vb_pos) ? 2 : 0;
  for (int dy = -2; dy < 6; dy += 2) {
    if ((row_vb == 1 && dy == 4) || (row_vb == 2 && dy == -2)) continue;
    for (int dx = -2; dx < 6; dx += 2) {
      const int x = bx + dx, y = by + dy;
      int down = y - 1, up = y + 1, up2 = y + 2;
      if (vb_h > 0 && y > 0) {
        const int yy = y % vb_h;
        if (vb_pos >= 2 && yy == vb_pos - 2) {
          down = y - 1; up = y + 1; up2 = y + 1;
        } else if (yy == vb_pos) {
          down = y; up = y + 1; up2 = y + 2;
        }
      }
      const int y0 = v.get(x, y) << 1, yu = v.get(x + 1, y + 1) << 1;
      sv += abs(y0 - v.get(x, down) - v.get(x, up)) + abs(yu - v.get(x + 1, y) - v.get(x + 1, up2));
      sh += abs(y0 - v.get(x + 1, y) - v.get(x - 1, y)) + abs(yu - v.get(x + 2, y + 1) - v.get(x, y + 1));
      d0 += abs(y0 - v.get(x - 1, down) - v.get(x + 1, up)) + abs(yu - v.get(x, y) - v.get(x + 2, up2));
      d1 += abs(y0 - v.get(x - 1, up) - v.get(x + 1, down)) + abs(yu - v.get(x, up2) - v.get(x + 2, y));
    }
  }
  int scale = 64;
  if (vb_h > 0 && vb_pos >= 4) {
    const int yy = by % vb_h;
    if (yy == vb_pos - 4 || yy == vb_pos) scale = 96;
  }
  const int act = std::min(15, std::max(0, ((sv + sh) * scale) >> (bd + 4)));
  int c = TH[act];
  int hv1, hv0, dhv, dd1, dd0, ddd;
  if (sv > sh) { hv1 = sv; hv0 = sh; dhv = 1; } else { hv1 = sh; hv0 = sv; dhv = 3; }
  if (d0 > d1) { dd1 = d0; dd0 = d1; ddd = 0; } else { dd1 = d1; dd0 = d0; ddd = 2; }
  int h1, h0, md, sd;
  if ((long long)dd1 * hv0 > (long long)hv1 * dd0) { h1 = dd1; h0 = dd0; md = ddd; sd = dhv; }
  else { h1 = hv1; h0 = hv0; md = dhv; sd = ddd; }
  int ds = 0;
  if (h1 > 2 * h0) ds = 1;
  if (h1 * 2 > 9 * h0) ds = 2;
  if (ds > 0) c += (((md & 1) << 1) + ds) * 5;
  *cls = c;
  *tr = TT[md * 2 + (sd >> 1)];
}

// decode_general.rs:5411-5565 alf_luma_block
void alf_luma_block(const View& src, uint16_t* dst, int dstride, int x0, int y0, int w, int h, int vb_h, int vb_pos,
                    const vvcg_alf_ctu& m, const vvcg_alf_params& a, int bd) {
  const int maxv = (1 << bd) - 1;
  const int* ct = clip_table(bd);
  static const int TERMS[12][4] = {{0, 5, 0, 6}, {1, 3, -1, 4}, {0, 3, 0, 4}, {-1, 3, 1, 4}, {2, 1, -2, 2}, {1, 1, -1, 2},
                                   {0, 1, 0, 2}, {-1, 1, 1, 2}, {-2, 1, 2, 2}, {3, 0, -3, 0}, {2, 0, -2, 0}, {1, 0, -1, 0}};
  for (int by = y0; by < y0 + h; by += 4)
    for (int bx = x0; bx < x0 + w; bx += 4) {
      int cls, tr;
      classify_vb(src, bx, by, vb_h, vb_pos, bd, &cls, &tr);
      int coeffs[12], clips[12] = {0};
      if (m.luma_mode == VVCG_ALF_FIXED) {
        const int fi = kAlfClassToFilter[std::min<int>(m.luma_set, 15) * 25 + std::min(cls, 24)];
        for (int k = 0; k < 12; k++) coeffs[k] = kAlfFixedCoeff[fi * 13 + k];
      } else {
        const int fi = std::min<int>(a.coeff_delta_idx[std::min(cls, 24)], std::max(1, (int)a.num_luma_filters) - 1);
        for (int k = 0; k < 12; k++) coeffs[k] = a.luma_coeff[fi][k];
        if (a.luma_clip && fi < a.num_luma_filters)
          for (int k = 0; k < 12; k++) clips[k] = a.luma_clip_idx[fi][k];
      }
      int fc[12], fcl[12];
      for (int k = 0; k < 12; k++) {
        const int p = kAlfTransposePerm[(tr & 3) * 12 + k];
        fc[k] = coeffs[p];
        fcl[k] = ct[clips[p] & 3];
      }
      const int xe = std::min(bx + 4, x0 + w), ye = std::min(by + 4, y0 + h);
      for (int y = by; y < ye; y++)
        for (int x = bx; x < xe; x++) {
          const int cur = src.get(x, y);
          const int yv = y % vb_h;
          int rows[7] = {y, y + 1, y - 1, y + 2, y - 2, y + 3, y - 3};
          if (yv < vb_pos && yv + 4 >= vb_pos) {
            if (yv == vb_pos - 1) { rows[1] = rows[0]; rows[2] = rows[0]; }
            if (yv + 2 >= vb_pos) { rows[3] = rows[1]; rows[4] = rows[2]; }
            if (yv + 3 >= vb_pos) { rows[5] = rows[3]; rows[6] = rows[4]; }
          } else if (yv >= vb_pos && yv <= vb_pos + 3) {
            if (yv == vb_pos) { rows[2] = rows[0]; rows[1] = rows[0]; }
            if (yv <= vb_pos + 1) { rows[4] = rows[2]; rows[3] = rows[1]; }
            if (yv <= vb_pos + 2) { rows[6] = rows[4]; rows[5] = rows[3]; }
          }
          const bool near = (yv < vb_pos && yv + 1 >= vb_pos) || yv == vb_pos;
          int sum = 0;
          for (int k = 0; k < 12; k++) {
            const int pa = src.get(x + TERMS[k][0], rows[TERMS[k][1]]);
            const int pb = src.get(x + TERMS[k][2], rows[TERMS[k][3]]);
            sum += fc[k] * (std::min(fcl[k], std::max(-fcl[k], pa - cur)) + std::min(fcl[k], std::max(-fcl[k], pb - cur)));
          }
          const int shift = near ? 10 : 7;
          dst[y * dstride + x] = (uint16_t)std::min(maxv, std::max(0, cur + ((sum + (1 << (shift - 1))) >> shift)));
        }
    }
}

// decode_general.rs:5568-5660 alf_chroma_block
void alf_chroma_block(const View& src, uint16_t* dst, int dstride, int dw, int dh, const vvcg_alf_params& a, int alt,
                      int x0, int y0, int w, int h, int vb_h, int vb_pos, int bd) {
  if (a.num_chroma_filters == 0) return;
  const int idx = std::min(alt, (int)a.num_chroma_filters - 1);
  const int maxv = (1 << bd) - 1;
  const int* ct = clip_table(bd);
  static const int TERMS[6][4] = {{0, 3, 0, 4}, {1, 1, -1, 2}, {0, 1, 0, 2}, {-1, 1, 1, 2}, {2, 0, -2, 0}, {1, 0, -1, 0}};
  for (int y = y0; y < std::min(y0 + h, dh); y++)
    for (int x = x0; x < std::min(x0 + w, dw); x++) {
      const int cur = src.get(x, y);
      const int yv = y % vb_h;
      int rows[5] = {y, y + 1, y - 1, y + 2, y - 2};
      if (yv < vb_pos && yv + 2 >= vb_pos) {
        if (yv + 1 == vb_pos) { rows[1] = rows[0]; rows[2] = rows[0]; }
        if (yv + 2 >= vb_pos) { rows[3] = rows[1]; rows[4] = rows[2]; }
      } else if (yv >= vb_pos && yv <= vb_pos + 1) {
        if (yv == vb_pos) { rows[2] = rows[0]; rows[1] = rows[0]; }
        if (yv <= vb_pos + 1) { rows[4] = rows[2]; rows[3] = rows[1]; }
      }
      const bool near = (yv < vb_pos && yv + 1 >= vb_pos) || yv == vb_pos;
      int sum = 0;
      for (int k = 0; k < 6; k++) {
        const int pa = src.get(x + TERMS[k][0], rows[TERMS[k][1]]);
        const int pb = src.get(x + TERMS[k][2], rows[TERMS[k][3]]);
        const int cl = ct[(a.chroma_clip ? a.chroma_clip_idx[idx][k] : 0) & 3];
        sum += a.chroma_coeff[idx][k] * (std::min(cl, std::max(-cl, pa - cur)) + std::min(cl, std::max(-cl, pb - cur)));
      }
      const int shift = near ? 10 : 7;
      dst[y * dstride + x] = (uint16_t)std::min(maxv, std::max(0, cur + ((sum + (1 << (shift - 1))) >> shift)));
    }
}

// decode_general.rs:5348-5408 ccalf_block (adds to dst in place)
void ccalf_block(const View& luma, uint16_t* chroma, int cstride, const int16_t* coeffs, int x0, int y0, int w, int h,
                 int cw, int ch, int ctu_l, int bd) {
  const int maxv = (1 << bd) - 1, offset = 1 << (bd - 1);
  const int vb_pos = std::max(0, ctu_l - 4);
  for (int y = y0; y < std::min(y0 + h, ch); y++) {
    const int ly = y * 2, pos = ly & (ctu_l - 1);
    int above, below, below2;
    if (pos == std::max(0, vb_pos - 2) || pos == vb_pos + 1) {
      above = ly - 1; below = ly + 1; below2 = ly + 1;
    } else if (pos == std::max(0, vb_pos - 1) || pos == vb_pos) {
      above = ly; below = ly; below2 = ly;
    } else {
      above = ly - 1; below = ly + 1; below2 = ly + 2;
    }
    for (int x = x0; x < std::min(x0 + w, cw); x++) {
      const int lx = x * 2, cur = luma.get(lx, ly);
      int sum = coeffs[0] * (luma.get(lx, above) - cur);
      sum += coeffs[1] * (luma.get(lx - 1, ly) - cur);
      sum += coeffs[2] * (luma.get(lx + 1, ly) - cur);
      sum += coeffs[3] * (luma.get(lx - 1, below) - cur);
      sum += coeffs[4] * (luma.get(lx, below) - cur);
      sum += coeffs[5] * (luma.get(lx + 1, below) - cur);
      sum += coeffs[6] * (luma.get(lx, below2) - cur);
      const int v = std::min(offset - 1, std::max(-offset, (sum + 64) >> 7));
      const int out = chroma[y * cstride + x] + v;
      chroma[y * cstride + x] = (uint16_t)std::min(maxv, std::max(0, out));
    }
  }
}

}  // namespace
}  // namespace orc

// decode_general.rs:5225-5345 apply_alf on a 4:2:0 picture: src / dst planes
// of width x height (chroma half size, strides = widths).
extern "C" void orc_alf_general(const uint16_t* sy, const uint16_t* su, const uint16_t* sv, uint16_t* dy,
                                uint16_t* du, uint16_t* dv, int pw, int ph, int vis_w, int vis_h, int bd, int ctu,
                                int ctu_cols, const vvcg_alf_ctu* ctus, const vvcg_alf_params* a) {
  using namespace orc;
  bd = std::min(12, std::max(8, bd));
  const int cw = (pw + 1) / 2, chh = (ph + 1) / 2;
  std::copy(sy, sy + pw * ph, dy);
  std::copy(su, su + cw * chh, du);
  std::copy(sv, sv + cw * chh, dv);
  const int cvis_w = (vis_w + 1) / 2, cvis_h = (vis_h + 1) / 2;
  View vy{sy, pw, std::min(vis_w, pw), std::min(vis_h, ph)};
  View vu{su, cw, std::min(cvis_w, cw), std::min(cvis_h, chh)};
  View vv{sv, cw, std::min(cvis_w, cw), std::min(cvis_h, chh)};
  for (int gy = 0; gy * ctu < vis_h; gy++)
    for (int gx = 0; gx * ctu < vis_w; gx++) {
      const vvcg_alf_ctu& m = ctus[gy * ctu_cols + gx];
      const int x0 = gx * ctu, y0 = gy * ctu;
      const int w = std::min(ctu, vis_w - x0), h = std::min(ctu, vis_h - y0);
      if (m.luma_mode != VVCG_ALF_OFF) alf_luma_block(vy, dy, pw, x0, y0, w, h, ctu, ctu - 4, m, *a, bd);
      for (int c = 1; c <= 2; c++) {
        const int alt = c == 1 ? m.cb_alt : m.cr_alt;
        if (alt == 0xFF) continue;
        alf_chroma_block(c == 1 ? vu : vv, c == 1 ? du : dv, cw, cw, chh, *a, alt, x0 / 2, y0 / 2, std::max(w / 2, 1),
                         std::max(h / 2, 1), ctu / 2, ctu / 2 - 2, bd);
      }
      for (int c = 1; c <= 2; c++) {
        const int idc = c == 1 ? m.cc_cb : m.cc_cr;
        const int nf = c == 1 ? a->num_cc_cb : a->num_cc_cr;
        if (idc == 0 || idc > nf) continue;
        const int16_t* co = c == 1 ? a->cc_cb[idc - 1] : a->cc_cr[idc - 1];
        ccalf_block(vy, c == 1 ? du : dv, cw, co, x0 / 2, y0 / 2, std::max(w / 2, 1), std::max(h / 2, 1), cvis_w,
                    cvis_h, ctu, bd);
      }
    }
}
