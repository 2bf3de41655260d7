// CPU oracle (test infrastructure only; see oracle.h): 8/10/12-bit intra
// prediction. Restates crates/rustmpeg-video/src/vvc/predict.rs of the
// reference (the Plane16 family used by the 10-bit frame encoder/decoder).
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "../rustmpeg-next_b200/csrc/vvc_tables.h"
#include "oracle.h"

namespace orc {
using namespace vvc_tables;

static const int PLANAR = 0, DC = 1, HOR = 18, DIA = 34, VER = 50, VDIA = 66;

static inline int ilog2(int v) { return __builtin_ctz((unsigned)v); }
static inline int floor_log2(unsigned v) { return 31 - __builtin_clz(v); }
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// predict.rs:1405-1422 get_modified_wide_angle
int get_modified_wide_angle(int w, int h, int mode) {
  if (mode > DC && mode <= VDIA) {
    static const int kShift[6] = {0, 6, 10, 12, 14, 15};
    int delta = std::abs(floor_log2(w) - floor_log2(h));
    if (delta < 6) {
      int s = kShift[delta];
      if (w > h && mode < 2 + s) return mode + (VDIA - 1);
      if (h > w && mode > VDIA - s) return mode - (VDIA - 1);
    }
  }
  return mode;
}

// predict.rs:1608-1685 init_angular_params
AngularParams init_angular_params(int dir_mode, int pu_w, int pu_h, int cu_w, int cu_h,
                                  bool is_luma, int mrl_idx, bool use_isp) {
  int bw = (use_isp && is_luma) ? cu_w : pu_w;
  int bh = (use_isp && is_luma) ? cu_h : pu_h;
  AngularParams p{};
  p.pred_mode = get_modified_wide_angle(bw, bh, dir_mode);
  p.is_mode_ver = p.pred_mode >= DIA;
  int mri = is_luma ? mrl_idx : 0;
  p.apply_pdpc = pu_w >= 4 && pu_h >= 4 && mri == 0;
  int ang_mode = p.is_mode_ver ? p.pred_mode - VER : -(p.pred_mode - HOR);
  int abs_mode = std::min(31, std::abs(ang_mode));
  int sign = ang_mode < 0 ? -1 : 1;
  int abs_ang = kAngTable[abs_mode];
  p.abs_inv_angle = kInvAngTable[abs_mode];
  p.intra_pred_angle = sign * abs_ang;
  p.angular_scale = 0;
  if (ang_mode < 0) {
    p.apply_pdpc = false;
  } else if (ang_mode > 0) {
    int side = p.is_mode_ver ? pu_h : pu_w;
    int inv_term = floor_log2((unsigned)std::max(1, 3 * p.abs_inv_angle - 2)) - 8;
    p.angular_scale = std::min(2, floor_log2((unsigned)side) - inv_term);
    if (p.angular_scale < 0) p.apply_pdpc = false;
  }
  p.ref_filter_flag = false;
  p.interpolation_flag = false;
  if (is_luma && !use_isp && mri == 0 && dir_mode != DC && dir_mode != PLANAR) {
    int diff = std::min(std::abs(p.pred_mode - HOR), std::abs(p.pred_mode - VER));
    int log2_size = (floor_log2(pu_w) + floor_log2(pu_h)) >> 1;
    if (diff > kIntraFilterThreshold[std::min(7, log2_size)]) {
      bool int_slope = (abs_ang & 0x1F) == 0;  // predict.rs:1396 is_integer_slope
      p.ref_filter_flag = int_slope;
      p.interpolation_flag = !int_slope;
    }
  }
  p.ref_w = (use_isp && is_luma) ? cu_w + pu_w : 2 * pu_w;
  p.ref_h = (use_isp && is_luma) ? cu_h + pu_h : 2 * pu_h;
  return p;
}

// predict.rs:2970-3005 ReferenceSamples16::filtered
static Refs16 filtered(const Refs16& r) {
  Refs16 o = r;
  int w2 = (int)r.above.size(), h2 = (int)r.left.size();
  o.top_left = (2 * r.top_left + r.above[0] + r.left[0] + 2) >> 2;
  for (int j = 0; j + 1 < w2; j++) {
    int prev = j == 0 ? r.top_left : r.above[j - 1];
    o.above[j] = (prev + 2 * r.above[j] + r.above[j + 1] + 2) >> 2;
  }
  for (int j = 0; j + 1 < h2; j++) {
    int prev = j == 0 ? r.top_left : r.left[j - 1];
    o.left[j] = (prev + 2 * r.left[j] + r.left[j + 1] + 2) >> 2;
  }
  return o;
}

// predict.rs:3016-3076 gather_references_16
Refs16 gather_references_16(const Plane16& p, int x, int y, int w, int h) {
  int bd = clampi(p.bd, 8, 12);
  int def = 1 << (bd - 1);
  Refs16 r;
  r.bd = p.bd;
  r.above.assign(2 * w, def);
  r.left.assign(2 * h, def);
  bool has_above = y > 0, has_left = x > 0;
  if (has_above) {
    int avail = std::min(std::max(0, p.width - x), 2 * w);
    for (int i = 0; i < avail; i++) r.above[i] = p.get(x + i, y - 1);
    int pad = r.above[std::max(0, avail - 1)];
    for (int i = avail; i < 2 * w; i++) r.above[i] = pad;
  }
  if (has_left) {
    int avail = std::min(std::max(0, p.height - y), h);
    for (int j = 0; j < avail; j++) r.left[j] = p.get(x - 1, y + j);
    int pad = r.left[std::max(0, avail - 1)];
    for (int j = avail; j < 2 * h; j++) r.left[j] = pad;
  }
  if (has_above && !has_left) {
    std::fill(r.left.begin(), r.left.end(), r.above[0]);
  } else if (!has_above && has_left) {
    std::fill(r.above.begin(), r.above.end(), r.left[0]);
  }
  if (has_above && has_left)
    r.top_left = p.get(x - 1, y - 1);
  else if (has_above)
    r.top_left = r.above[0];
  else if (has_left)
    r.top_left = r.left[0];
  else
    r.top_left = def;
  return r;
}

// predict.rs:3200-3215 apply_pdpc_16
static void apply_pdpc_16(uint16_t* pred, const Refs16& refs, int w, int h) {
  int s = ilog2(w) + ilog2(h);
  int scale = (s >= 2 ? s - 2 : 0) >> 2;
  int max_val = (1 << clampi(refs.bd, 8, 12)) - 1;
  for (int y = 0; y < h; y++) {
    int wt = 32 >> std::min(31, (y * 2) >> scale);
    int left = refs.left[y];
    for (int x = 0; x < w; x++) {
      int wl = 32 >> std::min(31, (x * 2) >> scale);
      int top = refs.above[x];
      int val = pred[y * w + x];
      pred[y * w + x] =
          (uint16_t)clampi(val + ((wl * (left - val) + wt * (top - val) + 32) >> 6), 0, max_val);
    }
  }
}

// predict.rs:3223-3410 predict_angular_16
static void predict_angular_16(const Refs16& refs, int w, int h, bool is_luma, int dir,
                               uint16_t* out) {
  int bd = clampi(refs.bd, 8, 12);
  int max_val = (1 << bd) - 1;
  int def = 1 << (bd - 1);
  AngularParams pa = init_angular_params(dir, w, h, w, h, is_luma, 0, false);
  Refs16 used = pa.ref_filter_flag ? filtered(refs) : refs;
  std::vector<int> row_above, row_left;
  row_above.push_back(used.top_left);
  row_above.insert(row_above.end(), used.above.begin(), used.above.end());
  row_left.push_back(used.top_left);
  row_left.insert(row_left.end(), used.left.begin(), used.left.end());
  bool is_ver = pa.is_mode_ver;
  int angle = pa.intra_pred_angle;
  int abs_inv = pa.abs_inv_angle;
  int mx = std::max(w, h);
  int base = mx + 4;
  int buf_len = base + 2 * mx + 64;
  std::vector<int> ref_above(buf_len, def), ref_left(buf_len, def);
  int na = (int)row_above.size(), nl = (int)row_left.size();
  if (angle < 0) {
    for (int x = 0; x <= w + 1; x++) ref_above[base + x] = row_above[std::min(x, na - 1)];
    for (int y = 0; y <= h + 1; y++) ref_left[base + y] = row_left[std::min(y, nl - 1)];
    int size_side = is_ver ? h : w;
    for (int k = -size_side; k <= -1; k++) {
      int proj = std::min((-k * abs_inv + 256) >> 9, size_side);
      if (is_ver)
        ref_above[base + k] = ref_left[base + proj];
      else
        ref_left[base + k] = ref_above[base + proj];
    }
  } else {
    for (int x = 0; x <= 2 * w; x++) ref_above[base + x] = row_above[std::min(x, na - 1)];
    for (int y = 0; y <= 2 * h; y++) ref_left[base + y] = row_left[std::min(y, nl - 1)];
    int ref_len = is_ver ? 2 * w : 2 * h;
    if (is_ver) {
      int v = ref_above[base + ref_len];
      for (int z = 1; z <= 2; z++) ref_above[base + ref_len + z] = v;
    } else {
      int v = ref_left[base + ref_len];
      for (int z = 1; z <= 2; z++) ref_left[base + ref_len + z] = v;
    }
  }
  const std::vector<int>& rm = is_ver ? ref_above : ref_left;
  const std::vector<int>& rs = is_ver ? ref_left : ref_above;
  int ww = is_ver ? w : h, wh = is_ver ? h : w;
  std::vector<int> temp((size_t)ww * wh, 0);
  if (angle == 0) {
    int scale = (ilog2(ww) + ilog2(wh) - 2) >> 2;
    int top_left = rm[base];
    for (int y = 0; y < wh; y++) {
      int row = y * ww;
      for (int x = 0; x < ww; x++) temp[row + x] = rm[base + x + 1];
      if (pa.apply_pdpc) {
        int left = rs[base + 1 + y];
        int limit = std::min(3 << scale, ww);
        for (int x = 0; x < limit; x++) {
          int wl = 32 >> ((2 * x) >> scale);
          int val = temp[row + x];
          temp[row + x] = clampi(val + ((wl * (left - top_left) + 32) >> 6), 0, max_val);
        }
      }
    }
  } else {
    bool int_slope = (std::abs(angle) & 0x1F) == 0;
    int delta_pos = angle;
    for (int y = 0; y < wh; y++) {
      int row = y * ww;
      int delta_int = delta_pos >> 5;
      int fr = delta_pos & 31;
      if (!int_slope) {
        int gauss[4] = {16 - (fr >> 1), 32 - (fr >> 1), 16 + (fr >> 1), fr >> 1};
        int f[4];
        for (int k = 0; k < 4; k++) f[k] = pa.interpolation_flag ? gauss[k] : kChromaTaps4[fr * 4 + k];
        if (is_luma) {
          for (int x = 0; x < ww; x++) {
            int i = base + delta_int + x;
            int s = f[0] * rm[i] + f[1] * rm[i + 1] + f[2] * rm[i + 2] + f[3] * rm[i + 3];
            temp[row + x] = clampi((s + 32) >> 6, 0, max_val);
          }
        } else {
          for (int x = 0; x < ww; x++) {
            int i = base + delta_int + x + 1;
            int p0 = rm[i], p1 = rm[i + 1];
            temp[row + x] = clampi(p0 + ((fr * (p1 - p0) + 16) >> 5), 0, max_val);
          }
        }
      } else {
        for (int x = 0; x < ww; x++) temp[row + x] = clampi(rm[base + delta_int + x + 1], 0, max_val);
      }
      if (pa.apply_pdpc) {
        int scale = std::max(0, pa.angular_scale);
        int inv_sum = 256;
        int limit = std::min(3 << scale, ww);
        for (int x = 0; x < limit; x++) {
          inv_sum += abs_inv;
          int wl = 32 >> ((2 * x) >> scale);
          int li = base + y + (inv_sum >> 9) + 1;
          int left = rs[std::min(li, buf_len - 1)];
          int val = temp[row + x];
          temp[row + x] = clampi(val + ((wl * (left - val) + 32) >> 6), 0, max_val);
        }
      }
      delta_pos += angle;
    }
  }
  if (is_ver) {
    for (int i = 0; i < w * h; i++) out[i] = (uint16_t)temp[i];
  } else {
    for (int y = 0; y < wh; y++)
      for (int x = 0; x < ww; x++) out[x * w + y] = (uint16_t)temp[y * ww + x];
  }
}

// predict.rs:3138-3196 predict_from_refs_16
void predict_from_refs_16(const Refs16& refs, int w, int h, bool is_luma, int mode,
                          uint16_t* out) {
  int max_val = (1 << clampi(refs.bd, 8, 12)) - 1;
  int lw = ilog2(w), lh = ilog2(h);
  if (mode == PLANAR) {
    // predict.rs:1287 uses_reference_filter: luma planar filters when w*h > 32
    Refs16 u = (is_luma && w * h > 32) ? filtered(refs) : refs;
    int shift = lw + lh + 1;
    int64_t offset = (int64_t)1 << (shift - 1);
    int64_t tr = u.above[w], bl = u.left[h];
    for (int ry = 0; ry < h; ry++) {
      int64_t left = u.left[ry];
      for (int rx = 0; rx < w; rx++) {
        int64_t ver = (int64_t)(h - 1 - ry) * u.above[rx] + (int64_t)(ry + 1) * bl;
        int64_t hor = (int64_t)(w - 1 - rx) * left + (int64_t)(rx + 1) * tr;
        int64_t v = ((ver << lw) + (hor << lh) + offset) >> shift;
        out[ry * w + rx] = (uint16_t)std::min<int64_t>(max_val, std::max<int64_t>(0, v));
      }
    }
    apply_pdpc_16(out, u, w, h);
    return;
  }
  if (mode == DC) {
    unsigned st = 0, sl = 0;
    for (int i = 0; i < w; i++) st += refs.above[i];
    for (int j = 0; j < h; j++) sl += refs.left[j];
    unsigned dc;
    if (w == h)
      dc = (st + sl + (unsigned)w) >> (lw + 1);
    else if (w > h)
      dc = (st + ((unsigned)w >> 1)) >> lw;
    else
      dc = (sl + ((unsigned)h >> 1)) >> lh;
    dc &= 0xFFFF;  // `as u16`
    uint16_t v = (uint16_t)std::min<unsigned>(dc, (unsigned)max_val);
    for (int i = 0; i < w * h; i++) out[i] = v;
    apply_pdpc_16(out, refs, w, h);
    return;
  }
  if (mode >= 2 && mode <= 66) {
    predict_angular_16(refs, w, h, is_luma, mode, out);
    return;
  }
  for (int i = 0; i < w * h; i++) out[i] = 0;  // CCLM/other modes: predict.rs:3194
}

// predict.rs:3079-3091 predict_block_16
void predict_block_16(const Plane16& p, int x, int y, int w, int h, bool is_luma, int mode,
                      uint16_t* out) {
  Refs16 r = gather_references_16(p, x, y, w, h);
  predict_from_refs_16(r, w, h, is_luma, mode, out);
}

// predict.rs:3101-3135 predict_coded_block_16
void predict_coded_block_16(const Plane16& p, int x, int y, int w, int h, bool is_luma, int mode,
                            int sx, int sy, const CodedMap& cm, uint16_t* out) {
  Refs16 r = gather_references_16(p, x, y, w, h);
  if (y > 0) {
    int pad = r.above[w - 1];
    for (int i = w; i < 2 * w; i++) {
      int px = x + i;
      if (px < p.width && !cm.is_coded_luma(px * sx, (y - 1) * sy)) r.above[i] = pad;
    }
  }
  if (x > 0) {
    for (int j = h; j < 2 * h; j++) {
      int py = y + j;
      if (py < p.height && cm.is_coded_luma((x - 1) * sx, py * sy)) r.left[j] = p.get(x - 1, py);
    }
  }
  predict_from_refs_16(r, w, h, is_luma, mode, out);
}

// predict.rs:2088-2177 derive_cclm_params_from_4_samples
void cclm_params(int sl[4], int sc[4], int cnt, int bd, int* a_out, int* b_out, int* shift_out) {
  if (cnt == 0) {
    *a_out = 0;
    *b_out = 1 << (bd > 0 ? bd - 1 : 0);
    *shift_out = 0;
    return;
  }
  if (cnt == 2) {
    sl[3] = sl[0];
    sc[3] = sc[0];
    sl[2] = sl[1];
    sc[2] = sc[1];
    sl[0] = sl[1];
    sc[0] = sc[1];
    sl[1] = sl[3];
    sc[1] = sc[3];
  }
  int mn[2] = {0, 2}, mxg[2] = {1, 3};
  if (sl[mn[0]] > sl[mn[1]]) std::swap(mn[0], mn[1]);
  if (sl[mxg[0]] > sl[mxg[1]]) std::swap(mxg[0], mxg[1]);
  if (sl[mn[0]] > sl[mxg[1]]) {
    std::swap(mn[0], mxg[0]);
    std::swap(mn[1], mxg[1]);
  }
  if (sl[mn[1]] > sl[mxg[0]]) std::swap(mn[1], mxg[0]);
  int min_l = (sl[mn[0]] + sl[mn[1]] + 1) >> 1;
  int min_c = (sc[mn[0]] + sc[mn[1]] + 1) >> 1;
  int max_l = (sl[mxg[0]] + sl[mxg[1]] + 1) >> 1;
  int max_c = (sc[mxg[0]] + sc[mxg[1]] + 1) >> 1;
  int diff = max_l - min_l;
  if (diff > 0) {
    int diff_c = max_c - min_c;
    int x = floor_log2((unsigned)diff);
    int norm = ((diff << 4) >> x) & 15;
    int v = (int)kCclmDivSig[norm] | 8;
    if (norm != 0) x += 1;
    int y = diff_c == 0 ? 1 : floor_log2((unsigned)std::abs(diff_c)) + 1;
    int add = (1 << y) >> 1;
    int a = (diff_c * v + add) >> y;
    int shift = 3 + x - y;
    if (shift < 1) {
      shift = 1;
      a = a == 0 ? 0 : (a < 0 ? -15 : 15);
    }
    *a_out = a;
    *b_out = min_c - ((a * min_l) >> shift);
    *shift_out = shift;
  } else {
    *a_out = 0;
    *b_out = min_c;
    *shift_out = 0;
  }
}

// predict.rs:3869-3990 downsample_luma_for_cclm_format_16 (4:2:0 and 4:4:4 forms)
static void cclm_downsample_16(const Plane16& luma, int bx, int by, int cw, int ch, int cf,
                               int ctu, std::vector<int>& blk, std::vector<int>& top,
                               std::vector<int>& left) {
  int bd = clampi(luma.bd, 8, 12);
  int mid = 1 << (bd - 1);
  auto gy = [&](int x, int y) {
    return (int)luma.get(clampi(x, 0, luma.width - 1), clampi(y, 0, luma.height - 1));
  };
  blk.assign((size_t)cw * ch, 0);
  top.assign(cw, mid);
  left.assign(ch, mid);
  if (cf == 1) {
    auto ds_region = [&](int rx, int ry, int rw, int rh, bool has_l, std::vector<int>& o) {
      o.assign((size_t)rw * rh, 0);
      for (int y = 0; y < rh; y++) {
        int ly = ry + 2 * y;
        for (int x = 0; x < rw; x++) {
          int lx = rx + 2 * x;
          int lxl = (x == 0 && !has_l) ? lx : lx - 1;
          int r0 = 2 * gy(lx, ly) + gy(lxl, ly) + gy(lx + 1, ly);
          int r1 = 2 * gy(lx, ly + 1) + gy(lxl, ly + 1) + gy(lx + 1, ly + 1);
          o[y * rw + x] = (r0 + r1 + 4) >> 3;
        }
      }
    };
    ds_region(bx, by, cw, ch, bx > 0, blk);
    bool first_row_of_ctu = ctu > 0 && (by & (ctu - 1)) == 0;
    if (by > 0 && first_row_of_ctu) {
      for (int x = 0; x < cw; x++) {
        int lx = bx + 2 * x;
        int y = by - 1;
        int x0 = clampi(lx, 0, luma.width - 1);
        int xr = clampi(lx + 1, 0, luma.width - 1);
        int xl = ((x == 0 && bx == 0) || x0 == 0) ? x0 : x0 - 1;
        top[x] = (2 * gy(x0, y) + gy(xl, y) + gy(xr, y) + 2) >> 2;
      }
    } else if (by >= 2) {
      std::vector<int> row;
      ds_region(bx, by - 2, cw, 1, bx > 0, row);
      for (int x = 0; x < cw; x++) top[x] = row[x];
    }
    if (bx >= 2) {
      std::vector<int> col;
      ds_region(bx - 2, by, 1, ch, true, col);
      for (int y = 0; y < ch; y++) left[y] = col[y];
    }
  } else if (cf == 2) {
    for (int y = 0; y < ch; y++) {
      int ly = by + y;
      for (int x = 0; x < cw; x++) {
        int lx = bx + 2 * x;
        int lxl = (x == 0 && bx == 0) ? lx : lx - 1;
        blk[y * cw + x] = (2 * gy(lx, ly) + gy(lxl, ly) + gy(lx + 1, ly) + 2) >> 2;
      }
    }
    if (by > 0) {
      int ly = by - 1;
      for (int x = 0; x < cw; x++) {
        int lx = bx + 2 * x;
        int lxl = (x == 0 && bx == 0) ? lx : lx - 1;
        top[x] = (2 * gy(lx, ly) + gy(lxl, ly) + gy(lx + 1, ly) + 2) >> 2;
      }
    }
    if (bx > 0) {
      for (int y = 0; y < ch; y++) {
        int ly = by + y;
        int lx = bx - 2;
        int lxl = bx >= 2 ? lx - 1 : lx;
        left[y] = (2 * gy(std::max(0, lx), ly) + gy(std::max(0, lxl), ly) + gy(bx - 1, ly) + 2) >> 2;
      }
    }
  } else {
    for (int y = 0; y < ch; y++)
      for (int x = 0; x < cw; x++) blk[y * cw + x] = gy(bx + x, by + y);
    if (by > 0)
      for (int x = 0; x < cw; x++) top[x] = gy(bx + x, by - 1);
    if (bx > 0)
      for (int y = 0; y < ch; y++) left[y] = gy(bx - 1, by + y);
  }
}

// predict.rs:3996-4066 predict_cclm_with_format_16
void predict_cclm_with_format_16(const Plane16& luma, const Plane16& chroma, int bxc, int byc,
                                 int cw, int ch, int cclm_mode, int cf, int ctu, uint16_t* out) {
  int bd = clampi(chroma.bd, 8, 12);
  int max_val = (1 << bd) - 1;
  int mid = 1 << (bd - 1);
  int sw = (cf == 1 || cf == 2) ? 2 : 1;
  int sh = (cf == 1) ? 2 : 1;
  std::vector<int> blk, top, left;
  cclm_downsample_16(luma, bxc * sw, byc * sh, cw, ch, cf, ctu, blk, top, left);
  Refs16 rc = gather_references_16(chroma, bxc, byc, cw, ch);
  bool has_top = byc > 0 && cclm_mode != 1;
  bool has_left = bxc > 0 && cclm_mode != 2;
  int lp[4] = {mid, mid, mid, mid}, cp[4] = {mid, mid, mid, mid};
  int cnt = 0;
  if (has_top && has_left) {
    int x0 = cw / 4, x1 = (3 * cw) / 4, y0 = ch / 4, y1 = (3 * ch) / 4;
    lp[0] = top[x0];
    lp[1] = top[x1];
    lp[2] = left[y0];
    lp[3] = left[y1];
    cp[0] = rc.above[x0];
    cp[1] = rc.above[x1];
    cp[2] = rc.left[y0];
    cp[3] = rc.left[y1];
    cnt = 4;
  } else if (has_top) {
    for (int i = 0; i < std::min(4, cw); i++) {
      int idx = std::min(((2 * i + 1) * cw) / 8, cw - 1);
      lp[i] = top[idx];
      cp[i] = rc.above[idx];
      cnt++;
    }
  } else if (has_left) {
    for (int i = 0; i < std::min(4, ch); i++) {
      int idx = std::min(((2 * i + 1) * ch) / 8, ch - 1);
      lp[i] = left[idx];
      cp[i] = rc.left[idx];
      cnt++;
    }
  }
  int a, b, shift;
  cclm_params(lp, cp, cnt, bd, &a, &b, &shift);
  for (int i = 0; i < cw * ch; i++) out[i] = (uint16_t)clampi(((blk[i] * a) >> shift) + b, 0, max_val);
}

// predict.rs:4069-4105 choose_intra_mode_16 (7 candidates, lowest SAD, first wins ties)
int choose_intra_mode_16(const Plane16& recon, const Plane16& src, int bx, int by, int w, int h,
                         bool is_luma) {
  static const int kCands[7] = {PLANAR, DC, 18, 50, 2, 34, 66};
  int best = PLANAR;
  uint64_t best_sad = UINT64_MAX;
  std::vector<uint16_t> pred((size_t)w * h);
  for (int c = 0; c < 7; c++) {
    predict_block_16(recon, bx, by, w, h, is_luma, kCands[c], pred.data());
    uint64_t sad = 0;
    for (int y = 0; y < h; y++) {
      int yy = std::min(by + y, std::max(0, src.height - 1));
      for (int x = 0; x < w; x++) {
        int xx = std::min(bx + x, std::max(0, src.width - 1));
        sad += (uint64_t)std::abs((int)src.get(xx, yy) - (int)pred[y * w + x]);
      }
    }
    if (sad < best_sad) {
      best_sad = sad;
      best = kCands[c];
    }
  }
  return best;
}

}  // namespace orc
