// CPU oracle (test infrastructure only; see oracle.h): the 8-bit intra
// predictors of the multi-tool encoder and its luma mode search. Restates
// crates/rustmpeg-video/src/vvc/predict.rs of the reference:
//   MrlRefSamples::from_ref_samples     predict.rs:1058-1075
//   gather_references                   predict.rs:1084-1134
//   gather_references_mrl               predict.rs:1141-1231
//   RefSamples::filtered                predict.rs:1233-1267
//   predict_planar / predict_dc         predict.rs:1688-1736
//   apply_pdpc                          predict.rs:1739-1754
//   predict_angular_with_params_bd      predict.rs:1776-1958
//   predict_block / predict_block_full  predict.rs:2619-2699 (predict_block for
//                                       both components, the full form for luma)
//   choose_luma_intra_pred_mode         predict.rs:2737-2801
// and the MRL candidate loop of encode_picture_multitool (slice.rs:2698-2731).
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "../rustmpeg-next_b200/csrc/vvc_tables.h"
#include "oracle.h"

namespace orc {
using namespace vvc_tables;

namespace {

const int PLANAR = 0, DC = 1;

inline int ilog2(int v) { return __builtin_ctz((unsigned)v); }
inline int floor_log2(unsigned v) { return 31 - __builtin_clz(v); }
inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

struct Refs8 {
  std::vector<int> above, left;  // 2w, 2h
  int top_left;
};

struct MrlRefs {
  int mrl_idx;
  std::vector<int> row_above, row_left;
};

// predict.rs:1084-1134 gather_references
Refs8 gather(const Plane8& r, int bx, int by, int w, int h) {
  Refs8 o;
  o.above.assign(2 * w, 0);
  o.left.assign(2 * h, 0);
  const int above_len = by == 0 ? 0 : std::min(r.width - bx, 2 * w);
  const int left_len = bx == 0 ? 0 : std::min(r.height - by, h);
  for (int i = 0; i < above_len; i++) o.above[i] = r.get(bx + i, by - 1);
  for (int i = 0; i < left_len; i++) o.left[i] = r.get(bx - 1, by + i);
  if (above_len > 0 && left_len > 0)
    o.top_left = r.get(bx - 1, by - 1);
  else if (above_len > 0)
    o.top_left = o.above[0];
  else if (left_len > 0)
    o.top_left = o.left[0];
  else
    o.top_left = 128;
  if (above_len == 0)
    std::fill(o.above.begin(), o.above.end(), left_len > 0 ? o.left[0] : 128);
  else
    for (int i = above_len; i < 2 * w; i++) o.above[i] = o.above[above_len - 1];
  if (left_len == 0)
    std::fill(o.left.begin(), o.left.end(), above_len > 0 ? o.above[0] : 128);
  else
    for (int i = left_len; i < 2 * h; i++) o.left[i] = o.left[left_len - 1];
  return o;
}

// predict.rs:1233-1267 RefSamples::filtered
Refs8 filtered(const Refs8& r) {
  Refs8 o = r;
  const int w2 = (int)r.above.size(), h2 = (int)r.left.size();
  o.top_left = (2 * r.top_left + r.above[0] + r.left[0] + 2) >> 2;
  for (int j = 0; j + 1 < w2; j++) {
    int prev = j == 0 ? r.top_left : r.above[j - 1];
    o.above[j] = (prev + 2 * r.above[j] + r.above[j + 1] + 2) >> 2;
  }
  if (w2 > 0) o.above[w2 - 1] = r.above[w2 - 1];
  for (int j = 0; j + 1 < h2; j++) {
    int prev = j == 0 ? r.top_left : r.left[j - 1];
    o.left[j] = (prev + 2 * r.left[j] + r.left[j + 1] + 2) >> 2;
  }
  if (h2 > 0) o.left[h2 - 1] = r.left[h2 - 1];
  return o;
}

// predict.rs:1058-1075 MrlRefSamples::from_ref_samples
MrlRefs from_refs(const Refs8& r) {
  MrlRefs m;
  m.mrl_idx = 0;
  m.row_above.push_back(r.top_left);
  m.row_above.insert(m.row_above.end(), r.above.begin(), r.above.end());
  m.row_above.resize(r.above.size() + 5, m.row_above.back());
  m.row_left.push_back(r.top_left);
  m.row_left.insert(m.row_left.end(), r.left.begin(), r.left.end());
  m.row_left.resize(r.left.size() + 5, m.row_left.back());
  return m;
}

// predict.rs:1141-1231 gather_references_mrl
MrlRefs gather_mrl(const Plane8& r, int bx, int by, int w, int h, int mrl_idx, int ctu_size) {
  const int eff = (ctu_size > 0 && (by & (ctu_size - 1)) == 0) ? 0 : std::min(mrl_idx, 2);
  if (eff == 0) return from_refs(gather(r, bx, by, w, h));
  const int offset = 1 + eff;
  MrlRefs m;
  m.mrl_idx = eff;
  m.row_above.assign(2 * w + offset + 4, 128);
  m.row_left.assign(2 * h + offset + 4, 128);
  const bool has_above = by >= offset, has_left = bx >= offset;
  if (has_above && has_left) {
    const int tl = r.get(bx - offset, by - offset);
    m.row_above[0] = tl;
    m.row_left[0] = tl;
    for (int i = 1; i <= eff; i++) {
      m.row_above[i] = r.get(bx - offset + i, by - offset);
      m.row_left[i] = r.get(bx - offset, by - offset + i);
    }
  }
  const int avail_above = has_above ? std::min(r.width - bx, 2 * w) : 0;
  const int avail_left = has_left ? std::min(r.height - by, h) : 0;
  if (avail_above > 0) {
    for (int x = 0; x < avail_above; x++) m.row_above[offset + x] = r.get(bx + x, by - offset);
    const int last = m.row_above[offset + avail_above - 1];
    for (size_t x = offset + avail_above; x < m.row_above.size(); x++) m.row_above[x] = last;
  }
  if (avail_left > 0) {
    for (int y = 0; y < avail_left; y++) m.row_left[offset + y] = r.get(bx - offset, by + y);
    const int last = m.row_left[offset + avail_left - 1];
    for (size_t y = offset + avail_left; y < m.row_left.size(); y++) m.row_left[y] = last;
  }
  if (!has_above || !has_left) {
    const int pad = avail_above > 0 ? m.row_above[offset] : (avail_left > 0 ? m.row_left[offset] : 128);
    for (int i = 0; i < offset; i++) {
      m.row_above[i] = pad;
      m.row_left[i] = pad;
    }
    if (avail_above == 0) std::fill(m.row_above.begin(), m.row_above.end(), pad);
    if (avail_left == 0) std::fill(m.row_left.begin(), m.row_left.end(), pad);
  }
  return m;
}

// predict.rs:1688-1719 predict_planar
std::vector<int> planar(const Refs8& r, int w, int h) {
  const int lw = ilog2(w), lh = ilog2(h);
  const int offset = 1 << (lw + lh), shift = 1 + lw + lh;
  std::vector<int> top(r.above.begin(), r.above.begin() + w + 1), left(r.left.begin(), r.left.begin() + h + 1);
  const int tr = top[w], bl = left[h];
  std::vector<int> bottom(w), right(h);
  for (int k = 0; k < w; k++) bottom[k] = bl - top[k];
  for (int k = 0; k < h; k++) right[k] = tr - left[k];
  for (auto& v : top) v <<= lh;
  for (auto& v : left) v <<= lw;
  std::vector<int> p(w * h);
  for (int y = 0; y < h; y++) {
    int hor = left[y];
    for (int x = 0; x < w; x++) {
      hor += right[y];
      top[x] += bottom[x];
      p[y * w + x] = ((hor << lh) + (top[x] << lw) + offset) >> shift;
    }
  }
  return p;
}

// predict.rs:1722-1736 predict_dc
std::vector<int> dc(const Refs8& r, int w, int h) {
  const int denom = w == h ? (w << 1) : std::max(w, h);
  int sum = 0;
  if (w >= h)
    for (int i = 0; i < w; i++) sum += r.above[i];
  if (w <= h)
    for (int i = 0; i < h; i++) sum += r.left[i];
  return std::vector<int>(w * h, (sum + (denom >> 1)) >> ilog2(denom));
}

// predict.rs:1739-1754 apply_pdpc
void pdpc(std::vector<int>& p, const Refs8& r, int w, int h) {
  const int scale = std::max(ilog2(w) + ilog2(h) - 2, 0) >> 2;
  for (int y = 0; y < h; y++) {
    const int wt = 32 >> std::min((y * 2) >> scale, 31);
    for (int x = 0; x < w; x++) {
      const int wl = 32 >> std::min((x * 2) >> scale, 31);
      const int v = p[y * w + x];
      p[y * w + x] = v + ((wl * (r.left[y] - v) + wt * (r.above[x] - v) + 32) >> 6);
    }
  }
}

// predict.rs:1776-1958 predict_angular_with_params_bd
std::vector<int> angular(const MrlRefs& m, int w, int h, bool is_luma, const AngularParams& P, int bit_depth) {
  const int bd = clampi(bit_depth, 8, 12);
  const int maxv = (1 << bd) - 1, def = 1 << (bd - 1);
  const bool ver = P.is_mode_ver;
  const int mri = is_luma ? m.mrl_idx : 0;
  const int angle = P.intra_pred_angle, inv = P.abs_inv_angle;
  const int base = std::max(h, w) + 4;
  const int len = base + 2 * std::max(w, h) + 2 * std::max(P.ref_w, P.ref_h) + 64;
  std::vector<int> ra(len, def), rl(len, def);
  const int na = (int)m.row_above.size(), nl = (int)m.row_left.size();
  if (angle < 0) {
    for (int x = 0; x <= w + 1 + mri; x++) ra[base + x] = m.row_above[std::min(x, na - 1)];
    for (int y = 0; y <= h + 1 + mri; y++) rl[base + y] = m.row_left[std::min(y, nl - 1)];
    const int side = ver ? h : w;
    for (int k = -side; k <= -1; k++) {
      const int proj = std::min((-k * inv + 256) >> 9, side);
      if (ver)
        ra[base + k] = rl[base + proj];
      else
        rl[base + k] = ra[base + proj];
    }
  } else {
    for (int x = 0; x <= P.ref_w + mri; x++) ra[base + x] = m.row_above[std::min(x, na - 1)];
    for (int y = 0; y <= P.ref_h + mri; y++) rl[base + y] = m.row_left[std::min(y, nl - 1)];
    const int log2_ratio = floor_log2(w) - floor_log2(h);
    const int s = std::max(0, ver ? log2_ratio : -log2_ratio);
    const int max_index = (mri << s) + 2;
    const int ref_length = ver ? P.ref_w : P.ref_h;
    std::vector<int>& r = ver ? ra : rl;
    const int v = r[base + ref_length + mri];
    for (int z = 1; z <= max_index; z++) r[base + ref_length + mri + z] = v;
  }
  const int mb = base + mri, sb = base + mri;
  const std::vector<int>& rm = ver ? ra : rl;
  const std::vector<int>& rs = ver ? rl : ra;
  const int ww = ver ? w : h, wh = ver ? h : w;
  std::vector<int> t(ww * wh);
  if (angle == 0) {
    const int scale = (floor_log2(ww) + floor_log2(wh) - 2) >> 2;
    const int tl = rm[mb];
    for (int y = 0; y < wh; y++) {
      for (int x = 0; x < ww; x++) t[y * ww + x] = rm[mb + x + 1];
      if (P.apply_pdpc && scale >= 0) {
        const int left = rs[sb + 1 + y];
        const int limit = std::min(3 << scale, ww);
        for (int x = 0; x < limit; x++) {
          const int wl = 32 >> ((2 * x) >> scale);
          t[y * ww + x] = clampi(t[y * ww + x] + ((wl * (left - tl) + 32) >> 6), 0, maxv);
        }
      }
    }
  } else {
    const bool int_slope = (std::abs(angle) & 0x1F) == 0;
    int delta_pos = angle * (1 + mri);
    for (int y = 0; y < wh; y++) {
      const int di = delta_pos >> 5, df = delta_pos & 31;
      if (!int_slope) {
        if (is_luma) {
          int g[4] = {16 - (df >> 1), 32 - (df >> 1), 16 + (df >> 1), df >> 1};
          const int* f = g;
          int c[4];
          if (!P.interpolation_flag) {
            for (int i = 0; i < 4; i++) c[i] = kChromaTaps4[df * 4 + i];
            f = c;
          }
          for (int x = 0; x < ww; x++) {
            const int b = mb + di + x;
            const int v = (f[0] * rm[b] + f[1] * rm[b + 1] + f[2] * rm[b + 2] + f[3] * rm[b + 3] + 32) >> 6;
            t[y * ww + x] = clampi(v, 0, maxv);
          }
        } else {
          for (int x = 0; x < ww; x++) {
            const int b = mb + di + x + 1;
            t[y * ww + x] = rm[b] + ((df * (rm[b + 1] - rm[b]) + 16) >> 5);
          }
        }
      } else {
        for (int x = 0; x < ww; x++) t[y * ww + x] = rm[mb + di + x + 1];
      }
      if (P.apply_pdpc) {
        const int scale = std::max(P.angular_scale, 0);
        int sum = 256;
        const int limit = std::min(3 << scale, ww);
        for (int x = 0; x < limit; x++) {
          sum += inv;
          const int wl = 32 >> ((2 * x) >> scale);
          const int li = std::min(sb + y + (sum >> 9) + 1, len - 1);
          const int v = t[y * ww + x];
          t[y * ww + x] = clampi(v + ((wl * (rs[li] - v) + 32) >> 6), 0, maxv);
        }
      }
      delta_pos += angle;
    }
  }
  if (ver) return t;
  std::vector<int> d(w * h);
  for (int y = 0; y < wh; y++)
    for (int x = 0; x < ww; x++) d[x * w + y] = t[y * ww + x];
  return d;
}

// predict.rs:2655-2699 predict_block_full for luma Planar / DC / angular
// (Planar / DC through predict_block, :2619-2650)
std::vector<int> predict_full(const Plane8& r, int bx, int by, int w, int h, int mode, int mrl, int ctu) {
  if (mode == PLANAR || mode == DC) {
    Refs8 refs = gather(r, bx, by, w, h);
    const Refs8 used = (mode == PLANAR && w * h > 32) ? filtered(refs) : refs;  // uses_reference_filter
    std::vector<int> p = mode == PLANAR ? planar(used, w, h) : dc(used, w, h);
    pdpc(p, used, w, h);
    return p;
  }
  if (mrl == 0) {  // predict_angular_bd (:1970-1987)
    AngularParams P = init_angular_params(mode, w, h, w, h, true, 0, false);
    Refs8 refs = gather(r, bx, by, w, h);
    return angular(from_refs(P.ref_filter_flag ? filtered(refs) : refs), w, h, true, P, 8);
  }
  MrlRefs m = gather_mrl(r, bx, by, w, h, mrl, ctu);
  AngularParams P = init_angular_params(mode, w, h, w, h, true, m.mrl_idx, false);
  return angular(m, w, h, true, P, 8);
}

// predict.rs:2619-2650 predict_block for either component: Planar / DC with
// the [1 2 1] filter on luma only (uses_reference_filter, :1287-1293) and
// PDPC, angular through predict_angular (:1962-1987) with is_luma selecting
// the interpolation and reference-filter rules.
std::vector<int> predict_block8(const Plane8& r, int bx, int by, int w, int h, bool is_luma, int mode) {
  Refs8 refs = gather(r, bx, by, w, h);
  if (mode == PLANAR || mode == DC) {
    const Refs8 used = (mode == PLANAR && is_luma && w * h > 32) ? filtered(refs) : refs;
    std::vector<int> p = mode == PLANAR ? planar(used, w, h) : dc(used, w, h);
    pdpc(p, used, w, h);
    return p;
  }
  AngularParams P = init_angular_params(mode, w, h, w, h, is_luma, 0, false);
  return angular(from_refs(P.ref_filter_flag ? filtered(refs) : refs), w, h, is_luma, P, 8);
}

uint64_t sad_of(const std::vector<int>& p, const Plane8& src, int bx, int by, int w, int h) {
  uint64_t s = 0;
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) s += (uint64_t)std::abs((int)src.get(bx + x, by + y) - p[y * w + x]);
  return s;
}

// ---- the general decoder (decode_general.rs) ----

struct Gen {
  const vvcg_gen_intra_state& S;
  int plane_w(int c) const { return c ? (int)S.width / 2 : (int)S.width; }
  int plane_h(int c) const { return c ? (int)S.height / 2 : (int)S.height; }
  int get(int c, int x, int y) const { return S.plane[c][(size_t)y * S.stride[c] + x]; }
  int dcv() const { return 1 << (clampi(S.bit_depth, 8, 12) - 1); }
  // Gen::decoded_at (decode_general.rs:4239-4251)
  bool decoded_at(bool luma, int x, int y) const {
    if (x < 0 || y < 0) return false;
    if (luma) {
      if (x >= (int)S.width || y >= (int)S.height) return false;
      return S.dec_y[(size_t)(y / 4) * (S.width / 4) + x / 4] != 0;
    }
    if (x >= (int)S.width / 2 || y >= (int)S.height / 2) return false;
    return S.dec_c[(size_t)y * (S.width / 2) + x] != 0;
  }
  // Gen::gather_len (decode_general.rs:4260-4341) on component c
  Refs8 gather_len(int c, bool luma, int x, int y, int top_len, int left_len) const {
    const int pw = plane_w(c), ph = plane_h(c), d = dcv();
    std::vector<char> aa(top_len, 0), la(left_len, 0);
    bool any = false;
    if (y > 0)
      for (int k = 0; k < top_len; k++)
        if (x + k < pw && decoded_at(luma, x + k, y - 1)) aa[k] = any = true;
    if (x > 0)
      for (int k = 0; k < left_len; k++)
        if (y + k < ph && decoded_at(luma, x - 1, y + k)) la[k] = any = true;
    const bool tl = x > 0 && y > 0 && decoded_at(luma, x - 1, y - 1);
    if (tl) any = true;
    int ft = -1, fl = -1;
    for (int k = 0; k < top_len && ft < 0; k++)
      if (aa[k]) ft = get(c, x + k, y - 1);
    for (int k = 0; k < left_len && fl < 0; k++)
      if (la[k]) fl = get(c, x - 1, y + k);
    Refs8 r;
    r.above.assign(top_len, d);
    r.left.assign(left_len, d);
    int prev = -1;
    for (int k = 0; k < top_len; k++) {
      if (aa[k]) {
        r.above[k] = prev = get(c, x + k, y - 1);
      } else {
        r.above[k] = prev >= 0 ? prev : ft >= 0 ? ft : fl >= 0 ? fl : d;
      }
    }
    prev = -1;
    for (int k = 0; k < left_len; k++) {
      if (la[k]) {
        r.left[k] = prev = get(c, x - 1, y + k);
      } else {
        r.left[k] = prev >= 0 ? prev : fl >= 0 ? fl : ft >= 0 ? ft : d;
      }
    }
    r.top_left = tl ? get(c, x - 1, y - 1) : (ft >= 0 ? ft : fl >= 0 ? fl : d);
    if (!any) {
      std::fill(r.above.begin(), r.above.end(), d);
      std::fill(r.left.begin(), r.left.end(), d);
    }
    return r;
  }
  // Gen::gather_mrl (decode_general.rs:4542-4632)
  MrlRefs gather_mrl(int x, int y, int w, int h, int mrl) const {
    const int d = dcv(), off = 1 + mrl, al = 2 * w, ll = 2 * h;
    MrlRefs m;
    m.mrl_idx = mrl;
    m.row_above.assign(al + off + 4, d);
    m.row_left.assign(ll + off + 4, d);
    const bool tl = x >= off && y >= off && decoded_at(true, x - off, y - off);
    if (tl) {
      m.row_above[0] = m.row_left[0] = get(0, x - off, y - off);
      for (int i = 1; i < off; i++) {
        m.row_above[i] = get(0, x - off + i, y - off);
        m.row_left[i] = get(0, x - off, y - off + i);
      }
    }
    std::vector<char> ta(al, 0), la(ll, 0);
    if (y >= off)
      for (int k = 0; k < al; k++)
        if (x + k < (int)S.width && decoded_at(true, x + k, y - off)) ta[k] = 1;
    if (x >= off)
      for (int k = 0; k < ll; k++)
        if (y + k < (int)S.height && decoded_at(true, x - off, y + k)) la[k] = 1;
    int ft = -1, fl = -1;
    for (int k = 0; k < al && ft < 0; k++)
      if (ta[k]) ft = get(0, x + k, y - off);
    for (int k = 0; k < ll && fl < 0; k++)
      if (la[k]) fl = get(0, x - off, y + k);
    int prev = -1;
    for (int k = 0; k < al; k++) {
      if (ta[k])
        m.row_above[off + k] = prev = get(0, x + k, y - off);
      else
        m.row_above[off + k] = prev >= 0 ? prev : ft >= 0 ? ft : fl >= 0 ? fl : d;
    }
    for (size_t k = off + al; k < m.row_above.size(); k++) m.row_above[k] = m.row_above[off + al - 1];
    prev = -1;
    for (int k = 0; k < ll; k++) {
      if (la[k])
        m.row_left[off + k] = prev = get(0, x - off, y + k);
      else
        m.row_left[off + k] = prev >= 0 ? prev : fl >= 0 ? fl : ft >= 0 ? ft : d;
    }
    for (size_t k = off + ll; k < m.row_left.size(); k++) m.row_left[k] = m.row_left[off + ll - 1];
    if (!tl) {
      const int fb = ft >= 0 ? ft : fl >= 0 ? fl : d;
      for (int i = 0; i < off; i++) m.row_above[i] = m.row_left[i] = fb;
    }
    return m;
  }
  // Gen::cclm_predict (decode_general.rs:4372-4537); mode 0 LM, 1 LM-L, 2 LM-T
  std::vector<int> cclm(int comp, int mode, int xc, int yc, int w, int h) const {
    const int mid = dcv(), maxv = (1 << clampi(S.bit_depth, 8, 12)) - 1;
    const int xtb = xc * 2, ytb = yc * 2;
    const bool al = xc > 0 && decoded_at(false, xc - 1, yc);
    const bool at = yc > 0 && decoded_at(false, xc, yc - 1);
    const bool ctb = S.ctu_size > 0 && (ytb & (S.ctu_size - 1)) == 0;
    const bool vc = S.vert_collocated != 0;
    auto py = [&](int x, int y) {
      if (y < 0 && !at) y = 0;
      if (x < 0 && !al) x = 0;
      return get(0, xtb + x, ytb + y);
    };
    int ntr = 0, nlb = 0;
    if (mode == 2 && at)
      for (int x = w; x < 2 * w && decoded_at(false, xc + x, yc - 1); x++) ntr++;
    if (mode == 1 && al)
      for (int y = h; y < 2 * h && decoded_at(false, xc - 1, yc + y); y++) nlb++;
    int nt, nl;
    if (mode == 0) {
      nt = at ? w : 0;
      nl = al ? h : 0;
    } else if (mode == 2) {
      nt = at ? w + std::min(ntr, h) : 0;
      nl = 0;
    } else {
      nt = 0;
      nl = al ? h + std::min(nlb, w) : 0;
    }
    const int is4n = !(at && al && mode == 0);
    int sl[4] = {mid, mid, mid, mid}, sc[4] = {mid, mid, mid, mid};
    int count = 0;
    auto top_ds = [&](int x) {
      const int lx = 2 * x;
      if (ctb) return (py(lx - 1, -1) + 2 * py(lx, -1) + py(lx + 1, -1) + 2) >> 2;
      if (vc) return (py(lx, -3) + py(lx - 1, -2) + 4 * py(lx, -2) + py(lx + 1, -2) + py(lx, -1) + 4) >> 3;
      return (py(lx - 1, -1) + py(lx - 1, -2) + 2 * py(lx, -1) + 2 * py(lx, -2) + py(lx + 1, -1) + py(lx + 1, -2) +
              4) >> 3;
    };
    auto left_ds = [&](int y) {
      const int ly = 2 * y;
      if (vc) return (py(-2, ly - 1) + py(-3, ly) + 4 * py(-2, ly) + py(-1, ly) + py(-2, ly + 1) + 4) >> 3;
      return (py(-3, ly) + py(-3, ly + 1) + 2 * py(-2, ly) + 2 * py(-2, ly + 1) + py(-1, ly) + py(-1, ly + 1) +
              4) >> 3;
    };
    if (nt > 0) {
      const int start = nt >> (2 + is4n), step = std::max(1, nt >> (1 + is4n)), cnt = std::min(nt, (1 + is4n) << 1);
      for (int pos = 0; pos < cnt; pos++) {
        const int x = start + pos * step;
        if (x >= nt) break;
        sl[count] = top_ds(x);
        sc[count] = get(comp, xc + x, yc - 1);
        count++;
      }
    }
    if (nl > 0) {
      const int start = nl >> (2 + is4n), step = std::max(1, nl >> (1 + is4n)), cnt = std::min(nl, (1 + is4n) << 1);
      for (int pos = 0; pos < cnt; pos++) {
        const int y = start + pos * step;
        if (y >= nl) break;
        sl[count] = left_ds(y);
        sc[count] = get(comp, xc - 1, yc + y);
        count++;
      }
    }
    if (count == 0) return std::vector<int>(w * h, mid);
    int a, b, shift;
    cclm_params(sl, sc, count, S.bit_depth, &a, &b, &shift);
    std::vector<int> out(w * h);
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++) {
        const int lx = 2 * x, ly = 2 * y;
        const int ds = vc ? (py(lx, ly - 1) + py(lx - 1, ly) + 4 * py(lx, ly) + py(lx + 1, ly) + py(lx, ly + 1) + 4) >> 3
                          : (py(lx - 1, ly) + py(lx - 1, ly + 1) + 2 * py(lx, ly) + 2 * py(lx, ly + 1) +
                             py(lx + 1, ly) + py(lx + 1, ly + 1) + 4) >> 3;
        out[y * w + x] = clampi(((ds * a) >> shift) + b, 0, maxv);
      }
    return out;
  }
  // predict_luma (decode_general.rs:4650-4732) for an intra CU
  std::vector<int> luma(const vvcg_gen_intra_req& r, int x, int y, int w, int h) const {
    const int mode = r.mode;
    if (r.bdpcm) {  // predict_bdpcm (predict.rs:1993-2010) on gather_avail
      Refs8 refs = gather_len(0, true, x, y, 2 * w, 2 * h);
      std::vector<int> p(w * h);
      for (int yy = 0; yy < h; yy++)
        for (int xx = 0; xx < w; xx++) p[yy * w + xx] = r.bdpcm == VVCG_BDPCM_VER ? refs.above[xx] : refs.left[yy];
      return p;
    }
    const bool isp = r.isp != VVCG_ISP_NONE;
    const int mrl = std::min<int>(r.mrl, 2);
    MrlRefs m = isp ? from_refs(gather_len(0, true, x, y, r.cu_w + w, r.cu_h + h))
                    : mrl == 0 ? from_refs(gather_len(0, true, x, y, 2 * w, 2 * h)) : gather_mrl(x, y, w, h, mrl);
    const int off = m.mrl_idx;
    Refs8 base;
    base.above.assign(m.row_above.begin() + off + 1, m.row_above.begin() + off + 1 + 2 * w);
    base.left.assign(m.row_left.begin() + off + 1, m.row_left.begin() + off + 1 + 2 * h);
    base.top_left = m.row_above[off];
    if (mode == PLANAR || mode == DC) {
      const Refs8 used = (mode == PLANAR && mrl == 0 && !isp && w * h > 32) ? filtered(base) : base;
      std::vector<int> p = mode == PLANAR ? planar(used, w, h) : dc(used, w, h);
      if (mrl == 0 && w >= 4 && h >= 4) pdpc(p, used, w, h);
      return p;
    }
    const int dir = std::min(mode, 66);
    AngularParams P = init_angular_params(dir, w, h, r.cu_w, r.cu_h, true, mrl, isp);
    if (mrl == 0 && !isp)
      return angular(from_refs(P.ref_filter_flag ? filtered(base) : base), w, h, true, P, S.bit_depth);
    return angular(m, w, h, true, P, S.bit_depth);
  }
  // predict_chroma (decode_general.rs:4734-4793) for an intra CU
  std::vector<int> chroma(const vvcg_gen_intra_req& r) const {
    const int c = r.comp, x = r.x, y = r.y, w = r.w, h = r.h, mode = r.mode;
    if (mode >= 81 && mode <= 83) return cclm(c, mode == 81 ? 0 : mode == 82 ? 1 : 2, x, y, w, h);
    Refs8 refs = gather_len(c, false, x, y, 2 * w, 2 * h);
    if (mode == PLANAR || mode == DC) {
      std::vector<int> p = mode == PLANAR ? planar(refs, w, h) : dc(refs, w, h);
      if (w >= 4 && h >= 4) pdpc(p, refs, w, h);
      return p;
    }
    AngularParams P = init_angular_params(std::min(mode, 66), w, h, w, h, false, 0, false);  // predict_angular_bd
    return angular(from_refs(refs), w, h, false, P, S.bit_depth);
  }
};

}  // namespace

// reconstruct_tu's prediction (decode_general.rs:3983-4024): the block's
// prediction into out (w * h); a narrow vertical ISP sub-partition takes its
// columns of the 4-wide region it shares.
void gen_intra_predict(const vvcg_gen_intra_state& st, const vvcg_gen_intra_req& r, int16_t* out) {
  Gen g{st};
  std::vector<int> p;
  if (r.comp == 0) {
    if (r.isp == VVCG_ISP_VER && (r.cu_w == 4 || (r.cu_w == 8 && r.cu_h > 4))) {
      const int rx = r.cu_x + ((r.x - r.cu_x) / 4) * 4;
      std::vector<int> full = g.luma(r, rx, r.y, 4, r.h);
      p.resize(r.w * r.h);
      for (int yy = 0; yy < r.h; yy++)
        for (int xx = 0; xx < r.w; xx++) p[yy * r.w + xx] = full[yy * 4 + (r.x - rx) + xx];
    } else {
      p = g.luma(r, r.x, r.y, r.w, r.h);
    }
  } else {
    p = g.chroma(r);
  }
  for (int i = 0; i < r.w * r.h; i++) out[i] = (int16_t)p[i];
}

// predict.rs:2737-2801 choose_luma_intra_pred_mode (Planar wins ties: the
// first candidate with the lowest SAD), then, with mrl, the MRL loop of
// encode_picture_multitool (slice.rs:2698-2731): lines 1 and 2 for
// mpm[1..5], each taken only when its SAD is strictly lower.
void luma_intra_search_8(const Plane8& recon, const Plane8& src, int bx, int by, int w, int h, const uint8_t mpm[6],
                         bool mpm_only, bool mrl, int ctu_size, int* best_mode, int* best_mrl, uint64_t* best_sad) {
  Refs8 refs = gather(recon, bx, by, w, h);
  Refs8 refs_f = filtered(refs);
  int bm = PLANAR;
  uint64_t bc = UINT64_MAX;
  const int n = mpm_only ? 6 : 67;
  for (int i = 0; i < n; i++) {
    const int mode = mpm_only ? mpm[i] : i;
    std::vector<int> p;
    if (mode == PLANAR) {
      const Refs8& u = w * h > 32 ? refs_f : refs;
      p = planar(u, w, h);
      pdpc(p, u, w, h);
    } else if (mode == DC) {
      p = dc(refs, w, h);
      pdpc(p, refs, w, h);
    } else {
      AngularParams P = init_angular_params(mode, w, h, w, h, true, 0, false);
      p = angular(from_refs(P.ref_filter_flag ? refs_f : refs), w, h, true, P, 8);
    }
    const uint64_t s = sad_of(p, src, bx, by, w, h);
    if (s < bc) {
      bc = s;
      bm = mode;
    }
  }
  int bmrl = 0;
  if (mrl) {
    for (int cand = 1; cand <= 2; cand++)
      for (int k = 1; k < 6; k++) {
        const uint64_t s = sad_of(predict_full(recon, bx, by, w, h, mpm[k], cand, ctu_size), src, bx, by, w, h);
        if (s < bc) {
          bc = s;
          bm = mpm[k];
          bmrl = cand;
        }
      }
  }
  *best_mode = bm;
  *best_mrl = bmrl;
  *best_sad = bc;
}

// predict_block (predict.rs:2619) of one component block into out (w * h).
void predict_block_8(const Plane8& recon, int bx, int by, int w, int h, bool is_luma, int mode, int32_t* out) {
  std::vector<int> p = predict_block8(recon, bx, by, w, h, is_luma, mode);
  std::copy(p.begin(), p.end(), out);
}

// predict_block_full (predict.rs:2655) of one luma mode into out (w * h).
void predict_luma_8(const Plane8& recon, int bx, int by, int w, int h, int mode, int mrl, int ctu_size, int32_t* out) {
  std::vector<int> p = predict_full(recon, bx, by, w, h, mode, mrl, ctu_size);
  std::copy(p.begin(), p.end(), out);
}

}  // namespace orc
