// Host-side CABAC parsing (ITU-T H.266 clause 9.3) of the library: the
// arithmetic decoder, residual_coding and residual_ts_coding, and the slice
// data of the strict 8-bit intra profile, emitting the frame path's CU
// records (per-TB transform tools) and levels, dense or sparse. Restates the
// reference's decoder side: cabac.rs (CtxModel :41-99, CtxStore :267-296,
// BinDecoder :761-1006), residual.rs (:85-240 context selection,
// :359-433 decode_last_sig_coeff, :534-881 decode_residual_with_options and
// decode_subblock), transform.rs:43-200 (CoeffScan), slice.rs
// (:458-627 decode_picture, :1003-1048 lfnst / mts idx, :1117-1130 and
// :1691-1717 intra mode, :1132-1191 and :1323-1435 residual_ts_coding,
// :920-992 the syntax-presence rules) and predict.rs:1455-1543 (MPM list).
//
// Everything here is plain C++ on the CPU: one picture's substream is
// parsed by one thread, pictures in parallel (vvcg_parse_strict).
#pragma once
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/vvcg.h"
#include "vvc_cabac.h"

namespace vvcg_parse {
using namespace vvc_cabac;

// ---------------------------------------------------------------- models --
// Two-rate probability estimate of one context (cabac.rs:41-99): two 15-bit
// states kept in 16 bits with their low bits masked, adapted at two rates.
struct Model {
  uint16_t s0, s1;
  uint8_t r0, r1;
  int state() const { return (s0 + s1) >> 8; }
  bool mps() const { return state() >= 128; }
  uint32_t lps(uint32_t range) const {
    int q = state();
    if (q & 0x80) q ^= 0xFF;
    return ((((uint32_t)q >> 2) * (range >> 5)) >> 1) + 4;
  }
  void adapt(bool bin) {
    constexpr uint32_t m0 = 0x7FE0, m1 = 0x7FFE;
    uint32_t a = s0 - ((s0 >> r0) & m0), b = s1 - ((s1 >> r1) & m1);
    if (bin) {
      a += (0x7FFFu >> r0) & m0;
      b += (0x7FFFu >> r1) & m1;
    }
    s0 = (uint16_t)a;
    s1 = (uint16_t)b;
  }
};

inline Model model_init(int qp, int init_id, int log2_window) {
  const int slope = (init_id >> 3) - 4, offset = (init_id & 7) * 18 + 1;
  const int st = std::min(127, std::max(1, ((slope * (qp - 16)) >> 1) + offset));
  const uint32_t p = (uint32_t)st << 8;
  Model m;
  m.s0 = (uint16_t)(p & 0x7FE0);
  m.s1 = (uint16_t)(p & 0x7FFE);
  m.r0 = (uint8_t)(2 + ((log2_window >> 2) & 3));
  m.r1 = (uint8_t)(3 + m.r0 + (log2_window & 3));
  return m;
}

struct Models {
  Model m[kNumContexts];
  // cabac.rs:276-308: one of the I / P / B initialisation tables at qp
  void init(int qp, const uint8_t (*table)[2]) {
    qp = std::min(63, std::max(0, qp));
    for (int i = 0; i < kNumContexts; i++) m[i] = model_init(qp, table[i][0], table[i][1]);
  }
  void init_i_slice(int qp) { init(qp, kCtxInitI); }
  Model& operator[](int i) { return m[i]; }
};

// ---------------------------------------------------- arithmetic decoder --
struct Reader {
  const uint8_t* data = nullptr;
  size_t size = 0, pos = 0;
  uint32_t range = 510, value = 0;
  int bits_needed = -8;
  uint8_t last = 0;

  void start(const uint8_t* d, size_t n) {
    data = d;
    size = n;
    const uint8_t b0 = n > 0 ? d[0] : 0, b1 = n > 1 ? d[1] : 0;
    pos = std::min<size_t>(n, 2);
    range = 510;
    value = ((uint32_t)b0 << 8) + b1;
    bits_needed = -8;
    last = b1;
  }
  uint32_t next_byte() {  // zero past the end of the substream
    if (pos >= size) return 0;
    last = data[pos++];
    return last;
  }
  bool bin(Model& c) {
    const bool mps = c.mps();
    const uint32_t l = c.lps(range);
    range -= l;
    const uint32_t scaled = range << 7;
    bool b;
    if (value < scaled) {
      b = mps;
      if (range < 256) {
        range <<= 1;
        value <<= 1;
        if (++bits_needed >= 0) {
          value += next_byte() << bits_needed;
          bits_needed -= 8;
        }
      }
    } else {
      b = !mps;
      const int nb = kRenormLps[l >> 3];
      value = (value - scaled) << nb;
      range = l << nb;
      bits_needed += nb;
      if (bits_needed >= 0) {
        value += next_byte() << bits_needed;
        bits_needed -= 8;
      }
    }
    c.adapt(b);
    return b;
  }
  bool bypass() {
    value <<= 1;
    if (++bits_needed >= 0) {
      value += next_byte();
      bits_needed = -8;
    }
    const uint32_t scaled = range << 7;
    if (value >= scaled) {
      value -= scaled;
      return true;
    }
    return false;
  }
  uint32_t bypass_bins(uint32_t n) {
    uint32_t v = 0;
    for (uint32_t i = 0; i < n; i++) v = (v << 1) | (bypass() ? 1u : 0u);
    return v;
  }
  // truncated binary code of a symbol below n (the shorter codes for the
  // first 2^(k+1) - n symbols)
  uint32_t trunc_bin(uint32_t n) {
    if (n <= 1) return 0;
    const uint32_t k = 31 - __builtin_clz(n), u = (1u << k) - (n - (1u << k));
    uint32_t s = bypass_bins(k);
    if (s >= u) s = 2 * s - u + (bypass() ? 1 : 0);
    return s;
  }
  uint32_t unary_max(uint32_t max) {
    uint32_t s = 0;
    while (s < max && bypass()) s++;
    return s;
  }
  bool terminate() {
    range -= 2;
    const uint32_t scaled = range << 7;
    if (value >= scaled) return true;
    if (range < 256) {
      range <<= 1;
      value <<= 1;
      if (++bits_needed == 0) {
        value += next_byte();
        bits_needed = -8;
      }
    }
    return false;
  }
  // the stop bit and byte alignment after the terminating bin
  bool aligned_end() const {
    const int shift = 8 + bits_needed;
    return !(shift >= 0 && (((uint32_t)last << shift) & 0xFF) != 0x80);
  }
  // Rice / exp-Golomb remainder (abs_remainder, dec_abs_level)
  uint32_t rem_abs(uint32_t k, uint32_t cutoff, uint32_t max_log2) {
    const uint32_t max_prefix = 32 - max_log2;
    uint32_t prefix = 0, bit;
    do {
      prefix++;
      bit = bypass() ? 1 : 0;
    } while (bit && prefix < max_prefix);
    prefix -= 1 - bit;
    uint32_t len = k, offset;
    if (prefix < cutoff) {
      offset = prefix << k;
    } else {
      offset = ((1u << (prefix - cutoff)) + cutoff - 1) << k;
      len += prefix == max_prefix ? max_log2 - k : prefix - cutoff;
    }
    return offset + bypass_bins(len);
  }
};

// ------------------------------------------------------ coefficient scan --
// Grouped up-right diagonal scan of a w x h block: coefficient groups (of
// the sizes below, by log2 w and log2 h) in diagonal order, positions in each
// group in diagonal order; only the top-left min(w, 32) x min(h, 32) region.
struct Scan {
  int w = 0, h = 0, log2_cg = 0, wg = 0, hg = 0, n = 0;
  std::vector<uint16_t> raster;   // scan position -> raster index
  std::vector<uint8_t> px, py;    // scan position -> x, y
  std::vector<uint16_t> cg;       // coefficient group (subset) -> raster index in the group grid
};

inline void diag_order(int w, int h, std::vector<std::pair<int, int>>& out) {
  out.clear();
  int line = 0, col = 0;
  for (int i = 0; i < w * h; i++) {
    out.emplace_back(col, line);
    if (col == w - 1 || line == 0) {
      line += col + 1;
      col = 0;
      if (line >= h) {
        col += line - (h - 1);
        line = h - 1;
      }
    } else {
      col++;
      line--;
    }
  }
}

inline Scan make_scan(int w, int h) {
  static const uint8_t kCgLog2[8][8][2] = {
      {{0, 0}, {0, 1}, {0, 2}, {0, 3}, {0, 4}, {0, 4}, {0, 4}, {0, 4}},
      {{1, 0}, {1, 1}, {1, 1}, {1, 3}, {1, 3}, {1, 3}, {1, 3}, {1, 3}},
      {{2, 0}, {1, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{3, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}}};
  Scan s;
  s.w = w;
  s.h = h;
  const int lx = std::min(7, __builtin_ctz((unsigned)w)), ly = std::min(7, __builtin_ctz((unsigned)h));
  const int cgw = 1 << kCgLog2[lx][ly][0], cgh = 1 << kCgLog2[lx][ly][1];
  s.log2_cg = kCgLog2[lx][ly][0] + kCgLog2[lx][ly][1];
  const int cw = std::min(w, 32), ch = std::min(h, 32);
  s.wg = cw / cgw;
  s.hg = ch / cgh;
  s.n = cw * ch;
  std::vector<std::pair<int, int>> groups, inner;
  diag_order(s.wg, s.hg, groups);
  diag_order(cgw, cgh, inner);
  for (auto& g : groups) {
    s.cg.push_back((uint16_t)(g.second * s.wg + g.first));
    for (auto& p : inner) {
      const int x = g.first * cgw + p.first, y = g.second * cgh + p.second;
      s.raster.push_back((uint16_t)(y * w + x));
      s.px.push_back((uint8_t)x);
      s.py.push_back((uint8_t)y);
    }
  }
  return s;
}

// ------------------------------------------------------- residual_coding --
enum ParseError { kOk = 0, kBadLast = 1, kBadRange = 2, kBadSyntax = 3, kTruncated = 4, kBadEnd = 5, kIntraInP = 6 };

struct Template {  // the last significance context's neighbourhood
  int diag = -1, sum1 = 0;
};

// Context of sig_coeff_flag from the 5-position neighbourhood (right, two
// right, below-right, below, two below) of the absolute levels decoded so
// far (residual.rs:142-188); records the neighbourhood for the level flags.
inline int sig_context(const Scan& s, const int32_t* c, int sp, bool luma, int state, Template& t) {
  const int x = s.px[sp], y = s.py[sp], w = s.w, h = s.h, at = y * w + x;
  int sum = 0, nz = 0;
  auto add = [&](int i) {
    const int a = std::abs(c[i]);
    sum += std::min(4 + (a & 1), a);
    nz += a != 0;
  };
  if (x + 1 < w) {
    add(at + 1);
    if (x + 2 < w) add(at + 2);
    if (y + 1 < h) add(at + w + 1);
  }
  if (y + 1 < h) {
    add(at + w);
    if (y + 2 < h) add(at + 2 * w);
  }
  const int d = x + y;
  int ofs = std::min((sum + 1) >> 1, 3) + (d < 2 ? 4 : 0);
  if (luma) ofs += d < 5 ? 4 : 0;
  t.diag = d;
  t.sum1 = sum - nz;
  const int set = std::min(2, std::max(0, state - 1));
  static const int kLuma[3] = {kCtxSigFlagLuma, kCtxSigFlagLuma1, kCtxSigFlagLuma2};
  static const int kChroma[3] = {kCtxSigFlagChroma, kCtxSigFlagChroma1, kCtxSigFlagChroma2};
  return (luma ? kLuma[set] : kChroma[set]) + ofs;
}

// Offset of the gt1 / parity / gt3 contexts (residual.rs:190-208).
inline int level_offset(const Template& t, bool luma) {
  if (t.diag < 0) return 0;
  int o = std::min(t.sum1, 4) + 1;
  if (t.diag == 0)
    o += luma ? 15 : 5;
  else if (luma)
    o += t.diag < 3 ? 10 : (t.diag < 10 ? 5 : 0);
  return o;
}

// Rice parameter from the absolute levels of the neighbourhood (residual.rs:210-239).
inline uint32_t rice_param(const Scan& s, const int32_t* c, int sp, int base) {
  const int x = s.px[sp], y = s.py[sp], w = s.w, h = s.h, at = y * w + x;
  int sum = 0;
  if (x + 1 < w) {
    sum += std::abs(c[at + 1]);
    if (x + 2 < w) sum += std::abs(c[at + 2]);
    if (y + 1 < h) sum += std::abs(c[at + w + 1]);
  }
  if (y + 1 < h) {
    sum += std::abs(c[at + w]);
    if (y + 2 < h) sum += std::abs(c[at + 2 * w]);
  }
  return kGoRicePars[std::min(31, std::max(0, sum - 5 * base))];
}

inline int next_dq_state(bool dq, int st, int level) {
  return dq ? (32040 >> ((st << 2) + ((level & 1) << 1))) & 3 : 0;
}

// last_sig_coeff_x / y prefix and suffix -> scan position of the last
// significant coefficient (residual.rs:359-433); -1 when malformed.
inline int last_position(Reader& r, Models& m, const Scan& s, bool luma) {
  const int maxx = kGroupIdx[std::min(s.w, 32) - 1], maxy = kGroupIdx[std::min(s.h, 32) - 1];
  const int bx = luma ? kCtxLastXLuma : kCtxLastXChroma, by = luma ? kCtxLastYLuma : kCtxLastYChroma;
  int ox, sx, oy, sy;
  if (luma) {
    const int lw = __builtin_ctz((unsigned)s.w), lh = __builtin_ctz((unsigned)s.h);
    ox = kPrefixCtx[lw];
    sx = (lw + 1) >> 2;
    oy = kPrefixCtx[lh];
    sy = (lh + 1) >> 2;
  } else {
    ox = oy = 0;
    sx = std::min(s.w >> 3, 2);
    sy = std::min(s.h >> 3, 2);
  }
  int x = 0, y = 0;
  while (x < maxx && r.bin(m[bx + ox + (x >> sx)])) x++;
  while (y < maxy && r.bin(m[by + oy + (y >> sy)])) y++;
  auto suffix = [&](int g) {
    if (g <= 3) return g;
    const int count = ((g - 2) >> 1) - 1;
    int v = 0;
    for (int i = count; i >= 0; i--) v += (r.bypass() ? 1 : 0) << i;
    return (int)kMinInGroup[g] + v;
  };
  x = suffix(x);
  y = suffix(y);
  if (x >= s.w || y >= s.h) return -1;
  const int at = y * s.w + x;
  for (int p = 0; p < s.n; p++)
    if (s.raster[p] == at) return p;
  return -1;
}

// residual_coding of one transform block into c (raster, w x h, zeroed
// here), regular (non transform-skip) coefficients, with dependent
// quantisation's state-dependent significance contexts and sign hiding as
// options (residual.rs:534-881).
inline int decode_residual(Reader& r, Models& m, const Scan& s, int32_t* c, bool luma, bool dq, bool sdh) {
  memset(c, 0, sizeof(int32_t) * s.w * s.h);
  const int last = last_position(r, m, s, luma);
  if (last < 0) return kBadLast;
  const int gsz = 1 << s.log2_cg;
  const int last_set = last >> s.log2_cg;
  int state = 0, remaining = (s.n * 28) >> 4;
  Template t;
  std::vector<uint8_t> sig_group(s.wg * s.hg, 0);
  const bool hide = sdh && !dq;
  for (int set = last_set; set >= 0; set--) {
    const int lo = set * gsz, hi = lo + gsz - 1;
    const bool is_last = set == last_set;
    const int cg = s.cg[set];
    bool coded = is_last || lo == 0;
    if (!coded) {
      const int gx = cg % s.wg, gy = cg / s.wg;
      const bool right = gx + 1 < s.wg && sig_group[cg + 1], below = gy + 1 < s.hg && sig_group[cg + s.wg];
      coded = r.bin(m[(luma ? kCtxSigCoeffGroupLuma : kCtxSigCoeffGroupChroma) + (right || below ? 1 : 0)]);
    }
    if (!coded) continue;
    sig_group[cg] = 1;
    // pass 1: significance, gt1, parity, gt3 (context coded)
    const int first = is_last ? last : hi;
    const int infer = first != last ? (set != 0 ? lo : -1) : first;
    int pos = first, nnz = 0, first_nz = first, last_nz = -1;
    int sig_at[16];
    while (pos >= lo && remaining >= 4) {
      const int at = s.raster[pos];
      bool sig = nnz == 0 && pos == infer;
      if (!sig) {
        sig = r.bin(m[sig_context(s, c, pos, luma, state, t)]);
        remaining--;
      } else if (pos != last) {
        sig_context(s, c, pos, luma, state, t);
      }
      if (sig) {
        const int o = level_offset(t, luma);
        sig_at[nnz++] = at;
        first_nz = pos;
        last_nz = std::max(last_nz, pos);
        const bool gt1 = r.bin(m[(luma ? kCtxGtx1Luma : kCtxGtx1Chroma) + o]);
        remaining--;
        int par = 0, gt3 = 0;
        if (gt1) {
          par = r.bin(m[(luma ? kCtxParFlagLuma : kCtxParFlagChroma) + o]) ? 1 : 0;
          gt3 = r.bin(m[(luma ? kCtxGtx2Luma : kCtxGtx2Chroma) + o]) ? 1 : 0;
          remaining -= 2;
        }
        c[at] += 1 + par + (gt1 ? 1 : 0) + (gt3 << 1);
      }
      state = next_dq_state(dq, state, c[at]);
      pos--;
    }
    const int stop2 = pos;
    // pass 2: remainders of levels that reached 4
    for (int p = first; p > stop2; p--) {
      const int at = s.raster[p];
      if (c[at] >= 4) c[at] += (int)r.rem_abs(rice_param(s, c, p, 4), 5, 15) << 1;
    }
    // pass 3: bypass-coded levels of the positions pass 1 did not reach
    for (int p = stop2; p >= lo; p--) {
      const uint32_t k = rice_param(s, c, p, 0);
      const int pos0 = (state < 2 ? 1 : 2) << k;
      const int rem = (int)r.rem_abs(k, 5, 15);
      const int lv = rem == pos0 ? 0 : (rem < pos0 ? rem + 1 : rem);
      state = next_dq_state(dq, state, lv);
      if (lv) {
        const int at = s.raster[p];
        sig_at[nnz++] = at;
        first_nz = p;
        last_nz = std::max(last_nz, p);
        c[at] = lv;
      }
    }
    // signs (the last one hidden in the parity of the sum with sign hiding)
    const bool hidden = hide && last_nz - first_nz > 3 && nnz > 0;
    const int nsign = hidden ? nnz - 1 : nnz;
    uint32_t pat = nsign ? r.bypass_bins(nsign) << (32 - nsign) : 0;
    int64_t sum = 0;
    for (int i = 0; i < nsign; i++) {
      const int a = c[sig_at[i]];
      if (a > 32767) return kBadRange;
      sum += a;
      c[sig_at[i]] = (pat & 0x80000000u) ? -a : a;
      pat <<= 1;
    }
    if (nnz > nsign) {
      const int a = c[sig_at[nsign]];
      if (a > 32767) return kBadRange;
      sum += a;
      c[sig_at[nsign]] = (sum & 1) ? -a : a;
    }
  }
  return kOk;
}

// ---------------------------------------------------- residual_ts_coding --
// residual_ts_coding of one transform-skip block into c (raster, zeroed
// here): coefficient groups in forward scan order, three passes per group
// (slice.rs:1323-1435 with the helpers :1132-1191). Levels are coded
// relative to the larger neighbouring magnitude (left / above).
inline void decode_ts_residual(Reader& r, Models& m, const Scan& s, int32_t* c) {
  memset(c, 0, sizeof(int32_t) * s.w * s.h);
  int remaining = (s.n * 7) >> 2;
  const int last_set = (s.n - 1) >> s.log2_cg, gsz = 1 << s.log2_cg;
  std::vector<uint8_t> gflag(s.wg * s.hg, 0);
  bool any_group = false;
  auto nb = [&](int x, int y, int* left, int* above) {
    *left = x > 0 ? c[y * s.w + x - 1] : 0;
    *above = y > 0 ? c[(y - 1) * s.w + x] : 0;
  };
  for (int set = 0; set <= last_set; set++) {
    const int lo = set * gsz, hi = lo + gsz - 1, cg = s.cg[set];
    const int gx = cg % s.wg, gy = cg / s.wg;
    const bool left_g = gx > 0 && gflag[cg - 1], above_g = gy > 0 && gflag[cg - s.wg];
    bool coded = set == last_set && !any_group;
    if (!coded) coded = r.bin(m[kCtxTsSigCoeffGroup + (left_g ? 1 : 0) + (above_g ? 1 : 0)]);
    gflag[cg] = coded ? 1 : 0;
    if (!coded) continue;
    any_group = true;
    // pass 1: significance, sign, gt1, parity
    int nnz = 0, last1 = -1;
    uint32_t signs = 0;
    int sig_at[16];
    for (int sp = lo; sp <= hi && remaining >= 4; sp++) {
      const int at = s.raster[sp], x = s.px[sp], y = s.py[sp];
      int left, above;
      nb(x, y, &left, &above);
      const int nn = (left != 0) + (above != 0);
      bool sig = nnz == 0 && sp == hi;
      if (!sig) {
        sig = r.bin(m[kCtxTsSigFlag + nn]);
        remaining--;
      }
      if (sig) {
        const int ls = (left > 0) - (left < 0), as = (above > 0) - (above < 0);
        const int sctx = ((ls == 0 && as == 0) || ls * as < 0) ? 0 : ((ls >= 0 && as >= 0) ? 1 : 2);
        const bool neg = r.bin(m[kCtxTsResidualSign + sctx]);
        remaining--;
        signs |= (neg ? 1u : 0u) << nnz;
        sig_at[nnz++] = at;
        const bool gt1 = r.bin(m[kCtxTsLrg1Flag + nn]);
        remaining--;
        bool par = false;
        if (gt1) {
          remaining--;
          par = r.bin(m[kCtxTsParFlag]);
        }
        c[at] = (1 + (gt1 ? 1 : 0) + (par ? 1 : 0)) * (neg ? -1 : 1);
      }
      last1 = sp;
    }
    // pass 2: gt3, gt5, gt7, gt9
    int last2 = -1;
    for (int sp = lo; sp <= hi && remaining >= 4; sp++) {
      const int at = s.raster[sp];
      int a = std::abs(c[at]);
      for (int i = 0; i < 4; i++) {
        const int cut = 2 + 2 * i;
        if (a >= cut) {
          a += (r.bin(m[kCtxTsGtxFlag + (cut >> 1)]) ? 1 : 0) << 1;
          remaining--;
        }
      }
      c[at] = a;
      last2 = sp;
    }
    // pass 3: remainders (and signs of the bypass-coded positions), then the
    // magnitudes back from their neighbour-relative form
    for (int sp = lo; sp <= hi; sp++) {
      const int at = s.raster[sp], x = s.px[sp], y = s.py[sp];
      const int cut = sp <= last2 ? 10 : (sp <= last1 ? 2 : 0);
      int a = std::abs(c[at]);
      if (a >= cut) {
        const int rem = (int)r.rem_abs(1, 5, 15);
        a += sp <= last1 ? rem << 1 : rem;
        if (a != 0 && sp > last1) {
          signs |= (r.bypass() ? 1u : 0u) << nnz;
          sig_at[nnz++] = at;
        }
      }
      if (cut != 0 && a > 0) {
        int left, above;
        nb(x, y, &left, &above);
        const int pred = std::max(std::abs(left), std::abs(above));
        a = (a == 1 && pred > 0) ? pred : a - (a <= pred ? 1 : 0);
      }
      c[at] = a;
    }
    for (int k = 0; k < nnz; k++) c[sig_at[k]] = ((signs >> k) & 1) ? -c[sig_at[k]] : c[sig_at[k]];
  }
}

// ------------------------------------------ strict profile slice data --
// The 6 MPM candidates without neighbours (predict.rs:1455-1476:
// Planar, DC, vertical, horizontal, vertical -4, vertical +4).
constexpr uint8_t kMpmNoNeighbours[6] = {0, 1, 50, 18, 46, 54};

// intra_luma_mpm_flag / planar flag / mpm_idx or the truncated-binary
// remainder (slice.rs:1691-1717 without MRL and ISP, predict.rs:1512-1522).
inline int decode_luma_mode(Reader& r, Models& m) {
  int mode;
  if (r.bin(m[kCtxIntraLumaMpmFlag])) {
    if (!r.bin(m[kCtxIntraLumaPlanarFlag + 1]))
      mode = kMpmNoNeighbours[0];
    else
      mode = kMpmNoNeighbours[std::min(5u, r.unary_max(4) + 1)];
  } else {
    uint8_t sorted[6];
    memcpy(sorted, kMpmNoNeighbours, 6);
    std::sort(sorted, sorted + 6);
    mode = (int)r.trunc_bin(61);
    for (int k = 0; k < 6; k++)
      if (mode >= sorted[k]) mode++;
  }
  return mode <= 1 ? mode : std::min(66, std::max(2, mode));
}

// The CU-level state residual_coding leaves for lfnst_idx / mts_idx
// (slice.rs:951-992): last scan positions and the MTS coefficient region.
struct CuSyntaxState {
  bool violates_lfnst[2] = {false, false};
  bool lfnst_last = false, violates_mts = false, mts_last = false;
  void update(const Scan& s, const int32_t* c, bool luma, bool ts) {
    int last = -1;
    for (int p = s.n - 1; p >= 0; p--)
      if (c[s.raster[p]] != 0) {
        last = p;
        break;
      }
    if (last < 0 || ts) return;
    const int w = s.w, h = s.n / s.w;
    if (w >= 4 && h >= 4) {
      const int maxpos = ((w == 4 && h == 4) || (w == 8 && h == 8)) ? 7 : 15;
      violates_lfnst[luma ? 0 : 1] |= last > maxpos;
      lfnst_last |= last >= 1;
    }
    if (luma) {
      mts_last |= last >= 1;
      for (int i = 0; i < s.w * s.h && !violates_mts; i++)
        if (c[i] != 0 && ((i % s.w) / 4 > 3 || (i / s.w) / 4 > 3)) violates_mts = true;
    }
  }
};

// Where a parsed TB's levels go: dense (w x h raster int16) or sparse (at
// an even offset the nonzero count, one unused word, then (raster index,
// level) pairs with rising indices).
struct LevelSink {
  int16_t* base;
  uint64_t cap, at = 0;
  bool sparse;
  // returns the TB's offset relative to base, or -1 when it does not fit
  int64_t put(const int32_t* c, int n) {
    if (!sparse) {
      if (at + n > cap) return -1;
      for (int i = 0; i < n; i++) base[at + i] = (int16_t)c[i];
      const int64_t o = (int64_t)at;
      at += n;
      return o;
    }
    if (at & 1) {
      if (at + 1 > cap) return -1;
      base[at++] = 0;
    }
    int nz = 0;
    for (int i = 0; i < n; i++) nz += c[i] != 0;
    if (at + 2 + 2 * (uint64_t)nz > cap) return -1;
    const int64_t o = (int64_t)at;
    base[at] = (int16_t)nz;
    base[at + 1] = 0;
    uint64_t q = at + 2;
    for (int i = 0; i < n; i++)
      if (c[i]) {
        base[q++] = (int16_t)i;
        base[q++] = (int16_t)c[i];
      }
    at = q;
    return o;
  }
};

// decode_picture's parse (slice.rs:458-575) of one strict 8-bit 4:2:0 IDR
// picture at CTU 32: per 32x32 coding unit in raster order the luma mode,
// the chroma mode (DM, or one of Planar / vertical / horizontal / DC with
// vertical-diagonal in place of the luma mode), the cbfs (Cb, Cr, Y), each
// coded TB's transform_skip_flag and residual, then lfnst_idx and mts_idx
// where their syntax is present; finally end_of_slice_one_bit and the byte
// alignment. Writes the CU records (tb-grid raster order, tu_tools as the
// frame path reads them) and the levels, level_off relative to `level_base`.
inline int parse_strict_picture(const uint8_t* data, size_t size, int qp, int width, int height,
                                vvcg_cu_rec* cus, LevelSink& sink, int64_t level_base) {
  thread_local const Scan luma_scan = make_scan(32, 32), chroma_scan = make_scan(16, 16);
  Reader r;
  r.start(data, size);
  Models m;
  m.init_i_slice(qp);
  int32_t cy[1024], cb[256], cr[256];
  int32_t* coef[3] = {cy, cb, cr};
  const int gw = width / 32, gh = height / 32;
  for (int k = 0; k < gw * gh; k++) {
    const int mode = decode_luma_mode(r, m);
    int cmode = mode;
    if (r.bin(m[kCtxIntraChromaPredMode])) {
      static const int kCand[4] = {0, 50, 18, 1};
      const int cand = kCand[r.bypass_bins(2) & 3];
      cmode = cand == mode ? 66 : cand;
    }
    const bool cbf_cb = r.bin(m[kCtxQtCbfCb]);
    const bool cbf_cr = r.bin(m[kCtxQtCbfCr + (cbf_cb ? 1 : 0)]);
    const bool cbf_y = r.bin(m[kCtxQtCbfY]);
    const bool cbf[3] = {cbf_y, cbf_cb, cbf_cr};
    bool ts[3] = {false, false, false};
    CuSyntaxState cu;
    for (int c = 0; c < 3; c++) {
      if (!cbf[c]) continue;
      const Scan& s = c ? chroma_scan : luma_scan;
      ts[c] = r.bin(m[kCtxTransformSkipFlag + (c ? 1 : 0)]);
      if (ts[c]) {
        decode_ts_residual(r, m, s, coef[c]);
      } else {
        const int e = decode_residual(r, m, s, coef[c], c == 0, false, false);
        if (e) return e;
      }
      cu.update(s, coef[c], c == 0, ts[c]);
    }
    const bool any_ts = (cbf_y && ts[0]) || (cbf_cb && ts[1]) || (cbf_cr && ts[2]);
    int lfnst = 0, mts = 0;
    if (!any_ts && cu.lfnst_last && !cu.violates_lfnst[0] && !cu.violates_lfnst[1] && r.bin(m[kCtxLfnstIdx]))
      lfnst = r.bin(m[kCtxLfnstIdx + 2]) ? 2 : 1;
    if (!(any_ts && ts[0]) && !cu.violates_mts && cu.mts_last && lfnst == 0 && r.bin(m[kCtxMtsIdx])) {
      mts = 1;
      for (int i = 0; i < 3 && r.bin(m[kCtxMtsIdx + 1 + i]); i++) mts++;
    }
    vvcg_cu_rec& rec = cus[k];
    rec.luma_mode = (uint8_t)mode;
    rec.chroma_mode = (uint8_t)cmode;
    rec.cbf = (uint8_t)((cbf_y ? 1 : 0) | (cbf_cb ? 2 : 0) | (cbf_cr ? 4 : 0));
    uint32_t tools = (uint32_t)(mts << VVCG_CU_MTS_SHIFT) | (uint32_t)(lfnst << VVCG_CU_LFNST_SHIFT);
    for (int c = 0; c < 3; c++) {
      rec.level_off[c] = -1;
      if (!cbf[c]) continue;
      if (ts[c]) tools |= 1u << c;
      const int64_t o = sink.put(coef[c], c ? 256 : 1024);
      if (o < 0) return kTruncated;
      const int64_t abs_off = level_base + o;
      if (abs_off > INT32_MAX) return kTruncated;
      rec.level_off[c] = (int32_t)abs_off;
    }
    rec.tu_tools = (uint8_t)tools;
  }
  if (!r.terminate() || !r.aligned_end()) return kBadEnd;
  return kOk;
}

}  // namespace vvcg_parse
