// CPU oracle (test infrastructure only; see oracle.h): the encoder side of the
// reference's CABAC, restated to write the bitstreams the library's host-side
// parser is checked on:
//   CtxModel / CtxStore::new_i_slice   cabac.rs:41-99, :267-296
//   BinEncoder                         cabac.rs:477-748 (with BitWriter,
//                                      bits.rs:48-117)
//   CoeffScan                          transform.rs:43-200
//   encode_residual_with_options       residual.rs:85-240, :280-357, :448-522,
//                                      :593-746 (encode_last_sig_coeff,
//                                      encode_subblock)
//   encode_ts_block                    slice.rs:1132-1321
//   encode_picture's syntax writes     slice.rs:370-455 with encode_intra_mode
//                                      :1106-1115 / encode_full_luma_intra_mode
//                                      :1658-1689, lfnst / mts idx :994-1029,
//                                      classify_luma_mode_mpm predict.rs:1527
//   encode_picture_multitool's writes  slice.rs:2867-2960 with
//                                      encode_chroma_intra_mode :1718-1754
//   encode_inter_picture's writes      slice.rs:3451-3536 with encode_mvd
//                                      :1782-1806, CtxStore::new_p_slice
// The context tables come from rustmpeg-next_b200/csrc/vvc_cabac.h, which a
// CPU test checks against the reference's literals.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../rustmpeg-next_b200/csrc/vvc_cabac.h"
#include "oracle.h"

namespace orc {
namespace {

using namespace vvc_cabac;

// cabac.rs:32-99 CtxModel
struct Ctx {
  uint16_t state0 = 0, state1 = 0;
  uint8_t rate0 = 0, rate1 = 0;
  void init(int qp, int init_id, int log2_window) {
    const int slope = (init_id >> 3) - 4;
    const int offset = (init_id & 7) * 18 + 1;
    int inistate = ((slope * (qp - 16)) >> 1) + offset;
    inistate = inistate < 1 ? 1 : (inistate > 127 ? 127 : inistate);
    const uint32_t p1 = (uint32_t)inistate << 8;
    rate0 = (uint8_t)(2 + ((log2_window >> 2) & 3));
    rate1 = (uint8_t)(3 + rate0 + (log2_window & 3));
    state0 = (uint16_t)(p1 & 0x7FE0);
    state1 = (uint16_t)(p1 & 0x7FFE);
  }
  uint32_t state() const { return ((uint32_t)state0 + state1) >> 8; }
  bool mps() const { return state() >= 128; }
  uint32_t get_lps(uint32_t range) const {
    uint32_t q = state();
    if (q & 0x80) q ^= 0xFF;
    return (((q >> 2) * (range >> 5)) >> 1) + 4;
  }
  void update(bool bin) {
    uint32_t n0 = state0 - ((state0 >> rate0) & 0x7FE0);
    uint32_t n1 = state1 - ((state1 >> rate1) & 0x7FFE);
    if (bin) {
      n0 += (0x7FFFu >> rate0) & 0x7FE0;
      n1 += (0x7FFFu >> rate1) & 0x7FFE;
    }
    state0 = (uint16_t)(n0 & 0xFFFF);
    state1 = (uint16_t)(n1 & 0xFFFF);
  }
};

// cabac.rs:267-308 CtxStore::from_table (I, P or B initialisation)
struct CtxStore {
  Ctx models[kNumContexts];
  explicit CtxStore(int qp, const uint8_t (*table)[2] = kCtxInitI) {
    qp = std::min(63, std::max(0, qp));
    for (int i = 0; i < kNumContexts; i++) models[i].init(qp, table[i][0], table[i][1]);
  }
};

// bits.rs BitWriter: MSB-first bits into bytes
struct Bits {
  std::vector<uint8_t> bytes;
  uint32_t cur = 0;
  int nbits = 0;
  void bit(bool b) {
    cur = (cur << 1) | (b ? 1 : 0);
    if (++nbits == 8) {
      bytes.push_back((uint8_t)cur);
      cur = 0;
      nbits = 0;
    }
  }
  void write(uint32_t v, uint32_t n) {
    for (int i = (int)n - 1; i >= 0; i--) bit((v >> i) & 1);
  }
  void byte_alignment() {
    bit(true);
    while (nbits) bit(false);
  }
};

// cabac.rs:477-748 BinEncoder
struct Encoder {
  uint32_t low = 0, range = 510, num_buffered = 0;
  uint8_t buffered = 0xFF;
  int bits_left = 23;
  Bits out;

  void write_out() {
    const uint32_t lead = low >> (24 - bits_left);
    bits_left += 8;
    low &= bits_left >= 32 ? 0u : (0xFFFFFFFFu >> bits_left);
    if (lead == 0xFF) {
      num_buffered++;
    } else if (num_buffered > 0) {
      const uint32_t carry = lead >> 8;
      out.write(buffered + carry, 8);
      buffered = (uint8_t)(lead & 0xFF);
      const uint32_t fill = (0xFF + carry) & 0xFF;
      for (; num_buffered > 1; num_buffered--) out.write(fill, 8);
    } else {
      num_buffered = 1;
      buffered = (uint8_t)lead;
    }
  }
  void bin(bool b, Ctx& c) {
    const uint32_t lps = c.get_lps(range);
    const bool mps = c.mps();
    range -= lps;
    if (b != mps) {
      const int nb = kRenormLps[lps >> 3];
      bits_left -= nb;
      low = (low + range) << nb;
      range = lps << nb;
      if (bits_left < 12) write_out();
    } else if (range < 256) {
      bits_left -= 1;
      low <<= 1;
      range <<= 1;
      if (bits_left < 12) write_out();
    }
    c.update(b);
  }
  void bypass(bool b) {
    low <<= 1;
    if (b) low += range;
    if (--bits_left < 12) write_out();
  }
  void bypass_bins(uint32_t bins, uint32_t n) {
    if (!n) return;
    if (range == 256) {  // aligned: whole bytes shift in
      uint32_t rem = n;
      while (rem) {
        const uint32_t k = std::min(rem, 8u);
        const uint32_t v = (bins >> (rem - k)) & ((1u << k) - 1);
        low = (low << k) + (v << 8);
        rem -= k;
        bits_left -= (int)k;
        if (bits_left < 12) write_out();
      }
      return;
    }
    uint32_t rem = n;
    while (rem > 8) {
      rem -= 8;
      const uint32_t pat = (bins >> rem) & 0xFF;
      low = (low << 8) + range * pat;
      bins -= pat << rem;
      bits_left -= 8;
      if (bits_left < 12) write_out();
    }
    low = (low << rem) + range * bins;
    bits_left -= (int)rem;
    if (bits_left < 12) write_out();
  }
  void trunc_bin(uint32_t sym, uint32_t n) {
    if (n <= 1) return;
    const uint32_t k = 31 - __builtin_clz(n), val = 1u << k, b = n - val;
    if (sym < val - b)
      bypass_bins(sym, k);
    else
      bypass_bins(sym + val - b, k + 1);
  }
  void unary_max(uint32_t sym, uint32_t max) {
    if (!max) return;
    for (uint32_t i = 0; i < std::min(sym, max); i++) bypass(true);
    if (sym < max) bypass(false);
  }
  void terminate(bool b) {
    range -= 2;
    if (b) {
      low = (low + range) << 7;
      range = 2 << 7;
      bits_left -= 7;
    } else if (range >= 256) {
      return;
    } else {
      low <<= 1;
      range <<= 1;
      bits_left -= 1;
    }
    if (bits_left < 12) write_out();
  }
  void rem_abs(uint32_t bins, uint32_t k, uint32_t cutoff, uint32_t max_log2) {
    const uint32_t threshold = cutoff << k;
    if (bins < threshold) {
      const uint32_t len = (bins >> k) + 1;
      bypass_bins((1u << len) - 2, len);
      bypass_bins(bins & ((1u << k) - 1), k);
      return;
    }
    const uint32_t max_prefix = 32 - cutoff - max_log2, code = (bins >> k) - cutoff;
    uint32_t plen, slen;
    if (code >= (1u << max_prefix) - 1) {
      plen = max_prefix;
      slen = max_log2;
    } else {
      plen = 0;
      while (code > ((2u << plen) - 2)) plen++;
      slen = plen + k + 1;
    }
    const uint32_t total = plen + cutoff;
    bypass_bins((1u << total) - 1, total);
    bypass_bins(((code - ((1u << plen) - 1)) << k) | (bins & ((1u << k) - 1)), slen);
  }
  std::vector<uint8_t> finish_and_align() {
    if (bits_left < 32 && (low >> (32 - bits_left)) != 0) {
      out.write(buffered + 1u, 8);
      for (; num_buffered > 1; num_buffered--) out.write(0x00, 8);
      low -= 1u << (32 - bits_left);
    } else {
      if (num_buffered > 0) out.write(buffered, 8);
      for (; num_buffered > 1; num_buffered--) out.write(0xFF, 8);
    }
    out.write(low >> 8, (uint32_t)(24 - bits_left));
    out.byte_alignment();
    return out.bytes;
  }
};

// transform.rs:43-200 CoeffScan
struct CScan {
  int width = 0, height = 0, log2_cg = 0, wig = 0, hig = 0, max_num = 0;
  std::vector<int> raster, xs, ys, gx, gy;
  int cg_raster(int sub) const { return gy[sub] * wig + gx[sub]; }
};

void diagonal(int w, int h, std::vector<int>& xs, std::vector<int>& ys) {
  xs.clear();
  ys.clear();
  int line = 0, column = 0;
  for (int i = 0; i < w * h; i++) {
    xs.push_back(column);
    ys.push_back(line);
    if (column == w - 1 || line == 0) {
      line += column + 1;
      column = 0;
      if (line >= h) {
        column += line - (h - 1);
        line = h - 1;
      }
    } else {
      column++;
      line--;
    }
  }
}

CScan coeff_scan(int w, int h) {
  // transform.rs coefficient_group_log2 (rows: log2 width, columns: log2 height)
  static const int T[8][8][2] = {
      {{0, 0}, {0, 1}, {0, 2}, {0, 3}, {0, 4}, {0, 4}, {0, 4}, {0, 4}},
      {{1, 0}, {1, 1}, {1, 1}, {1, 3}, {1, 3}, {1, 3}, {1, 3}, {1, 3}},
      {{2, 0}, {1, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{3, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}}};
  CScan s;
  s.width = w;
  s.height = h;
  const int lx = std::min(7, __builtin_ctz((unsigned)w)), ly = std::min(7, __builtin_ctz((unsigned)h));
  const int cw = 1 << T[lx][ly][0], ch = 1 << T[lx][ly][1];
  s.log2_cg = T[lx][ly][0] + T[lx][ly][1];
  s.wig = std::min(w, 32) / cw;
  s.hig = std::min(h, 32) / ch;
  s.max_num = std::min(w, 32) * std::min(h, 32);
  std::vector<int> ix, iy;
  diagonal(s.wig, s.hig, s.gx, s.gy);
  diagonal(cw, ch, ix, iy);
  for (size_t g = 0; g < s.gx.size(); g++)
    for (size_t k = 0; k < ix.size(); k++) {
      const int x = s.gx[g] * cw + ix[k], y = s.gy[g] * ch + iy[k];
      s.raster.push_back(y * w + x);
      s.xs.push_back(x);
      s.ys.push_back(y);
    }
  return s;
}

// residual.rs:142-188 sig_ctx_id_abs, :190-208 ctx_offset_abs, :210-239 derive_rice
struct Tmpl {
  int diag = -1, sum1 = 0;
};

int sig_ctx(const CScan& s, const int32_t* c, int sp, bool luma, int state, Tmpl& t) {
  const int x = s.xs[sp], y = s.ys[sp], w = s.width, h = s.height, base = y * w + x;
  int sum_abs = 0, num_pos = 0;
  auto upd = [&](int i) {
    const int a = abs(c[i]);
    sum_abs += std::min(4 + (a & 1), a);
    num_pos += a != 0;
  };
  if (x + 1 < w) {
    upd(base + 1);
    if (x + 2 < w) upd(base + 2);
    if (y + 1 < h) upd(base + w + 1);
  }
  if (y + 1 < h) {
    upd(base + w);
    if (y + 2 < h) upd(base + 2 * w);
  }
  const int diag = x + y;
  int ofs = std::min((sum_abs + 1) >> 1, 3) + (diag < 2 ? 4 : 0);
  if (luma) ofs += diag < 5 ? 4 : 0;
  t.diag = diag;
  t.sum1 = sum_abs - num_pos;
  const int set = std::min(2, std::max(0, state - 1));
  const int lb[3] = {kCtxSigFlagLuma, kCtxSigFlagLuma1, kCtxSigFlagLuma2};
  const int cb[3] = {kCtxSigFlagChroma, kCtxSigFlagChroma1, kCtxSigFlagChroma2};
  return (luma ? lb[set] : cb[set]) + ofs;
}

int abs_ctx_offset(const Tmpl& t, bool luma) {
  if (t.diag < 0) return 0;
  int o = std::min(t.sum1, 4) + 1;
  if (t.diag == 0)
    o += luma ? 15 : 5;
  else if (luma)
    o += t.diag < 3 ? 10 : (t.diag < 10 ? 5 : 0);
  return o;
}

uint32_t rice(const CScan& s, const int32_t* c, int sp, int base_level) {
  const int x = s.xs[sp], y = s.ys[sp], w = s.width, h = s.height, base = y * w + x;
  int sum = 0;
  if (x + 1 < w) {
    sum += abs(c[base + 1]);
    if (x + 2 < w) sum += abs(c[base + 2]);
    if (y + 1 < h) sum += abs(c[base + w + 1]);
  }
  if (y + 1 < h) {
    sum += abs(c[base + w]);
    if (y + 2 < h) sum += abs(c[base + 2 * w]);
  }
  sum -= 5 * base_level;
  return kGoRicePars[sum < 0 ? 0 : (sum > 31 ? 31 : sum)];
}

int dq_next(int table, int st, int level) { return (table >> ((st << 2) + ((level & 1) << 1))) & 3; }

// residual.rs:280-357 encode_last_sig_coeff
void write_last(Encoder& e, CtxStore& m, const CScan& s, int last, bool luma) {
  const int px = s.xs[last], py = s.ys[last];
  const int gxi = kGroupIdx[px], gyi = kGroupIdx[py];
  const int maxx = kGroupIdx[std::min(s.width, 32) - 1], maxy = kGroupIdx[std::min(s.height, 32) - 1];
  const int bx = luma ? kCtxLastXLuma : kCtxLastXChroma, by = luma ? kCtxLastYLuma : kCtxLastYChroma;
  int ox, sx, oy, sy;
  if (luma) {
    const int lw = __builtin_ctz((unsigned)s.width), lh = __builtin_ctz((unsigned)s.height);
    ox = kPrefixCtx[lw];
    sx = (lw + 1) >> 2;
    oy = kPrefixCtx[lh];
    sy = (lh + 1) >> 2;
  } else {
    ox = oy = 0;
    sx = std::min(s.width >> 3, 2);
    sy = std::min(s.height >> 3, 2);
  }
  int k = 0;
  for (; k < gxi; k++) e.bin(true, m.models[bx + ox + (k >> sx)]);
  if (gxi < maxx) e.bin(false, m.models[bx + ox + (k >> sx)]);
  for (k = 0; k < gyi; k++) e.bin(true, m.models[by + oy + (k >> sy)]);
  if (gyi < maxy) e.bin(false, m.models[by + oy + (k >> sy)]);
  if (gxi > 3) {
    const int v = px - kMinInGroup[gxi], cnt = ((gxi - 2) >> 1) - 1;
    for (int i = cnt; i >= 0; i--) e.bypass((v >> i) & 1);
  }
  if (gyi > 3) {
    const int v = py - kMinInGroup[gyi], cnt = ((gyi - 2) >> 1) - 1;
    for (int i = cnt; i >= 0; i--) e.bypass((v >> i) & 1);
  }
}

// residual.rs:593-746 encode_subblock
void write_subblock(Encoder& e, CtxStore& m, const CScan& s, const int32_t* c, int min_sub, int max_sub, int last,
                    bool luma, int table, int* state, bool sdh, Tmpl& t, int* remaining) {
  const bool is_last = (last >> s.log2_cg) == (min_sub >> s.log2_cg);
  const int first_sig = is_last ? last : max_sub;
  const int sub_set = min_sub >> s.log2_cg;
  const int infer = first_sig != last ? (sub_set != 0 ? min_sub : -1) : first_sig;
  int next = first_sig, first_nz = next, last_nz = -1, first2 = min_sub - 1;
  uint32_t nnz = 0, signs = 0;
  while (next >= min_sub && *remaining >= 4) {
    const int at = s.raster[next];
    const int level = c[at];
    const bool sig = level != 0;
    if (nnz != 0 || next != infer) {
      e.bin(sig, m.models[sig_ctx(s, c, next, luma, *state, t)]);
      (*remaining)--;
    } else if (next != last) {
      sig_ctx(s, c, next, luma, *state, t);
    }
    if (sig) {
      const int o = abs_ctx_offset(t, luma);
      nnz++;
      first_nz = next;
      last_nz = std::max(last_nz, next);
      const int a = abs(level);
      if (next != last) signs <<= 1;
      if (level < 0) signs += 1;
      const bool gt1 = a > 1;
      e.bin(gt1, m.models[(luma ? kCtxGtx1Luma : kCtxGtx1Chroma) + o]);
      (*remaining)--;
      if (gt1) {
        e.bin(a & 1, m.models[(luma ? kCtxParFlagLuma : kCtxParFlagChroma) + o]);
        const bool gt3 = a > 3;
        e.bin(gt3, m.models[(luma ? kCtxGtx2Luma : kCtxGtx2Chroma) + o]);
        *remaining -= 2;
        if (gt3) first2 = std::max(first2, next);
      }
    }
    *state = dq_next(table, *state, level);
    next--;
  }
  const int min2 = next;
  for (int sp = first2; sp > min2; sp--) {
    const int a = abs(c[s.raster[sp]]);
    if (a >= 4) e.rem_abs((uint32_t)((a - 4) >> 1), rice(s, c, sp, 4), 5, 15);
  }
  for (int sp = min2; sp >= min_sub; sp--) {
    const int at = s.raster[sp];
    const int a = abs(c[at]);
    const uint32_t k = rice(s, c, sp, 0);
    const int pos0 = (*state < 2 ? 1 : 2) << k;
    const int rem = a == 0 ? pos0 : (a <= pos0 ? a - 1 : a);
    e.rem_abs((uint32_t)rem, k, 5, 15);
    *state = dq_next(table, *state, a);
    if (a) {
      nnz++;
      first_nz = sp;
      last_nz = std::max(last_nz, sp);
      signs <<= 1;
      if (c[at] < 0) signs += 1;
    }
  }
  uint32_t nsign = nnz;
  if (sdh && last_nz - first_nz > 3 && nsign > 0) {
    nsign--;
    signs >>= 1;
  }
  e.bypass_bins(signs, nsign);
}

// residual.rs:448-522 encode_residual_with_options (a block with a nonzero level)
void write_residual(Encoder& e, CtxStore& m, const CScan& s, const int32_t* c, bool luma, bool dq, bool sdh) {
  int last = -1;
  for (int p = s.max_num - 1; p >= 0; p--)
    if (c[s.raster[p]] != 0) {
      last = p;
      break;
    }
  write_last(e, m, s, last, luma);
  const int gsz = 1 << s.log2_cg, lastg = last >> s.log2_cg;
  std::vector<char> coded(s.wig * s.hig, 0), flags(s.wig * s.hig, 0);
  for (int p = 0; p < s.max_num; p++)
    if (c[s.raster[p]] != 0) coded[p >> s.log2_cg] = 1;
  const int table = dq ? 32040 : 0;
  int state = 0, remaining = (s.max_num * 28) >> 4;
  Tmpl t;
  for (int sub = lastg; sub >= 0; sub--) {
    const int min_sub = sub * gsz, max_sub = min_sub + gsz - 1, cg = s.cg_raster(sub);
    flags[cg] = coded[sub];
    if (sub != 0 && sub != lastg) {
      const int gx = cg % s.wig, gy = cg / s.wig;
      const bool right = gx + 1 < s.wig && flags[cg + 1], lower = gy + 1 < s.hig && flags[cg + s.wig];
      e.bin(coded[sub], m.models[(luma ? kCtxSigCoeffGroupLuma : kCtxSigCoeffGroupChroma) + (right || lower)]);
      if (!coded[sub]) continue;
    }
    write_subblock(e, m, s, c, min_sub, max_sub, last, luma, table, &state, sdh && !dq, t, &remaining);
  }
}

// slice.rs:1132-1191 neighbours / sign_context / derive_mod_coeff
void ts_neighbours(const int32_t* c, int w, int x, int y, int* left, int* above) {
  *left = x > 0 ? c[y * w + x - 1] : 0;
  *above = y > 0 ? c[(y - 1) * w + x] : 0;
}
int ts_mod(int left, int above, int a, bool identity) {
  if (a == 0) return 0;
  if (identity) return a;
  const int pred = std::max(abs(left), abs(above));
  return a == pred ? 1 : (a < pred ? a + 1 : a);
}

// slice.rs:1193-1321 encode_ts_block (a block with a nonzero level)
void write_ts(Encoder& e, CtxStore& m, const CScan& s, const int32_t* c) {
  int remaining = (s.max_num * 7) >> 2;
  const int lastg = (s.max_num - 1) >> s.log2_cg, gsz = 1 << s.log2_cg;
  std::vector<char> flags(s.wig * s.hig, 0);
  bool any = false;
  for (int sub = 0; sub <= lastg; sub++) {
    const int lo = sub * gsz, hi = lo + gsz - 1, cg = s.cg_raster(sub);
    bool has = false;
    for (int sp = lo; sp <= hi; sp++) has |= c[s.raster[sp]] != 0;
    const int gx = cg % s.wig, gy = cg / s.wig;
    const bool sl = gx > 0 && flags[cg - 1], sa = gy > 0 && flags[cg - s.wig];
    flags[cg] = has;
    if (sub != lastg || any) {
      e.bin(has, m.models[kCtxTsSigCoeffGroup + sl + sa]);
      if (!has) continue;
    }
    int nnz = 0, last1 = -1;
    for (int sp = lo; sp <= hi && remaining >= 4; sp++) {
      const int v = c[s.raster[sp]];
      int left, above;
      ts_neighbours(c, s.width, s.xs[sp], s.ys[sp], &left, &above);
      const int nn = (left != 0) + (above != 0);
      if (nnz != 0 || sp != hi) {
        e.bin(v != 0, m.models[kCtxTsSigFlag + nn]);
        remaining--;
      }
      if (v != 0) {
        const int ls = (left > 0) - (left < 0), as = (above > 0) - (above < 0);
        const int sctx = ((ls == 0 && as == 0) || ls * as < 0) ? 0 : ((ls >= 0 && as >= 0) ? 1 : 2);
        e.bin(v < 0, m.models[kCtxTsResidualSign + sctx]);
        remaining--;
        nnz++;
        const int rem_abs = ts_mod(left, above, abs(v), false) - 1;
        e.bin(rem_abs != 0, m.models[kCtxTsLrg1Flag + nn]);
        remaining--;
        if (rem_abs != 0) {
          e.bin((rem_abs - 1) & 1, m.models[kCtxTsParFlag]);
          remaining--;
        }
      }
      last1 = sp;
    }
    int last2 = -1;
    for (int sp = lo; sp <= hi && remaining >= 4; sp++) {
      int left, above;
      ts_neighbours(c, s.width, s.xs[sp], s.ys[sp], &left, &above);
      const int a = ts_mod(left, above, abs(c[s.raster[sp]]), false);
      for (int i = 0; i < 4; i++) {
        const int cut = 2 + 2 * i;
        if (a >= cut) {
          e.bin(a >= cut + 2, m.models[kCtxTsGtxFlag + (cut >> 1)]);
          remaining--;
        }
      }
      last2 = sp;
    }
    for (int sp = lo; sp <= hi; sp++) {
      const int cut = sp <= last2 ? 10 : (sp <= last1 ? 2 : 0);
      int left, above;
      ts_neighbours(c, s.width, s.xs[sp], s.ys[sp], &left, &above);
      const int v = c[s.raster[sp]];
      const int a = ts_mod(left, above, abs(v), cut == 0);
      if (a >= cut) {
        e.rem_abs((uint32_t)(sp <= last1 ? (a - cut) >> 1 : a), 1, 5, 15);
        if (a != 0 && sp > last1) e.bypass(v < 0);
      }
    }
    if (has) any = true;
  }
}

// slice.rs:951-992 CuConstraints and the presence rules of lfnst_idx / mts_idx
struct Constraints {
  bool vl[2] = {false, false}, lfnst_last = false, vmts = false, mts_last = false;
  void update(const CScan& s, const int32_t* c, bool luma, bool ts) {
    int last = -1;
    for (int p = s.max_num - 1; p >= 0; p--)
      if (c[s.raster[p]] != 0) {
        last = p;
        break;
      }
    if (last < 0 || ts) return;
    const int h = s.max_num / s.width;
    if (s.width >= 4 && h >= 4) {
      const int mx = ((s.width == 4 && h == 4) || (s.width == 8 && h == 8)) ? 7 : 15;
      vl[luma ? 0 : 1] |= last > mx;
      lfnst_last |= last >= 1;
    }
    if (luma) {
      mts_last |= last >= 1;
      for (int i = 0; i < s.width * s.width; i++)
        if (c[i] != 0 && ((i % s.width) / 4 > 3 || (i / s.width) / 4 > 3)) vmts = true;
    }
  }
};

// slice.rs:1658-1689 encode_full_luma_intra_mode with the neighbour-free MPM
// list (predict.rs:1455-1476) and classify_luma_mode_mpm (predict.rs:1527)
void write_luma_mode(Encoder& e, CtxStore& m, int mode) {
  static const int mpm[6] = {0, 1, 50, 18, 46, 54};
  for (int i = 0; i < 6; i++)
    if (mpm[i] == mode) {
      e.bin(true, m.models[kCtxIntraLumaMpmFlag]);
      if (i == 0) {
        e.bin(false, m.models[kCtxIntraLumaPlanarFlag + 1]);
      } else {
        e.bin(true, m.models[kCtxIntraLumaPlanarFlag + 1]);
        e.unary_max((uint32_t)(i - 1), 4);
      }
      return;
    }
  int sorted[6];
  memcpy(sorted, mpm, sizeof(sorted));
  std::sort(sorted, sorted + 6);
  int rem = mode;
  for (int i = 5; i >= 0; i--)
    if (rem > sorted[i]) rem--;
  e.bin(false, m.models[kCtxIntraLumaMpmFlag]);
  e.trunc_bin((uint32_t)rem, 61);
}

// slice.rs:1658-1689 encode_full_luma_intra_mode (intra_luma_ref_idx 0, no
// ISP) against an MPM list
void write_full_luma_mode(Encoder& e, CtxStore& m, int mode, const uint8_t mpm[6]) {
  for (int i = 0; i < 6; i++)
    if (mpm[i] == mode) {
      e.bin(true, m.models[kCtxIntraLumaMpmFlag]);
      e.bin(i != 0, m.models[kCtxIntraLumaPlanarFlag + 1]);
      if (i) e.unary_max((uint32_t)(i - 1), 4);
      return;
    }
  uint8_t sorted[6];
  memcpy(sorted, mpm, 6);
  std::sort(sorted, sorted + 6);
  int rem = mode;
  for (int i = 5; i >= 0; i--)
    if (rem > sorted[i]) rem--;
  e.bin(false, m.models[kCtxIntraLumaMpmFlag]);
  e.trunc_bin((uint32_t)rem, 61);
}

// slice.rs:1718-1754 encode_chroma_intra_mode without CCLM; false when the
// mode is neither DM nor a Table 24 candidate.
bool write_chroma_mode(Encoder& e, CtxStore& m, int chroma, int luma) {
  if (chroma == luma) {
    e.bin(false, m.models[kCtxIntraChromaPredMode]);
    return true;
  }
  static const int cand[4] = {0, 50, 18, 1};
  for (int i = 0; i < 4; i++)
    if ((cand[i] == luma ? 66 : cand[i]) == chroma) {
      e.bin(true, m.models[kCtxIntraChromaPredMode]);
      e.bypass_bins((uint32_t)i, 2);
      return true;
    }
  return false;
}

// slice.rs:1782-1806 encode_mvd
void write_mvd(Encoder& e, CtxStore& m, const int32_t mvd[2]) {
  for (int i = 0; i < 2; i++) e.bin(mvd[i] != 0, m.models[kCtxMvd]);
  for (int i = 0; i < 2; i++)
    if (mvd[i] != 0) e.bin(std::abs(mvd[i]) > 1, m.models[kCtxMvd + 1]);
  for (int i = 0; i < 2; i++)
    if (mvd[i] != 0) {
      if (std::abs(mvd[i]) > 1) e.rem_abs((uint32_t)std::abs(mvd[i]) - 2, 1, 0, 17);
      e.bypass(mvd[i] < 0);
    }
}

// A coded TB's levels (n of them, at least one nonzero) and its
// transform_skip_flag and residual syntax.
int write_tb(Encoder& e, CtxStore& m, const CScan& s, const int16_t* levels, uint64_t num_levels, int32_t off, int n,
             bool luma, bool ts, bool dq, bool sdh, std::vector<int32_t>& c) {
  if (off < 0 || (uint64_t)off + n > num_levels) return -4;
  c.assign(n, 0);
  bool any = false;
  for (int i = 0; i < n; i++) {
    c[i] = levels[off + i];
    any |= c[i] != 0;
  }
  if (!any) return -5;
  e.bin(ts, m.models[kCtxTransformSkipFlag + (luma ? 0 : 1)]);
  if (ts)
    write_ts(e, m, s, c.data());
  else
    write_residual(e, m, s, c.data(), luma, dq, sdh);
  return 0;
}

}  // namespace

// The slice data encode_picture_multitool writes (slice.rs:2867-2960 with
// every optional tool but dep_quant / sign_data_hiding off) for 32 x 32
// coding units in raster order: luma mode against the MPM list of the left
// neighbour's mode, chroma mode, cbfs (Cb, Cr, Y), then per coded TB its
// transform_skip_flag and residual. Returns 0, or a negative code for
// records the syntax cannot carry.
int mt_write(const vvcg_cu_rec* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
             uint32_t opts, std::vector<uint8_t>* out) {
  if (w % 32 || h % 32 || w <= 0 || h <= 0) return -1;
  const bool dq = opts & VVCG_SLICE_DEP_QUANT, sdh = opts & VVCG_SLICE_SIGN_HIDING;
  const CScan ls = coeff_scan(32, 32), cs = coeff_scan(16, 16);
  Encoder e;
  CtxStore m(qp);
  std::vector<int32_t> c;
  const int gw = w / 32, gh = h / 32;
  for (int k = 0; k < gw * gh; k++) {
    const vvcg_cu_rec& r = cus[k];
    if (r.luma_mode > 66 || (r.tu_tools >> 3)) return -2;
    uint8_t mpm[6];
    derive_intra_mpms(k % gw ? cus[k - 1].luma_mode : -1, -1, mpm);
    write_full_luma_mode(e, m, r.luma_mode, mpm);
    if (!write_chroma_mode(e, m, r.chroma_mode, r.luma_mode)) return -3;
    const bool cbf[3] = {(r.cbf & 1) != 0, (r.cbf & 2) != 0, (r.cbf & 4) != 0};
    e.bin(cbf[1], m.models[kCtxQtCbfCb]);
    e.bin(cbf[2], m.models[kCtxQtCbfCr + (cbf[1] ? 1 : 0)]);
    e.bin(cbf[0], m.models[kCtxQtCbfY]);
    for (int q = 0; q < 3; q++) {
      if (!cbf[q]) continue;
      const int rc = write_tb(e, m, q ? cs : ls, levels, num_levels, r.level_off[q], q ? 256 : 1024, q == 0,
                              (r.tu_tools >> q) & 1, dq, sdh, c);
      if (rc) return rc;
    }
  }
  e.terminate(true);
  *out = e.finish_and_align();
  return 0;
}

// The slice data encode_inter_picture writes (slice.rs:3451-3536, P slice,
// SAO / ALF / joint Cb-Cr off) for one coding unit per 32 x 32 CTU: the skip
// flag (context from the left and above CTUs' skip flags), and unless
// skipped pred_mode_flag (inter), general_merge_flag, for AMVP coding units
// the mvd, mvp_l0_flag and rqt_root_cbf, then the cbfs (tu_y_coded_flag only
// when a chroma cbf is set, else inferred 1) and each coded TB's
// transform_skip_flag and residual. A record is a skip coding unit when it
// is merge with no cbf. A record with flags bit 0x80 (not a vvcg_inter_cu
// flag) writes pred_mode_flag 1 instead, an intra coding unit, and ends the
// slice data there: the input of the parser's rejection test. Returns 0, or
// a negative code for records the syntax cannot carry.
int p_write(const vvcg_inter_cu* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
            uint32_t opts, std::vector<uint8_t>* out) {
  if (w % 32 || h % 32 || w <= 0 || h <= 0) return -1;
  const bool dq = opts & VVCG_SLICE_DEP_QUANT, sdh = opts & VVCG_SLICE_SIGN_HIDING;
  const CScan ls = coeff_scan(32, 32), cs = coeff_scan(16, 16);
  Encoder e;
  CtxStore m(qp, kCtxInitP);
  std::vector<int32_t> c;
  const int gw = w / 32, gh = h / 32;
  std::vector<char> skip(gw * gh, 0);
  for (int k = 0; k < gw * gh; k++) {
    const vvcg_inter_cu& r = cus[k];
    const int gx = k % gw, gy = k / gw;
    const bool merge = (r.flags & VVCG_INTER_CU_MERGE) != 0, any_cbf = (r.cbf & 7) != 0;
    const bool cu_skip = merge && !any_cbf;
    if (((r.flags & VVCG_INTER_CU_SKIP) != 0) != cu_skip || (r.tu_tools >> 3) || r.mvp_idx > 1) return -2;
    const int sctx = kCtxSkipFlag + (gx > 0 && skip[k - 1]) + (gy > 0 && skip[k - gw]);
    if (r.flags & 0x80) {  // test hook: an intra coding unit (pred_mode_flag 1), where the syntax ends
      e.bin(false, m.models[sctx]);
      e.bin(true, m.models[kCtxPredMode]);
      break;
    }
    e.bin(cu_skip, m.models[sctx]);
    skip[k] = cu_skip;
    if (cu_skip) continue;
    e.bin(false, m.models[kCtxPredMode]);
    e.bin(merge, m.models[kCtxMergeFlag]);
    if (!merge) {
      write_mvd(e, m, r.mvd);
      e.bin(r.mvp_idx != 0, m.models[kCtxMvpIdx]);
      e.bin(any_cbf, m.models[kCtxQtRootCbf]);
    }
    if (!any_cbf) continue;
    const bool cbf[3] = {(r.cbf & 1) != 0, (r.cbf & 2) != 0, (r.cbf & 4) != 0};
    e.bin(cbf[1], m.models[kCtxQtCbfCb]);
    e.bin(cbf[2], m.models[kCtxQtCbfCr + (cbf[1] ? 1 : 0)]);
    if (cbf[1] || cbf[2])
      e.bin(cbf[0], m.models[kCtxQtCbfY]);
    else if (!cbf[0])
      return -3;  // cannot happen: any_cbf
    for (int q = 0; q < 3; q++) {
      if (!cbf[q]) continue;
      const int rc = write_tb(e, m, q ? cs : ls, levels, num_levels, r.level_off[q], q ? 256 : 1024, q == 0,
                              (r.tu_tools >> q) & 1, dq, sdh, c);
      if (rc) return rc;
    }
  }
  e.terminate(true);
  *out = e.finish_and_align();
  return 0;
}

// The slice data encode_picture writes (slice.rs:407-455) for records in the
// frame path's strict layout. Returns 0, or a negative code for records the
// syntax cannot carry.
int strict_write(const vvcg_cu_rec* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                 std::vector<uint8_t>* out) {
  if (w % 32 || h % 32) return -1;
  const CScan ls = coeff_scan(32, 32), cs = coeff_scan(16, 16);
  Encoder e;
  CtxStore m(qp);
  std::vector<int32_t> c[3] = {std::vector<int32_t>(1024), std::vector<int32_t>(256), std::vector<int32_t>(256)};
  for (int k = 0; k < (w / 32) * (h / 32); k++) {
    const vvcg_cu_rec& r = cus[k];
    if (r.luma_mode > 66 || r.chroma_mode > 66) return -2;
    write_luma_mode(e, m, r.luma_mode);
    if (r.chroma_mode == r.luma_mode) {
      e.bin(false, m.models[kCtxIntraChromaPredMode]);
    } else {
      static const int cand[4] = {0, 50, 18, 1};
      int idx = -1;
      for (int i = 0; i < 4; i++)
        if ((cand[i] == r.luma_mode ? 66 : cand[i]) == r.chroma_mode) idx = i;
      if (idx < 0) return -3;
      e.bin(true, m.models[kCtxIntraChromaPredMode]);
      e.bypass_bins((uint32_t)idx, 2);
    }
    const bool cbf[3] = {(r.cbf & 1) != 0, (r.cbf & 2) != 0, (r.cbf & 4) != 0};
    e.bin(cbf[1], m.models[kCtxQtCbfCb]);
    e.bin(cbf[2], m.models[kCtxQtCbfCr + (cbf[1] ? 1 : 0)]);
    e.bin(cbf[0], m.models[kCtxQtCbfY]);
    const uint32_t t = r.tu_tools;
    bool ts[3];
    Constraints con;
    for (int q = 0; q < 3; q++) {
      ts[q] = cbf[q] && ((t >> q) & 1);
      if (!cbf[q]) continue;
      const int n = q ? 256 : 1024;
      if (r.level_off[q] < 0 || (uint64_t)r.level_off[q] + n > num_levels) return -4;
      bool any = false;
      for (int i = 0; i < n; i++) {
        c[q][i] = levels[r.level_off[q] + i];
        any |= c[q][i] != 0;
      }
      if (!any) return -5;  // a coded TB needs a nonzero level
      const CScan& s = q ? cs : ls;
      e.bin(ts[q], m.models[kCtxTransformSkipFlag + (q ? 1 : 0)]);
      if (ts[q])
        write_ts(e, m, s, c[q].data());
      else
        write_residual(e, m, s, c[q].data(), q == 0, false, false);
      con.update(s, c[q].data(), q == 0, ts[q]);
    }
    const int mts = (t >> VVCG_CU_MTS_SHIFT) & 7, lfnst = t >> VVCG_CU_LFNST_SHIFT;
    const bool any_ts = ts[0] || ts[1] || ts[2];
    if (!any_ts && con.lfnst_last && !con.vl[0] && !con.vl[1]) {
      e.bin(lfnst != 0, m.models[kCtxLfnstIdx]);
      if (lfnst) e.bin(lfnst == 2, m.models[kCtxLfnstIdx + 2]);
    } else if (lfnst) {
      return -6;
    }
    if (!(any_ts && ts[0]) && !con.vmts && con.mts_last && lfnst == 0) {
      e.bin(mts != 0, m.models[kCtxMtsIdx]);
      if (mts)
        for (int i = 0; i < 3; i++) {
          const bool more = mts > 1 + i;
          e.bin(more, m.models[kCtxMtsIdx + 1 + i]);
          if (!more) break;
        }
    } else if (mts) {
      return -7;
    }
  }
  e.terminate(true);
  *out = e.finish_and_align();
  return 0;
}

// One residual_coding or residual_ts_coding of a w x h block (raster levels,
// at least one nonzero) on fresh I-slice contexts at qp, then the
// terminating bin and the byte alignment.
int block_write(const int32_t* c, int w, int h, bool luma, bool dq, bool sdh, bool ts, int qp,
                std::vector<uint8_t>* out) {
  const CScan s = coeff_scan(w, h);
  bool any = false;
  for (int i = 0; i < w * h; i++) any |= c[i] != 0;
  if (!any) return -1;
  Encoder e;
  CtxStore m(qp);
  if (ts)
    write_ts(e, m, s, c);
  else
    write_residual(e, m, s, c, luma, dq, sdh);
  e.terminate(true);
  *out = e.finish_and_align();
  return 0;
}

}  // namespace orc
