// Intra prediction of the general decoding path (crates/rustmpeg-video/src/
// vvc/decode_general.rs), one warp per transform block: reference samples
// with the decoded-map availability and nearest-available substitution of
// Gen::gather_len (:4260-4341) and Gen::gather_mrl (:4542-4632), the ISP
// reference lengths of isp_refs (:4634-4648), predict_luma (:4650-4732),
// predict_chroma (:4734-4793), Gen::cclm_predict (:4372-4537) and the
// shared 4-wide region of narrow vertical ISP sub-partitions (reconstruct_tu,
// :4001-4024). The predictors are those of predict.rs (planar :1688, DC
// :1722, PDPC :1739, predict_angular_with_params_bd :1776-1958, BDPCM :1993).
#pragma once
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

constexpr int kGiWarps = 4;
constexpr int kGiRef = 136;   // longest reference row: 128 ISP samples + 5, or 2 x 64 + 3 + 4 (MRL)
constexpr int kGiBuf = 520;   // angular buffer: base + 2 max(w, h) + 2 max(refW, refH) + 64 <= 516

struct GenIntraArgs {
  vvcg_gen_intra_state st;
  const vvcg_gen_intra_req* reqs;
  int32_t n;
  int16_t* out;
};

struct GiWs {
  int16_t ra[kGiBuf], rl[kGiBuf];  // angular main / side buffers
  int16_t above[kGiRef], left[kGiRef];  // gathered references (gather_len)
  int16_t rowa[kGiRef], rowl[kGiRef];   // MrlRefSamples rows
  int16_t ba[kGiRef], bl[kGiRef];       // base refs for planar / DC (filtered or not)
  int tl, btl, nrowa, nrowl, off;
};

struct GiAng {
  int angle, abs_inv, scale, ref_w, ref_h;
  bool ver, ref_filter, interp, pdpc;
};

// init_angular_params (predict.rs:1608-1685)
__device__ __forceinline__ GiAng gi_ang_params(int dir, int pw, int ph, int cw, int ch, bool luma, int mrl, bool isp) {
  GiAng p;
  const int bw = (isp && luma) ? cw : pw, bh = (isp && luma) ? ch : ph;
  int mode = dir;
  if (dir > 1 && dir <= 66) {  // get_modified_wide_angle (predict.rs:1405-1422)
    const int delta = abs(floor_log2(bw) - floor_log2(bh));
    if (delta < 6) {
      const int s = delta == 0 ? 0 : delta == 1 ? 6 : delta == 2 ? 10 : delta == 3 ? 12 : delta == 4 ? 14 : 15;
      if (bw > bh && dir < 2 + s)
        mode = dir + 65;
      else if (bh > bw && dir > 66 - s)
        mode = dir - 65;
    }
  }
  p.ver = mode >= 34;
  const int mri = luma ? mrl : 0;
  p.pdpc = pw >= 4 && ph >= 4 && mri == 0;
  const int am = p.ver ? mode - 50 : -(mode - 18);
  const int absm = min(31, abs(am));
  const int abs_ang = c_ang_table[absm];
  p.abs_inv = c_inv_ang_table[absm];
  p.angle = (am < 0 ? -1 : 1) * abs_ang;
  p.scale = 0;
  if (am < 0) {
    p.pdpc = false;
  } else if (am > 0) {
    const int side = p.ver ? ph : pw;
    const int inv_term = floor_log2((unsigned)max(1, 3 * p.abs_inv - 2)) - 8;
    p.scale = min(2, floor_log2((unsigned)side) - inv_term);
    if (p.scale < 0) p.pdpc = false;
  }
  p.ref_filter = false;
  p.interp = false;
  if (luma && !isp && mri == 0 && dir > 1) {
    const int diff = min(abs(mode - 18), abs(mode - 50));
    const int l2 = (floor_log2(pw) + floor_log2(ph)) >> 1;
    if (diff > c_intra_filter_thr[min(7, l2)]) {
      const bool integer = (abs_ang & 0x1F) == 0;
      p.ref_filter = integer;
      p.interp = !integer;
    }
  }
  p.ref_w = (isp && luma) ? cw + pw : 2 * pw;
  p.ref_h = (isp && luma) ? ch + ph : 2 * ph;
  return p;
}

__device__ __forceinline__ bool gi_decoded(const vvcg_gen_intra_state& S, bool luma, int x, int y) {
  if (x < 0 || y < 0) return false;
  if (luma) {
    if (x >= (int)S.width || y >= (int)S.height) return false;
    return S.dec_y[(size_t)(y >> 2) * (S.width >> 2) + (x >> 2)] != 0;
  }
  if (x >= (int)(S.width >> 1) || y >= (int)(S.height >> 1)) return false;
  return S.dec_c[(size_t)y * (S.width >> 1) + x] != 0;
}

__device__ __forceinline__ int gi_get(const vvcg_gen_intra_state& S, int c, int x, int y) {
  return S.plane[c][(size_t)y * S.stride[c] + x];
}

// One side of Gen::gather_len / gather_mrl: dst[k] (k < len) = the sample at
// position k when available, else the nearest available one before it, else
// `fb` (the other fallbacks, resolved by the caller). `av` / `pos` give a
// position's availability and plane coordinates. Returns the first available
// sample (or -1) through *first.
template <class Avail, class Pos>
__device__ void gi_fill_side(const vvcg_gen_intra_state& S, int c, int len, int16_t* dst, Avail av, Pos pos,
                             int* first_val) {
  const int lane = threadIdx.x & 31;
  int carry = -1;  // value of the last available position of earlier chunks
  int first = -1;
  const int pw = c ? (int)S.width >> 1 : (int)S.width, ph = c ? (int)S.height >> 1 : (int)S.height;
  for (int k0 = 0; k0 < len; k0 += 32) {
    const int k = k0 + lane;
    // the sample is loaded with the availability lookup, not after it (one
    // memory round trip instead of two); unavailable ones are dropped
    int px = 0, py = 0;
    if (k < len) pos(k, &px, &py);
    const bool inplane = k < len && px >= 0 && py >= 0 && px < pw && py < ph;
    int v = inplane ? gi_get(S, c, px, py) : -1;
    const bool a = k < len && av(k);
    if (!a) v = -1;
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, a);
    if (first < 0 && m) first = __shfl_sync(0xFFFFFFFFu, v, __ffs(m) - 1);
    const uint32_t below = m & ((1u << lane) - 1u);
    const int src = below ? 31 - __clz(below) : -1;
    const int pv = __shfl_sync(0xFFFFFFFFu, v, src < 0 ? 0 : src);
    if (k < len) dst[k] = (int16_t)(a ? v : (src >= 0 ? pv : carry));
    if (m) carry = __shfl_sync(0xFFFFFFFFu, v, 31 - __clz(m));
  }
  *first_val = first;
  __syncwarp();
}

// Gen::gather_len (decode_general.rs:4260-4341) into W.above / W.left / W.tl.
__device__ void gi_gather_len(const vvcg_gen_intra_state& S, int c, bool luma, int x, int y, int top_len,
                              int left_len, GiWs& W) {
  const int lane = threadIdx.x & 31;
  const int pw = c ? (int)S.width >> 1 : (int)S.width, ph = c ? (int)S.height >> 1 : (int)S.height;
  const int d = 1 << (S.bit_depth - 1);
  int ft, fl;
  gi_fill_side(S, c, top_len, W.above,
               [&](int k) { return y > 0 && x + k < pw && gi_decoded(S, luma, x + k, y - 1); },
               [&](int k, int* px, int* py) { *px = x + k; *py = y - 1; }, &ft);
  gi_fill_side(S, c, left_len, W.left,
               [&](int k) { return x > 0 && y + k < ph && gi_decoded(S, luma, x - 1, y + k); },
               [&](int k, int* px, int* py) { *px = x - 1; *py = y + k; }, &fl);
  const bool tl = x > 0 && y > 0 && gi_decoded(S, luma, x - 1, y - 1);
  const bool any = ft >= 0 || fl >= 0 || tl;
  // positions with nothing available before them: first_top / first_left / dc
  const int fa = ft >= 0 ? ft : fl >= 0 ? fl : d, flb = fl >= 0 ? fl : ft >= 0 ? ft : d;
  for (int k = lane; k < top_len; k += 32)
    if (!any) W.above[k] = (int16_t)d; else if (W.above[k] < 0) W.above[k] = (int16_t)fa;
  for (int k = lane; k < left_len; k += 32)
    if (!any) W.left[k] = (int16_t)d; else if (W.left[k] < 0) W.left[k] = (int16_t)flb;
  if (lane == 0) W.tl = tl ? gi_get(S, c, x - 1, y - 1) : fa;
  __syncwarp();
}

// MrlRefSamples::from_ref_samples (predict.rs:1058-1075) of W.above / W.left.
__device__ void gi_rows_from_refs(int top_len, int left_len, GiWs& W) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < top_len + 5; i += 32) W.rowa[i] = i == 0 ? (int16_t)W.tl : W.above[min(i - 1, top_len - 1)];
  for (int i = lane; i < left_len + 5; i += 32) W.rowl[i] = i == 0 ? (int16_t)W.tl : W.left[min(i - 1, left_len - 1)];
  if (lane == 0) {
    W.nrowa = top_len + 5;
    W.nrowl = left_len + 5;
    W.off = 0;
  }
  __syncwarp();
}

// Gen::gather_mrl (decode_general.rs:4542-4632) into W.rowa / W.rowl.
__device__ void gi_gather_mrl(const vvcg_gen_intra_state& S, int x, int y, int w, int h, int mrl, GiWs& W) {
  const int lane = threadIdx.x & 31;
  const int d = 1 << (S.bit_depth - 1), off = 1 + mrl, al = 2 * w, ll = 2 * h;
  int ft, fl;
  gi_fill_side(S, 0, al, W.above,
               [&](int k) { return y >= off && x + k < (int)S.width && gi_decoded(S, true, x + k, y - off); },
               [&](int k, int* px, int* py) { *px = x + k; *py = y - off; }, &ft);
  gi_fill_side(S, 0, ll, W.left,
               [&](int k) { return x >= off && y + k < (int)S.height && gi_decoded(S, true, x - off, y + k); },
               [&](int k, int* px, int* py) { *px = x - off; *py = y + k; }, &fl);
  const bool tl = x >= off && y >= off && gi_decoded(S, true, x - off, y - off);
  const int fa = ft >= 0 ? ft : fl >= 0 ? fl : d, flb = fl >= 0 ? fl : ft >= 0 ? ft : d;
  const int fb = fa;  // the corner fallback: first_top, first_left, dc
  for (int i = lane; i < al + off + 4; i += 32) {
    int v;
    if (i < off) {
      v = tl ? gi_get(S, 0, x - off + i, y - off) : fb;
    } else {
      const int k = min(i - off, al - 1);
      v = W.above[k] < 0 ? fa : W.above[k];
    }
    W.rowa[i] = (int16_t)v;
  }
  for (int i = lane; i < ll + off + 4; i += 32) {
    int v;
    if (i < off) {
      v = tl ? gi_get(S, 0, x - off, y - off + i) : fb;
    } else {
      const int k = min(i - off, ll - 1);
      v = W.left[k] < 0 ? flb : W.left[k];
    }
    W.rowl[i] = (int16_t)v;
  }
  if (lane == 0) {
    W.nrowa = al + off + 4;
    W.nrowl = ll + off + 4;
    W.off = mrl;
  }
  __syncwarp();
}

// predict_angular_with_params_bd (predict.rs:1776-1958) from W.rowa / W.rowl
// with reference line mri; sink(i, v) per sample (raster of the w x h block).
template <class Sink>
__device__ void gi_angular(const GiAng& P, int w, int h, bool luma, int mri, int bd, GiWs& W, Sink sink) {
  const int lane = threadIdx.x & 31;
  const int def = 1 << (bd - 1), maxv = (1 << bd) - 1;
  const int base = max(h, w) + 4;
  const int len = base + 2 * max(w, h) + 2 * max(P.ref_w, P.ref_h) + 64;
  const int na = W.nrowa, nl = W.nrowl;
  const int a_hi = P.angle < 0 ? w + 1 + mri : P.ref_w + mri;
  const int l_hi = P.angle < 0 ? h + 1 + mri : P.ref_h + mri;
  for (int i = lane; i < len; i += 32) {
    const int x = i - base;
    W.ra[i] = (x >= 0 && x <= a_hi) ? W.rowa[min(x, na - 1)] : (int16_t)def;
    W.rl[i] = (x >= 0 && x <= l_hi) ? W.rowl[min(x, nl - 1)] : (int16_t)def;
  }
  __syncwarp();
  const bool ver = P.ver;
  if (P.angle < 0) {
    const int side = ver ? h : w;
    for (int k = -side + lane; k <= -1; k += 32) {
      const int proj = min((-k * P.abs_inv + 256) >> 9, side);
      if (ver)
        W.ra[base + k] = W.rl[base + proj];
      else
        W.rl[base + k] = W.ra[base + proj];
    }
  } else {
    const int lr = floor_log2(w) - floor_log2(h);
    const int s = max(0, ver ? lr : -lr);
    const int max_index = (mri << s) + 2;
    const int ref_length = ver ? P.ref_w : P.ref_h;
    int16_t* r = ver ? W.ra : W.rl;
    const int16_t v = r[base + ref_length + mri];
    for (int z = 1 + lane; z <= max_index; z += 32) r[base + ref_length + mri + z] = v;
  }
  __syncwarp();
  const int mb = base + mri, sb = base + mri;
  const int16_t* rm = ver ? W.ra : W.rl;
  const int16_t* rs = ver ? W.rl : W.ra;
  const int ww = ver ? w : h, wh = ver ? h : w;
  const bool int_slope = (abs(P.angle) & 0x1F) == 0;
  const int pscale = max(P.scale, 0);
  const int plimit = min(3 << pscale, ww);
  const int scale0 = (floor_log2(ww) + floor_log2(wh) - 2) >> 2;
  for (int i = lane; i < w * h; i += 32) {
    const int r = i / w, c = i - r * w;
    const int x = ver ? c : r, y = ver ? r : c;
    int v;
    if (P.angle == 0) {
      v = rm[mb + x + 1];
      if (P.pdpc && scale0 >= 0 && x < min(3 << scale0, ww)) {
        const int wl = 32 >> ((2 * x) >> scale0);
        v = clampi(v + ((wl * (rs[sb + 1 + y] - rm[mb]) + 32) >> 6), 0, maxv);
      }
    } else {
      const int dp = P.angle * (y + 1 + mri);
      const int di = dp >> 5, df = dp & 31;
      if (!int_slope) {
        if (luma) {
          int f0, f1, f2, f3;
          if (P.interp) {
            f0 = 16 - (df >> 1);
            f1 = 32 - (df >> 1);
            f2 = 16 + (df >> 1);
            f3 = df >> 1;
          } else {
            f0 = c_chroma_taps4[df * 4];
            f1 = c_chroma_taps4[df * 4 + 1];
            f2 = c_chroma_taps4[df * 4 + 2];
            f3 = c_chroma_taps4[df * 4 + 3];
          }
          const int b = mb + di + x;
          v = clampi((f0 * rm[b] + f1 * rm[b + 1] + f2 * rm[b + 2] + f3 * rm[b + 3] + 32) >> 6, 0, maxv);
        } else {
          const int b = mb + di + x + 1;
          v = rm[b] + ((df * (rm[b + 1] - rm[b]) + 16) >> 5);
        }
      } else {
        v = rm[mb + di + x + 1];
      }
      if (P.pdpc && x < plimit) {
        const int sum = 256 + (x + 1) * P.abs_inv;
        const int wl = 32 >> ((2 * x) >> pscale);
        const int li = min(sb + y + (sum >> 9) + 1, len - 1);
        v = clampi(v + ((wl * (rs[li] - v) + 32) >> 6), 0, maxv);
      }
    }
    sink(i, v);
  }
  __syncwarp();
}

// Planar / DC (predict.rs:1688-1736) on W.ba / W.bl / W.btl, PDPC when asked.
template <class Sink>
__device__ void gi_planar_dc(bool planar, int w, int h, bool pdpc, GiWs& W, Sink sink) {
  const int lane = threadIdx.x & 31;
  const int lw = floor_log2(w), lh = floor_log2(h);
  const int tr = W.ba[w], bl = W.bl[h];
  int dcv = 0;
  if (!planar) {
    const int denom = w == h ? (w << 1) : max(w, h);
    int s = 0;
    if (w >= h)
      for (int i = lane; i < w; i += 32) s += W.ba[i];
    if (w <= h)
      for (int i = lane; i < h; i += 32) s += W.bl[i];
    s = __reduce_add_sync(0xFFFFFFFFu, s);
    dcv = (s + (denom >> 1)) >> floor_log2(denom);
  }
  const int sc = max(lw + lh - 2, 0) >> 2;
  for (int i = lane; i < w * h; i += 32) {
    const int y = i >> lw, x = i & (w - 1);
    int v;
    if (planar) {
      const int hor = (W.bl[y] << lw) + (x + 1) * (tr - W.bl[y]);
      const int vert = (W.ba[x] << lh) + (y + 1) * (bl - W.ba[x]);
      v = ((hor << lh) + (vert << lw) + (1 << (lw + lh))) >> (1 + lw + lh);
    } else {
      v = dcv;
    }
    if (pdpc) {
      const int wt = 32 >> min((y * 2) >> sc, 31), wl = 32 >> min((x * 2) >> sc, 31);
      v = v + ((wl * (W.bl[y] - v) + wt * (W.ba[x] - v) + 32) >> 6);
    }
    sink(i, v);
  }
  __syncwarp();
}

// RefSamples::filtered (predict.rs:1233-1267) of `n` above / left samples
// from src arrays (with top-left) into W.ba / W.bl / W.btl.
__device__ void gi_filter_into_base(const int16_t* sa, const int16_t* sl, int tlv, int na, int nl, GiWs& W) {
  const int lane = threadIdx.x & 31;
  for (int j = lane; j < na; j += 32)
    W.ba[j] = j + 1 < na ? (int16_t)(((j == 0 ? tlv : sa[j - 1]) + 2 * sa[j] + sa[j + 1] + 2) >> 2) : sa[j];
  for (int j = lane; j < nl; j += 32)
    W.bl[j] = j + 1 < nl ? (int16_t)(((j == 0 ? tlv : sl[j - 1]) + 2 * sl[j] + sl[j + 1] + 2) >> 2) : sl[j];
  if (lane == 0) W.btl = (2 * tlv + sa[0] + sl[0] + 2) >> 2;
  __syncwarp();
}

// derive_cclm_params_from_4_samples (predict.rs:2088-2177); sl / sc of count
__device__ __forceinline__ void gi_cclm_params(int* sl, int* sc, int cnt, int bd, int* a, int* b, int* shift) {
  if (cnt == 0) {
    *a = 0;
    *b = 1 << (bd - 1);
    *shift = 0;
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
  int mn0 = 0, mn1 = 2, mx0 = 1, mx1 = 3, t;
  if (sl[mn0] > sl[mn1]) { t = mn0; mn0 = mn1; mn1 = t; }
  if (sl[mx0] > sl[mx1]) { t = mx0; mx0 = mx1; mx1 = t; }
  if (sl[mn0] > sl[mx1]) {
    t = mn0; mn0 = mx0; mx0 = t;
    t = mn1; mn1 = mx1; mx1 = t;
  }
  if (sl[mn1] > sl[mx0]) { t = mn1; mn1 = mx0; mx0 = t; }
  const int min_l = (sl[mn0] + sl[mn1] + 1) >> 1, min_c = (sc[mn0] + sc[mn1] + 1) >> 1;
  const int max_l = (sl[mx0] + sl[mx1] + 1) >> 1, max_c = (sc[mx0] + sc[mx1] + 1) >> 1;
  const int diff = max_l - min_l;
  if (diff > 0) {
    const int diff_c = max_c - min_c;
    int x = floor_log2((unsigned)diff);
    const int norm = ((diff << 4) >> x) & 15;
    const int v = (int)c_cclm_div_sig[norm] | 8;
    if (norm != 0) x += 1;
    const int y = diff_c == 0 ? 1 : floor_log2((unsigned)abs(diff_c)) + 1;
    const int add = (1 << y) >> 1;
    int aa = (diff_c * v + add) >> y;
    int sh = 3 + x - y;
    if (sh < 1) {
      sh = 1;
      aa = aa == 0 ? 0 : (aa < 0 ? -15 : 15);
    }
    *a = aa;
    *b = min_c - ((aa * min_l) >> sh);
    *shift = sh;
  } else {
    *a = 0;
    *b = min_c;
    *shift = 0;
  }
}

// Gen::cclm_predict (decode_general.rs:4372-4537); mode 0 LM, 1 LM-L, 2 LM-T.
template <class Sink>
__device__ void gi_cclm(const vvcg_gen_intra_state& S, int comp, int mode, int xc, int yc, int w, int h, Sink sink) {
  const int lane = threadIdx.x & 31;
  const int bd = S.bit_depth, mid = 1 << (bd - 1), maxv = (1 << bd) - 1;
  const int xtb = xc * 2, ytb = yc * 2;
  const bool al = xc > 0 && gi_decoded(S, false, xc - 1, yc);
  const bool at = yc > 0 && gi_decoded(S, false, xc, yc - 1);
  const bool ctb = S.ctu_size > 0 && (ytb & (S.ctu_size - 1)) == 0;
  const bool vc = S.vert_collocated != 0;
  auto py = [&](int x, int y) -> int {
    if (y < 0 && !at) y = 0;
    if (x < 0 && !al) x = 0;
    return gi_get(S, 0, xtb + x, ytb + y);
  };
  // numTopRight / numLeftBelow: the run of decoded samples from w / h on
  int ntr = 0, nlb = 0;
  if (mode == 2 && at) {
    const bool dd = lane < w && gi_decoded(S, false, xc + w + lane, yc - 1);
    const uint32_t m = ~__ballot_sync(0xFFFFFFFFu, dd);
    ntr = min(w, __ffs(m) - 1 < 0 ? 32 : __ffs(m) - 1);
  }
  if (mode == 1 && al) {
    const bool dd = lane < h && gi_decoded(S, false, xc - 1, yc + h + lane);
    const uint32_t m = ~__ballot_sync(0xFFFFFFFFu, dd);
    nlb = min(h, __ffs(m) - 1 < 0 ? 32 : __ffs(m) - 1);
  }
  int nt, nl;
  if (mode == 0) {
    nt = at ? w : 0;
    nl = al ? h : 0;
  } else if (mode == 2) {
    nt = at ? w + min(ntr, h) : 0;
    nl = 0;
  } else {
    nt = 0;
    nl = al ? h + min(nlb, w) : 0;
  }
  const int is4n = !(at && al && mode == 0) ? 1 : 0;
  int sl[4] = {mid, mid, mid, mid}, sc[4] = {mid, mid, mid, mid};
  int count = 0;
  if (nt > 0) {
    const int start = nt >> (2 + is4n), step = max(1, nt >> (1 + is4n)), cnt = min(nt, (1 + is4n) << 1);
    for (int pos = 0; pos < cnt; pos++) {
      const int x = start + pos * step;
      if (x >= nt) break;
      const int lx = 2 * x;
      int ds;
      if (ctb)
        ds = (py(lx - 1, -1) + 2 * py(lx, -1) + py(lx + 1, -1) + 2) >> 2;
      else if (vc)
        ds = (py(lx, -3) + py(lx - 1, -2) + 4 * py(lx, -2) + py(lx + 1, -2) + py(lx, -1) + 4) >> 3;
      else
        ds = (py(lx - 1, -1) + py(lx - 1, -2) + 2 * py(lx, -1) + 2 * py(lx, -2) + py(lx + 1, -1) + py(lx + 1, -2) +
              4) >> 3;
      sl[count] = ds;
      sc[count] = gi_get(S, comp, xc + x, yc - 1);
      count++;
    }
  }
  if (nl > 0) {
    const int start = nl >> (2 + is4n), step = max(1, nl >> (1 + is4n)), cnt = min(nl, (1 + is4n) << 1);
    for (int pos = 0; pos < cnt; pos++) {
      const int y = start + pos * step;
      if (y >= nl) break;
      const int ly = 2 * y;
      int ds;
      if (vc)
        ds = (py(-2, ly - 1) + py(-3, ly) + 4 * py(-2, ly) + py(-1, ly) + py(-2, ly + 1) + 4) >> 3;
      else
        ds = (py(-3, ly) + py(-3, ly + 1) + 2 * py(-2, ly) + 2 * py(-2, ly + 1) + py(-1, ly) + py(-1, ly + 1) + 4) >> 3;
      sl[count] = ds;
      sc[count] = gi_get(S, comp, xc - 1, yc + y);
      count++;
    }
  }
  int a = 0, b = mid, shift = 0;
  if (count > 0) gi_cclm_params(sl, sc, count, bd, &a, &b, &shift);
  for (int i = lane; i < w * h; i += 32) {
    const int y = i / w, x = i - y * w;
    int v = mid;
    if (count > 0) {
      const int lx = 2 * x, ly = 2 * y;
      const int ds = vc ? (py(lx, ly - 1) + py(lx - 1, ly) + 4 * py(lx, ly) + py(lx + 1, ly) + py(lx, ly + 1) + 4) >> 3
                        : (py(lx - 1, ly) + py(lx - 1, ly + 1) + 2 * py(lx, ly) + 2 * py(lx, ly + 1) + py(lx + 1, ly) +
                           py(lx + 1, ly + 1) + 4) >> 3;
      v = clampi(((ds * a) >> shift) + b, 0, maxv);
    }
    sink(i, v);
  }
  __syncwarp();
}

// The prediction of one request, by the calling warp: emit(i, v) per sample
// (i: raster index in the w x h block), once every reference is in W.
template <class Emit>
__device__ void gi_predict_emit(const vvcg_gen_intra_state& S, const vvcg_gen_intra_req& R, GiWs& W, Emit emit) {
  const int lane = threadIdx.x & 31;
  const int bd = S.bit_depth;
  if (R.comp == 0) {
    // the 4-wide region of narrow vertical ISP sub-partitions
    const bool region = R.isp == VVCG_ISP_VER && (R.cu_w == 4 || (R.cu_w == 8 && R.cu_h > 4));
    const int px = region ? R.cu_x + ((R.x - R.cu_x) / 4) * 4 : R.x;
    const int pw = region ? 4 : R.w, ph = R.h, col0 = R.x - px;
    auto put = [&](int i, int v) {
      const int yy = i / pw, xx = i - yy * pw - col0;
      if (xx >= 0 && xx < R.w) emit(yy * R.w + xx, v);
    };
    if (R.bdpcm) {
      gi_gather_len(S, 0, true, px, R.y, 2 * pw, 2 * ph, W);
      for (int i = lane; i < pw * ph; i += 32) {
        const int yy = i / pw, xx = i - yy * pw;
        put(i, R.bdpcm == VVCG_BDPCM_VER ? W.above[xx] : W.left[yy]);
      }
      __syncwarp();
      return;
    }
    const bool isp = R.isp != VVCG_ISP_NONE;
    const int mrl = min((int)R.mrl, 2);
    if (isp) {
      gi_gather_len(S, 0, true, px, R.y, R.cu_w + pw, R.cu_h + ph, W);
      gi_rows_from_refs(R.cu_w + pw, R.cu_h + ph, W);
    } else if (mrl == 0) {
      gi_gather_len(S, 0, true, px, R.y, 2 * pw, 2 * ph, W);
      gi_rows_from_refs(2 * pw, 2 * ph, W);
    } else {
      gi_gather_mrl(S, px, R.y, pw, ph, mrl, W);
    }
    const int off = W.off;
    const int mode = R.mode;
    if (mode <= 1) {
      const bool filt = mode == 0 && mrl == 0 && !isp && pw * ph > 32;
      if (filt) {
        gi_filter_into_base(W.rowa + off + 1, W.rowl + off + 1, W.rowa[off], 2 * pw, 2 * ph, W);
      } else {
        for (int i = lane; i < 2 * pw; i += 32) W.ba[i] = W.rowa[off + 1 + i];
        for (int i = lane; i < 2 * ph; i += 32) W.bl[i] = W.rowl[off + 1 + i];
        __syncwarp();
      }
      gi_planar_dc(mode == 0, pw, ph, mrl == 0 && pw >= 4 && ph >= 4, W, put);
      return;
    }
    const GiAng P = gi_ang_params(min(mode, 66), pw, ph, R.cu_w, R.cu_h, true, mrl, isp);
    if (mrl == 0 && !isp && P.ref_filter) {
      // rows from the filtered base refs
      gi_filter_into_base(W.rowa + 1, W.rowl + 1, W.rowa[0], 2 * pw, 2 * ph, W);
      for (int i = lane; i < 2 * pw + 5; i += 32) W.rowa[i] = i == 0 ? (int16_t)W.btl : W.ba[min(i - 1, 2 * pw - 1)];
      for (int i = lane; i < 2 * ph + 5; i += 32) W.rowl[i] = i == 0 ? (int16_t)W.btl : W.bl[min(i - 1, 2 * ph - 1)];
      __syncwarp();
    }
    gi_angular(P, pw, ph, true, W.off, bd, W, put);  // the rows' reference line
    return;
  }
  // chroma
  auto put = [&](int i, int v) { emit(i, v); };
  const int w = R.w, h = R.h;
  if (R.mode >= 81 && R.mode <= 83) {
    gi_cclm(S, R.comp, R.mode - 81, R.x, R.y, w, h, put);
    return;
  }
  gi_gather_len(S, R.comp, false, R.x, R.y, 2 * w, 2 * h, W);
  if (R.mode <= 1) {
    for (int i = lane; i < 2 * w; i += 32) W.ba[i] = W.above[i];
    for (int i = lane; i < 2 * h; i += 32) W.bl[i] = W.left[i];
    __syncwarp();
    gi_planar_dc(R.mode == 0, w, h, w >= 4 && h >= 4, W, put);
    return;
  }
  gi_rows_from_refs(2 * w, 2 * h, W);
  const GiAng P = gi_ang_params(min((int)R.mode, 66), w, h, w, h, false, 0, false);
  gi_angular(P, w, h, false, 0, bd, W, put);
}

// The prediction of one request into out (w x h int16, row-major).
__device__ void gi_predict(const vvcg_gen_intra_state& S, const vvcg_gen_intra_req& R, int16_t* out, GiWs& W) {
  gi_predict_emit(S, R, W, [&](int i, int v) { out[i] = (int16_t)v; });
}

__global__ void __launch_bounds__(kGiWarps * 32) k_gen_intra(const __grid_constant__ GenIntraArgs A) {
  __shared__ GiWs ws[kGiWarps];
  const int warp = threadIdx.x >> 5;
  for (int q = blockIdx.x * kGiWarps + warp; q < A.n; q += gridDim.x * kGiWarps) {
    const vvcg_gen_intra_req R = A.reqs[q];
    gi_predict(A.st, R, A.out + R.out_off, ws[warp]);
  }
}

// Sequential reconstruction of groups of transform blocks (one group per
// warp, its blocks in order; groups are independent): each block is
// predicted (gi_predict), its residual added, clipped to the bit depth and
// stored into its plane, and its samples marked decoded, so the next block of
// the group (the next ISP sub-partition) predicts from them. Follows
// reconstruct_tu (decode_general.rs:3985-4096; the add / clip / set loop
// :4087-4093) and the decoded maps of mark_tu (:4891-4906).
struct GenReconArgs {
  vvcg_gen_intra_state st;
  const vvcg_gen_intra_req* reqs;
  const uint32_t* group_start;  // num_groups + 1 entries
  int32_t num_groups;
  const int16_t* res;           // per request w x h at out_off; null = no residual
  int16_t* pred;                // receives the predictions (w x h at out_off)
};

// One block of a sequential reconstruction: predicted (gi_predict), its
// residual added, clipped to the bit depth and stored into its plane, and its
// samples marked decoded for the blocks after it.
__device__ void gi_recon_block(const vvcg_gen_intra_state& S, const vvcg_gen_intra_req& R, int16_t* pred,
                               const int16_t* res, GiWs& ws, int lane) {
  const int maxv = (1 << S.bit_depth) - 1;
  gi_predict(S, R, pred, ws);
  __syncwarp();
  uint16_t* pl = const_cast<uint16_t*>(S.plane[R.comp]);
  const int st = (int)S.stride[R.comp];
  for (int i = lane; i < R.w * R.h; i += 32) {
    const int yy = i / R.w, xx = i - yy * R.w;
    const int v = (int)pred[i] + (res ? (int)res[i] : 0);
    pl[(size_t)(R.y + yy) * st + R.x + xx] = (uint16_t)clampi(v, 0, maxv);
  }
  // mark_tu's decoded maps: luma per 4x4 cell touched, chroma per sample
  if (R.comp == 0) {
    uint8_t* dm = const_cast<uint8_t*>(S.dec_y);
    const int cw = (int)S.width >> 2;
    const int x0 = R.x >> 2, x1 = min((R.x + R.w + 3) >> 2, cw), y0 = R.y >> 2;
    const int y1 = min((R.y + R.h + 3) >> 2, (int)S.height >> 2);
    for (int i = lane; i < (x1 - x0) * (y1 - y0); i += 32)
      dm[(size_t)(y0 + i / (x1 - x0)) * cw + x0 + i % (x1 - x0)] = 1;
  } else {
    uint8_t* dm = const_cast<uint8_t*>(S.dec_c);
    const int cw = (int)S.width >> 1;
    for (int i = lane; i < R.w * R.h; i += 32) dm[(size_t)(R.y + i / R.w) * cw + R.x + i % R.w] = 1;
  }
  __threadfence_block();
  __syncwarp();
}

// gi_recon_block without the prediction buffer: each predicted sample goes
// straight into the plane with its residual added and clipped.
__device__ void gi_recon_block_fused(const vvcg_gen_intra_state& S, const vvcg_gen_intra_req& R,
                                     const int16_t* __restrict__ res, GiWs& ws, int lane) {
  const int maxv = (1 << S.bit_depth) - 1;
  uint16_t* pl = const_cast<uint16_t*>(S.plane[R.comp]);
  const int st = (int)S.stride[R.comp];
  gi_predict_emit(S, R, ws, [&](int i, int v) {
    const int yy = i / R.w, xx = i - yy * R.w;
    pl[(size_t)(R.y + yy) * st + R.x + xx] = (uint16_t)clampi(v + (int)res[i], 0, maxv);
  });
  __syncwarp();
  if (R.comp == 0) {
    uint8_t* dm = const_cast<uint8_t*>(S.dec_y);
    const int cw = (int)S.width >> 2;
    const int x0 = R.x >> 2, x1 = min((R.x + R.w + 3) >> 2, cw), y0 = R.y >> 2;
    const int y1 = min((R.y + R.h + 3) >> 2, (int)S.height >> 2);
    for (int i = lane; i < (x1 - x0) * (y1 - y0); i += 32)
      dm[(size_t)(y0 + i / (x1 - x0)) * cw + x0 + i % (x1 - x0)] = 1;
  } else {
    uint8_t* dm = const_cast<uint8_t*>(S.dec_c);
    const int cw = (int)S.width >> 1;
    for (int i = lane; i < R.w * R.h; i += 32) dm[(size_t)(R.y + i / R.w) * cw + R.x + i % R.w] = 1;
  }
  __threadfence_block();
  __syncwarp();
}

__global__ void __launch_bounds__(kGiWarps * 32) k_gen_intra_recon(const __grid_constant__ GenReconArgs A) {
  __shared__ GiWs ws[kGiWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int g = blockIdx.x * kGiWarps + warp; g < A.num_groups; g += gridDim.x * kGiWarps)
    for (uint32_t q = A.group_start[g]; q < A.group_start[g + 1]; q++) {
      const vvcg_gen_intra_req R = A.reqs[q];
      gi_recon_block(A.st, R, A.pred + R.out_off, A.res ? A.res + R.out_off : nullptr, ws[warp], lane);
    }
}

// One dependency level of the general picture pass: each warp takes coding
// units (groups of blocks in decode order) of the level, from any picture of
// the batch, and reconstructs their blocks in order. The host puts a group
// in a later level than every earlier group whose samples it may read and
// every earlier group that may read its samples, so the decoded maps each
// block sees are those of the picture's sequential decode.
struct GenLevelArgs {
  const vvcg_gen_intra_state* states;  // per picture
  const vvcg_gen_intra_req* reqs;      // all blocks of the batch
  const uint32_t* group_first;         // per group: first block; group_first[g + 1] ends it
  const uint32_t* group_pic;           // per group: picture
  const uint32_t* level_groups;        // the groups of this level
  uint32_t n;
  const int16_t* res;                  // residuals at out_off (zero where uncoded)
  int16_t* pred;                       // predictions at out_off
};

__global__ void __launch_bounds__(kGiWarps * 32) k_gen_recon_level(const __grid_constant__ GenLevelArgs A) {
  __shared__ GiWs ws[kGiWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t i = blockIdx.x * kGiWarps + warp; i < A.n; i += gridDim.x * kGiWarps) {
    const uint32_t g = A.level_groups[i];
    const vvcg_gen_intra_state& S = A.states[A.group_pic[g]];
    for (uint32_t q = A.group_first[g]; q < A.group_first[g + 1]; q++) {
      const vvcg_gen_intra_req R = A.reqs[q];
      gi_recon_block_fused(S, R, A.res + R.out_off, ws[warp], lane);
    }
  }
}

}  // namespace vvcg
