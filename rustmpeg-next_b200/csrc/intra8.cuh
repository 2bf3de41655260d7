// Luma intra mode search of the 8-bit multi-tool encoder on the GPU:
// choose_luma_intra_pred_mode (crates/rustmpeg-video/src/vvc/predict.rs:
// 2737-2801) over Planar, DC and the 65 angular modes (or the 6 MPMs), then
// the encoder's MRL candidates (slice.rs:2698-2731): reference lines 1 and 2
// for mpm[1..5]. One CTA per block, one warp per candidate at a time; each
// warp builds the candidate's extended reference arrays in its own shared
// buffers exactly as predict_angular_with_params_bd (predict.rs:1776-1958)
// lays them out, then sums |source - prediction| over the block. The block's
// winner is the first candidate with the lowest sum (Planar wins ties), and an
// MRL candidate replaces it only with a strictly lower sum.
#pragma once
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

constexpr int kIsrWarps = 8;
constexpr int kIsrRow = 136;  // 2 * 64 + 3 + 4 + 1: longest MRL row
constexpr int kIsrBuf = 520;  // base + 2 max(w, h) + 2 max(refW, refH) + 64 for 64x64 (516)
constexpr int kIsrMaxCand = 67 + 10;

struct IsrArgs {
  const uint8_t* recon;
  const uint8_t* src;
  int64_t recon_stride, src_stride;
  int32_t width, height, n;
  const vvcg_intra_search_req* reqs;
  vvcg_intra_search_res* res;
};

// init_angular_params (predict.rs:1608-1685) for a luma w x h block without
// ISP and reference line mri.
struct Ang8 {
  int angle, abs_inv, scale;
  bool ver, ref_filter, interp, pdpc;
};
__device__ __forceinline__ Ang8 ang8_params(int dir, int w, int h, int mri) {
  Ang8 p;
  int mode = dir;
  if (dir > 1 && dir <= 66) {  // get_modified_wide_angle (predict.rs:1405-1422)
    const int delta = abs(floor_log2(w) - floor_log2(h));
    if (delta < 6) {
      const int shifts[6] = {0, 6, 10, 12, 14, 15};
      const int s = shifts[delta];
      if (w > h && dir < 2 + s)
        mode = dir + 65;
      else if (h > w && dir > 66 - s)
        mode = dir - 65;
    }
  }
  p.ver = mode >= 34;
  p.pdpc = mri == 0;  // w, h >= 4 here
  const int am = p.ver ? mode - 50 : -(mode - 18);
  const int absm = min(31, abs(am));
  const int abs_ang = c_ang_table[absm];
  p.abs_inv = c_inv_ang_table[absm];
  p.angle = (am < 0 ? -1 : 1) * abs_ang;
  p.scale = 0;
  if (am < 0) {
    p.pdpc = false;
  } else if (am > 0) {
    const int side = p.ver ? h : w;
    const int inv_term = floor_log2((unsigned)max(1, 3 * p.abs_inv - 2)) - 8;
    p.scale = min(2, floor_log2((unsigned)side) - inv_term);
    if (p.scale < 0) p.pdpc = false;
  }
  p.ref_filter = false;
  p.interp = false;
  if (mri == 0 && dir > 1) {
    const int diff = min(abs(mode - 18), abs(mode - 50));
    const int l2 = (floor_log2(w) + floor_log2(h)) >> 1;
    if (diff > c_intra_filter_thr[min(7, l2)]) {
      const bool integer = (abs_ang & 0x1F) == 0;
      p.ref_filter = integer;
      p.interp = !integer;
    }
  }
  return p;
}

struct IsrShared {
  uint8_t src[64 * 64];
  // reference rows as MrlRefSamples: [set][0 above / 1 left]; sets 0 / 1 are
  // line 0 unfiltered / filtered, 2 / 3 are lines 1 / 2
  int16_t row[4][2][kIsrRow];
  int16_t row_len[4][2];
  int16_t ref[2][2][128];  // RefSamples above / left, [unfiltered / filtered]
  int16_t tl[2];
  int16_t mrl_eff[2];
  int32_t dc;
  uint32_t sad[kIsrMaxCand];
  int16_t buf[kIsrWarps][2][kIsrBuf];  // a warp's ref_above / ref_left
};

// |source - prediction| summed over the block for one angular candidate
// (predict_angular_with_params_bd with 8-bit samples), by one warp.
__device__ uint32_t isr_angular_sad(IsrShared& S, int warp, int lane, int w, int h, int dir, int set, int mri) {
  const Ang8 P = ang8_params(dir, w, h, mri);
  int16_t* ra = S.buf[warp][0];
  int16_t* rl = S.buf[warp][1];
  const int16_t* rowa = S.row[set][0];
  const int16_t* rowl = S.row[set][1];
  const int na = S.row_len[set][0], nl = S.row_len[set][1];
  const int base = max(h, w) + 4;
  const int ref_w = 2 * w, ref_h = 2 * h;
  const int len = base + 2 * max(w, h) + 2 * max(ref_w, ref_h) + 64;
  const bool ver = P.ver;
  // copy ranges of the two arrays (everything else holds the 8-bit default 128)
  const int a_hi = P.angle < 0 ? w + 1 + mri : ref_w + mri;
  const int l_hi = P.angle < 0 ? h + 1 + mri : ref_h + mri;
  for (int i = lane; i < len; i += 32) {
    const int x = i - base;
    ra[i] = (x >= 0 && x <= a_hi) ? rowa[min(x, na - 1)] : (int16_t)128;
    rl[i] = (x >= 0 && x <= l_hi) ? rowl[min(x, nl - 1)] : (int16_t)128;
  }
  __syncwarp();
  if (P.angle < 0) {
    const int side = ver ? h : w;
    for (int k = -side + lane; k <= -1; k += 32) {
      const int proj = min((-k * P.abs_inv + 256) >> 9, side);
      if (ver)
        ra[base + k] = rl[base + proj];
      else
        rl[base + k] = ra[base + proj];
    }
  } else {
    const int lr = floor_log2(w) - floor_log2(h);
    const int s = max(0, ver ? lr : -lr);
    const int max_index = (mri << s) + 2;
    const int ref_length = ver ? ref_w : ref_h;
    int16_t* r = ver ? ra : rl;
    const int16_t v = r[base + ref_length + mri];
    for (int z = 1 + lane; z <= max_index; z += 32) r[base + ref_length + mri + z] = v;
  }
  __syncwarp();
  const int mb = base + mri, sb = base + mri;
  const int16_t* rm = ver ? ra : rl;
  const int16_t* rs = ver ? rl : ra;
  const int ww = ver ? w : h, wh = ver ? h : w;
  const bool int_slope = (abs(P.angle) & 0x1F) == 0;
  const int pscale = max(P.scale, 0);
  const int plimit = min(3 << pscale, ww);
  const int scale0 = (floor_log2(ww) + floor_log2(wh) - 2) >> 2;
  uint32_t sad = 0;
  for (int i = lane; i < w * h; i += 32) {
    const int r = i / w, c = i - r * w;  // block row / column
    const int x = ver ? c : r, y = ver ? r : c;
    int v;
    if (P.angle == 0) {
      v = rm[mb + x + 1];
      if (P.pdpc && scale0 >= 0 && x < min(3 << scale0, ww)) {
        const int wl = 32 >> ((2 * x) >> scale0);
        v = clampi(v + ((wl * (rs[sb + 1 + y] - rm[mb]) + 32) >> 6), 0, 255);
      }
    } else {
      const int dp = P.angle * (y + 1 + mri);
      const int di = dp >> 5, df = dp & 31;
      if (!int_slope) {
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
        v = clampi((f0 * rm[b] + f1 * rm[b + 1] + f2 * rm[b + 2] + f3 * rm[b + 3] + 32) >> 6, 0, 255);
      } else {
        v = rm[mb + di + x + 1];
      }
      if (P.pdpc && x < plimit) {
        const int sum = 256 + (x + 1) * P.abs_inv;
        const int wl = 32 >> ((2 * x) >> pscale);
        const int li = min(sb + y + (sum >> 9) + 1, len - 1);
        v = clampi(v + ((wl * (rs[li] - v) + 32) >> 6), 0, 255);
      }
    }
    sad += (uint32_t)abs((int)S.src[i] - v);
  }
  __syncwarp();  // the buffers are rebuilt for the warp's next candidate
  return sad;
}

// Planar (predict.rs:1688-1719) or DC (:1722-1736) with PDPC (:1739-1754).
__device__ uint32_t isr_planar_dc_sad(IsrShared& S, int lane, int w, int h, bool planar) {
  const int f = (planar && w * h > 32) ? 1 : 0;  // uses_reference_filter for luma Planar
  const int16_t* top = S.ref[f][0];
  const int16_t* left = S.ref[f][1];
  const int lw = floor_log2(w), lh = floor_log2(h);
  const int pscale = max(lw + lh - 2, 0) >> 2;
  const int tr = top[w], bl = left[h];
  uint32_t sad = 0;
  for (int i = lane; i < w * h; i += 32) {
    const int y = i >> lw, x = i & (w - 1);
    int v;
    if (planar) {
      const int hor = (left[y] << lw) + (x + 1) * (tr - left[y]);
      const int vert = (top[x] << lh) + (y + 1) * (bl - top[x]);
      v = ((hor << lh) + (vert << lw) + (1 << (lw + lh))) >> (1 + lw + lh);
    } else {
      v = S.dc;
    }
    const int wt = 32 >> min((y * 2) >> pscale, 31), wl = 32 >> min((x * 2) >> pscale, 31);
    v = v + ((wl * (left[y] - v) + wt * (top[x] - v) + 32) >> 6);
    sad += (uint32_t)abs((int)S.src[i] - v);
  }
  return sad;
}

__global__ void __launch_bounds__(kIsrWarps * 32) k_luma_intra_search_8(const __grid_constant__ IsrArgs A) {
  __shared__ IsrShared S;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int q = blockIdx.x; q < A.n; q += gridDim.x) {
    const vvcg_intra_search_req R = A.reqs[q];
    const int w = 1 << R.log2_w, h = 1 << R.log2_h, bx = (int)R.x, by = (int)R.y;
    const uint8_t* rec = A.recon;
    const int64_t rs = A.recon_stride;
    for (int i = t; i < w * h; i += blockDim.x)
      S.src[i] = A.src[(int64_t)(by + i / w) * A.src_stride + bx + (i % w)];
    // gather_references (predict.rs:1084-1134)
    const int above_len = by == 0 ? 0 : min(A.width - bx, 2 * w);
    const int left_len = bx == 0 ? 0 : min(A.height - by, h);
    const int a0 = above_len > 0 ? rec[(int64_t)(by - 1) * rs + bx] : 0;
    const int l0 = left_len > 0 ? rec[(int64_t)by * rs + bx - 1] : 0;
    for (int i = t; i < 2 * w; i += blockDim.x)
      S.ref[0][0][i] = above_len == 0 ? (left_len > 0 ? l0 : 128)
                                      : rec[(int64_t)(by - 1) * rs + bx + min(i, above_len - 1)];
    for (int i = t; i < 2 * h; i += blockDim.x)
      S.ref[0][1][i] = left_len == 0 ? (above_len > 0 ? a0 : 128)
                                     : rec[(int64_t)(by + min(i, left_len - 1)) * rs + bx - 1];
    if (t == 0)
      S.tl[0] = (above_len > 0 && left_len > 0) ? rec[(int64_t)(by - 1) * rs + bx - 1]
                : above_len > 0                  ? a0
                : left_len > 0                   ? l0
                                                 : 128;
    // MRL rows (gather_references_mrl, predict.rs:1141-1231) for lines 1, 2
    const bool mrl = (R.flags & VVCG_ISR_MRL) != 0;
    const int ctu = 1 << R.log2_ctu;
    const bool ctu_top = (by & (ctu - 1)) == 0;
    if (mrl && !ctu_top) {
      for (int e = 1; e <= 2; e++) {
        const int off = 1 + e, set = 1 + e;
        const int la = 2 * w + off + 4, ll = 2 * h + off + 4;
        const bool has_above = by >= off, has_left = bx >= off;
        const int av_a = has_above ? min(A.width - bx, 2 * w) : 0;
        const int av_l = has_left ? min(A.height - by, h) : 0;
        const int pad = av_a > 0 ? rec[(int64_t)(by - off) * rs + bx]
                        : av_l > 0 ? rec[(int64_t)by * rs + bx - off]
                                   : 128;
        for (int i = t; i < la; i += blockDim.x) {
          int v = 128;
          if (i < off) {
            if (has_above && has_left) v = rec[(int64_t)(by - off) * rs + bx - off + i];
          } else if (av_a > 0) {
            v = rec[(int64_t)(by - off) * rs + bx + min(i - off, av_a - 1)];
          }
          if (!has_above || !has_left) {
            if (i < off || av_a == 0) v = pad;
          }
          S.row[set][0][i] = (int16_t)v;
        }
        for (int i = t; i < ll; i += blockDim.x) {
          int v = 128;
          if (i < off) {
            if (has_above && has_left) v = rec[(int64_t)(by - off + i) * rs + bx - off];
          } else if (av_l > 0) {
            v = rec[(int64_t)(by + min(i - off, av_l - 1)) * rs + bx - off];
          }
          if (!has_above || !has_left) {
            if (i < off || av_l == 0) v = pad;
          }
          S.row[set][1][i] = (int16_t)v;
        }
        if (t == 0) {
          S.row_len[set][0] = (int16_t)la;
          S.row_len[set][1] = (int16_t)ll;
        }
      }
    }
    __syncthreads();
    // RefSamples::filtered (predict.rs:1233-1267) and the line-0 rows
    // (MrlRefSamples::from_ref_samples, predict.rs:1058-1075)
    for (int i = t; i < 2 * w; i += blockDim.x) {
      const int prev = i == 0 ? S.tl[0] : S.ref[0][0][i - 1];
      S.ref[1][0][i] = i == 2 * w - 1 ? S.ref[0][0][i] : (int16_t)((prev + 2 * S.ref[0][0][i] + S.ref[0][0][i + 1] + 2) >> 2);
    }
    for (int i = t; i < 2 * h; i += blockDim.x) {
      const int prev = i == 0 ? S.tl[0] : S.ref[0][1][i - 1];
      S.ref[1][1][i] = i == 2 * h - 1 ? S.ref[0][1][i] : (int16_t)((prev + 2 * S.ref[0][1][i] + S.ref[0][1][i + 1] + 2) >> 2);
    }
    if (t == 0) S.tl[1] = (int16_t)((2 * S.tl[0] + S.ref[0][0][0] + S.ref[0][1][0] + 2) >> 2);
    if (t == 32) {
      const int denom = w == h ? (w << 1) : max(w, h);
      int sum = 0;
      if (w >= h)
        for (int i = 0; i < w; i++) sum += S.ref[0][0][i];
      if (w <= h)
        for (int i = 0; i < h; i++) sum += S.ref[0][1][i];
      S.dc = (sum + (denom >> 1)) >> floor_log2(denom);
    }
    __syncthreads();
    for (int f = 0; f < 2; f++) {
      for (int i = t; i < 2 * w + 5; i += blockDim.x)
        S.row[f][0][i] = i == 0 ? S.tl[f] : S.ref[f][0][min(i - 1, 2 * w - 1)];
      for (int i = t; i < 2 * h + 5; i += blockDim.x)
        S.row[f][1][i] = i == 0 ? S.tl[f] : S.ref[f][1][min(i - 1, 2 * h - 1)];
      if (t == 0) {
        S.row_len[f][0] = (int16_t)(2 * w + 5);
        S.row_len[f][1] = (int16_t)(2 * h + 5);
      }
    }
    __syncthreads();
    const bool mpm_only = (R.flags & VVCG_ISR_MPM_ONLY) != 0;
    const int n_main = mpm_only ? 6 : 67;
    const int n_cand = n_main + (mrl ? 10 : 0);
    for (int c = warp; c < n_cand; c += kIsrWarps) {
      int mode, set, mri;
      if (c < n_main) {
        mode = mpm_only ? R.mpm[c] : c;
        mri = 0;
        set = (mode > 1 && ang8_params(mode, w, h, 0).ref_filter) ? 1 : 0;
      } else {
        const int k = c - n_main, line = 1 + k / 5;
        mode = R.mpm[1 + k % 5];
        mri = ctu_top ? 0 : line;  // the first CTU row keeps line 0, unfiltered
        set = ctu_top ? 0 : 1 + line;
      }
      const uint32_t s = mode <= 1 ? isr_planar_dc_sad(S, lane, w, h, mode == 0)
                                   : isr_angular_sad(S, warp, lane, w, h, mode, set, mri);
      const uint32_t tot = __reduce_add_sync(0xFFFFFFFFu, s);
      if (lane == 0) S.sad[c] = tot;
    }
    __syncthreads();
    if (t == 0) {
      uint32_t best = 0xFFFFFFFFu;
      int bm = 0, bl = 0;
      for (int c = 0; c < n_main; c++)
        if (S.sad[c] < best) {
          best = S.sad[c];
          bm = mpm_only ? R.mpm[c] : c;
        }
      for (int c = n_main; c < n_cand; c++)
        if (S.sad[c] < best) {
          const int k = c - n_main;
          best = S.sad[c];
          bm = R.mpm[1 + k % 5];
          bl = 1 + k / 5;
        }
      vvcg_intra_search_res o;
      o.sad = best;
      o.mode = (uint8_t)bm;
      o.mrl_idx = (uint8_t)bl;
      for (int i = 0; i < 6; i++) o.reserved[i] = 0;
      A.res[q] = o;
    }
    __syncthreads();
  }
}

}  // namespace vvcg
