// Luma intra mode searches on the GPU.
//
// 1. The 8-bit multi-tool encoder's decision: choose_luma_intra_pred_mode
//    (crates/rustmpeg-video/src/vvc/predict.rs:2737-2801) over Planar, DC and
//    the 65 angular modes (or the 6 MPMs), then the encoder's MRL candidates
//    (slice.rs:2698-2731): reference lines 1 and 2 for mpm[1..5]. Cost: SAD.
// 2. The CTU full search of the GPU encoder: every block of the six split
//    types of a 32x32 CTU, each over the 67 modes (or a candidate list), on
//    8..12-bit samples with the predictors of predict_block_16
//    (predict.rs:3079-3410), cost = 8x8 Hadamard SATD + lambda * mode bits.
//
// One CTA per block, one warp per candidate at a time; each warp builds the
// candidate's extended reference arrays in its own shared buffers exactly as
// predict_angular_with_params_bd (predict.rs:1776-1958) lays them out, then
// evaluates every sample of the block. The winner is the first candidate
// with the lowest cost (Planar wins ties); an MRL candidate replaces it only
// with a strictly lower cost.
#pragma once
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

constexpr int kIsrWarps = 8;
constexpr int kIsrRow = 136;  // 2 * 64 + 3 + 4 + 1: longest MRL row
constexpr int kIsrBuf = 520;  // base + 2 max(w, h) + 2 max(refW, refH) + 64 for 64x64 (516)
constexpr int kIsrMaxCand = 67 + 10;
constexpr int kSatdMaxSamples = 1024;

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
      const int s = delta == 0 ? 0 : delta == 1 ? 6 : delta == 2 ? 10 : delta == 3 ? 12 : delta == 4 ? 14 : 15;
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

template <bool kSatd>
struct IsrShared {
  uint16_t src[64 * 64];
  // reference rows as MrlRefSamples: [set][0 above / 1 left]; sets 0 / 1 are
  // line 0 unfiltered / filtered, 2 / 3 are lines 1 / 2
  int16_t row[4][2][kIsrRow];
  int16_t row_len[4][2];
  int16_t ref[2][2][128];  // RefSamples above / left, [unfiltered / filtered]
  int16_t tl[2];
  int32_t dc;
  uint32_t cost[kIsrMaxCand];
  int16_t buf[kIsrWarps][2][kIsrBuf];                               // a warp's ref_above / ref_left
  int16_t res[kSatd ? kIsrWarps : 1][kSatd ? kSatdMaxSamples : 1];  // a warp's residual block
};

// Calls sink(i, v) with the prediction v of every sample i (raster) of a w x h
// block for one angular candidate (predict_angular_with_params_bd), by one warp.
template <bool kSatd, typename Sink>
__device__ void isr_angular(IsrShared<kSatd>& S, int warp, int lane, int w, int h, int dir, int set, int mri, int bd,
                            Sink sink) {
  const Ang8 P = ang8_params(dir, w, h, mri);
  const int def = 1 << (bd - 1), maxv = (1 << bd) - 1;
  int16_t* ra = S.buf[warp][0];
  int16_t* rl = S.buf[warp][1];
  const int16_t* rowa = S.row[set][0];
  const int16_t* rowl = S.row[set][1];
  const int na = S.row_len[set][0], nl = S.row_len[set][1];
  const int base = max(h, w) + 4;
  const int ref_w = 2 * w, ref_h = 2 * h;
  const int len = base + 2 * max(w, h) + 2 * max(ref_w, ref_h) + 64;
  const bool ver = P.ver;
  // copy ranges of the two arrays (everything else holds the default sample)
  const int a_hi = P.angle < 0 ? w + 1 + mri : ref_w + mri;
  const int l_hi = P.angle < 0 ? h + 1 + mri : ref_h + mri;
  for (int i = lane; i < len; i += 32) {
    const int x = i - base;
    ra[i] = (x >= 0 && x <= a_hi) ? rowa[min(x, na - 1)] : (int16_t)def;
    rl[i] = (x >= 0 && x <= l_hi) ? rowl[min(x, nl - 1)] : (int16_t)def;
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
  for (int i = lane; i < w * h; i += 32) {
    const int r = i / w, c = i - r * w;  // block row / column
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
  __syncwarp();  // the buffers are rebuilt for the warp's next candidate
}

// Planar (predict.rs:1688-1719) or DC (:1722-1736) with PDPC (:1739-1754).
template <bool kSatd, typename Sink>
__device__ void isr_planar_dc(IsrShared<kSatd>& S, int lane, int w, int h, bool planar, Sink sink) {
  const int f = (planar && w * h > 32) ? 1 : 0;  // uses_reference_filter for luma Planar
  const int16_t* top = S.ref[f][0];
  const int16_t* left = S.ref[f][1];
  const int lw = floor_log2(w), lh = floor_log2(h);
  const int pscale = max(lw + lh - 2, 0) >> 2;
  const int tr = top[w], bl = left[h];
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
    sink(i, v);
  }
}

// gather_references (predict.rs:1084-1134; gather_references_16 :3016-3076
// at 8..12 bits), RefSamples::filtered (:1233-1267), the line-0 rows
// (MrlRefSamples::from_ref_samples, :1058-1075) and the DC value. With
// `mrl`, also lines 1 and 2 (gather_references_mrl, :1141-1231).
template <bool kSatd, typename T>
__device__ void isr_prepare(IsrShared<kSatd>& S, const T* rec, int64_t rs, int width, int height, int bx, int by,
                            int w, int h, int bd, bool mrl, bool ctu_top) {
  const int t = threadIdx.x;
  const int def = 1 << (bd - 1);
  const int above_len = by == 0 ? 0 : min(width - bx, 2 * w);
  const int left_len = bx == 0 ? 0 : min(height - by, h);
  const int a0 = above_len > 0 ? (int)rec[(int64_t)(by - 1) * rs + bx] : 0;
  const int l0 = left_len > 0 ? (int)rec[(int64_t)by * rs + bx - 1] : 0;
  for (int i = t; i < 2 * w; i += blockDim.x)
    S.ref[0][0][i] = above_len == 0 ? (left_len > 0 ? l0 : def)
                                    : rec[(int64_t)(by - 1) * rs + bx + min(i, above_len - 1)];
  for (int i = t; i < 2 * h; i += blockDim.x)
    S.ref[0][1][i] = left_len == 0 ? (above_len > 0 ? a0 : def)
                                   : rec[(int64_t)(by + min(i, left_len - 1)) * rs + bx - 1];
  if (t == 0)
    S.tl[0] = (above_len > 0 && left_len > 0) ? (int)rec[(int64_t)(by - 1) * rs + bx - 1]
              : above_len > 0                  ? a0
              : left_len > 0                   ? l0
                                               : def;
  if (mrl && !ctu_top) {
    for (int e = 1; e <= 2; e++) {
      const int off = 1 + e, set = 1 + e;
      const int la = 2 * w + off + 4, ll = 2 * h + off + 4;
      const bool has_above = by >= off, has_left = bx >= off;
      const int av_a = has_above ? min(width - bx, 2 * w) : 0;
      const int av_l = has_left ? min(height - by, h) : 0;
      const int pad = av_a > 0 ? (int)rec[(int64_t)(by - off) * rs + bx]
                      : av_l > 0 ? (int)rec[(int64_t)by * rs + bx - off]
                                 : def;
      for (int i = t; i < la; i += blockDim.x) {
        int v = def;
        if (i < off) {
          if (has_above && has_left) v = rec[(int64_t)(by - off) * rs + bx - off + i];
        } else if (av_a > 0) {
          v = rec[(int64_t)(by - off) * rs + bx + min(i - off, av_a - 1)];
        }
        if ((!has_above || !has_left) && (i < off || av_a == 0)) v = pad;
        S.row[set][0][i] = (int16_t)v;
      }
      for (int i = t; i < ll; i += blockDim.x) {
        int v = def;
        if (i < off) {
          if (has_above && has_left) v = rec[(int64_t)(by - off + i) * rs + bx - off];
        } else if (av_l > 0) {
          v = rec[(int64_t)(by + min(i - off, av_l - 1)) * rs + bx - off];
        }
        if ((!has_above || !has_left) && (i < off || av_l == 0)) v = pad;
        S.row[set][1][i] = (int16_t)v;
      }
      if (t == 0) {
        S.row_len[set][0] = (int16_t)la;
        S.row_len[set][1] = (int16_t)ll;
      }
    }
  }
  __syncthreads();
  for (int i = t; i < 2 * w; i += blockDim.x) {
    const int prev = i == 0 ? S.tl[0] : S.ref[0][0][i - 1];
    S.ref[1][0][i] =
        i == 2 * w - 1 ? S.ref[0][0][i] : (int16_t)((prev + 2 * S.ref[0][0][i] + S.ref[0][0][i + 1] + 2) >> 2);
  }
  for (int i = t; i < 2 * h; i += blockDim.x) {
    const int prev = i == 0 ? S.tl[0] : S.ref[0][1][i - 1];
    S.ref[1][1][i] =
        i == 2 * h - 1 ? S.ref[0][1][i] : (int16_t)((prev + 2 * S.ref[0][1][i] + S.ref[0][1][i + 1] + 2) >> 2);
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
}

// ---------------------------------------------------------------- 8-bit SAD --

struct IsrArgs {
  const uint8_t* recon;
  const uint8_t* src;
  int64_t recon_stride, src_stride;
  int32_t width, height, n;
  const vvcg_intra_search_req* reqs;
  vvcg_intra_search_res* res;
};

__global__ void __launch_bounds__(kIsrWarps * 32) k_luma_intra_search_8(const __grid_constant__ IsrArgs A) {
  __shared__ IsrShared<false> S;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int q = blockIdx.x; q < A.n; q += gridDim.x) {
    const vvcg_intra_search_req R = A.reqs[q];
    const int w = 1 << R.log2_w, h = 1 << R.log2_h, bx = (int)R.x, by = (int)R.y;
    for (int i = t; i < w * h; i += blockDim.x)
      S.src[i] = A.src[(int64_t)(by + i / w) * A.src_stride + bx + (i % w)];
    const bool mrl = (R.flags & VVCG_ISR_MRL) != 0;
    const bool ctu_top = (by & ((1 << R.log2_ctu) - 1)) == 0;
    isr_prepare(S, A.recon, A.recon_stride, A.width, A.height, bx, by, w, h, 8, mrl, ctu_top);
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
      uint32_t sad = 0;
      auto acc = [&](int i, int v) { sad += (uint32_t)abs((int)S.src[i] - v); };
      if (mode <= 1)
        isr_planar_dc(S, lane, w, h, mode == 0, acc);
      else
        isr_angular(S, warp, lane, w, h, mode, set, mri, 8, acc);
      const uint32_t tot = __reduce_add_sync(0xFFFFFFFFu, sad);
      if (lane == 0) S.cost[c] = tot;
    }
    __syncthreads();
    if (t == 0) {
      uint32_t best = 0xFFFFFFFFu;
      int bm = 0, bl = 0;
      for (int c = 0; c < n_main; c++)
        if (S.cost[c] < best) {
          best = S.cost[c];
          bm = mpm_only ? R.mpm[c] : c;
        }
      for (int c = n_main; c < n_cand; c++)
        if (S.cost[c] < best) {
          const int k = c - n_main;
          best = S.cost[c];
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

// ------------------------------------------------------- CTU full search ----

// Bits a block is charged in the search cost: a header of 8 bits (split
// flags, cbf and the like) plus its mode, ordered by the default MPM list
// (derive_intra_mpms with no neighbours, predict.rs): MPM i costs 2 + i bits,
// any other mode 7.
__device__ __forceinline__ int search_mode_bits(int m) {
  return 8 + (m == 0 ? 2 : m == 1 ? 3 : m == 50 ? 4 : m == 18 ? 5 : m == 46 ? 6 : 7);
}

// One block of one split type of one CTU.
struct CostReq {
  uint32_t x, y;
  uint8_t log2_w, log2_h, n_cand, reserved;
  uint8_t cand[6];
  uint16_t slot;  // block slot of the CTU, 0..14
  uint32_t ctu;   // index of the CTU request
};

struct CostArgs {
  const uint16_t* src;
  int64_t stride;
  int32_t width, height, bd, n;
  uint32_t lambda_q8;
  const CostReq* reqs;
  uint32_t* block_cost;  // [ctu][15]
  uint8_t* block_mode;   // [ctu][15]
  uint32_t* mode_costs;  // optional [ctu][67]: every mode's cost of the unsplit CU (slot 0, full set)
};

// 8x8 Hadamard SATD of a w x h residual block (w, h multiples of 8) in the
// warp's buffer: each 8-lane group transforms one 8x8 tile (rows, then
// columns); a tile's SATD is (sum |coefficient| + 2) >> 2.
__device__ __forceinline__ uint32_t satd8x8_warp(int16_t* res, int lane, int w, int h) {
  const int tiles = (w >> 3) * (h >> 3);
  const int g = lane >> 3, r = lane & 7;
  uint32_t total = 0;
  for (int t0 = 0; t0 < tiles; t0 += 4) {
    const int tile = t0 + g;
    const bool act = tile < tiles;
    const int tx = act ? (tile % (w >> 3)) * 8 : 0, ty = act ? (tile / (w >> 3)) * 8 : 0;
    int v[8];
    if (act) {
#pragma unroll
      for (int k = 0; k < 8; k++) v[k] = res[(ty + r) * w + tx + k];
      // 8-point Hadamard of row r
#pragma unroll
      for (int s = 1; s < 8; s <<= 1)
#pragma unroll
        for (int k = 0; k < 8; k++)
          if (!(k & s)) {
            const int a = v[k], b = v[k + s];
            v[k] = a + b;
            v[k + s] = a - b;
          }
    }
    // rows back to the buffer, then each lane takes column r of its tile
    if (act) {
#pragma unroll
      for (int k = 0; k < 8; k++) res[(ty + r) * w + tx + k] = (int16_t)v[k];
    }
    __syncwarp();
    int col[8];
    if (act) {
#pragma unroll
      for (int k = 0; k < 8; k++) col[k] = res[(ty + k) * w + tx + r];
    }
    __syncwarp();
    uint32_t s_abs = 0;
    if (act) {
#pragma unroll
      for (int s = 1; s < 8; s <<= 1)
#pragma unroll
        for (int k = 0; k < 8; k++)
          if (!(k & s)) {
            const int a = col[k], b = col[k + s];
            col[k] = a + b;
            col[k + s] = a - b;
          }
#pragma unroll
      for (int k = 0; k < 8; k++) s_abs += (uint32_t)abs(col[k]);
    }
    // the tile's sum over its 8 lanes
    s_abs += __shfl_xor_sync(0xFFFFFFFFu, s_abs, 1);
    s_abs += __shfl_xor_sync(0xFFFFFFFFu, s_abs, 2);
    s_abs += __shfl_xor_sync(0xFFFFFFFFu, s_abs, 4);
    if (act && r == 0) total += (s_abs + 2) >> 2;
  }
  return __reduce_add_sync(0xFFFFFFFFu, total);
}

__global__ void __launch_bounds__(kIsrWarps * 32) k_cost_search(const __grid_constant__ CostArgs A) {
  __shared__ IsrShared<true> S;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int q = blockIdx.x; q < A.n; q += gridDim.x) {
    const CostReq R = A.reqs[q];
    if (R.log2_w == 0) continue;  // an unused slot (pruned search)
    const int w = 1 << R.log2_w, h = 1 << R.log2_h, bx = (int)R.x, by = (int)R.y;
    for (int i = t; i < w * h; i += blockDim.x) S.src[i] = A.src[(int64_t)(by + i / w) * A.stride + bx + (i % w)];
    isr_prepare(S, A.src, A.stride, A.width, A.height, bx, by, w, h, A.bd, false, true);
    const int n_cand = R.n_cand ? R.n_cand : 67;
    int16_t* res = S.res[warp];
    for (int c = warp; c < n_cand; c += kIsrWarps) {
      const int mode = R.n_cand ? R.cand[c] : c;
      auto put = [&](int i, int v) { res[i] = (int16_t)((int)S.src[i] - v); };
      if (mode <= 1)
        isr_planar_dc(S, lane, w, h, mode == 0, put);
      else
        isr_angular(S, warp, lane, w, h, mode, (ang8_params(mode, w, h, 0).ref_filter) ? 1 : 0, 0, A.bd, put);
      __syncwarp();
      const uint32_t satd = satd8x8_warp(res, lane, w, h);
      __syncwarp();
      if (lane == 0) S.cost[c] = satd + (uint32_t)(((uint64_t)A.lambda_q8 * search_mode_bits(mode)) >> 8);
    }
    __syncthreads();
    if (t == 0) {
      uint32_t best = 0xFFFFFFFFu;
      int bm = 0;
      for (int c = 0; c < n_cand; c++)
        if (S.cost[c] < best) {
          best = S.cost[c];
          bm = R.n_cand ? R.cand[c] : c;
        }
      A.block_cost[(size_t)R.ctu * 15 + R.slot] = best;
      A.block_mode[(size_t)R.ctu * 15 + R.slot] = (uint8_t)bm;
    }
    if (A.mode_costs && R.slot == 0 && R.n_cand == 0)
      for (int c = t; c < 67; c += blockDim.x) A.mode_costs[(size_t)R.ctu * 67 + c] = S.cost[c];
    __syncthreads();
  }
}

// Slots of the 15 blocks of a 32x32 CTU per split type and the split bits.
__constant__ uint8_t c_split_first[6] = {0, 1, 5, 7, 9, 12};
__constant__ uint8_t c_split_count[6] = {1, 4, 2, 2, 3, 3};
__constant__ uint8_t c_split_bits[6] = {1, 2, 3, 3, 4, 4};

// Per CTU: each evaluated split's cost (its blocks' costs + lambda * split
// bits), the first lowest wins.
__global__ void k_ctu_search_combine(const vvcg_ctu_search_req* reqs, int n, uint32_t lambda_q8,
                                     const uint32_t* block_cost, const uint8_t* block_mode,
                                     vvcg_ctu_search_res* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t mask = reqs[i].split_mask;
  vvcg_ctu_search_res o;
  o.cost = 0xFFFFFFFFu;
  o.split = 0xFF;
  o.cu_mode = 0xFF;
  for (int k = 0; k < 4; k++) o.modes[k] = 0xFF;
  o.reserved[0] = o.reserved[1] = 0;
  for (int s = 0; s < 6; s++) {
    o.split_cost[s] = 0xFFFFFFFFu;
    if (!(mask & (1u << s))) continue;
    uint64_t c = ((uint64_t)lambda_q8 * c_split_bits[s]) >> 8;
    for (int k = 0; k < c_split_count[s]; k++) c += block_cost[(size_t)i * 15 + c_split_first[s] + k];
    o.split_cost[s] = c < 0xFFFFFFFEull ? (uint32_t)c : 0xFFFFFFFEu;
    if (o.split_cost[s] < o.cost) {
      o.cost = o.split_cost[s];
      o.split = (uint8_t)s;
      for (int k = 0; k < 4; k++)
        o.modes[k] = k < c_split_count[s] ? block_mode[(size_t)i * 15 + c_split_first[s] + k] : 0xFF;
    }
  }
  if (mask & 1u) o.cu_mode = block_mode[(size_t)i * 15];
  out[i] = o;
}

}  // namespace vvcg
