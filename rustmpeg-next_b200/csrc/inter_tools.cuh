// Inter-prediction tools of the reference beyond plain motion compensation,
// batched over independent blocks (crates/rustmpeg-video/src/vvc/inter.rs):
// BDOF (apply_bdof_luma :1218-1339), DMVR (refine_dmvr_subblock :1371-1471,
// dmvr_subpel_1d :1341), affine subblock motion and PROF deltas
// (derive_affine_subblock_mvs :1502-1579 with
// is_subblock_vector_spread_over_limit :1473), PROF (apply_prof_4x4
// :1581-1609), CIIP (apply_ciip_blend :1615-1630) and GPM
// (derive_gpm_params_table / predict_gpm_block :1641-1731). Integer
// arithmetic only, in the reference's order; outputs of the sample tools are
// the reference's 8-bit ones.
#pragma once
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

namespace vvcg {

__constant__ int c_geo_dis[32];
__constant__ int c_geo_angle_to_mask[32];
__constant__ int c_bilinear4[32];

constexpr int kMvMinStorage = -(1 << 17), kMvMaxStorage = (1 << 17) - 1;

__device__ __forceinline__ int right_shift_msb_d(int numer, int denom) {
  return denom <= 0 ? 0 : numer >> (31 - __clz(denom));
}

// Mv::shr_round (inter.rs:183-195)
__device__ __forceinline__ int shr_round_d(int v, int shift) {
  return shift == 0 ? v : (v + (1 << (shift - 1)) + ((~v) >> 31)) >> shift;
}

// --------------------------------------------------------------- BDOF ----
// One CTA per block, one thread per 4x4 subblock. The reference pads each
// prediction by one sample (edge copies) and its gradients likewise, so every
// position of the 6x6 window reads the sample or gradient at its coordinates
// clamped into the block.
__global__ void __launch_bounds__(128) k_bdof(const vvcg_bdof_req* __restrict__ reqs, const int32_t* __restrict__ pred0,
                                              const int32_t* __restrict__ pred1, int32_t* __restrict__ out) {
  const vvcg_bdof_req R = reqs[blockIdx.x];
  const int w = R.w, h = R.h;
  const int32_t* a = pred0 + R.off;
  const int32_t* b = pred1 + R.off;
  int32_t* o = out + R.off;
  auto P = [&](const int32_t* p, int x, int y) { return p[clampi(y, 0, h - 1) * w + clampi(x, 0, w - 1)]; };
  auto gx = [&](const int32_t* p, int x, int y) { return (P(p, x + 1, y) >> 6) - (P(p, x - 1, y) >> 6); };
  auto gy = [&](const int32_t* p, int x, int y) { return (P(p, x, y + 1) >> 6) - (P(p, x, y - 1) >> 6); };
  const int sbw = w >> 2, nsb = sbw * (h >> 2);
  const int shift_num = 7, offset = (1 << (shift_num - 1)) + 2 * (1 << 13), limit = 15;
  for (int s = threadIdx.x; s < nsb; s += blockDim.x) {
    const int xu = s % sbw, yu = s / sbw;
    int sgx = 0, sgy = 0, sdx = 0, sdy = 0, sgygx = 0;
    for (int dy = 0; dy < 6; dy++)
      for (int dx = 0; dx < 6; dx++) {
        const int x = clampi(xu * 4 + dx - 1, 0, w - 1), y = clampi(yu * 4 + dy - 1, 0, h - 1);
        const int tgx = (gx(a, x, y) + gx(b, x, y)) >> 1, tgy = (gy(a, x, y) + gy(b, x, y)) >> 1;
        const int tdi = (b[y * w + x] >> 4) - (a[y * w + x] >> 4);
        sgx += abs(tgx);
        sgy += abs(tgy);
        sdx += tgx < 0 ? -tdi : (tgx == 0 ? 0 : tdi);
        sdy += tgy < 0 ? -tdi : (tgy == 0 ? 0 : tdi);
        sgygx += tgy < 0 ? -tgx : (tgy == 0 ? 0 : tgx);
      }
    const int tmpx = sgx == 0 ? 0 : clampi(right_shift_msb_d(4 * sdx, sgx), -limit, limit);
    const int tmp_data = (sgygx * tmpx) >> 1;
    const int tmpy = sgy == 0 ? 0 : clampi(right_shift_msb_d(4 * sdy - tmp_data, sgy), -limit, limit);
    for (int dy = 0; dy < 4; dy++)
      for (int dx = 0; dx < 4; dx++) {
        const int x = xu * 4 + dx, y = yu * 4 + dy;
        const int bb = tmpx * (gx(a, x, y) - gx(b, x, y)) + tmpy * (gy(a, x, y) - gy(b, x, y));
        o[y * w + x] = clampi((a[y * w + x] + b[y * w + x] + bb + offset) >> shift_num, 0, 255);
      }
  }
}

// --------------------------------------------------------------- DMVR ----
__device__ __forceinline__ int dmvr_subpel_1d_d(long long s0, long long s1, long long s2) {
  const long long den = s1 + s2 - 2 * s0;
  if (den == 0) return 0;
  if (s1 != s0 && s2 != s0) {
    const long long num = ((s1 - s2) << 4) >> 1;
    long long rem = num < 0 ? -num : num;
    int q = 0;
    for (int i = 2; i >= 0; i--) {
      const long long div = den << i;
      if (rem >= div) {
        rem -= div;
        q += 1 << i;
      }
    }
    return num < 0 ? -q : q;
  }
  return s1 == s0 ? -8 : 8;
}

struct DmvrArgs {
  const uint8_t* ref0;
  const uint8_t* ref1;
  int32_t w, h, stride, n;
  const vvcg_dmvr_req* reqs;
  int32_t* mv_out;  // 4 per request
};

// One warp per subblock: the 25 bilateral costs of the integer offsets, each
// reduced over the warp; lane 0 keeps the reference's evaluation order.
__global__ void __launch_bounds__(128) k_dmvr(const __grid_constant__ DmvrArgs A) {
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (q >= A.n) return;
  const vvcg_dmvr_req R = A.reqs[q];
  const int dx = R.dx, dy = R.dy;
  auto sc = [&](const uint8_t* p, int x, int y) {
    return (int)p[(size_t)clampi(y, 0, A.h - 1) * A.stride + clampi(x, 0, A.w - 1)];
  };
  auto bil = [&](const uint8_t* p, int mvh, int mvv, int ox, int oy, int x, int y) {
    const int px = R.bx + (mvh >> 4) + ox + x, py = R.by + (mvv >> 4) + oy + y;
    const int* wx = &c_bilinear4[2 * (mvh & 15)];
    const int* wy = &c_bilinear4[2 * (mvv & 15)];
    const int h0 = (sc(p, px, py) * wx[0] + sc(p, px + 1, py) * wx[1] + 8) >> 4;
    const int h1 = (sc(p, px, py + 1) * wx[0] + sc(p, px + 1, py + 1) * wx[1] + 8) >> 4;
    return (h0 * wy[0] + h1 * wy[1] + 8) >> 4;
  };
  auto cost = [&](int ox, int oy) -> long long {
    long long c = 0;
    const int rows = (dy + 1) / 2;
    for (int i = lane; i < rows * dx; i += 32) {
      const int y = 2 * (i / dx), x = i % dx;
      c += abs(bil(A.ref0, R.mv[0][0], R.mv[0][1], ox, oy, x, y) - bil(A.ref1, R.mv[1][0], R.mv[1][1], -ox, -oy, x, y));
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    return c;
  };
  long long sads[5][5];
  long long min_cost = cost(0, 0);
  min_cost -= min_cost >> 2;
  sads[2][2] = min_cost;
  int dh = 0, dv = 0;
  if (min_cost >= (long long)dx * dy) {
    int bix = 0, biy = 0;
    for (int oy = -2; oy <= 2; oy++)
      for (int ox = -2; ox <= 2; ox++) {
        if (ox == 0 && oy == 0) continue;
        const long long c = cost(ox, oy);
        sads[oy + 2][ox + 2] = c;
        if (c < min_cost) {
          min_cost = c;
          bix = ox;
          biy = oy;
        }
      }
    dh = bix * 16;
    dv = biy * 16;
    if (abs(bix) < 2 && abs(biy) < 2) {
      const int ux = bix + 2, uy = biy + 2;
      dh += dmvr_subpel_1d_d(sads[uy][ux], sads[uy][ux - 1], sads[uy][ux + 1]);
      dv += dmvr_subpel_1d_d(sads[uy][ux], sads[uy - 1][ux], sads[uy + 1][ux]);
    }
  }
  if (lane == 0) {
    int32_t* o = A.mv_out + 4 * (size_t)q;
    o[0] = clampi(R.mv[0][0] + dh, kMvMinStorage, kMvMaxStorage);
    o[1] = clampi(R.mv[0][1] + dv, kMvMinStorage, kMvMaxStorage);
    o[2] = clampi(R.mv[1][0] - dh, kMvMinStorage, kMvMaxStorage);
    o[3] = clampi(R.mv[1][1] - dv, kMvMinStorage, kMvMaxStorage);
  }
}

// ------------------------------------------------------- affine + PROF ----
__device__ __forceinline__ bool spread_over_limit_d(int a, int b, int c, int d, int pred_type) {
  const int s4 = 4 << 11, tap = 6;
  if (pred_type == 3) {
    const int max_w = max(max(0, 4 * a + s4), max(4 * c, 4 * a + 4 * c + s4));
    const int min_w = min(min(0, 4 * a + s4), min(4 * c, 4 * a + 4 * c + s4));
    const int max_h = max(max(0, 4 * b), max(4 * d + s4, 4 * b + 4 * d + s4));
    const int min_h = min(min(0, 4 * b), min(4 * d + s4, 4 * b + 4 * d + s4));
    return (((max_w - min_w) >> 11) + tap + 3) * (((max_h - min_h) >> 11) + tap + 3) > (tap + 9) * (tap + 9);
  }
  if (((abs(4 * a + s4) >> 11) + tap + 3) * ((abs(4 * b) >> 11) + tap + 3) > (tap + 9) * (tap + 5)) return true;
  return ((abs(4 * c) >> 11) + tap + 3) * ((abs(4 * d + s4) >> 11) + tap + 3) > (tap + 5) * (tap + 9);
}

// One thread per coding unit: its 4x4 subblock MVs (at sub_mv + 2 * sub_off)
// and PROF deltas (prof + 33 * request: 16 horizontal, 16 vertical, flag).
__global__ void k_affine_mvs(const vvcg_affine_req* __restrict__ reqs, int n, int32_t* __restrict__ sub_mv,
                             int32_t* __restrict__ prof) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const vvcg_affine_req R = reqs[q];
  const int prec = 7, w = R.w, h = R.h, lw = __ffs(w) - 1, lh = __ffs(h) - 1;
  const int dhx = (R.cp[1][0] - R.cp[0][0]) << (prec - lw), dhy = (R.cp[1][1] - R.cp[0][1]) << (prec - lw);
  const int dvx = R.six_param ? (R.cp[2][0] - R.cp[0][0]) << (prec - lh) : -dhy;
  const int dvy = R.six_param ? (R.cp[2][1] - R.cp[0][1]) << (prec - lh) : dhx;
  const bool large = spread_over_limit_d(dhx, dhy, dvx, dvy, R.inter_dir);
  const bool en = !large && (dhx || dhy || dvx || dvy);
  const int bh = R.cp[0][0] << prec, bv = R.cp[0][1] << prec;
  int32_t* o = sub_mv + 2 * (size_t)R.sub_off;
  int k = 0;
  for (int sy = 0; sy < h / 4; sy++)
    for (int sx = 0; sx < w / 4; sx++) {
      const int wh = large ? (w >> 1) : 2 + sx * 4, wv = large ? (h >> 1) : 2 + sy * 4;
      o[2 * k] = clampi(shr_round_d(bh + dhx * wh + dvx * wv, prec), kMvMinStorage, kMvMaxStorage);
      o[2 * k + 1] = clampi(shr_round_d(bv + dhy * wh + dvy * wv, prec), kMvMinStorage, kMvMaxStorage);
      k++;
    }
  int32_t* pf = prof + 33 * (size_t)q;
  const int lim = (1 << 5) - 1;
  for (int y = 0; y < 4; y++)
    for (int x = 0; x < 4; x++) {
      const int wx = 2 * x - 3, wy = 2 * y - 3;
      pf[y * 4 + x] = en ? clampi(shr_round_d(wx * dhx + wy * dvx, 7), -lim, lim) : 0;
      pf[16 + y * 4 + x] = en ? clampi(shr_round_d(wx * dhy + wy * dvy, 7), -lim, lim) : 0;
    }
  pf[32] = en ? 1 : 0;
}

// One thread per sample of a 4x4 PROF subblock (16 per request).
__global__ void k_prof(const vvcg_prof_req* __restrict__ reqs, int n, const int32_t* __restrict__ src,
                       const int32_t* __restrict__ dmv, int32_t* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 16 * n) return;
  const vvcg_prof_req R = reqs[t >> 4];
  const int i = t & 15, y = i >> 2, x = i & 3;
  const int32_t* s = src + R.src_off;
  const int c = (y + 1) * 6 + x + 1;
  const int gx = (s[c + 1] >> 6) - (s[c - 1] >> 6), gy = (s[c + 6] >> 6) - (s[c - 6] >> 6);
  const int di = clampi(dmv[R.dmv_off + i] * gx + dmv[R.dmv_off + 16 + i] * gy, -(1 << 13), (1 << 13) - 1);
  const int v = s[c] + di;
  out[R.out_off + i] = R.bi ? v : clampi((v + (1 << 5) + (1 << 13)) >> 6, 0, 255);
}

// ---------------------------------------------------------------- CIIP ----
// One CTA per block.
__global__ void k_ciip(const vvcg_ciip_req* __restrict__ reqs, const int32_t* __restrict__ inter,
                       const int32_t* __restrict__ intra, int32_t* __restrict__ out) {
  const vvcg_ciip_req R = reqs[blockIdx.x];
  const int wi = 1 + (R.left_intra ? 1 : 0) + (R.above_intra ? 1 : 0);
  for (uint32_t i = threadIdx.x; i < R.n; i += blockDim.x) {
    const int pi = inter[R.off + i];
    out[R.off + i] = clampi(pi + ((wi * (intra[R.off + i] - pi) + 2) >> 2), 0, 255);
  }
}

// ----------------------------------------------------------------- GPM ----
// One CTA per block; the split direction's (angle, distance) from the
// derive_gpm_params_table order, found by the first thread.
__global__ void k_gpm(const vvcg_gpm_req* __restrict__ reqs, const int32_t* __restrict__ p0,
                      const int32_t* __restrict__ p1, int32_t* __restrict__ out) {
  __shared__ int s_angle, s_dist;
  const vvcg_gpm_req R = reqs[blockIdx.x];
  if (threadIdx.x == 0) {
    int m = 0, want = R.split_dir & 63, ang = 0, dis = 0;
    for (int a = 0; a < 32 && m <= want; a++)
      for (int d = 0; d < 4 && m <= want; d++) {
        const int mask = c_geo_angle_to_mask[a];
        if ((d == 0 && a >= 16) || ((d == 2 || d == 0) && (mask == 0 || mask == 5)) || mask == -1) continue;
        if (m == want) {
          ang = a;
          dis = d;
        }
        m++;
      }
    s_angle = ang;
    s_dist = dis;
  }
  __syncthreads();
  const int angle = s_angle, distance = s_dist;
  const int w = R.w, h = R.h, lw = w << R.scale_x, lh = h << R.scale_y;
  int ox = -(lw >> 1), oy = -(lh >> 1);
  if (distance > 0) {
    const int am = angle % 16;
    if (am == 8 || (am != 0 && lh >= lw))
      oy += angle < 16 ? (distance * lh) >> 3 : -((distance * lh) >> 3);
    else
      ox += angle < 16 ? (distance * lw) >> 3 : -((distance * lw) >> 3);
  }
  const int gdx = c_geo_dis[angle], gdy = c_geo_dis[(angle + 8) % 32];
  for (int i = threadIdx.x; i < w * h; i += blockDim.x) {
    const int y = i / w, x = i - y * w;
    const int wi = ((((x << R.scale_x) + ox) << 1) + 1) * gdx + ((((y << R.scale_y) + oy) << 1) + 1) * gdy;
    const int w0 = clampi((32 + wi + 4) >> 3, 0, 8), w1 = 8 - w0;
    out[R.off + i] = clampi((w0 * p0[R.off + i] + w1 * p1[R.off + i] + 4) >> 3, 0, 255);
  }
}

}  // namespace vvcg
