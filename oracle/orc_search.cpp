// CPU oracle (test infrastructure only; see oracle.h): the CTU full search of
// the GPU encoder (vvcg_ctu_search_dev). It is new work, not a reference
// function: every block of the six split types of a 32x32 CTU takes the
// luma mode of lowest cost, with predictions from the source plane itself by
// predict_block_16 (predict.rs:3079-3091, restated in orc_intra.cpp), cost =
// 8x8 Hadamard SATD + lambda * mode bits, and the CTU takes the split type of
// lowest total cost (+ lambda * split bits). First lowest wins throughout.
#include <stdlib.h>

#include <vector>

#include "oracle.h"

namespace orc {

namespace {

const int kBlocks[15][4] = {{0, 0, 32, 32}, {0, 0, 16, 16}, {16, 0, 16, 16}, {0, 16, 16, 16}, {16, 16, 16, 16},
                            {0, 0, 32, 16}, {0, 16, 32, 16}, {0, 0, 16, 32}, {16, 0, 16, 32}, {0, 0, 32, 8},
                            {0, 8, 32, 16}, {0, 24, 32, 8}, {0, 0, 8, 32}, {8, 0, 16, 32}, {24, 0, 8, 32}};
const int kFirst[6] = {0, 1, 5, 7, 9, 12}, kCount[6] = {1, 4, 2, 2, 3, 3}, kSplitBits[6] = {1, 2, 3, 3, 4, 4};

// an 8-bit block header plus the mode: MPM i of the default list 2 + i bits, others 7
int mode_bits(int m) {
  static const int mpm[6] = {0, 1, 50, 18, 46, 54};
  for (int i = 0; i < 6; i++)
    if (mpm[i] == m) return 8 + 2 + i;
  return 8 + 7;
}

// per 8x8 tile: (sum |H8 * D * H8^T| + 2) >> 2, H8 the unnormalised
// Sylvester-ordered Hadamard matrix
uint32_t satd8(const int* d, int w, int h) {
  uint32_t total = 0;
  for (int ty = 0; ty < h; ty += 8)
    for (int tx = 0; tx < w; tx += 8) {
      int m[8][8];
      for (int r = 0; r < 8; r++)
        for (int c = 0; c < 8; c++) {
          int s = 0;
          for (int k = 0; k < 8; k++) s += ((__builtin_popcount(c & k) & 1) ? -1 : 1) * d[(ty + r) * w + tx + k];
          m[r][c] = s;
        }
      uint32_t sum = 0;
      for (int c = 0; c < 8; c++)
        for (int r = 0; r < 8; r++) {
          int s = 0;
          for (int k = 0; k < 8; k++) s += ((__builtin_popcount(r & k) & 1) ? -1 : 1) * m[k][c];
          sum += (uint32_t)std::abs(s);
        }
      total += (sum + 2) >> 2;
    }
  return total;
}

}  // namespace

void ctu_search(const Plane16& src, int cx, int cy, int split_mask, int n_cand, const uint8_t* cand,
                uint32_t lambda_q8, uint32_t* cost, uint32_t split_cost[6], int* split, int* cu_mode, int modes[4]) {
  uint32_t bcost[15] = {0};
  int bmode[15] = {0};
  std::vector<uint16_t> pred(32 * 32);
  std::vector<int> d(32 * 32);
  for (int s = 0; s < 6; s++) {
    if (!(split_mask & (1 << s))) continue;
    for (int k = 0; k < kCount[s]; k++) {
      const int slot = kFirst[s] + k;
      const int bx = cx + kBlocks[slot][0], by = cy + kBlocks[slot][1], w = kBlocks[slot][2], h = kBlocks[slot][3];
      uint32_t best = 0xFFFFFFFFu;
      int bm = 0;
      const int n = n_cand ? n_cand : 67;
      for (int c = 0; c < n; c++) {
        const int mode = n_cand ? cand[c] : c;
        predict_block_16(src, bx, by, w, h, true, mode, pred.data());
        for (int y = 0; y < h; y++)
          for (int x = 0; x < w; x++) d[y * w + x] = (int)src.get(bx + x, by + y) - (int)pred[y * w + x];
        const uint32_t c0 = satd8(d.data(), w, h) + (uint32_t)(((uint64_t)lambda_q8 * mode_bits(mode)) >> 8);
        if (c0 < best) {
          best = c0;
          bm = mode;
        }
      }
      bcost[slot] = best;
      bmode[slot] = bm;
    }
  }
  *cost = 0xFFFFFFFFu;
  *split = 0xFF;
  *cu_mode = (split_mask & 1) ? bmode[0] : 0xFF;
  for (int k = 0; k < 4; k++) modes[k] = 0xFF;
  for (int s = 0; s < 6; s++) {
    split_cost[s] = 0xFFFFFFFFu;
    if (!(split_mask & (1 << s))) continue;
    uint64_t c = ((uint64_t)lambda_q8 * kSplitBits[s]) >> 8;
    for (int k = 0; k < kCount[s]; k++) c += bcost[kFirst[s] + k];
    split_cost[s] = c < 0xFFFFFFFEull ? (uint32_t)c : 0xFFFFFFFEu;
    if (split_cost[s] < *cost) {
      *cost = split_cost[s];
      *split = s;
      for (int k = 0; k < 4; k++) modes[k] = k < kCount[s] ? bmode[kFirst[s] + k] : 0xFF;
    }
  }
}

// choose_qt_mtt_partition_rdo_16 (slice.rs:4111-4121) over
// choose_qt_mtt_partition_rdo (slice.rs:4126-4167): the region's samples are
// first rounded to 8 bits as Plane16::to_plane_8bit does (predict.rs:2914-2926:
// (v saturating+ 2^(bd-9)) >> (bd-8), at most 255); each quadrant's mean is
// its sum over the samples inside the plane divided by the full quadrant area;
// the mean differences across the horizontal and vertical midlines, against
// max(qp, 4) / 2 + 8, choose quad, horizontal binary, vertical binary or no
// split. Returns 0 none, 1 quad, 2 binary horizontal, 3 binary vertical.
int qt_mtt_split(const Plane16& src, int64_t bx, int64_t by, int64_t w, int64_t h, int qp, int64_t min_cb) {
  const int64_t lim = min_cb > 8 ? min_cb : 8;
  if (w <= lim || h <= lim) return 0;
  const int shift = src.bd > 8 ? src.bd - 8 : 0;
  const uint32_t add = shift > 0 ? 1u << (shift - 1) : 0u;
  auto to8 = [&](uint16_t v) -> int64_t {
    uint32_t t = (uint32_t)v + add;
    if (t > 65535u) t = 65535u;
    t >>= shift;
    return t > 255u ? 255 : (int64_t)t;
  };
  const int64_t hw = w / 2, hh = h / 2;
  auto quad_mean = [&](int64_t qx, int64_t qy, int64_t qw, int64_t qh) -> int64_t {
    int64_t sum = 0;
    const int64_t ye = qy + qh < src.height ? qy + qh : src.height;
    const int64_t xe = qx + qw < src.width ? qx + qw : src.width;
    for (int64_t y = qy; y < ye; y++)
      for (int64_t x = qx; x < xe; x++) sum += to8(src.get((int)x, (int)y));
    const int64_t area = qw * qh > 1 ? qw * qh : 1;
    return sum / area;
  };
  const int64_t m00 = quad_mean(bx, by, hw, hh), m10 = quad_mean(bx + hw, by, hw, hh);
  const int64_t m01 = quad_mean(bx, by + hh, hw, hh), m11 = quad_mean(bx + hw, by + hh, hw, hh);
  const int64_t hor = llabs(m00 - m01) + llabs(m10 - m11);
  const int64_t ver = llabs(m00 - m10) + llabs(m01 - m11);
  const int64_t thr = (qp > 4 ? qp : 4) / 2 + 8;
  if (w == h && hor > thr && ver > thr) return 1;
  if (hor > ver && hor > thr) return 2;
  if (ver > thr) return 3;
  return 0;
}

}  // namespace orc
