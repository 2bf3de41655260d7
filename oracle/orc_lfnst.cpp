// CPU oracle (test infrastructure only; see oracle.h): low-frequency
// non-separable transform. Restates crates/rustmpeg-video/src/vvc/lfnst.rs.
#include <algorithm>

#include "../rustmpeg-next_b200/csrc/vvc_tables.h"
#include "oracle.h"

namespace orc {
using namespace vvc_tables;

// lfnst.rs:85-95 get_lfnst_intra_mode (wide-angle mode -> LFNST mode index)
int get_lfnst_intra_mode(int m) {
  if (m < 0) return m + 14 + 67;
  if (m >= 67) return m + 14;
  return m;
}

// lfnst.rs:97-99 transposes
static bool transposes(int m) { return (m >= 35 && m < 67) || m >= 81; }

// lfnst.rs:108-125 parameters_rect
static int params(int w, int h, int idx, int* sb, int* tr, int* zo) {
  if (idx == 0 || idx > 2) return -1;
  if (w < 4 || h < 4) return -1;
  *sb = (w >= 8 && h >= 8) ? 8 : 4;
  bool small = (w == 4 && h == 4) || (w == 8 && h == 8);
  *tr = *sb == 4 ? 16 : 48;
  *zo = small ? 8 : 16;
  return 0;
}

// Top-left 8x8 region in 4x4-group diagonal order (lfnst.rs:16-81
// TOP_LEFT_DIAG_SCAN_8X8): the grouped scan of an 8x8 block.
static void scan8(int* xs, int* ys) {
  int32_t r[64];
  coeff_scan_raster(8, 8, r);
  for (int k = 0; k < 64; k++) {
    xs[k] = r[k] % 8;
    ys[k] = r[k] / 8;
  }
}

static inline int coef(int sb, int set, int idx, int row, int col) {
  return sb == 4 ? kLfnst4x4[((set * 2 + idx) * 16 + row) * 16 + col]
                 : kLfnst8x8[((set * 2 + idx) * 16 + row) * 48 + col];
}

// lfnst.rs:131-205 forward_lfnst_rect
int forward_lfnst_rect(int32_t* c, int w, int h, int idx, int mode) {
  int sb, tr, zo;
  if (params(w, h, idx, &sb, &tr, &zo)) return -1;
  if (mode < 0 || mode >= 95) return -2;
  int set = kLfnstLut[mode];
  int id = idx - 1;
  int32_t src[48] = {0};
  if (transposes(mode)) {
    if (sb == 4) {
      for (int y = 0; y < 4; y++)
        for (int k = 0; k < 4; k++) src[y + 4 * k] = c[y * w + k];
    } else {
      for (int y = 0; y < 8; y++) {
        for (int k = 0; k < 4; k++) src[y + 8 * k] = c[y * w + k];
        if (y < 4)
          for (int k = 0; k < 4; k++) src[y + 32 + 4 * k] = c[y * w + 4 + k];
      }
    }
  } else {
    int pos = 0;
    for (int y = 0; y < sb; y++) {
      int stride = y < 4 ? sb : 4;
      for (int x = 0; x < stride; x++) src[pos++] = c[y * w + x];
    }
  }
  int32_t out[48] = {0};
  for (int j = 0; j < zo; j++) {
    int64_t s = 0;
    for (int i = 0; i < tr; i++) s += (int64_t)src[i] * coef(sb, set, id, j, i);
    out[j] = (int32_t)((s + 64) >> 7);
  }
  int xs[64], ys[64];
  scan8(xs, ys);
  for (int k = 0; k < tr; k++) c[ys[k] * w + xs[k]] = out[k];
  return 0;
}

// lfnst.rs:219-294 inverse_lfnst_rect
int inverse_lfnst_rect(int32_t* c, int w, int h, int idx, int mode) {
  int sb, tr, zo;
  if (params(w, h, idx, &sb, &tr, &zo)) return -1;
  if (mode < 0 || mode >= 95) return -2;
  int set = kLfnstLut[mode];
  int id = idx - 1;
  int xs[64], ys[64];
  scan8(xs, ys);
  int32_t src[16];
  for (int i = 0; i < 16; i++) src[i] = c[ys[i] * w + xs[i]];
  int32_t out[48] = {0};
  for (int j = 0; j < tr; j++) {
    int64_t s = 0;
    for (int i = 0; i < zo; i++) s += (int64_t)src[i] * coef(sb, set, id, i, j);
    out[j] = (int32_t)std::min<int64_t>(32767, std::max<int64_t>(-32768, (s + 64) >> 7));
  }
  if (transposes(mode)) {
    if (sb == 4) {
      for (int y = 0; y < 4; y++)
        for (int k = 0; k < 4; k++) c[y * w + k] = out[y + 4 * k];
    } else {
      for (int y = 0; y < 8; y++) {
        for (int k = 0; k < 4; k++) c[y * w + k] = out[y + 8 * k];
        if (y < 4)
          for (int k = 0; k < 4; k++) c[y * w + 4 + k] = out[y + 32 + 4 * k];
      }
    }
  } else {
    int pos = 0;
    for (int y = 0; y < sb; y++) {
      int stride = y < 4 ? sb : 4;
      for (int x = 0; x < stride; x++) c[y * w + x] = out[pos++];
    }
  }
  return 0;
}

}  // namespace orc
