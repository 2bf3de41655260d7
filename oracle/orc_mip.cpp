// CPU oracle (test infrastructure only; see oracle.h): matrix-based intra
// prediction. Restates crates/rustmpeg-video/src/vvc/predict.rs:
//   get_mip_size_id / get_num_modes_mip     :2355-2372
//   mip_boundary_downsampling_1d            :2374-2391
//   mip_prediction_upsampling_1d            :2393-2429
//   predict_mip_bd                          :2461-2611 (predict_mip_16 :4109)
//   choose_best_mip_mode_16                 :4166-4199
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "../rustmpeg-next_b200/csrc/vvc_tables.h"
#include "oracle.h"

namespace orc {
using namespace vvc_tables;

static int size_id(int w, int h) { return (w == 4 && h == 4) ? 0 : (w == 4 || h == 4 || (w == 8 && h == 8)) ? 1 : 2; }
static int num_modes(int w, int h) { int s = size_id(w, h); return s == 0 ? 16 : s == 1 ? 8 : 6; }
static int ilog2(int v) { return __builtin_ctz((unsigned)v); }

static std::vector<int> downsample(const int* src, int src_len, int dst_len) {
  std::vector<int> r(dst_len);
  if (dst_len < src_len) {
    int f = src_len / dst_len, lf = ilog2(f), ro = 1 << (lf - 1);
    for (int d = 0; d < dst_len; d++) {
      int s = 0;
      for (int k = 0; k < f; k++) s += src[d * f + k];
      r[d] = (s + ro) >> lf;
    }
  } else {
    for (int d = 0; d < dst_len; d++) r[d] = src[d];
  }
  return r;
}

static void upsample(int* dst, int dst_base, const int* src, int src_base, const int* bndry, int up_dim, int orth_dim,
                     int src_step, int src_stride, int dst_step, int dst_stride, int bndry_step, int f) {
  const int lf = ilog2(f), ro = 1 << (lf - 1);
  for (int o = 0; o < orth_dim; o++) {
    const int sl = src_base + o * src_stride, dl = dst_base + o * dst_stride;
    int before = bndry[o * bndry_step + bndry_step - 1];
    for (int u = 0; u < up_dim; u++) {
      const int behind = src[sl + u * src_step];
      int sb = before << lf, sh = 0, cur = dl + u * f * dst_step;
      for (int p = 1; p <= f; p++) {
        sb -= before;
        sh += behind;
        dst[cur] = (sb + sh + ro) >> lf;
        cur += dst_step;
      }
      before = behind;
    }
  }
}

void predict_mip_bd(const int* above, const int* left, int w, int h, int mode_idx, bool transpose, int bd, int* out) {
  const int sid = size_id(w, h);
  const int rbs = sid == 0 ? 2 : 4, rps = sid == 2 ? 8 : 4;
  const int uh = w / rps, uv = h / rps;
  std::vector<int> top = downsample(above, w, rbs), lft = downsample(left, h, rbs);
  std::vector<int> b;
  if (transpose) {
    b.insert(b.end(), lft.begin(), lft.end());
    b.insert(b.end(), top.begin(), top.end());
  } else {
    b.insert(b.end(), top.begin(), top.end());
    b.insert(b.end(), lft.begin(), lft.end());
  }
  const int in_off = b[0];
  bd = std::min(12, std::max(8, bd));
  const int centre = 1 << (bd - 1), maxv = (1 << bd) - 1;
  b[0] = sid != 2 ? centre - in_off : 0;
  for (size_t i = 1; i < b.size(); i++) b[i] -= in_off;
  int sum = 0;
  for (int v : b) sum += v;
  const int offset = (1 << (6 - 1)) - 32 * sum;
  const int np = rps * rps, m = mode_idx % num_modes(w, h);
  std::vector<int> raw(np);
  for (int pos = 0; pos < np; pos++) {
    int dot = 0;
    if (sid == 0)
      for (int i = 0; i < 4; i++) dot += b[i] * kMip4x4[(m * 16 + pos) * 4 + i];
    else if (sid == 1)
      for (int i = 0; i < 8; i++) dot += b[i] * kMip8x8[(m * 16 + pos) * 8 + i];
    else
      for (int i = 0; i < 7; i++) dot += b[i + 1] * kMip16x16[(m * 64 + pos) * 7 + i];
    raw[pos] = std::min(maxv, std::max(0, ((dot + offset) >> 6) + in_off));
  }
  std::vector<int> red(np);
  for (int y = 0; y < rps; y++)
    for (int x = 0; x < rps; x++) red[y * rps + x] = transpose ? raw[x * rps + y] : raw[y * rps + x];
  if (uh == 1 && uv == 1) {
    for (int i = 0; i < np; i++) out[i] = red[i];
    return;
  }
  std::vector<int> dst(w * h, 0);
  if (uh > 1 && uv == 1) {
    upsample(dst.data(), 0, red.data(), 0, left, rps, rps, 1, rps, 1, w, 1, uh);
  } else if (uh == 1 && uv > 1) {
    upsample(dst.data(), 0, red.data(), 0, above, rps, w, w, 1, w, 1, 1, uv);
  } else {
    const int hb = (uv - 1) * w, vs = w * uv;
    upsample(dst.data(), hb, red.data(), 0, left, rps, rps, 1, rps, 1, vs, uv, uh);
    std::vector<int> tmp = dst;
    upsample(dst.data(), 0, tmp.data(), hb, above, rps, w, vs, 1, w, 1, 1, uv);
  }
  for (int i = 0; i < w * h; i++) out[i] = dst[i];
}

}  // namespace orc

// predict_mip_16 of one block from its w above and h left reference samples.
extern "C" void orc_mip_predict(const int32_t* above, const int32_t* left, int w, int h, int mode, int transposed,
                                int bd, int32_t* out) {
  orc::predict_mip_bd(above, left, w, h, mode, transposed != 0, bd, out);
}

// choose_best_mip_mode_16 over the references and the source block; returns
// (transposed << 8) | mode and the SAD, and writes the best prediction.
extern "C" int orc_mip_search(const int32_t* above, const int32_t* left, const int32_t* src, int w, int h, int bd,
                              int32_t* best_pred, uint64_t* best_sad) {
  const int nm = orc::num_modes(w, h);
  std::vector<int> pred(w * h);
  int best = 0;
  uint64_t bs = UINT64_MAX;
  for (int tr = 0; tr < 2; tr++)
    for (int m = 0; m < nm; m++) {
      orc::predict_mip_bd(above, left, w, h, m, tr != 0, bd, pred.data());
      uint64_t sad = 0;
      for (int i = 0; i < w * h; i++) sad += (uint64_t)std::abs(src[i] - std::min(65535, std::max(0, pred[i])));
      if (sad < bs) {
        bs = sad;
        best = (tr << 8) | m;
        for (int i = 0; i < w * h; i++) best_pred[i] = pred[i];
      }
    }
  *best_sad = bs;
  return best;
}
