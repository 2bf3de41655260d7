// CNN-pruned CTU search: the pruner's logits choose, per CTU, the intra
// candidates (the top_modes most probable modes) and the split types (the
// top_splits most probable) that the full search of intra_search.cuh then
// evaluates; a head whose chosen candidates hold less than the threshold of
// its softmax probability mass (for a calibrated network: the chance that
// the full search's choice is among them), or under the max-probability
// rule whose most probable entry is below the threshold, keeps its full set
// (all 67 modes / all 6 splits). Everything
// stays on the device: requests are built from the logits by one thread per
// CTU and expanded into the 15 block slots of the search.
#pragma once
#include "cnn.cuh"
#include "intra_search.cuh"

namespace vvcg {

// Positions of the 15 blocks of a 32x32 CTU (x, y, log2 w, log2 h) by slot.
__constant__ uint8_t c_search_blocks[15][4] = {
    {0, 0, 5, 5},  {0, 0, 4, 4},  {16, 0, 4, 4}, {0, 16, 4, 4}, {16, 16, 4, 4}, {0, 0, 5, 4},  {0, 16, 5, 4}, {0, 0, 4, 5},
    {16, 0, 4, 5}, {0, 0, 5, 3},  {0, 8, 5, 4},  {0, 24, 5, 3}, {0, 0, 3, 5},   {8, 0, 4, 5},  {24, 0, 3, 5}};

// indices of the k largest of v[0..n) (ties: the lower index first)
__device__ __forceinline__ void top_k(const float* v, int n, int k, uint8_t* out) {
  uint64_t used[2] = {0, 0};
  for (int r = 0; r < k; r++) {
    int best = -1;
    for (int j = 0; j < n; j++) {
      if ((used[j >> 6] >> (j & 63)) & 1) continue;
      if (best < 0 || v[j] > v[best]) best = j;
    }
    used[best >> 6] |= 1ull << (best & 63);
    out[r] = (uint8_t)best;
  }
}

// softmax probability mass of the k entries idx[0..k) of v[0..n); idx[0] is
// the largest entry
__device__ __forceinline__ float top_mass(const float* v, int n, const uint8_t* idx, int k) {
  const float mx = v[idx[0]];
  float s = 0.0f, t = 0.0f;
  for (int j = 0; j < n; j++) s += __expf(v[j] - mx);
  for (int r = 0; r < k; r++) t += __expf(v[idx[r]] - mx);
  return t / s;
}

__global__ void k_prune_requests(const float* __restrict__ logits, const uint32_t* __restrict__ xy, int n, int width,
                                 int height, int top_modes, int top_splits, float thr, bool max_prob,
                                 vvcg_ctu_search_req* reqs, CostReq* blocks) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  vvcg_ctu_search_req r{};
  r.x = xy[2 * i];
  r.y = xy[2 * i + 1];
  const bool inside = width >= 32 && height >= 32 && r.x <= (uint32_t)width - 32 && r.y <= (uint32_t)height - 32;
  r.split_mask = inside ? 0x3F : 0;
  r.n_cand = 0;
  if (inside && logits) {
    const float* lg = logits + (size_t)i * kCnnOut;
    uint8_t cand[6];
    top_k(lg, kCnnModes, top_modes, cand);
    if (top_mass(lg, kCnnModes, cand, max_prob ? 1 : top_modes) >= thr) {
      r.n_cand = (uint8_t)top_modes;
      for (int k = 0; k < top_modes; k++) r.cand[k] = cand[k];
    }
    uint8_t sp[6];
    top_k(lg + kCnnModes, kCnnSplits, top_splits, sp);
    if (top_mass(lg + kCnnModes, kCnnSplits, sp, max_prob ? 1 : top_splits) >= thr) {
      r.split_mask = 0;
      for (int k = 0; k < top_splits; k++) r.split_mask |= (uint8_t)(1u << sp[k]);
    }
  }
  reqs[i] = r;
  for (int s = 0; s < 6; s++) {
    const int first = c_split_first[s], count = c_split_count[s];
    for (int k = 0; k < count; k++) {
      const int slot = first + k;
      CostReq b{};
      if (r.split_mask & (1u << s)) {
        b.x = r.x + c_search_blocks[slot][0];
        b.y = r.y + c_search_blocks[slot][1];
        b.log2_w = c_search_blocks[slot][2];
        b.log2_h = c_search_blocks[slot][3];
        b.n_cand = r.n_cand;
        for (int c = 0; c < 6; c++) b.cand[c] = r.cand[c];
      }  // else log2_w = 0: the slot is skipped
      b.slot = (uint16_t)slot;
      b.ctu = (uint32_t)i;
      blocks[(size_t)i * 15 + slot] = b;
    }
  }
}

}  // namespace vvcg
