// P pictures of the multi-tool stream on the GPU (vvcg_decode_p_batch) and
// the context's picture buffer (vvcg_dpb_*). Included at the end of vvcg.cu.
//
// decode_inter_picture (slice.rs:3677-3834) reconstructs every CTU as one
// coding unit: the inter prediction of its motion (predict_inter_pu,
// inter.rs:1734: 8-bit uni-prediction with the luma 8-tap / chroma 4-tap
// filters of interpolate_luma_block :896 and interpolate_chroma_block_420
// :1056, reference reads clamped to the picture), each component's residual
// (reconstruct_component_full, slice.rs:1920: DCT-2 or transform skip,
// regular or dependent dequantisation) and the clipped sum. Every CTU of a
// picture depends only on the reference pictures, so one CTA per CTU runs
// them all at once: warp 0 turns the Y levels into the residual (the TU
// path's warp_tu_inverse) while warps 1 and 2 do Cb and Cr and then, with
// warp 3, stage each component's reference window and filter it into a
// prediction in shared memory; all four warps then store the clipped sums
// into the picture's buffer slot. apply_inter_loop_filters'
// CTU-boundary deblocking (slice.rs:2291) follows for pictures that enable
// it. Pictures are grouped into levels by their slots (a picture waits for
// the pictures before it that write a slot it reads or writes, or read the
// slot it writes); one launch runs a level.

namespace vvcg {

constexpr int kPWarps = 4;

struct PPicDev {
  const vvcg_inter_cu* cus;
  uint16_t* out[3];
  const uint16_t* ref[4][3];
  int32_t stride[3];
  int32_t w, h, gw, gh, lqp, cqp, num_refs;
  uint32_t flags;  // bit0 dependent quantisation, bit1 sparse levels
};

// The MC window of one component (the luma 39 x 39, or chroma 19 x 19) and
// the horizontal pass's rows. 16 bits suffice: samples are 8-bit and the
// horizontal sums of the 8-tap / 4-tap filters stay within +-32767.
struct PMcSmem {
  int16_t win[39][40];
  int16_t tmp[39][32];
};

// Barrier of warps 1..3, the prediction warps of a CTA.
__device__ __forceinline__ void p_mc_sync() { asm volatile("bar.sync 1, 96;" ::: "memory"); }

// The inter prediction of one component of a coding unit into `pred` (int16,
// n x n raster), by the prediction warps (thread `tid` of 96).
__device__ void p_predict_component(const PPicDev& P, const vvcg_inter_cu& rec, int comp, int bx, int by,
                                    int16_t* __restrict__ pred, PMcSmem& S, int tid) {
  constexpr int nth = 96;
  const bool luma = comp == 0;
  const int n = luma ? 32 : 16, ntap = luma ? 8 : 4, half = luma ? 3 : 1;
  const int pw = luma ? P.w : P.w / 2, ph = luma ? P.h : P.h / 2;
  const int x0 = luma ? bx : bx / 2, y0 = luma ? by : by / 2;
  const int rstride = P.stride[comp];
  const bool has = (rec.inter_dir & 1) && rec.ref_idx[0] >= 0;
  if (!has) {  // predict_inter_pu without a usable list: 128
    for (int i = tid; i < n * n; i += nth) pred[i] = 128;
    return;
  }
  const uint16_t* ref = P.ref[min((int)rec.ref_idx[0], P.num_refs - 1)][comp];
  // 1/16-sample luma motion; 4:2:0 chroma reads it as 1/32 of a chroma sample
  const int mx = rec.mv[0][0], my = rec.mv[0][1];
  const int dx = luma ? mx >> 4 : mx >> 5, dy = luma ? my >> 4 : my >> 5;
  const int fx = luma ? mx & 15 : mx & 31, fy = luma ? my & 15 : my & 31;
  const bool alt = (rec.flags & VVCG_INTER_CU_ALT_HPEL) != 0;
  int fh[8], fv[8];
  for (int k = 0; k < ntap; k++) {
    if (luma) {
      fh[k] = (alt && fx == 8) ? c_luma_alt_hpel[k] : c_luma_taps8[fx * 8 + k];
      fv[k] = (alt && fy == 8) ? c_luma_alt_hpel[k] : c_luma_taps8[fy * 8 + k];
    } else {
      fh[k] = c_chroma_taps4[fx * 4 + k];
      fv[k] = c_chroma_taps4[fy * 4 + k];
    }
  }
  const int wx0 = x0 + dx - half, wy0 = y0 + dy - half, ww = n + ntap - 1;
  p_mc_sync();  // the window buffer is free
  for (int i = tid; i < ww * ww; i += nth) {
    const int yy = i / ww, xx = i % ww;
    const int gx = clampi(wx0 + xx, 0, pw - 1), gy = clampi(wy0 + yy, 0, ph - 1);
    S.win[yy][xx] = (int16_t)ref[(size_t)gy * rstride + gx];
  }
  p_mc_sync();
  if (fx != 0 && fy != 0) {  // horizontal pass over every window row (shift1 is 0 at 8 bits)
    for (int i = tid; i < n * ww; i += nth) {
      const int x = i % n, yy = i / n;
      int s = 0;
      for (int k = 0; k < ntap; k++) s += fh[k] * S.win[yy][x + k];
      S.tmp[yy][x] = (int16_t)s;
    }
    p_mc_sync();
  }
  for (int i = tid; i < n * n; i += nth) {
    const int x = i % n, y = i / n;
    int p;
    if (fx == 0 && fy == 0) {
      p = S.win[y + half][x + half];
    } else if (fy == 0) {
      int s = 0;
      for (int k = 0; k < ntap; k++) s += fh[k] * S.win[y + half][x + k];
      p = clampi((s + 32) >> 6, 0, 255);
    } else if (fx == 0) {
      int s = 0;
      for (int k = 0; k < ntap; k++) s += fv[k] * S.win[y + k][x + half];
      p = clampi((s + 32) >> 6, 0, 255);
    } else {
      int s = 0;
      for (int k = 0; k < ntap; k++) s += fv[k] * S.tmp[y + k][x];
      p = clampi((s + 2048) >> 12, 0, 255);
    }
    pred[i] = (int16_t)p;
  }
}

// Grid: (CTUs of the largest picture of the level, pictures of the level).
// Warp 0 turns the luma levels into the residual while warps 1 and 2 do the
// chroma ones and then, with warp 3, the three predictions; all four warps
// then add, clip and store.
__global__ void __launch_bounds__(kPWarps * 32, 7)
k_p_cu(const PPicDev* __restrict__ pics, const int16_t* __restrict__ levels, uint64_t n_levels, uint32_t* status) {
  __shared__ __align__(16) int32_t ws_luma[2][1024 + kTuPad];     // the luma warp's transform tiles
  __shared__ __align__(16) int32_t ws_chroma[2][2][256 + kTuPad];  // the chroma warps' tiles
  __shared__ __align__(16) PMcSmem mc;
  __shared__ __align__(16) int16_t res[1024 + 2 * 256];
  __shared__ __align__(16) int16_t pred[1024 + 2 * 256];
  __shared__ __align__(16) int16_t dense[1024 + 2 * 256];  // sparse TBs expanded (same layout as res)
  const PPicDev& P = pics[blockIdx.y];
  const int cu = blockIdx.x;
  if (cu >= P.gw * P.gh) return;
  const vvcg_inter_cu rec = P.cus[cu];
  const int bx = (cu % P.gw) * 32, by = (cu / P.gw) * 32;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (wid < 3) {
    const int c = wid, n = c ? 256 : 1024, off_res = c == 0 ? 0 : (c == 1 ? 1024 : 1280);
    int16_t* r = res + off_res;
    bool coded = (rec.cbf >> c) & 1;
    if (coded) {
      const int off = rec.level_off[c];
      const int16_t* src = levels + off;
      bool ok = off >= 0 && !(rec.tu_tools >> 3);
      if (ok && (P.flags & 2)) {  // sparse: count, unused word, (index, level) pairs
        const int cnt = (off & 1) || (uint64_t)off + 2 > n_levels ? -1 : levels[off];
        ok = cnt >= 0 && cnt <= n && (uint64_t)off + 2 + 2 * (uint64_t)cnt <= n_levels &&
             expand_sparse(levels + off, cnt, n, dense + off_res, lane);
        src = dense + off_res;
      } else if (ok) {
        ok = (uint64_t)off + (uint64_t)n <= n_levels;
      }
      if (!ok) {
        if (lane == 0) atomicOr(status, kStatusBadRecord);
        coded = false;
      } else {
        const bool ts = (rec.tu_tools >> c) & 1;
        const int q = c ? P.cqp : P.lqp;
        vvcg_tu_rec t;
        t.log2_w = t.log2_h = (uint8_t)(c ? 4 : 5);
        t.bit_depth = 8;
        t.qp = (uint8_t)(ts ? max(4, q) : q);
        t.flags = ts ? VVCG_TU_TRANSFORM_SKIP : ((P.flags & 1) ? VVCG_TU_DEP_QUANT : 0);
        t.mts_idx = t.lfnst_idx = t.lfnst_mode = 0;
        t.in_off = t.out_off = 0;
        int32_t* A = c ? ws_chroma[c - 1][0] : ws_luma[0];
        int32_t* B = c ? ws_chroma[c - 1][1] : ws_luma[1];
        warp_tu_inverse(t, src, r, A, B, lane);
      }
    }
    if (!coded)
      for (int i = lane; i < n; i += 32) r[i] = 0;
  }
  if (wid >= 1)
    for (int c = 0; c < 3; c++)
      p_predict_component(P, rec, c, bx, by, pred + (c == 0 ? 0 : (c == 1 ? 1024 : 1280)), mc, threadIdx.x - 32);
  __syncthreads();
  // reconstruction: clip(prediction + residual), two samples per store
  for (int i = threadIdx.x; i < (1024 + 512) / 2; i += blockDim.x) {
    const int e = 2 * i;
    const int comp = e < 1024 ? 0 : (e < 1280 ? 1 : 2);
    const int n = comp ? 16 : 32, base = comp == 0 ? 0 : (comp == 1 ? 1024 : 1280);
    const int k = e - base, x = k % n, y = k / n;
    const int x0 = comp ? bx / 2 : bx, y0 = comp ? by / 2 : by;
    const uint32_t pv = *reinterpret_cast<const uint32_t*>(&pred[e]);
    const uint32_t rv = *reinterpret_cast<const uint32_t*>(&res[e]);
    const int v0 = clampi((int)(int16_t)(pv & 0xFFFFu) + (int)(int16_t)(rv & 0xFFFFu), 0, 255);
    const int v1 = clampi((int)(int16_t)(pv >> 16) + (int)(int16_t)(rv >> 16), 0, 255);
    *reinterpret_cast<uint32_t*>(P.out[comp] + (size_t)(y0 + y) * P.stride[comp] + x0 + x) =
        (uint32_t)v0 | ((uint32_t)v1 << 16);
  }
}

}  // namespace vvcg

// ---------------------------------------------------------------------------
// Picture buffer and P-picture state of a context.
// ---------------------------------------------------------------------------
struct PState {
  uint32_t slots = 0, w = 0, h = 0, stride[3] = {0, 0, 0};
  uint64_t slot_samples = 0;
  DevBuf arena, d_cus, d_levels, d_cells, d_pics, d_status;
  uint16_t* plane(uint32_t slot, int comp) const {
    uint16_t* base = (uint16_t*)arena.p + slot * slot_samples;
    if (comp == 0) return base;
    return base + (uint64_t)stride[0] * h + (comp == 2 ? (uint64_t)stride[1] * (h / 2) : 0);
  }
};

void p_state_free(PState* s) {
  if (!s) return;
  for (DevBuf* b : {&s->arena, &s->d_cus, &s->d_levels, &s->d_cells, &s->d_pics, &s->d_status}) b->release();
  delete s;
}

static_assert(sizeof(vvcg_inter_cu) == 48, "inter CU layout");
static_assert(sizeof(vvcg_p_pic) == 36, "P picture layout");

extern "C" vvcg_status vvcg_dpb_reserve(vvcg_ctx* ctx, uint32_t slots, uint32_t width, uint32_t height) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!slots || slots > 1024 || !width || !height || (width & 1) || (height & 1))
    return fail(ctx, VVCG_INVALID_INPUT, "picture buffer: 1..1024 slots of a nonzero even size");
  if ((uint64_t)width * height > kMaxLumaSamples) return fail(ctx, VVCG_LIMIT_EXCEEDED, "picture too large");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "sync");
  if (!ctx->p) ctx->p = new PState();
  PState& s = *ctx->p;
  s.w = width;
  s.h = height;
  s.stride[0] = (width + 63) & ~63u;
  s.stride[1] = s.stride[2] = ((width / 2) + 63) & ~63u;
  s.slot_samples = (uint64_t)s.stride[0] * height + 2ull * s.stride[1] * (height / 2);
  s.slots = 0;
  CK(s.arena.reserve(slots * s.slot_samples * sizeof(uint16_t)), "cudaMalloc");
  s.slots = slots;
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_dpb_plane(vvcg_ctx* ctx, uint32_t slot, uint32_t comp, void** dev_ptr, uint32_t* stride) {
  if (!ctx || !dev_ptr || !ctx->p || slot >= ctx->p->slots || comp > 2) return VVCG_INVALID_INPUT;
  *dev_ptr = ctx->p->plane(slot, (int)comp);
  if (stride) *stride = ctx->p->stride[comp];
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_dpb_store(vvcg_ctx* ctx, uint32_t pic, uint32_t slot) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!ctx->p || slot >= ctx->p->slots) return fail(ctx, VVCG_INVALID_INPUT, "no such picture-buffer slot");
  if (!ctx->prepared || pic >= ctx->num_pics) return fail(ctx, VVCG_INVALID_INPUT, "no such batch picture");
  const PicLayout& L = ctx->layout[pic];
  const DevPic& D = ctx->pics[pic];
  PState& s = *ctx->p;
  if (D.bd != 8 || D.cf != 1 || (uint32_t)L.pw[0] != s.w || (uint32_t)L.ph[0] != s.h)
    return fail(ctx, VVCG_INVALID_INPUT, "batch picture %u is not an 8-bit 4:2:0 picture of the buffer's size", pic);
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  for (int c = 0; c < 3; c++) {
    void* src = nullptr;
    uint32_t sstride = 0;
    vvcg_batch_plane(ctx, pic, (uint32_t)c, &src, &sstride);
    CK(cudaMemcpy2DAsync(s.plane(slot, c), s.stride[c] * 2, src, (size_t)sstride * 2, (size_t)L.pw[c] * 2, L.ph[c],
                         cudaMemcpyDeviceToDevice, ctx->stream),
       "copy");
  }
  return VVCG_OK;
}

static vvcg_status dpb_copy(vvcg_ctx* ctx, uint32_t slot, const void* const* ptr, const uint32_t* strides, bool in) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!ctx->p || slot >= ctx->p->slots) return fail(ctx, VVCG_INVALID_INPUT, "no such picture-buffer slot");
  PState& s = *ctx->p;
  for (int c = 0; c < 3; c++)
    if (!ptr[c] || strides[c] < (c ? s.w / 2 : s.w)) return fail(ctx, VVCG_INVALID_INPUT, "plane %d", c);
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  for (int c = 0; c < 3; c++) {
    const uint32_t pw = c ? s.w / 2 : s.w, ph = c ? s.h / 2 : s.h;
    if (in)
      CK(cudaMemcpy2DAsync(s.plane(slot, c), s.stride[c] * 2, ptr[c], (size_t)strides[c] * 2, (size_t)pw * 2, ph,
                           cudaMemcpyDefault, ctx->stream),
         "upload");
    else
      CK(cudaMemcpy2DAsync(const_cast<void*>(ptr[c]), (size_t)strides[c] * 2, s.plane(slot, c), s.stride[c] * 2,
                           (size_t)pw * 2, ph, cudaMemcpyDefault, ctx->stream),
         "download");
  }
  CK(cudaStreamSynchronize(ctx->stream), "sync");
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_dpb_upload(vvcg_ctx* ctx, uint32_t slot, const vvcg_plane_in planes[3]) {
  if (!ctx || !planes) return VVCG_INVALID_INPUT;
  const void* p[3] = {planes[0].data, planes[1].data, planes[2].data};
  const uint32_t st[3] = {planes[0].stride, planes[1].stride, planes[2].stride};
  return dpb_copy(ctx, slot, p, st, true);
}

extern "C" vvcg_status vvcg_dpb_download(vvcg_ctx* ctx, uint32_t slot, const vvcg_plane_out planes[3]) {
  if (!ctx || !planes) return VVCG_INVALID_INPUT;
  const void* p[3] = {planes[0].data, planes[1].data, planes[2].data};
  const uint32_t st[3] = {planes[0].stride, planes[1].stride, planes[2].stride};
  return dpb_copy(ctx, slot, p, st, false);
}

extern "C" vvcg_status vvcg_decode_p_batch(vvcg_ctx* ctx, const vvcg_p_pic* pics, uint32_t num_pics,
                                           const vvcg_inter_cu* cus, uint32_t num_cus, const int16_t* levels,
                                           uint64_t num_levels) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_pics) return VVCG_OK;
  if (!pics || !cus || (!levels && num_levels)) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  if (num_pics > 65535) return fail(ctx, VVCG_LIMIT_EXCEEDED, "more than 65535 pictures in one call");
  if (!ctx->p || !ctx->p->slots) return fail(ctx, VVCG_INVALID_INPUT, "no picture buffer (vvcg_dpb_reserve)");
  PState& s = *ctx->p;
  const uint32_t gw = s.w / 32, gh = s.h / 32;
  if (s.w % 32 || s.h % 32) return fail(ctx, VVCG_INVALID_INPUT, "picture buffer size is not a multiple of 32");
  // validation of pictures and records, and the dependency level of each picture
  std::vector<int> level(num_pics, 0);
  int num_levels_dep = 0;
  for (uint32_t i = 0; i < num_pics; i++) {
    const vvcg_p_pic& p = pics[i];
    if (p.width != s.w || p.height != s.h) return fail(ctx, VVCG_INVALID_INPUT, "picture %u: size", i);
    if (p.qp > 63 || (p.options & ~(uint32_t)(VVCG_SLICE_DEP_QUANT | VVCG_SLICE_DEBLOCK | VVCG_SLICE_SIGN_HIDING)))
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: QP or options", i);
    if (p.num_refs < 1 || p.num_refs > 4 || p.out_slot < 0 || (uint32_t)p.out_slot >= s.slots)
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: reference count or output slot", i);
    for (int r = 0; r < p.num_refs; r++)
      if (p.ref_slot[r] < 0 || (uint32_t)p.ref_slot[r] >= s.slots || p.ref_slot[r] == p.out_slot)
        return fail(ctx, VVCG_INVALID_INPUT, "picture %u: reference slot %d", i, r);
    if ((uint64_t)p.cu_offset + (uint64_t)gw * gh > num_cus)
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: records past the array", i);
    for (uint32_t k = 0; k < gw * gh; k++) {
      const vvcg_inter_cu& r = cus[p.cu_offset + k];
      if (r.tu_tools >> 3 || (r.cbf >> 3)) return fail(ctx, VVCG_INVALID_INPUT, "picture %u CU %u: flags", i, k);
      for (int c = 0; c < 3; c++)
        if (((r.cbf >> c) & 1) &&
            (r.level_off[c] < 0 ||
             !tb_level_extent(levels, num_levels, (uint64_t)r.level_off[c], c ? 256 : 1024, p.sparse != 0)))
          return fail(ctx, VVCG_INVALID_INPUT, "picture %u CU %u: levels of component %d", i, k, c);
    }
    auto reads = [&](const vvcg_p_pic& q, int32_t slot) {
      for (int r = 0; r < q.num_refs; r++)
        if (q.ref_slot[r] == slot) return true;
      return false;
    };
    for (uint32_t j = 0; j < i; j++)
      if (reads(p, pics[j].out_slot) || pics[j].out_slot == p.out_slot || reads(pics[j], p.out_slot))
        level[i] = std::max(level[i], level[j] + 1);
    num_levels_dep = std::max(num_levels_dep, level[i] + 1);
  }
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  // uploads: records, levels, deblocking cells, the per-picture descriptors
  const uint64_t ncu = (uint64_t)num_cus;
  CK(s.d_cus.reserve(ncu * sizeof(vvcg_inter_cu)), "cudaMalloc");
  CK(s.d_levels.reserve(std::max<uint64_t>(num_levels, 1) * sizeof(int16_t)), "cudaMalloc");
  CK(s.d_cells.reserve((uint64_t)num_pics * gw * gh * sizeof(vvcg_ctu_motion)), "cudaMalloc");
  CK(s.d_pics.reserve(num_pics * sizeof(vvcg::PPicDev)), "cudaMalloc");
  CK(s.d_status.reserve(sizeof(uint32_t)), "cudaMalloc");
  CK(cudaMemcpyAsync(s.d_cus.p, cus, ncu * sizeof(vvcg_inter_cu), cudaMemcpyHostToDevice, ctx->stream), "upload");
  if (num_levels)
    CK(cudaMemcpyAsync(s.d_levels.p, levels, num_levels * sizeof(int16_t), cudaMemcpyHostToDevice, ctx->stream),
       "upload");
  CK(cudaMemsetAsync(s.d_status.p, 0, sizeof(uint32_t), ctx->stream), "memset");
  std::vector<vvcg_ctu_motion> cells((size_t)num_pics * gw * gh);
  std::vector<std::vector<vvcg::PPicDev>> by_level(num_levels_dep);
  for (uint32_t i = 0; i < num_pics; i++) {
    const vvcg_p_pic& p = pics[i];
    vvcg::PPicDev d{};
    d.cus = (const vvcg_inter_cu*)s.d_cus.p + p.cu_offset;
    for (int c = 0; c < 3; c++) {
      d.out[c] = s.plane((uint32_t)p.out_slot, c);
      d.stride[c] = (int32_t)s.stride[c];
      for (int r = 0; r < 4; r++) d.ref[r][c] = s.plane((uint32_t)p.ref_slot[std::min(r, p.num_refs - 1)], c);
    }
    d.w = (int32_t)s.w;
    d.h = (int32_t)s.h;
    d.gw = (int32_t)gw;
    d.gh = (int32_t)gh;
    // slice.rs:3568-3569: max(SliceQpY, 4) and max(derived_chroma_qp, 4) (hls.rs:778)
    d.lqp = std::max<int>(p.qp, 4);
    d.cqp = std::max(4, p.qp <= 26 ? (int)p.qp : (int)p.qp - 1);
    d.num_refs = p.num_refs;
    d.flags = ((p.options & VVCG_SLICE_DEP_QUANT) ? 1u : 0u) | (p.sparse ? 2u : 0u);
    by_level[level[i]].push_back(d);
    // slice.rs:2319-2326 / :2438-2444: each CTU's own L0 motion and cbfs
    for (uint32_t k = 0; k < gw * gh; k++) {
      const vvcg_inter_cu& r = cus[p.cu_offset + k];
      vvcg_ctu_motion& m = cells[(size_t)i * gw * gh + k];
      memset(&m, 0, sizeof(m));
      for (int j = 0; j < 3; j++) {
        m.mv[j][0] = r.mv[0][0];
        m.mv[j][1] = r.mv[0][1];
        m.ref[j] = r.ref_idx[0];
      }
      m.cbf = r.cbf & 7;
    }
  }
  CK(cudaMemcpyAsync(s.d_cells.p, cells.data(), cells.size() * sizeof(vvcg_ctu_motion), cudaMemcpyHostToDevice,
                     ctx->stream),
     "upload");
  std::vector<vvcg::PPicDev> flat;
  std::vector<size_t> start;
  for (auto& L : by_level) {
    start.push_back(flat.size());
    flat.insert(flat.end(), L.begin(), L.end());
  }
  CK(cudaMemcpyAsync(s.d_pics.p, flat.data(), flat.size() * sizeof(vvcg::PPicDev), cudaMemcpyHostToDevice,
                     ctx->stream),
     "upload");
  const vvcg::PPicDev* dp = (const vvcg::PPicDev*)s.d_pics.p;
  for (int L = 0; L < num_levels_dep; L++) {
    vvcg::k_p_cu<<<dim3(gw * gh, (unsigned)by_level[L].size()), vvcg::kPWarps * 32, 0, ctx->stream>>>(
        dp + start[L], (const int16_t*)s.d_levels.p, num_levels, (uint32_t*)s.d_status.p);
    ctx->launches++;
    CK(cudaGetLastError(), "P-picture launch");
    for (uint32_t i = 0; i < num_pics; i++) {
      if (level[i] != L || !(pics[i].options & VVCG_SLICE_DEBLOCK)) continue;
      uint16_t* planes[3] = {s.plane((uint32_t)pics[i].out_slot, 0), s.plane((uint32_t)pics[i].out_slot, 1),
                             s.plane((uint32_t)pics[i].out_slot, 2)};
      vvcg_status st = vvcg_deblock_ctu_edges_dev(ctx, planes, s.stride, s.w, s.h, 32, pics[i].qp,
                                                  (const vvcg_ctu_motion*)s.d_cells.p + (size_t)i * gw * gh);
      if (st != VVCG_OK) return st;
    }
  }
  uint32_t status = 0;
  CK(cudaMemcpyAsync(&status, s.d_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream), "status");
  CK(cudaStreamSynchronize(ctx->stream), "sync");
  if (status) return fail(ctx, VVCG_INVALID_INPUT, "malformed records or levels (status 0x%x)", status);
  return VVCG_OK;
}
