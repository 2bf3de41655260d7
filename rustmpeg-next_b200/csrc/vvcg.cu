// libvvcg: C ABI of the B200 VVC reconstruction / loop-filter / MC library.
// One translation unit: the kernels live in the included .cuh headers.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/vvcg.h"
#include "alf_general.cuh"
#include "annexb.h"
#include "cnn.cuh"
#include "dbk_general.cuh"
#include "enc.cuh"
#include "filters.cuh"
#include "gen_intra.cuh"
#include "intra_search.cuh"
#include "inter_search.cuh"
#include "inter_tools.cuh"
#include "prune.cuh"
#include "split.cuh"
#include "lmcs.cuh"
#include "mc.cuh"
#include "metrics.cuh"
#include "mip.cuh"
#include "recon.cuh"
#include "tu.cuh"
#include "txsearch.cuh"
#include "umma.cuh"
#include "vvc_tables.h"
#include "vvcg_device.cuh"
#include "vvcg_tables_dev.cuh"

using namespace vvcg;

namespace {

// Picture size limit of the reference (mod.rs:91 MAX_LUMA_SAMPLES).
constexpr uint64_t kMaxLumaSamples = 35651584ull;
constexpr uint32_t kDefaultSpinLimit = 1u << 22;  // ~0.5-1 s of polling

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t reserve(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(bytes, (size_t)256);
    want += want / 4;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// Grow-only pinned host buffer (staging for asynchronous uploads). Grow it
// only when no copy from it is in flight.
struct PinnedBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t reserve(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(bytes, (size_t)4096);
    want += want / 4;
    cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

struct PicLayout {
  uint64_t plane_off[3], scratch_off[3];  // in samples within the plane arena
  int32_t stride[3], pw[3], ph[3];
  int final_in_scratch[3];
  int vis_w[3], vis_h[3];
};

}  // namespace

struct GenPass;  // the general decoder's picture pass (gen_picture.cuh)
void gen_pass_free(GenPass* g);
struct PState;  // picture buffer and P-picture state (p_picture.cuh)
void p_state_free(PState* s);

struct vvcg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  std::string err;
  uint64_t launches = 0;
  uint32_t spin_limit = kDefaultSpinLimit;
  uint32_t epoch = 0;
  int num_sms = 0;
  // batch state
  bool prepared = false;
  bool any_tu_tools = false;  // a prepared picture carries VVCG_TOOL_TU_TOOLS
  uint32_t num_pics = 0;
  std::vector<PicLayout> layout;
  std::vector<DevPic> pics;
  std::vector<RowItem> items;
  std::vector<DbfPass> dbf[4];  // luma V, luma H, chroma V, chroma H
  std::vector<SaoPass> sao;
  std::vector<AlfPass> alf;
  std::vector<SaoAlfPass> sao_alf;  // luma SAO + ALF in one pass (pictures with both)
  std::vector<CUtensorMap> tmaps;   // one per sao_alf pass: its deblocked luma plane
  uint64_t num_cus = 0, num_levels = 0, num_ctus = 0, num_aps = 0;
  // device memory
  DevBuf planes, flags, d_pics, d_items, d_dbf[4], d_sao, d_alf, d_sao_alf, d_tmaps, d_cus, d_levels, d_ctus,
      d_aps, d_ctrl;  // d_ctrl: [0] queue counter, [1] status word
  // transform-unit batches; tu_pick[forward][size bin] indexes the bin's CTA
  // widths (kTuTable), chosen by vvcg_tu_autotune (default: the middle one)
  std::vector<uint32_t> tu_idx;
  DevBuf d_tu_recs, d_tu_idx;
  uint8_t tu_pick[2][3] = {{1, 1, 1}, {1, 1, 1}};
  DevBuf d_lmcs;  // a device copy of the LMCS tables of the last call
  DevBuf d_alfp, d_alfc;  // general-decoder ALF parameters and CTU switches
  DevBuf d_search_reqs, d_search_cost, d_search_mode, d_search_ctus;  // CTU full search
  DevBuf d_cnn_pack, d_cnn_packT;  // packed bf16 convolution weights of the CNN (forward / transposed)
  DevBuf d_cnn_acts, d_cnn_logits, d_cnn_gap, d_cnn_partial;  // CNN training workspace
  DevBuf d_me_reqs, d_me_cands;  // motion-estimation requests and merge candidates
  std::vector<DbfPass> dbf_ctu;  // CTU-boundary deblocking passes of inter pictures
  DevBuf d_dbf_ctu;
  uint64_t flags_count = 0;
  int recon_per_sm = 0;  // resident k_recon_rows CTAs per SM
  // CUDA graph of vvcg_batch_run_graph for the prepared batch and one stage mask
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  uint32_t graph_mask = 0;
  uint32_t graph_launches = 0;
  // sub-contexts (own streams and arenas) of vvcg_decode_batch_pipelined
  std::vector<vvcg_ctx*> lanes;
  // pinned staging of prepare's uploads (cursor in bytes), and of the
  // rebased records of a pipelined chunk
  PinnedBuf stage, stage_cus;
  size_t stage_used = 0;
  GenPass* gen = nullptr;  // state of vvcg_gen_prepare / vvcg_gen_run
  PState* p = nullptr;     // picture buffer and P-picture state (vvcg_dpb_*, vvcg_decode_p_batch)
};

namespace {

std::mutex g_tables_mu;
bool g_tables_ready[64] = {false};

// The int16 words a TB's levels take at off: its n coefficients when dense;
// when sparse the count word, one unused word and count (index, level)
// pairs. Zero for a malformed record: past the array, an odd sparse offset
// or a count outside 0..n. The index range of each pair is checked on the
// device, where the pairs are read.
// Why a CU's tu_tools byte is outside vvcg_cu_rec's ranges, or null.
const char* cu_tu_tools_error(uint32_t t) {
  const uint32_t mts = (t >> VVCG_CU_MTS_SHIFT) & 7, lfnst = t >> VVCG_CU_LFNST_SHIFT;
  if (mts > 4) return "mts_idx above 4";
  if (lfnst > 2) return "lfnst_idx above 2";
  if (mts && lfnst) return "MTS combined with LFNST";
  if ((t & VVCG_CU_TS_Y) && (mts || lfnst)) return "luma transform skip with MTS or LFNST";
  return nullptr;
}

uint64_t tb_level_extent(const int16_t* levels, uint64_t num_levels, uint64_t off, uint64_t n, bool sparse) {
  if (!sparse) return off + n <= num_levels ? n : 0;
  if ((off & 1) || off + 2 > num_levels) return 0;
  const int cnt = levels[off];
  if (cnt < 0 || (uint64_t)cnt > n || off + 2 + 2 * (uint64_t)cnt > num_levels) return 0;
  return 2 + 2 * (uint64_t)cnt;
}

// cuTensorMapEncodeTiled, fetched from the driver through the runtime (no
// link-time dependency on libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return (EncodeTiledFn)p;
  }();
  return fn;
}

// Tensor map of a w x h plane of 16-bit samples (row pitch `stride` samples,
// a multiple of 8) whose loads copy box_w x box_h samples; false when the
// driver has no encoder or rejects the plane.
bool plane_tensor_map(CUtensorMap* m, void* base, int w, int h, int stride, int box_w, int box_h) {
  EncodeTiledFn enc = encode_tiled_fn();
  if (!enc || (reinterpret_cast<uintptr_t>(base) & 15) || (stride & 7)) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)w, (cuuint64_t)h};
  const cuuint64_t strides[1] = {(cuuint64_t)stride * 2};
  const cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)box_h};
  const cuuint32_t elem[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, base, dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

vvcg_status fail(vvcg_ctx* ctx, vvcg_status st, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return st;
}

vvcg_status cuda_fail(vvcg_ctx* ctx, cudaError_t e, const char* what) {
  return fail(ctx, VVCG_EXECUTION, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call, what)                                   \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, what); \
  } while (0)

// Grouped diagonal scan of a w x h TB (VTM ScanGenerator DIAG over 4x4-style
// coefficient groups sized by g_log2TxSubblockSize, H.266 6.5.3-6.5.4),
// raster index per scan position, capped to the top-left 32x32.
int build_scan(int w, int h, int16_t* out) {
  static const uint8_t T[8][8][2] = {
      {{0, 0}, {0, 1}, {0, 2}, {0, 3}, {0, 4}, {0, 4}, {0, 4}, {0, 4}},
      {{1, 0}, {1, 1}, {1, 1}, {1, 3}, {1, 3}, {1, 3}, {1, 3}, {1, 3}},
      {{2, 0}, {1, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{3, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
      {{4, 0}, {3, 1}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}},
  };
  int a = std::min(7, __builtin_ctz(w)), b = std::min(7, __builtin_ctz(h));
  int cgw = 1 << T[a][b][0], cgh = 1 << T[a][b][1];
  int gw = std::min(w, 32) / cgw, gh = std::min(h, 32) / cgh;
  auto diag = [](int W, int H, std::vector<std::pair<int, int>>& o) {
    o.clear();
    int line = 0, col = 0;
    for (int i = 0; i < W * H; i++) {
      o.push_back({col, line});
      if (col == W - 1 || line == 0) {
        line += col + 1;
        col = 0;
        if (line >= H) {
          col += line - (H - 1);
          line = H - 1;
        }
      } else {
        col++;
        line--;
      }
    }
  };
  std::vector<std::pair<int, int>> g, in;
  diag(gw, gh, g);
  diag(cgw, cgh, in);
  int k = 0;
  for (auto& G : g)
    for (auto& I : in) out[k++] = (int16_t)((G.second * cgh + I.second) * w + G.first * cgw + I.first);
  return k;
}

vvcg_status upload_tables(vvcg_ctx* ctx) {
  std::lock_guard<std::mutex> lk(g_tables_mu);
  if (ctx->device < 64 && g_tables_ready[ctx->device]) return VVCG_OK;
  using namespace vvc_tables;
  int ang[32], inv[32], thr[8];
  for (int i = 0; i < 32; i++) {
    ang[i] = kAngTable[i];
    inv[i] = kInvAngTable[i];
  }
  for (int i = 0; i < 8; i++) thr[i] = kIntraFilterThreshold[i];
  CK(cudaMemcpyToSymbol(c_ang_table, ang, sizeof(ang)), "tables");
  CK(cudaMemcpyToSymbol(c_inv_ang_table, inv, sizeof(inv)), "tables");
  CK(cudaMemcpyToSymbol(c_intra_filter_thr, thr, sizeof(thr)), "tables");
  CK(cudaMemcpyToSymbol(c_chroma_taps4, kChromaTaps4, sizeof(kChromaTaps4)), "tables");
  CK(cudaMemcpyToSymbol(c_cclm_div_sig, kCclmDivSig, sizeof(kCclmDivSig)), "tables");
  CK(cudaMemcpyToSymbol(c_inv_quant_scale, kInvQuantScale, sizeof(kInvQuantScale)), "tables");
  CK(cudaMemcpyToSymbol(c_quant_scale, kQuantScale, sizeof(kQuantScale)), "tables");
  CK(cudaMemcpyToSymbol(c_dbf_tc, kDbfTc, sizeof(kDbfTc)), "tables");
  CK(cudaMemcpyToSymbol(c_dbf_beta, kDbfBeta, sizeof(kDbfBeta)), "tables");
  CK(cudaMemcpyToSymbol(c_luma_taps8, kLumaTaps8, sizeof(kLumaTaps8)), "tables");
  CK(cudaMemcpyToSymbol(c_affine_taps8, kAffineTaps8, sizeof(kAffineTaps8)), "tables");
  CK(cudaMemcpyToSymbol(c_luma_alt_hpel, kLumaAltHpel, sizeof(kLumaAltHpel)), "tables");
  CK(cudaMemcpyToSymbol(c_bcw_weights, kBcwWeights, sizeof(kBcwWeights)), "tables");
  CK(cudaMemcpyToSymbol(c_geo_dis, kGeoDis, sizeof(kGeoDis)), "tables");
  CK(cudaMemcpyToSymbol(c_geo_angle_to_mask, kGeoAngleToMask, sizeof(kGeoAngleToMask)), "tables");
  CK(cudaMemcpyToSymbol(c_bilinear4, kBilinear4, sizeof(kBilinear4)), "tables");
  CK(cudaMemcpyToSymbol(c_alf_clip, kAlfClip, sizeof(kAlfClip)), "tables");
  CK(cudaMemcpyToSymbol(c_alf_fixed, kAlfFixedCoeff, sizeof(kAlfFixedCoeff)), "tables");
  CK(cudaMemcpyToSymbol(c_alf_class_to_filter, kAlfClassToFilter, sizeof(kAlfClassToFilter)), "tables");
  CK(cudaMemcpyToSymbol(c_alf_transpose_perm, kAlfTransposePerm, sizeof(kAlfTransposePerm)), "tables");
  static const int8_t* d2[6] = {kDct2N2, kDct2N4, kDct2N8, kDct2N16, kDct2N32, kDct2N64};
  for (int i = 0; i < 6; i++) {
    int n = 2 << i;
    CK(cudaMemcpyToSymbol(g_dct2_m, d2[i], n * n, (size_t)i * 64 * 64), "tables");
  }
  static const int8_t* s7[4] = {kDst7N4, kDst7N8, kDst7N16, kDst7N32};
  static const int8_t* c8[4] = {kDct8N4, kDct8N8, kDct8N16, kDct8N32};
  for (int i = 0; i < 4; i++) {
    int n = 4 << i;
    CK(cudaMemcpyToSymbol(g_dst7_m, s7[i], n * n, (size_t)i * 32 * 32), "tables");
    CK(cudaMemcpyToSymbol(g_dct8_m, c8[i], n * n, (size_t)i * 32 * 32), "tables");
  }
  std::vector<int16_t> scans(36 * 1024, 0);
  int32_t offs[36];
  int pos = 0;
  for (int a = 1; a <= 6; a++)
    for (int b = 1; b <= 6; b++) {
      offs[(a - 1) * 6 + (b - 1)] = pos;
      pos += build_scan(1 << a, 1 << b, scans.data() + pos);
    }
  CK(cudaMemcpyToSymbol(g_scan, scans.data(), sizeof(int16_t) * pos), "tables");
  CK(cudaMemcpyToSymbol(g_scan_off, offs, sizeof(offs)), "tables");
  std::vector<int16_t> scan_pos(36 * 1024, 0);
  for (int a = 1; a <= 5; a++)
    for (int b = 1; b <= 5; b++) {
      const int o = offs[(a - 1) * 6 + (b - 1)], n = (1 << a) * (1 << b);
      for (int k = 0; k < n; k++) scan_pos[o + scans[o + k]] = (int16_t)k;
    }
  CK(cudaMemcpyToSymbol(g_scan_pos, scan_pos.data(), sizeof(int16_t) * scan_pos.size()), "tables");
  // every (log2 w, log2 h) in 0..6 for the transform-unit kernels
  std::vector<int16_t> tu_scans(kTuScanTotal, 0);
  int32_t tu_offs[49];
  pos = 0;
  for (int a = 0; a <= 6; a++)
    for (int b = 0; b <= 6; b++) {
      tu_offs[a * 7 + b] = pos;
      pos += build_scan(1 << a, 1 << b, tu_scans.data() + pos);
    }
  if (pos != kTuScanTotal) return fail(ctx, VVCG_EXECUTION, "scan table size %d", pos);
  CK(cudaMemcpyToSymbol(g_tu_scan, tu_scans.data(), sizeof(int16_t) * pos), "tables");
  CK(cudaMemcpyToSymbol(g_tu_scan_off, tu_offs, sizeof(tu_offs)), "tables");
  CK(cudaMemcpyToSymbol(g_lfnst8, kLfnst8x8, sizeof(kLfnst8x8)), "tables");
  CK(cudaMemcpyToSymbol(g_lfnst4, kLfnst4x4, sizeof(kLfnst4x4)), "tables");
  CK(cudaMemcpyToSymbol(g_lfnst_lut, kLfnstLut, sizeof(kLfnstLut)), "tables");
  CK(cudaMemcpyToSymbol(g_mip4, kMip4x4, sizeof(kMip4x4)), "tables");
  CK(cudaMemcpyToSymbol(g_mip8, kMip8x8, sizeof(kMip8x8)), "tables");
  CK(cudaMemcpyToSymbol(g_mip16, kMip16x16, sizeof(kMip16x16)), "tables");
  CK(cudaDeviceSynchronize(), "tables");
  if (ctx->device < 64) g_tables_ready[ctx->device] = true;
  return VVCG_OK;
}

uint32_t align_up(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }
bool encode_geometry(const vvcg_pic_desc& d, uint32_t* cus, uint64_t* levels);  // defined with the encoder
int ilog2_host(int v) { return __builtin_ctz((unsigned)v); }

// Copies v to the device through the pinned staging buffer when it has room
// (an asynchronous copy that does not hold the host), else directly.
template <typename T>
vvcg_status upload_vec(vvcg_ctx* ctx, DevBuf& buf, const std::vector<T>& v) {
  if (v.empty()) return VVCG_OK;
  const size_t bytes = sizeof(T) * v.size();
  CK(buf.reserve(bytes), "cudaMalloc");
  const void* src = v.data();
  if (ctx->stage.p && ctx->stage_used + bytes <= ctx->stage.cap) {
    void* dst = (char*)ctx->stage.p + ctx->stage_used;
    memcpy(dst, v.data(), bytes);
    ctx->stage_used += (bytes + 255) & ~(size_t)255;
    src = dst;
  }
  CK(cudaMemcpyAsync(buf.p, src, bytes, cudaMemcpyHostToDevice, ctx->stream), "upload");
  return VVCG_OK;
}

bool tu_set_smem_limits();  // every transform-unit kernel variant may use its shared memory

}  // namespace

extern "C" {

vvcg_status vvcg_ctx_create(const vvcg_config* cfg, vvcg_ctx** out) {
  if (!out) return VVCG_INVALID_INPUT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return VVCG_UNAVAILABLE;
  }
  int dev = cfg ? cfg->device : 0;
  if (dev < 0 || dev >= ndev) return VVCG_INVALID_INPUT;
  vvcg_ctx* ctx = new vvcg_ctx();
  ctx->device = dev;
  if (cfg && cfg->spin_limit) ctx->spin_limit = cfg->spin_limit;
  if (cudaSetDevice(dev) != cudaSuccess) {
    delete ctx;
    return VVCG_UNAVAILABLE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    delete ctx;
    return VVCG_UNAVAILABLE;
  }
  ctx->num_sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return VVCG_UNAVAILABLE;
  }
  ctx->stream = ctx->own_stream;
  if (cudaFuncSetAttribute(k_recon_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(kWarpsPerCta * sizeof(WaveWs))) != cudaSuccess) {
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return VVCG_UNAVAILABLE;
  }
  if (cudaFuncSetAttribute(k_encode_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(kEncWarps * sizeof(EncWs))) != cudaSuccess) {
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return VVCG_UNAVAILABLE;
  }
  if (cudaFuncSetAttribute(k_luma_tx_search, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(TxsWs)) != cudaSuccess) {
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return VVCG_UNAVAILABLE;
  }
  if (!tu_set_smem_limits()) {
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return VVCG_UNAVAILABLE;
  }
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->recon_per_sm, k_recon_rows, kWarpsPerCta * 32,
                                                    kWarpsPerCta * sizeof(WaveWs)) != cudaSuccess) {
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return VVCG_UNAVAILABLE;
  }
  if (upload_tables(ctx) != VVCG_OK) {
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return VVCG_UNAVAILABLE;
  }
  if (cfg && cfg->reserve_bytes) ctx->planes.reserve(cfg->reserve_bytes);
  if (ctx->d_ctrl.reserve(64) != cudaSuccess) {
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return VVCG_UNAVAILABLE;
  }
  cudaMemset(ctx->d_ctrl.p, 0, 64);
  *out = ctx;
  return VVCG_OK;
}

void vvcg_ctx_destroy(vvcg_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  for (vvcg_ctx* l : ctx->lanes) vvcg_ctx_destroy(l);
  gen_pass_free(ctx->gen);
  p_state_free(ctx->p);
  ctx->stage.release();
  ctx->stage_cus.release();
  for (DevBuf* b : {&ctx->planes, &ctx->flags, &ctx->d_pics, &ctx->d_items, &ctx->d_dbf[0],
                    &ctx->d_dbf[1], &ctx->d_dbf[2], &ctx->d_dbf[3], &ctx->d_sao, &ctx->d_alf, &ctx->d_sao_alf, &ctx->d_tmaps,
                    &ctx->d_cus, &ctx->d_levels, &ctx->d_ctus, &ctx->d_aps, &ctx->d_ctrl,
                    &ctx->d_tu_recs, &ctx->d_tu_idx, &ctx->d_lmcs, &ctx->d_alfp, &ctx->d_alfc,
                    &ctx->d_search_reqs, &ctx->d_search_cost, &ctx->d_search_mode, &ctx->d_search_ctus,
                    &ctx->d_cnn_pack, &ctx->d_cnn_packT, &ctx->d_cnn_acts, &ctx->d_cnn_logits, &ctx->d_cnn_gap,
                    &ctx->d_cnn_partial, &ctx->d_me_reqs, &ctx->d_me_cands, &ctx->d_dbf_ctu})
    b->release();
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

const char* vvcg_last_error(const vvcg_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

vvcg_status vvcg_set_stream(vvcg_ctx* ctx, void* stream) {
  if (!ctx) return VVCG_INVALID_INPUT;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return VVCG_OK;
}

uint64_t vvcg_kernel_launches(const vvcg_ctx* ctx) {
  if (!ctx) return 0;
  uint64_t n = ctx->launches;
  for (const vvcg_ctx* l : ctx->lanes) n += l->launches;
  return n;
}

vvcg_status vvcg_batch_prepare(vvcg_ctx* ctx, const vvcg_batch* b) {
  if (!ctx) return VVCG_INVALID_INPUT;
  ctx->prepared = false;
  // a captured graph holds this batch's buffers and launch shapes
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  ctx->graph_exec = nullptr;
  ctx->graph = nullptr;
  if (!b || !b->pics || b->num_pics == 0) return fail(ctx, VVCG_INVALID_INPUT, "empty batch");
  if (b->num_cus && !b->cus) return fail(ctx, VVCG_INVALID_INPUT, "missing CU records");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  // earlier work of this context may still read the staging buffer or the arena
  CK(cudaStreamSynchronize(ctx->stream), "prepare");
  ctx->stage_used = 0;
  const uint32_t np = b->num_pics;
  ctx->num_pics = np;
  ctx->layout.assign(np, PicLayout{});
  ctx->pics.assign(np, DevPic{});
  ctx->items.clear();
  for (auto& v : ctx->dbf) v.clear();
  ctx->sao.clear();
  ctx->alf.clear();
  ctx->sao_alf.clear();
  ctx->tmaps.clear();
  ctx->num_cus = b->num_cus;
  ctx->num_levels = b->num_levels;
  ctx->num_ctus = b->num_ctus;
  ctx->num_aps = b->num_aps;
  uint64_t plane_samples = 0;
  bool any_tools = false;
  for (uint32_t i = 0; i < np; i++) {
    const vvcg_pic_desc& d = b->pics[i];
    if (d.ctu_log2 < 5 || d.ctu_log2 > 7)
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: CTU size outside 32..=128", i);
    const uint32_t ctu = 1u << d.ctu_log2;
    if (d.width < ctu || d.height < ctu || d.width % ctu || d.height % ctu)
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: coded size not aligned to the CTU grid", i);
    if ((uint64_t)d.width * d.height > kMaxLumaSamples)
      return fail(ctx, VVCG_LIMIT_EXCEEDED, "picture %u: %ux%u exceeds %llu luma samples", i,
                  d.width, d.height, (unsigned long long)kMaxLumaSamples);
    if (d.bit_depth < 8 || d.bit_depth > 12 || d.chroma_format > 3)
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: bit depth or chroma format", i);
    if (d.visible_width > d.width || d.visible_height > d.height || !d.visible_width || !d.visible_height)
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: visible size", i);
    if (d.alf_aps >= 0 && (uint32_t)d.alf_aps >= b->num_aps)
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: ALF APS index", i);
    const int tb = std::min<int>(ctu, 32);
    const int cf = d.chroma_format;
    const int sw = (cf == 1 || cf == 2) ? 2 : 1, sh = cf == 1 ? 2 : 1;
    const int tcw = cf ? std::max(tb / sw, 2) : 0, tch = cf ? std::max(tb / sh, 2) : 0;
    const uint32_t gw = d.width / tb, gh = d.height / tb;
    const uint32_t cw_ = d.width / ctu, ch_ = d.height / ctu;
    if ((uint64_t)d.cu_offset + (uint64_t)gw * gh > b->num_cus)
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: CU records out of range", i);
    const bool filt = d.tools & (VVCG_TOOL_SAO | VVCG_TOOL_ALF);
    if (filt && (!b->ctus || (uint64_t)d.ctu_offset + (uint64_t)cw_ * ch_ > b->num_ctus))
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: CTU filter records out of range", i);
    const bool tu_tools = (d.tools & VVCG_TOOL_TU_TOOLS) != 0;
    if (tu_tools)
      for (uint32_t k = 0; k < gw * gh; k++) {
        const char* why = cu_tu_tools_error(b->cus[d.cu_offset + k].tu_tools);
        if (why) return fail(ctx, VVCG_INVALID_INPUT, "picture %u CU %u: %s", i, k, why);
      }
    any_tools |= tu_tools;
    // level offsets
    const bool sparse = (d.tools & VVCG_TOOL_SPARSE_LEVELS) != 0;
    for (uint32_t k = 0; k < gw * gh; k++) {
      const vvcg_cu_rec& r = b->cus[d.cu_offset + k];
      for (int c = 0; c < (cf ? 3 : 1); c++) {
        if (!((r.cbf >> c) & 1) || r.level_off[c] < 0) continue;
        uint64_t n = c ? (uint64_t)tcw * tch : (uint64_t)tb * tb;
        if (!b->levels || !tb_level_extent(b->levels, b->num_levels, (uint64_t)r.level_off[c], n, sparse))
          return fail(ctx, VVCG_INVALID_INPUT, "picture %u CU %u: level offset out of range", i, k);
      }
    }
    PicLayout& L = ctx->layout[i];
    const int ncomp = cf ? 3 : 1;
    for (int c = 0; c < 3; c++) {
      L.pw[c] = c == 0 ? d.width : (cf ? (d.width + sw - 1) / sw : 0);
      L.ph[c] = c == 0 ? d.height : (cf ? (d.height + sh - 1) / sh : 0);
      L.vis_w[c] = c == 0 ? d.visible_width : (cf ? (d.visible_width + sw - 1) / sw : 0);
      L.vis_h[c] = c == 0 ? d.visible_height : (cf ? (d.visible_height + sh - 1) / sh : 0);
      L.stride[c] = c < ncomp ? (int32_t)align_up(L.pw[c], 64) : 0;
      L.plane_off[c] = plane_samples;
      plane_samples += c < ncomp ? (uint64_t)L.stride[c] * L.ph[c] : 0;
      L.scratch_off[c] = plane_samples;
      plane_samples += c < ncomp ? (uint64_t)L.stride[c] * L.ph[c] : 0;
      L.final_in_scratch[c] = 0;
    }
    DevPic& P = ctx->pics[i];
    P.bd = d.bit_depth;
    P.cf = cf;
    P.ctu_log2 = d.ctu_log2;
    P.ctu = ctu;
    P.tb = tb;
    P.tb_cw = tcw;
    P.tb_ch = tch;
    P.sub_w = sw;
    P.sub_h = sh;
    P.grid_w = gw;
    P.grid_h = gh;
    P.ctu_w = cw_;
    P.ctu_h = ch_;
    // slice.rs:4681-4682 Qp'Y and Qp'C, both at least 4
    const int off = 6 * (d.bit_depth - 8);
    P.lqp = std::max(std::min(63 + off, std::max(0, (int)d.slice_qp + off)), 4);
    P.cqp = std::max((int)d.chroma_qp_scaled, 4);
    P.slice_qp = d.slice_qp;
    P.tools = d.tools;
    P.aps = d.alf_aps;
    for (int c = 0; c < 3; c++) {
      P.stride[c] = L.stride[c];
      P.pw[c] = L.pw[c];
      P.ph[c] = L.ph[c];
    }
  }
  // wavefront work: CTU rows, row-major across the pictures, so a row is only
  // handed out after the row above it
  uint64_t total_rows = 0;
  std::vector<uint64_t> row_base(np);
  {
    int hmax = 0;
    for (uint32_t i = 0; i < np; i++) {
      row_base[i] = total_rows;
      total_rows += ctx->pics[i].ctu_h;
      hmax = std::max(hmax, ctx->pics[i].ctu_h);
    }
    for (int cy = 0; cy < hmax; cy++)
      for (uint32_t i = 0; i < np; i++)
        if (cy < ctx->pics[i].ctu_h) ctx->items.push_back(RowItem{i, (uint32_t)cy});
  }
  // device memory
  CK(ctx->planes.reserve(plane_samples * sizeof(uint16_t)), "cudaMalloc planes");
  const size_t flag_bytes = total_rows * kRowFlagStride * sizeof(uint64_t);
  if (ctx->flags.cap < flag_bytes) {
    CK(ctx->flags.reserve(flag_bytes), "cudaMalloc flags");
    CK(cudaMemsetAsync(ctx->flags.p, 0, ctx->flags.cap, ctx->stream), "memset flags");
  }
  ctx->flags_count = total_rows;
  CK(ctx->d_cus.reserve(std::max<uint64_t>(1, b->num_cus) * sizeof(vvcg_cu_rec)), "cudaMalloc");
  CK(ctx->d_levels.reserve(std::max<uint64_t>(1, b->num_levels) * sizeof(int16_t)), "cudaMalloc");
  CK(ctx->d_ctus.reserve(std::max<uint64_t>(1, b->num_ctus) * sizeof(vvcg_ctu_filter)), "cudaMalloc");
  CK(ctx->d_aps.reserve(std::max<uint64_t>(1, b->num_aps) * sizeof(vvcg_alf_aps)), "cudaMalloc");
  uint16_t* base = (uint16_t*)ctx->planes.p;
  for (uint32_t i = 0; i < np; i++) {
    const vvcg_pic_desc& d = b->pics[i];
    DevPic& P = ctx->pics[i];
    PicLayout& L = ctx->layout[i];
    for (int c = 0; c < 3; c++) {
      P.plane[c] = base + L.plane_off[c];
      P.scratch[c] = base + L.scratch_off[c];
    }
    P.cus = (const vvcg_cu_rec*)ctx->d_cus.p + d.cu_offset;
    P.ctus = (const vvcg_ctu_filter*)ctx->d_ctus.p + d.ctu_offset;
    P.row_done = (uint64_t*)ctx->flags.p + row_base[i] * kRowFlagStride;
    const int ncomp = P.cf ? 3 : 1;
    if (d.tools & VVCG_TOOL_DEBLOCK) {
      // slice.rs:4990-5020: luma lattice tb, CTB ctu, SliceQpY; chroma lattice
      // tb_cw, CTB height ctu / SubHeightC, QP derived_chroma_qp(SliceQpY)
      const int step = std::max(P.tb, 8), ctb = std::max(P.ctu, step);
      const int lml = step <= 4 ? 1 : (step >= 32 ? 7 : 3);
      DbfPass v{P.plane[0], P.stride[0], P.pw[0], P.ph[0], P.bd, step, ctb, (int)d.slice_qp, 2, 0, 0,
                lml, lml, 1, 0, 0};
      v.n_edges = (P.pw[0] - 8) / step;
      v.n_segs = P.ph[0] / 4;
      DbfPass h = v;
      h.n_edges = (P.ph[0] - 8) / step;
      h.n_segs = P.pw[0] / 4;
      if (v.n_edges > 0 && v.n_segs > 0) ctx->dbf[0].push_back(v);
      if (h.n_edges > 0 && h.n_segs > 0) ctx->dbf[1].push_back(h);
      if (P.cf) {
        const int cqp = std::min(63, std::max(0, (int)d.slice_qp <= 26 ? (int)d.slice_qp
                                                                        : (int)d.slice_qp - 1));
        const int cstep = std::max(P.tb_cw, 8);
        const int cctb = std::max(P.ctu / P.sub_h, cstep);
        const int clen = cstep >= 8 ? 3 : 1;
        for (int c = 1; c <= 2; c++) {
          DbfPass cv{P.plane[c], P.stride[c], P.pw[c], P.ph[c], P.bd, cstep, cctb, cqp, 2, 0, 0,
                     clen, clen, P.sub_h, 0, 0};
          cv.n_edges = P.pw[c] >= 8 ? (P.pw[c] - 4) / cstep : 0;
          cv.n_segs = P.ph[c] / (P.sub_h == 1 ? 4 : 2);
          DbfPass ch = cv;
          ch.sub = P.sub_w;
          ch.n_edges = P.ph[c] >= 8 ? (P.ph[c] - 4) / cstep : 0;
          ch.n_segs = P.pw[c] / (P.sub_w == 1 ? 4 : 2);
          if (cv.n_edges > 0 && cv.n_segs > 0) ctx->dbf[2].push_back(cv);
          if (ch.n_edges > 0 && ch.n_segs > 0) ctx->dbf[3].push_back(ch);
        }
      }
    }
    bool alf_any = false;
    if (d.tools & VVCG_TOOL_ALF)
      for (uint64_t k = 0; k < (uint64_t)P.ctu_w * P.ctu_h; k++) alf_any |= b->ctus[d.ctu_offset + k].alf_luma != 0;
    const bool sao = (d.tools & VVCG_TOOL_SAO) != 0;
    const vvcg_alf_aps* aps_dev = d.alf_aps >= 0 ? (const vvcg_alf_aps*)ctx->d_aps.p + d.alf_aps : nullptr;
    if (sao && alf_any) {
      // luma: SAO and ALF in one pass (slice.rs:5022-5069 order), deblocked
      // plane -> scratch; the tensor map is fixed up once the maps' device
      // copy exists (a null map means plain loads)
      CUtensorMap m;
      const bool ok = plane_tensor_map(&m, P.plane[0], P.pw[0], P.ph[0], P.stride[0], kSaStW, kSaStH);
      if (!ok) memset(&m, 0, sizeof(m));
      SaoAlfPass f{P.plane[0], P.scratch[0], P.ctus, aps_dev, ok ? reinterpret_cast<const CUtensorMap*>(1) : nullptr,
                   P.stride[0], P.pw[0], P.ph[0], P.bd, ilog2_host(P.ctu), P.ctu_w};
      ctx->sao_alf.push_back(f);
      ctx->tmaps.push_back(m);
      L.final_in_scratch[0] = 1;
    }
    if (sao) {
      for (int c = (alf_any ? 1 : 0); c < ncomp; c++) {
        SaoPass s{P.plane[c], P.scratch[c], P.ctus, P.stride[c], P.pw[c], P.ph[c], P.bd, c,
                  ilog2_host(c ? P.ctu / P.sub_w : P.ctu), ilog2_host(c ? P.ctu / P.sub_h : P.ctu), P.ctu_w,
                  (uint32_t)(((1ull << 32) + (uint64_t)P.ctu_w - 1) / (uint64_t)P.ctu_w)};
        ctx->sao.push_back(s);
        L.final_in_scratch[c] = 1;
      }
    } else if (alf_any) {
      AlfPass a{P.plane[0], P.scratch[0], aps_dev, P.stride[0], P.pw[0], P.ph[0], P.bd};
      ctx->alf.push_back(a);
      L.final_in_scratch[0] = 1;
    }
  }
  if (!ctx->tmaps.empty()) {
    CK(ctx->d_tmaps.reserve(sizeof(CUtensorMap) * ctx->tmaps.size()), "cudaMalloc");
    for (size_t i = 0; i < ctx->sao_alf.size(); i++)
      if (ctx->sao_alf[i].tmap) ctx->sao_alf[i].tmap = (const CUtensorMap*)ctx->d_tmaps.p + i;
  }
  // pinned staging for the uploads below (and one more picture table, which
  // the encoder uploads again)
  {
    size_t need = 2 * (sizeof(DevPic) * ctx->pics.size() + 256) + sizeof(RowItem) * ctx->items.size() + 256 +
                  sizeof(SaoPass) * ctx->sao.size() + 256 + sizeof(AlfPass) * ctx->alf.size() + 256 +
                  sizeof(SaoAlfPass) * ctx->sao_alf.size() + 256 + sizeof(CUtensorMap) * ctx->tmaps.size() + 256;
    for (int k = 0; k < 4; k++) need += sizeof(DbfPass) * ctx->dbf[k].size() + 256;
    CK(ctx->stage.reserve(need), "cudaHostAlloc");
  }
  vvcg_status st;
  if ((st = upload_vec(ctx, ctx->d_pics, ctx->pics)) != VVCG_OK) return st;
  if ((st = upload_vec(ctx, ctx->d_items, ctx->items)) != VVCG_OK) return st;
  for (int k = 0; k < 4; k++)
    if ((st = upload_vec(ctx, ctx->d_dbf[k], ctx->dbf[k])) != VVCG_OK) return st;
  if ((st = upload_vec(ctx, ctx->d_sao, ctx->sao)) != VVCG_OK) return st;
  if ((st = upload_vec(ctx, ctx->d_alf, ctx->alf)) != VVCG_OK) return st;
  if ((st = upload_vec(ctx, ctx->d_tmaps, ctx->tmaps)) != VVCG_OK) return st;
  if ((st = upload_vec(ctx, ctx->d_sao_alf, ctx->sao_alf)) != VVCG_OK) return st;
  // no wait here: the copies read pinned staging (or pageable memory the
  // driver has already staged), and the next prepare waits for the stream
  // before it reuses the staging buffer
  ctx->any_tu_tools = any_tools;
  ctx->prepared = true;
  return VVCG_OK;
}

vvcg_status vvcg_batch_upload(vvcg_ctx* ctx, const vvcg_batch* b) {
  if (!ctx || !b) return VVCG_INVALID_INPUT;
  if (!ctx->prepared) return fail(ctx, VVCG_INVALID_INPUT, "batch not prepared");
  if (b->num_cus != ctx->num_cus || b->num_levels > ctx->d_levels.cap / sizeof(int16_t) ||
      b->num_ctus != ctx->num_ctus || b->num_aps != ctx->num_aps)
    return fail(ctx, VVCG_INVALID_INPUT, "batch shape differs from the prepared one");
  ctx->num_levels = b->num_levels;
  if (b->num_cus)
    CK(cudaMemcpyAsync(ctx->d_cus.p, b->cus, sizeof(vvcg_cu_rec) * b->num_cus, cudaMemcpyHostToDevice, ctx->stream), "upload CUs");
  if (b->num_levels)
    CK(cudaMemcpyAsync(ctx->d_levels.p, b->levels, sizeof(int16_t) * b->num_levels, cudaMemcpyHostToDevice, ctx->stream), "upload levels");
  if (b->num_ctus && b->ctus)
    CK(cudaMemcpyAsync(ctx->d_ctus.p, b->ctus, sizeof(vvcg_ctu_filter) * b->num_ctus, cudaMemcpyHostToDevice, ctx->stream), "upload CTUs");
  if (b->num_aps && b->aps)
    CK(cudaMemcpyAsync(ctx->d_aps.p, b->aps, sizeof(vvcg_alf_aps) * b->num_aps, cudaMemcpyHostToDevice, ctx->stream), "upload APS");
  return VVCG_OK;
}

}  // extern "C"

namespace {

// Epoch of graph replays: the graph clears the progress words itself, and
// direct runs never use this value.
constexpr uint32_t kGraphEpoch = 0xFFFFFFFFu;

// Enqueues the stages of `mask` for the prepared batch on the context's
// stream. `epoch` tags the wavefront's progress words; with `clear_flags` the
// words are zeroed first (graph replays). Counts the launches in *launches.
vvcg_status enqueue_run(vvcg_ctx* ctx, uint32_t mask, uint32_t epoch, bool clear_flags, uint32_t* launches) {
  uint32_t* ctrl = (uint32_t*)ctx->d_ctrl.p;
  CK(cudaMemsetAsync(ctrl, 0, 2 * sizeof(uint32_t), ctx->stream), "memset");
  if ((mask & VVCG_STAGE_RECON) && clear_flags)
    CK(cudaMemsetAsync(ctx->flags.p, 0, ctx->flags_count * kRowFlagStride * sizeof(uint64_t), ctx->stream),
       "memset flags");
  if (mask & VVCG_STAGE_RECON) {
    // residuals of every coded TB (no dependencies), into the scratch planes
    uint32_t max_cus = 0;
    for (auto& P : ctx->pics) max_cus = std::max<uint32_t>(max_cus, (uint32_t)(P.grid_w * P.grid_h));
    k_residual<<<dim3((max_cus + kWarpsPerCta - 1) / kWarpsPerCta, ctx->num_pics), kWarpsPerCta * 32, 0,
                 ctx->stream>>>((const DevPic*)ctx->d_pics.p, (const int16_t*)ctx->d_levels.p,
                                ctx->num_levels, ctrl + 1);
    CK(cudaGetLastError(), "residual launch");
    (*launches)++;
    if (ctx->any_tu_tools) {  // TBs with transform skip, MTS or LFNST
      k_residual_tools<<<dim3((max_cus + kResToolWarps - 1) / kResToolWarps, ctx->num_pics), kResToolWarps * 32, 0,
                         ctx->stream>>>((const DevPic*)ctx->d_pics.p, (const int16_t*)ctx->d_levels.p,
                                        ctx->num_levels, ctrl + 1);
      CK(cudaGetLastError(), "residual (TU tools) launch");
      (*launches)++;
    }
    // prediction + reconstruction in CTU wavefront order
    const uint32_t n = (uint32_t)ctx->items.size();
    const size_t wave_smem = kWarpsPerCta * sizeof(WaveWs);
    const uint32_t warps = (uint32_t)ctx->num_sms * std::max(1, ctx->recon_per_sm) * kWarpsPerCta;
    const uint32_t grid = (std::min<uint32_t>(n, warps) + kWarpsPerCta - 1) / kWarpsPerCta;
    k_recon_rows<<<grid, kWarpsPerCta * 32, wave_smem, ctx->stream>>>(
        (const DevPic*)ctx->d_pics.p, (const RowItem*)ctx->d_items.p, n, ctrl, epoch, ctx->spin_limit, ctrl + 1);
    CK(cudaGetLastError(), "recon launch");
    (*launches)++;
  }
  if (mask & VVCG_STAGE_DEBLOCK) {
    for (int k = 0; k < 4; k++) {
      const auto& v = ctx->dbf[k];
      if (v.empty()) continue;
      uint32_t maxw = 0;
      for (auto& p : v) maxw = std::max<uint32_t>(maxw, (uint32_t)(p.n_edges * p.n_segs));
      dim3 grid((maxw + 127) / 128, (unsigned)v.size());
      const DbfPass* d = (const DbfPass*)ctx->d_dbf[k].p;
      if (k == 0) k_deblock_luma<true><<<grid, 128, 0, ctx->stream>>>(d, (int)v.size());
      if (k == 1) k_deblock_luma<false><<<grid, 128, 0, ctx->stream>>>(d, (int)v.size());
      if (k == 2) k_deblock_chroma<true><<<grid, 128, 0, ctx->stream>>>(d, (int)v.size());
      if (k == 3) k_deblock_chroma<false><<<grid, 128, 0, ctx->stream>>>(d, (int)v.size());
      CK(cudaGetLastError(), "deblock launch");
      (*launches)++;
    }
  }
  if ((mask & VVCG_STAGE_SAO) && !ctx->sao.empty()) {
    // warps: one per (CTU, group of rows), see k_sao
    uint64_t items = 0;
    for (auto& s : ctx->sao) {
      const int tpr = std::max(1, (1 << s.ctu_w_log2) >> 2), rpw = 32 / tpr, ctu_h = 1 << s.ctu_h_log2;
      const uint64_t n_ctu = (uint64_t)s.ctu_cols * ((s.h + ctu_h - 1) / ctu_h);
      items = std::max<uint64_t>(items, n_ctu * ((ctu_h + rpw - 1) / rpw));
    }
    k_sao<<<dim3((unsigned)((items + 7) / 8), (unsigned)ctx->sao.size()), 256, 0, ctx->stream>>>(
        (const SaoPass*)ctx->d_sao.p, ctrl + 1);
    CK(cudaGetLastError(), "sao launch");
    (*launches)++;
  }
  if ((mask & VVCG_STAGE_SAO) && !ctx->sao_alf.empty()) {
    // luma SAO + ALF of the pictures that use both (part of the SAO stage)
    uint32_t gx = 0, gy = 0;
    for (auto& a : ctx->sao_alf) {
      gx = std::max<uint32_t>(gx, (a.w + kAlfTw - 1) / kAlfTw);
      gy = std::max<uint32_t>(gy, (a.h + kAlfTh - 1) / kAlfTh);
    }
    k_sao_alf_luma<<<dim3(gx, gy, (unsigned)ctx->sao_alf.size()), 256, 0, ctx->stream>>>(
        (const SaoAlfPass*)ctx->d_sao_alf.p, ctx->spin_limit, ctrl + 1);
    CK(cudaGetLastError(), "sao+alf launch");
    (*launches)++;
  }
  if ((mask & VVCG_STAGE_ALF) && !ctx->alf.empty()) {
    uint32_t gx = 0, gy = 0;
    for (auto& a : ctx->alf) {
      gx = std::max<uint32_t>(gx, (a.w + kAlfTw - 1) / kAlfTw);
      gy = std::max<uint32_t>(gy, (a.h + kAlfTh - 1) / kAlfTh);
    }
    k_alf_luma<<<dim3(gx, gy, (unsigned)ctx->alf.size()), 256, 0, ctx->stream>>>(
        (const AlfPass*)ctx->d_alf.p, ctrl + 1);
    CK(cudaGetLastError(), "alf launch");
    (*launches)++;
  }
  return VVCG_OK;
}

}  // namespace

extern "C" {

vvcg_status vvcg_batch_run(vvcg_ctx* ctx, uint32_t mask) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!ctx->prepared) return fail(ctx, VVCG_INVALID_INPUT, "batch not prepared");
  bool clear = false;
  if (mask & VVCG_STAGE_RECON) {
    if (++ctx->epoch == kGraphEpoch) {  // never reuse the graph's tag
      ctx->epoch = 1;
      clear = true;
    }
  }
  uint32_t n = 0;
  vvcg_status st = enqueue_run(ctx, mask, ctx->epoch, clear, &n);
  ctx->launches += n;
  return st;
}

vvcg_status vvcg_batch_run_graph(vvcg_ctx* ctx, uint32_t mask) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!ctx->prepared) return fail(ctx, VVCG_INVALID_INPUT, "batch not prepared");
  if (!ctx->graph_exec || ctx->graph_mask != mask) {
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    if (ctx->graph) cudaGraphDestroy(ctx->graph);
    ctx->graph_exec = nullptr;
    ctx->graph = nullptr;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    uint32_t n = 0;
    vvcg_status st = enqueue_run(ctx, mask, kGraphEpoch, true, &n);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (st != VVCG_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "end capture");
    e = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      return cuda_fail(ctx, e, "graph instantiate");
    }
    ctx->graph = g;
    ctx->graph_mask = mask;
    ctx->graph_launches = n;
  }
  CK(cudaGraphLaunch(ctx->graph_exec, ctx->stream), "graph launch");
  ctx->launches += ctx->graph_launches;
  return VVCG_OK;
}

vvcg_status vvcg_batch_sync(vvcg_ctx* ctx) {
  if (!ctx) return VVCG_INVALID_INPUT;
  uint32_t status = 0;
  CK(cudaMemcpyAsync(&status, (uint32_t*)ctx->d_ctrl.p + 1, sizeof(status), cudaMemcpyDeviceToHost, ctx->stream), "status");
  CK(cudaStreamSynchronize(ctx->stream), "synchronize");
  if (status & kStatusTimeout)
    return fail(ctx, VVCG_TIMEOUT, "a wavefront wait gave up after %u polls", ctx->spin_limit);
  if (status & kStatusBadRecord) return fail(ctx, VVCG_INVALID_INPUT, "a level offset or sparse level entry was out of range");
  if (status & kStatusAlfAbort)
    return fail(ctx, VVCG_INVALID_INPUT,
                "fixed-filter ALF reached a class >= 16, where the reference aborts");
  if (status & kStatusSaoAbort)
    return fail(ctx, VVCG_INVALID_INPUT,
                "SAO edge class 3 on the first or last picture row, where the reference aborts");
  return VVCG_OK;
}

}  // extern "C"

namespace {

// The copies of vvcg_batch_download, without waiting for them. A plane whose
// rows are contiguous on both sides (both pitches equal the visible width)
// goes as one linear copy, which the copy engine moves faster than the same
// bytes as a pitched copy.
vvcg_status enqueue_download(vvcg_ctx* ctx, const vvcg_plane_out* out) {
  for (uint32_t i = 0; i < ctx->num_pics; i++) {
    const PicLayout& L = ctx->layout[i];
    const DevPic& P = ctx->pics[i];
    for (int c = 0; c < (P.cf ? 3 : 1); c++) {
      const vvcg_plane_out& o = out[i * 3 + c];
      if (!o.data) continue;
      if (o.stride < (uint32_t)L.vis_w[c]) return fail(ctx, VVCG_INVALID_INPUT, "output stride too small");
      const uint16_t* src = L.final_in_scratch[c] ? P.scratch[c] : P.plane[c];
      const uint32_t w = (uint32_t)L.vis_w[c];
      if (o.stride == w && (uint32_t)L.stride[c] == w)
        CK(cudaMemcpyAsync(o.data, src, (size_t)w * L.vis_h[c] * 2, cudaMemcpyDeviceToHost, ctx->stream),
           "download");
      else
        CK(cudaMemcpy2DAsync(o.data, (size_t)o.stride * 2, src, (size_t)L.stride[c] * 2, (size_t)w * 2,
                             L.vis_h[c], cudaMemcpyDeviceToHost, ctx->stream),
           "download");
    }
  }
  return VVCG_OK;
}

}  // namespace

extern "C" {

vvcg_status vvcg_batch_download(vvcg_ctx* ctx, const vvcg_plane_out* out) {
  if (!ctx || !out) return VVCG_INVALID_INPUT;
  if (!ctx->prepared) return fail(ctx, VVCG_INVALID_INPUT, "batch not prepared");
  const vvcg_status st = enqueue_download(ctx, out);
  if (st != VVCG_OK) return st;
  CK(cudaStreamSynchronize(ctx->stream), "download");
  return VVCG_OK;
}

vvcg_status vvcg_batch_plane(vvcg_ctx* ctx, uint32_t pic, uint32_t comp, void** ptr, uint32_t* stride) {
  if (!ctx || !ptr || !ctx->prepared || pic >= ctx->num_pics || comp > 2) return VVCG_INVALID_INPUT;
  const PicLayout& L = ctx->layout[pic];
  const DevPic& P = ctx->pics[pic];
  if (comp > 0 && !P.cf) return VVCG_INVALID_INPUT;
  *ptr = L.final_in_scratch[comp] ? P.scratch[comp] : P.plane[comp];
  if (stride) *stride = (uint32_t)L.stride[comp];
  return VVCG_OK;
}

vvcg_status vvcg_decode_batch(vvcg_ctx* ctx, const vvcg_batch* b, const vvcg_plane_out* out) {
  vvcg_status st;
  if ((st = vvcg_batch_prepare(ctx, b)) != VVCG_OK) return st;
  if ((st = vvcg_batch_upload(ctx, b)) != VVCG_OK) return st;
  if ((st = vvcg_batch_run(ctx, VVCG_STAGE_ALL)) != VVCG_OK) return st;
  if ((st = vvcg_batch_sync(ctx)) != VVCG_OK) return st;
  return vvcg_batch_download(ctx, out);
}

vvcg_status vvcg_decode_batch_async(vvcg_ctx* ctx, const vvcg_batch* b, const vvcg_plane_out* out) {
  vvcg_status st;
  if ((st = vvcg_batch_prepare(ctx, b)) != VVCG_OK) return st;  // waits for this context's previous work
  if ((st = vvcg_batch_upload(ctx, b)) != VVCG_OK) return st;
  if ((st = vvcg_batch_run(ctx, VVCG_STAGE_ALL)) != VVCG_OK) return st;
  if (!out) return fail(ctx, VVCG_INVALID_INPUT, "missing output planes");
  return enqueue_download(ctx, out);
}

vvcg_status vvcg_decode_batch_pipelined(vvcg_ctx* ctx, const vvcg_batch* b, const vvcg_plane_out* out,
                                        uint32_t chunk_pictures, uint32_t num_lanes) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!b || !b->pics || !b->num_pics || !out) return fail(ctx, VVCG_INVALID_INPUT, "empty batch");
  if (!chunk_pictures || chunk_pictures >= b->num_pics) return vvcg_decode_batch(ctx, b, out);
  if (b->num_cus && !b->cus) return fail(ctx, VVCG_INVALID_INPUT, "missing CU records");
  num_lanes = std::max<uint32_t>(1, std::min<uint32_t>(num_lanes ? num_lanes : 3, 8));
  while (ctx->lanes.size() < num_lanes) {
    vvcg_config cfg{ctx->device, 0, 0, ctx->spin_limit, 0};
    vvcg_ctx* l = nullptr;
    vvcg_status st = vvcg_ctx_create(&cfg, &l);
    if (st != VVCG_OK) return fail(ctx, st, "lane context could not be created");
    ctx->lanes.push_back(l);
  }
  // Each chunk is a batch of its own: its pictures' records, CTU records and
  // the range of the level pool they index, with the offsets rebased.
  const uint32_t nchunks = (b->num_pics + chunk_pictures - 1) / chunk_pictures;
  std::vector<std::vector<vvcg_pic_desc>> cpics(nchunks);
  std::vector<uint64_t> c_cu0(nchunks), c_lv0(nchunks);
  std::vector<vvcg_batch> cb(nchunks);
  for (uint32_t k = 0; k < nchunks; k++) {
    const uint32_t p0 = k * chunk_pictures, p1 = std::min(b->num_pics, p0 + chunk_pictures);
    uint64_t cu0 = UINT64_MAX, cu1 = 0, ct0 = UINT64_MAX, ct1 = 0, lv0 = UINT64_MAX, lv1 = 0;
    for (uint32_t i = p0; i < p1; i++) {
      const vvcg_pic_desc& d = b->pics[i];
      uint32_t ncu;
      uint64_t nl;
      if (!encode_geometry(d, &ncu, &nl))
        return fail(ctx, VVCG_INVALID_INPUT, "picture %u: CTU size or coded size outside the frame path", i);
      const uint32_t ctu = 1u << d.ctu_log2, tb = std::min<uint32_t>(ctu, 32);
      const uint64_t nctu = (uint64_t)(d.width / ctu) * (d.height / ctu);
      if ((uint64_t)d.cu_offset + ncu > b->num_cus)
        return fail(ctx, VVCG_INVALID_INPUT, "picture %u: CU records out of range", i);
      cu0 = std::min<uint64_t>(cu0, d.cu_offset);
      cu1 = std::max<uint64_t>(cu1, (uint64_t)d.cu_offset + ncu);
      if (b->ctus) {
        ct0 = std::min<uint64_t>(ct0, d.ctu_offset);
        ct1 = std::max<uint64_t>(ct1, (uint64_t)d.ctu_offset + nctu);
      }
      const int cf = d.chroma_format, sw = (cf == 1 || cf == 2) ? 2 : 1, sh = cf == 1 ? 2 : 1;
      const uint64_t nch = cf ? (uint64_t)std::max<int>(tb / sw, 2) * std::max<int>(tb / sh, 2) : 0;
      const uint64_t nlc[3] = {(uint64_t)tb * tb, nch, nch};
      const bool sparse = (d.tools & VVCG_TOOL_SPARSE_LEVELS) != 0;
      for (uint32_t c = 0; c < ncu; c++) {
        const vvcg_cu_rec& r = b->cus[d.cu_offset + c];
        for (int q = 0; q < (cf ? 3 : 1); q++)
          if (((r.cbf >> q) & 1) && r.level_off[q] >= 0) {
            const uint64_t off = (uint64_t)r.level_off[q];
            const uint64_t ext = b->levels ? tb_level_extent(b->levels, b->num_levels, off, nlc[q], sparse) : 0;
            if (!ext) return fail(ctx, VVCG_INVALID_INPUT, "picture %u CU %u: level offset out of range", i, c);
            lv0 = std::min<uint64_t>(lv0, off);
            lv1 = std::max<uint64_t>(lv1, off + ext);
          }
      }
    }
    if (lv0 == UINT64_MAX) lv0 = lv1 = 0;
    lv0 &= ~1ull;  // sparse TBs start at even offsets, also after rebasing
    if (ct0 == UINT64_MAX) ct0 = ct1 = 0;
    if (lv1 > b->num_levels) return fail(ctx, VVCG_INVALID_INPUT, "chunk %u: level offsets out of range", k);
    cpics[k].assign(b->pics + p0, b->pics + p1);
    for (auto& d : cpics[k]) {
      d.cu_offset -= (uint32_t)cu0;
      d.ctu_offset -= (uint32_t)ct0;
    }
    c_cu0[k] = cu0;
    c_lv0[k] = lv0;
    cb[k] = vvcg_batch{cpics[k].data(), p1 - p0, (uint32_t)(cu1 - cu0), nullptr,
                       b->levels ? b->levels + lv0 : nullptr, lv1 - lv0,
                       b->ctus ? b->ctus + ct0 : nullptr, (uint32_t)(ct1 - ct0), b->num_aps, b->aps};
  }
  // round robin over the lanes: a lane takes its next chunk once its previous
  // one has finished, while the other lanes' copies and kernels run
  vvcg_status st = VVCG_OK;
  for (uint32_t k = 0; k < nchunks && st == VVCG_OK; k++) {
    vvcg_ctx* l = ctx->lanes[k % num_lanes];
    // the lane's previous chunk must be done with the lane's pinned records
    CK(cudaSetDevice(l->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(l->stream), "lane");
    CK(l->stage_cus.reserve(std::max<size_t>(1, cb[k].num_cus) * sizeof(vvcg_cu_rec)), "cudaHostAlloc");
    vvcg_cu_rec* rc = (vvcg_cu_rec*)l->stage_cus.p;
    const uint64_t lv0 = c_lv0[k];
    for (uint32_t i = 0; i < cb[k].num_cus; i++) {
      vvcg_cu_rec r = b->cus[c_cu0[k] + i];
      for (int q = 0; q < 3; q++)
        if (r.level_off[q] >= 0 && (uint64_t)r.level_off[q] >= lv0) r.level_off[q] -= (int32_t)lv0;
      rc[i] = r;
    }
    cb[k].cus = rc;
    if ((st = vvcg_batch_prepare(l, &cb[k])) != VVCG_OK) break;
    if ((st = vvcg_batch_upload(l, &cb[k])) != VVCG_OK) break;
    if ((st = vvcg_batch_run(l, VVCG_STAGE_ALL)) != VVCG_OK) break;
    st = enqueue_download(l, out + (size_t)k * chunk_pictures * 3);
  }
  for (uint32_t i = 0; i < num_lanes; i++) {
    vvcg_status s2 = vvcg_batch_sync(ctx->lanes[i]);
    if (st == VVCG_OK && s2 != VVCG_OK) st = s2;
  }
  if (st != VVCG_OK) {
    for (vvcg_ctx* l : ctx->lanes)
      if (!l->err.empty()) return fail(ctx, st, "%s", l->err.c_str());
    return st;
  }
  return VVCG_OK;
}

static vvcg_status mc_common(vvcg_ctx* ctx, const uint16_t* ref, uint32_t w, uint32_t h,
                             uint32_t stride, uint8_t bd, int chroma, const vvcg_mc_block* blocks,
                             uint32_t n, int32_t* out) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!ref || !out || (n && !blocks) || !w || !h || stride < w || bd < 8 || bd > 12)
    return fail(ctx, VVCG_INVALID_INPUT, "invalid MC arguments");
  if (n == 0) return VVCG_OK;
  McParams pm{ref, nullptr, (int32_t)w, (int32_t)h, (int32_t)stride, bd, chroma};
  k_mc<<<n, 256, 0, ctx->stream>>>(pm, blocks, n, out, (uint32_t*)ctx->d_ctrl.p + 1);
  CK(cudaGetLastError(), "mc launch");
  ctx->launches++;
  return VVCG_OK;
}

static vvcg_status mc_common_8(vvcg_ctx* ctx, const uint8_t* ref, uint32_t w, uint32_t h, uint32_t stride,
                               int chroma, const vvcg_mc_block* blocks, uint32_t n, int32_t* out) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!ref || !out || (n && !blocks) || !w || !h || stride < w)
    return fail(ctx, VVCG_INVALID_INPUT, "invalid MC arguments");
  if (n == 0) return VVCG_OK;
  McParams pm{nullptr, ref, (int32_t)w, (int32_t)h, (int32_t)stride, 8, chroma};
  k_mc<<<n, 256, 0, ctx->stream>>>(pm, blocks, n, out, (uint32_t*)ctx->d_ctrl.p + 1);
  CK(cudaGetLastError(), "mc launch");
  ctx->launches++;
  return VVCG_OK;
}

vvcg_status vvcg_mc_luma_8_dev(vvcg_ctx* ctx, const uint8_t* ref, uint32_t w, uint32_t h, uint32_t stride,
                               const vvcg_mc_block* blocks, uint32_t n, int32_t* out) {
  return mc_common_8(ctx, ref, w, h, stride, 0, blocks, n, out);
}

vvcg_status vvcg_mc_chroma_420_8_dev(vvcg_ctx* ctx, const uint8_t* ref, uint32_t w, uint32_t h, uint32_t stride,
                                     const vvcg_mc_block* blocks, uint32_t n, int32_t* out) {
  return mc_common_8(ctx, ref, w, h, stride, 1, blocks, n, out);
}

vvcg_status vvcg_mc_luma_16_dev(vvcg_ctx* ctx, const uint16_t* ref, uint32_t w, uint32_t h,
                                uint32_t stride, uint8_t bd, const vvcg_mc_block* blocks,
                                uint32_t n, int32_t* out) {
  return mc_common(ctx, ref, w, h, stride, bd, 0, blocks, n, out);
}

vvcg_status vvcg_mc_chroma_16_dev(vvcg_ctx* ctx, const uint16_t* ref, uint32_t w, uint32_t h,
                                  uint32_t stride, uint8_t bd, uint8_t cf,
                                  const vvcg_mc_block* blocks, uint32_t n, int32_t* out) {
  if (cf < 1 || cf > 3) return fail(ctx, VVCG_INVALID_INPUT, "chroma format");
  return mc_common(ctx, ref, w, h, stride, bd, cf, blocks, n, out);
}

vvcg_status vvcg_mc_bi_average_16_dev(vvcg_ctx* ctx, const int32_t* p0, const int32_t* p1,
                                      uint64_t count, uint8_t bcw, uint8_t bd, uint16_t* out) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!p0 || !p1 || !out || bd < 8 || bd > 12 || bcw > 4)
    return fail(ctx, VVCG_INVALID_INPUT, "invalid bi-average arguments");
  if (!count) return VVCG_OK;
  uint32_t grid = (uint32_t)std::min<uint64_t>((count + 255) / 256, (uint64_t)ctx->num_sms * 16);
  k_bi_average<<<grid, 256, 0, ctx->stream>>>(p0, p1, count, bcw, bd, out);
  CK(cudaGetLastError(), "bi average launch");
  ctx->launches++;
  return VVCG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Luma transform search (vvcg_luma_tx_search_dev).
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_luma_tx_search_dev(vvcg_ctx* ctx, const vvcg_tx_search_req* reqs, uint32_t num_reqs,
                                               const int16_t* pred, const int16_t* src, uint64_t in_count,
                                               int16_t* levels, int16_t* samples, uint64_t out_count,
                                               vvcg_tx_search_res* res) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (num_reqs == 0) return VVCG_OK;
  if (!reqs || !pred || !src || !levels || !samples || !res)
    return fail(ctx, VVCG_INVALID_INPUT, "missing requests or buffers");
  for (uint32_t i = 0; i < num_reqs; i++) {
    const vvcg_tx_search_req& q = reqs[i];
    if (q.log2_size < 2 || q.log2_size > 5) return fail(ctx, VVCG_INVALID_INPUT, "request %u: size outside 4..32", i);
    if (q.qp > 63) return fail(ctx, VVCG_INVALID_INPUT, "request %u: QP above 63", i);
    if (q.mode > 66) return fail(ctx, VVCG_INVALID_INPUT, "request %u: intra mode above 66", i);
    const uint64_t nn = 1ull << (2 * q.log2_size);
    if (q.in_off + nn > in_count || q.out_off + nn > out_count)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: sample range past the buffers", i);
  }
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_tu_recs.reserve(sizeof(vvcg_tx_search_req) * num_reqs), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_tu_recs.p, reqs, sizeof(vvcg_tx_search_req) * num_reqs, cudaMemcpyHostToDevice,
                     ctx->stream),
     "upload");
  k_luma_tx_search<<<num_reqs, kTxsWarps * 32, sizeof(TxsWs), ctx->stream>>>(
      (const vvcg_tx_search_req*)ctx->d_tu_recs.p, pred, src, levels, samples, res);
  CK(cudaGetLastError(), "transform search launch");
  ctx->launches++;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// LMCS and joint chroma residuals.
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_lmcs_build(const vvcg_lmcs_aps* aps, uint8_t bit_depth, vvcg_lmcs_tables* t) {
  // LmcsReshaper16::from_aps (filter.rs:2628-2705)
  if (!aps || !t) return VVCG_INVALID_INPUT;
  memset(t, 0, sizeof(*t));
  const int bd = std::min(12, std::max(8, (int)bit_depth));
  const int max_val = (1 << bd) - 1, log2_cw = bd - 4, init_cw = 1 << log2_cw;
  const int min_bin = std::min<int>(aps->min_bin_idx, 15);
  const int max_bin = std::max(std::min<int>(aps->max_bin_idx, 15), min_bin);
  int bin_cw[16] = {0}, in_piv[17] = {0}, re_piv[17] = {0}, fwd_sc[16], inv_sc[16], adj[16];
  for (int i = min_bin; i <= max_bin; i++) bin_cw[i] = std::max(0, init_cw + aps->bin_cw_delta[i]);
  for (int i = 0; i < 16; i++) {
    re_piv[i + 1] = re_piv[i] + bin_cw[i];
    in_piv[i + 1] = in_piv[i] + init_cw;
    fwd_sc[i] = ((bin_cw[i] << kLmcsFpPrec) + (1 << (log2_cw - 1))) >> log2_cw;
    inv_sc[i] = bin_cw[i] ? (init_cw << kLmcsFpPrec) / bin_cw[i] : 0;
    adj[i] = bin_cw[i] ? (init_cw << kLmcsFpPrec) / std::max(1, bin_cw[i] + aps->chroma_res_scaling_offset)
                       : 1 << kLmcsFpPrec;
  }
  const int half = 1 << (kLmcsFpPrec - 1);
  for (int v = 0; v <= max_val; v++) {
    const int iy = std::min(15, v >> log2_cw);
    t->fwd_lut[v] = (uint16_t)std::min(max_val, std::max(0, re_piv[iy] + ((fwd_sc[iy] * (v - in_piv[iy]) + half) >> kLmcsFpPrec)));
    int ii = min_bin;
    while (ii <= max_bin && v >= re_piv[ii + 1]) ii++;
    ii = std::min(ii, 15);
    t->inv_lut[v] = (uint16_t)std::min(max_val, std::max(0, in_piv[ii] + ((inv_sc[ii] * (v - re_piv[ii]) + half) >> kLmcsFpPrec)));
  }
  t->bit_depth = (uint8_t)bd;
  t->min_bin_idx = (uint8_t)min_bin;
  t->max_bin_idx = (uint8_t)max_bin;
  memcpy(t->reshape_pivot, re_piv, sizeof(re_piv));
  memcpy(t->chroma_adj_lut, adj, sizeof(adj));
  return VVCG_OK;
}

namespace {
vvcg_status upload_lmcs(vvcg_ctx* ctx, const vvcg_lmcs_tables* t) {
  if (!t || t->bit_depth < 8 || t->bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "LMCS tables");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_lmcs.reserve(sizeof(vvcg_lmcs_tables)), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_lmcs.p, t, sizeof(vvcg_lmcs_tables), cudaMemcpyHostToDevice, ctx->stream), "upload");
  return VVCG_OK;
}
}  // namespace

extern "C" vvcg_status vvcg_lmcs_map_plane_16_dev(vvcg_ctx* ctx, const vvcg_lmcs_tables* t, int inverse,
                                                  uint16_t* plane, uint32_t stride, uint32_t w, uint32_t h) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (w && h && (!plane || stride < w)) return fail(ctx, VVCG_INVALID_INPUT, "plane");
  vvcg_status st = upload_lmcs(ctx, t);
  if (st != VVCG_OK || !w || !h) return st;
  const vvcg_lmcs_tables* d = (const vvcg_lmcs_tables*)ctx->d_lmcs.p;
  const uint64_t work = (uint64_t)((w + 3) / 4) * h;
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((work + 255) / 256, (uint64_t)ctx->num_sms * 8));
  k_lut_plane<<<grid, 256, 0, ctx->stream>>>(inverse ? d->inv_lut : d->fwd_lut, t->bit_depth, plane, stride, w, h);
  CK(cudaGetLastError(), "lmcs launch");
  ctx->launches++;
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_lmcs_chroma_scales_dev(vvcg_ctx* ctx, const vvcg_lmcs_tables* t, const uint16_t* luma,
                                                   uint32_t stride, uint32_t pw, uint32_t ph, uint32_t ctu,
                                                   const uint32_t* pos, uint32_t num, int32_t* out) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (num && (!luma || !pos || !out || !pw || !ph || stride < pw))
    return fail(ctx, VVCG_INVALID_INPUT, "missing or invalid buffers");
  if (ctu != 32 && ctu != 64 && ctu != 128) return fail(ctx, VVCG_INVALID_INPUT, "CTU size");
  vvcg_status st = upload_lmcs(ctx, t);
  if (st != VVCG_OK || !num) return st;
  k_lmcs_chroma_scales<<<(num + 7) / 8, 256, 0, ctx->stream>>>((const vvcg_lmcs_tables*)ctx->d_lmcs.p, luma, stride,
                                                              (int)pw, (int)ph, (int)ctu, pos, num, out);
  CK(cudaGetLastError(), "lmcs launch");
  ctx->launches++;
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_chroma_residuals_dev(vvcg_ctx* ctx, const vvcg_cres_rec* recs, uint32_t num,
                                                 int16_t* res, uint64_t count) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num) return VVCG_OK;
  if (!recs || !res) return fail(ctx, VVCG_INVALID_INPUT, "missing records or residuals");
  for (uint32_t i = 0; i < num; i++) {
    const vvcg_cres_rec& r = recs[i];
    if (r.log2_w > 5 || r.log2_h > 5 || r.bit_depth < 8 || r.bit_depth > 12 || r.joint < -3 || r.joint > 3)
      return fail(ctx, VVCG_INVALID_INPUT, "record %u: size, bit depth or joint mode", i);
    const uint64_t n = 1ull << (r.log2_w + r.log2_h);
    if (r.cb_off + n > count || (!(r.flags & VVCG_CRES_SINGLE) && r.cr_off + n > count))
      return fail(ctx, VVCG_INVALID_INPUT, "record %u: residual range past the buffer", i);
  }
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_tu_recs.reserve(sizeof(vvcg_cres_rec) * num), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_tu_recs.p, recs, sizeof(vvcg_cres_rec) * num, cudaMemcpyHostToDevice, ctx->stream), "upload");
  k_chroma_residuals<<<(num + 7) / 8, 256, 0, ctx->stream>>>((const vvcg_cres_rec*)ctx->d_tu_recs.p, num, res);
  CK(cudaGetLastError(), "chroma residual launch");
  ctx->launches++;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// Matrix-based intra prediction (vvcg_mip_predict_dev).
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_mip_predict_dev(vvcg_ctx* ctx, const vvcg_mip_req* reqs, uint32_t num_reqs,
                                            const int16_t* refs, uint64_t ref_count, const int16_t* src,
                                            int16_t* pred, uint64_t count, vvcg_mip_res* res) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!reqs || !refs || !pred) return fail(ctx, VVCG_INVALID_INPUT, "missing requests or buffers");
  for (uint32_t i = 0; i < num_reqs; i++) {
    const vvcg_mip_req& q = reqs[i];
    if (q.log2_w < 2 || q.log2_w > 6 || q.log2_h < 2 || q.log2_h > 6)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: block size outside 4..64", i);
    if (q.bit_depth < 8 || q.bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "request %u: bit depth", i);
    const uint64_t w = 1u << q.log2_w, h = 1u << q.log2_h;
    if (q.ref_off + w + h > ref_count || q.out_off + w * h > count)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: sample range past the buffers", i);
    if (q.mode == VVCG_MIP_SEARCH && (!src || !res))
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: a search needs the source and results", i);
  }
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_tu_recs.reserve(sizeof(vvcg_mip_req) * num_reqs), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_tu_recs.p, reqs, sizeof(vvcg_mip_req) * num_reqs, cudaMemcpyHostToDevice, ctx->stream),
     "upload");
  k_mip<<<(num_reqs + kMipWarps - 1) / kMipWarps, kMipWarps * 32, 0, ctx->stream>>>(
      (const vvcg_mip_req*)ctx->d_tu_recs.p, num_reqs, refs, src, pred, res);
  CK(cudaGetLastError(), "mip launch");
  ctx->launches++;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// General-decoder ALF (vvcg_alf_general_dev).
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_alf_general_dev(vvcg_ctx* ctx, const uint16_t* const src[3], uint16_t* const dst[3],
                                            const uint32_t stride[3], uint32_t width, uint32_t height,
                                            uint32_t vis_width, uint32_t vis_height, uint8_t bit_depth,
                                            uint32_t ctu_size, uint32_t ctu_cols, const vvcg_alf_ctu* ctus,
                                            const vvcg_alf_params* a) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!src || !dst || !stride || !ctus || !a) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  if (!width || !height) return VVCG_OK;
  for (int c = 0; c < 3; c++) {
    const uint32_t pw = c ? (width + 1) / 2 : width;
    if (!src[c] || !dst[c] || src[c] == dst[c] || stride[c] < pw)
      return fail(ctx, VVCG_INVALID_INPUT, "plane %d: missing, in place, or stride too small", c);
  }
  if (bit_depth < 8 || bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "bit depth");
  if (ctu_size < 16 || ctu_size > 128 || (ctu_size & (ctu_size - 1)))
    return fail(ctx, VVCG_INVALID_INPUT, "CTU size must be a power of two in 16..128");
  if (!vis_width || !vis_height || vis_width > width || vis_height > height)
    return fail(ctx, VVCG_INVALID_INPUT, "visible size");
  const uint32_t gw = (vis_width + ctu_size - 1) / ctu_size, gh = (vis_height + ctu_size - 1) / ctu_size;
  if (ctu_cols < gw) return fail(ctx, VVCG_INVALID_INPUT, "CTU columns");
  if (a->num_luma_filters > 25 || a->num_chroma_filters > 8 || a->num_cc_cb > 4 || a->num_cc_cr > 4)
    return fail(ctx, VVCG_INVALID_INPUT, "ALF filter counts");
  for (uint32_t gy = 0; gy < gh; gy++)
    for (uint32_t gx = 0; gx < gw; gx++) {
      const vvcg_alf_ctu& m = ctus[gy * ctu_cols + gx];
      if (m.luma_mode > VVCG_ALF_APS) return fail(ctx, VVCG_INVALID_INPUT, "CTU %u,%u: luma mode", gx, gy);
      if (m.luma_mode == VVCG_ALF_APS && a->num_luma_filters == 0)
        return fail(ctx, VVCG_INVALID_INPUT, "CTU %u,%u: ALF APS mode without luma filters", gx, gy);
    }
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  const size_t nctu = (size_t)gh * ctu_cols;
  CK(ctx->d_alfp.reserve(sizeof(vvcg_alf_params)), "cudaMalloc");
  CK(ctx->d_alfc.reserve(sizeof(vvcg_alf_ctu) * nctu), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_alfp.p, a, sizeof(vvcg_alf_params), cudaMemcpyHostToDevice, ctx->stream), "upload");
  CK(cudaMemcpyAsync(ctx->d_alfc.p, ctus, sizeof(vvcg_alf_ctu) * nctu, cudaMemcpyHostToDevice, ctx->stream),
     "upload");
  AlfGenPass P;
  const int pw = (int)width, ph = (int)height, cw = (pw + 1) / 2, ch = (ph + 1) / 2;
  const int cvw = ((int)vis_width + 1) / 2, cvh = ((int)vis_height + 1) / 2;
  P.y = AlfGenView{src[0], (int32_t)stride[0], min((int)vis_width, pw), min((int)vis_height, ph)};
  P.u = AlfGenView{src[1], (int32_t)stride[1], min(cvw, cw), min(cvh, ch)};
  P.v = AlfGenView{src[2], (int32_t)stride[2], min(cvw, cw), min(cvh, ch)};
  for (int c = 0; c < 3; c++) {
    P.dst[c] = dst[c];
    P.dstride[c] = (int32_t)stride[c];
  }
  P.pw = pw;
  P.ph = ph;
  P.cw = cw;
  P.ch = ch;
  P.vis_w = (int)vis_width;
  P.vis_h = (int)vis_height;
  P.cvis_w = cvw;
  P.cvis_h = cvh;
  P.bd = bit_depth;
  P.ctu = (int)ctu_size;
  P.ctu_cols = (int)ctu_cols;
  P.ctus = (const vvcg_alf_ctu*)ctx->d_alfc.p;
  P.a = (const vvcg_alf_params*)ctx->d_alfp.p;
  const uint64_t nb = (uint64_t)((pw + 3) / 4) * ((ph + 3) / 4);
  k_alf_general_luma<<<(uint32_t)std::min<uint64_t>((nb + 127) / 128, (uint64_t)ctx->num_sms * 16), 128, 0,
                       ctx->stream>>>(P);
  CK(cudaGetLastError(), "alf launch");
  const uint64_t nc = 2ull * cw * ch;
  k_alf_general_chroma<<<(uint32_t)std::min<uint64_t>((nc + 255) / 256, (uint64_t)ctx->num_sms * 16), 256, 0,
                         ctx->stream>>>(P);
  CK(cudaGetLastError(), "alf launch");
  ctx->launches += 2;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// 8-bit luma intra mode search (vvcg_luma_intra_search_8_dev).
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_luma_intra_search_8_dev(vvcg_ctx* ctx, const uint8_t* recon, uint64_t recon_stride,
                                                    const uint8_t* src, uint64_t src_stride, uint32_t width,
                                                    uint32_t height, const vvcg_intra_search_req* reqs,
                                                    uint32_t num_reqs, vvcg_intra_search_res* res) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!recon || !src || !reqs || !res) return fail(ctx, VVCG_INVALID_INPUT, "missing planes, requests or results");
  if (recon_stride < width || src_stride < width) return fail(ctx, VVCG_INVALID_INPUT, "stride smaller than width");
  if (width > (1u << 20) || height > (1u << 20)) return fail(ctx, VVCG_LIMIT_EXCEEDED, "plane larger than 2^20");
  for (uint32_t i = 0; i < num_reqs; i++) {
    const vvcg_intra_search_req& q = reqs[i];
    if (q.log2_w < 2 || q.log2_w > 6 || q.log2_h < 2 || q.log2_h > 6)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: block size outside 4..64", i);
    if ((uint64_t)q.x + (1u << q.log2_w) > width || (uint64_t)q.y + (1u << q.log2_h) > height)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: block outside the plane", i);
    if (q.flags & ~(uint32_t)(VVCG_ISR_MPM_ONLY | VVCG_ISR_MRL))
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: unknown flags", i);
    if ((q.flags & VVCG_ISR_MRL) && (q.log2_ctu < 4 || q.log2_ctu > 7))
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: CTU size outside 16..128", i);
    for (int k = 0; k < 6; k++)
      if (q.mpm[k] > 66) return fail(ctx, VVCG_INVALID_INPUT, "request %u: MPM %d is not a mode", i, k);
  }
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_tu_recs.reserve(sizeof(vvcg_intra_search_req) * num_reqs), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_tu_recs.p, reqs, sizeof(vvcg_intra_search_req) * num_reqs, cudaMemcpyHostToDevice,
                     ctx->stream),
     "upload");
  IsrArgs A{recon, src, (int64_t)recon_stride, (int64_t)src_stride, (int32_t)width, (int32_t)height,
            (int32_t)num_reqs, (const vvcg_intra_search_req*)ctx->d_tu_recs.p, res};
  const uint32_t grid = std::min<uint32_t>(num_reqs, (uint32_t)ctx->num_sms * 8);
  k_luma_intra_search_8<<<grid, kIsrWarps * 32, 0, ctx->stream>>>(A);
  CK(cudaGetLastError(), "intra search launch");
  ctx->launches++;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// Partition hook of the reference encoders (vvcg_qt_mtt_split_dev).
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_qt_mtt_split_dev(vvcg_ctx* ctx, const uint16_t* plane, uint64_t stride, uint32_t width,
                                             uint32_t height, uint8_t bit_depth, const vvcg_split_req* reqs,
                                             uint32_t num_reqs, uint8_t* res) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!plane || !reqs || !res) return fail(ctx, VVCG_INVALID_INPUT, "missing plane, requests or results");
  if (stride < width || bit_depth < 8 || bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "plane geometry");
  if (width > (1u << 20) || height > (1u << 20) || num_reqs > (1u << 24))
    return fail(ctx, VVCG_LIMIT_EXCEEDED, "plane or request count too large");
  for (uint32_t i = 0; i < num_reqs; i++) {
    const vvcg_split_req& q = reqs[i];
    if (q.w < 1 || q.h < 1 || q.w > 4096 || q.h > 4096)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: region size outside 1..4096", i);
    if (q.qp > 63) return fail(ctx, VVCG_INVALID_INPUT, "request %u: QP above 63", i);
  }
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_tu_recs.reserve(sizeof(vvcg_split_req) * num_reqs), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_tu_recs.p, reqs, sizeof(vvcg_split_req) * num_reqs, cudaMemcpyHostToDevice, ctx->stream),
     "upload");
  SplitArgs A{plane, (int64_t)stride, (int32_t)width, (int32_t)height, (int32_t)bit_depth, (int32_t)num_reqs,
              (const vvcg_split_req*)ctx->d_tu_recs.p, res};
  const uint32_t grid =
      std::min<uint32_t>((num_reqs + kSplitWarps - 1) / kSplitWarps, (uint32_t)ctx->num_sms * 8);
  k_qt_mtt_split<<<grid, kSplitWarps * 32, 0, ctx->stream>>>(A);
  CK(cudaGetLastError(), "split launch");
  ctx->launches++;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// Motion-estimation hook of the reference encoders (vvcg_inter_search_8_dev).
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_inter_search_8_dev(vvcg_ctx* ctx, const uint8_t* src, uint64_t stride, uint32_t width,
                                               uint32_t height, const uint8_t* const* ref_l0, uint32_t num_l0,
                                               const uint8_t* const* ref_l1, uint32_t num_l1,
                                               const vvcg_mv_cand* cands, uint32_t num_cands,
                                               const vvcg_me_req* reqs, uint32_t num_reqs, vvcg_me_res* res) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!src || !reqs || !res) return fail(ctx, VVCG_INVALID_INPUT, "missing plane, requests or results");
  if (!width || !height || stride < width) return fail(ctx, VVCG_INVALID_INPUT, "plane geometry");
  if (width > (1u << 20) || height > (1u << 20) || num_reqs > (1u << 24))
    return fail(ctx, VVCG_LIMIT_EXCEEDED, "plane or request count too large");
  if (num_l0 > (uint32_t)kMeMaxRefs || num_l1 > (uint32_t)kMeMaxRefs)
    return fail(ctx, VVCG_LIMIT_EXCEEDED, "more than %d references in a list", kMeMaxRefs);
  if ((num_l0 && !ref_l0) || (num_l1 && !ref_l1) || (num_cands && !cands))
    return fail(ctx, VVCG_INVALID_INPUT, "missing reference list or candidates");
  MeArgs A{};
  for (uint32_t i = 0; i < num_l0; i++)
    if (!(A.l0[i] = ref_l0[i])) return fail(ctx, VVCG_INVALID_INPUT, "L0 reference %u is null", i);
  for (uint32_t i = 0; i < num_l1; i++)
    if (!(A.l1[i] = ref_l1[i])) return fail(ctx, VVCG_INVALID_INPUT, "L1 reference %u is null", i);
  for (uint32_t i = 0; i < num_reqs; i++) {
    const vvcg_me_req& q = reqs[i];
    if (q.w < 1 || q.h < 1 || q.w > 128 || q.h > 128)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: block size outside 1..128", i);
    if ((uint64_t)q.x + q.w > width || (uint64_t)q.y + q.h > height)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: block outside the plane", i);
    if ((uint64_t)q.cand_off + q.num_cands > num_cands)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: merge candidates past the array", i);
  }
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_me_reqs.reserve(sizeof(vvcg_me_req) * num_reqs), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_me_reqs.p, reqs, sizeof(vvcg_me_req) * num_reqs, cudaMemcpyHostToDevice, ctx->stream),
     "upload");
  if (num_cands) {
    CK(ctx->d_me_cands.reserve(sizeof(vvcg_mv_cand) * num_cands), "cudaMalloc");
    CK(cudaMemcpyAsync(ctx->d_me_cands.p, cands, sizeof(vvcg_mv_cand) * num_cands, cudaMemcpyHostToDevice,
                       ctx->stream),
       "upload");
  }
  A.src = src;
  A.stride = (int64_t)stride;
  A.width = (int32_t)width;
  A.height = (int32_t)height;
  A.n0 = (int32_t)num_l0;
  A.n1 = (int32_t)num_l1;
  A.cands = num_cands ? (const vvcg_mv_cand*)ctx->d_me_cands.p : nullptr;
  A.reqs = (const vvcg_me_req*)ctx->d_me_reqs.p;
  A.n = (int32_t)num_reqs;
  A.res = res;
  const uint32_t grid = std::min<uint32_t>(num_reqs, (uint32_t)ctx->num_sms * 8);
  k_inter_search_8<<<grid, kMeThreads, 0, ctx->stream>>>(A);
  CK(cudaGetLastError(), "motion search launch");
  ctx->launches++;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// CTU full search of the GPU encoder (vvcg_ctu_search_dev).
// ---------------------------------------------------------------------------
// Blocks of a 32x32 CTU: (x, y, log2 w, log2 h) per slot; the slots of split
// s are c_split_first[s] .. + c_split_count[s] - 1.
static const uint8_t kSearchBlocks[15][4] = {
    {0, 0, 5, 5},                                                   // none
    {0, 0, 4, 4},  {16, 0, 4, 4}, {0, 16, 4, 4}, {16, 16, 4, 4},    // quad
    {0, 0, 5, 4},  {0, 16, 5, 4},                                   // binary, horizontal split
    {0, 0, 4, 5},  {16, 0, 4, 5},                                   // binary, vertical split
    {0, 0, 5, 3},  {0, 8, 5, 4},  {0, 24, 5, 3},                    // ternary, horizontal split
    {0, 0, 3, 5},  {8, 0, 4, 5},  {24, 0, 3, 5}};                   // ternary, vertical split
static const uint8_t kSearchSplitFirst[6] = {0, 1, 5, 7, 9, 12};
static const uint8_t kSearchSplitCount[6] = {1, 4, 2, 2, 3, 3};

extern "C" vvcg_status vvcg_ctu_search_dev(vvcg_ctx* ctx, const uint16_t* src, uint64_t stride, uint32_t width,
                                           uint32_t height, uint8_t bit_depth, uint32_t lambda_q8,
                                           const vvcg_ctu_search_req* reqs, uint32_t num_reqs,
                                           vvcg_ctu_search_res* res) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!src || !reqs || !res) return fail(ctx, VVCG_INVALID_INPUT, "missing plane, requests or results");
  if (stride < width) return fail(ctx, VVCG_INVALID_INPUT, "stride smaller than width");
  if (bit_depth < 8 || bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "bit depth");
  if (width > (1u << 20) || height > (1u << 20)) return fail(ctx, VVCG_LIMIT_EXCEEDED, "plane larger than 2^20");
  if (num_reqs > (1u << 24)) return fail(ctx, VVCG_LIMIT_EXCEEDED, "more than 2^24 CTUs");
  std::vector<CostReq> blocks;
  blocks.reserve((size_t)num_reqs * 15);
  for (uint32_t i = 0; i < num_reqs; i++) {
    const vvcg_ctu_search_req& q = reqs[i];
    if ((uint64_t)q.x + 32 > width || (uint64_t)q.y + 32 > height)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: CTU outside the plane", i);
    if (!q.split_mask || q.split_mask > 0x3F) return fail(ctx, VVCG_INVALID_INPUT, "request %u: split mask", i);
    if (q.n_cand > 6) return fail(ctx, VVCG_INVALID_INPUT, "request %u: more than 6 candidates", i);
    for (int k = 0; k < q.n_cand; k++)
      if (q.cand[k] > 66) return fail(ctx, VVCG_INVALID_INPUT, "request %u: candidate %d is not a mode", i, k);
    for (int sp = 0; sp < 6; sp++) {
      if (!(q.split_mask & (1u << sp))) continue;
      for (int k = 0; k < kSearchSplitCount[sp]; k++) {
        const int slot = kSearchSplitFirst[sp] + k;
        CostReq b{};
        b.x = q.x + kSearchBlocks[slot][0];
        b.y = q.y + kSearchBlocks[slot][1];
        b.log2_w = kSearchBlocks[slot][2];
        b.log2_h = kSearchBlocks[slot][3];
        b.n_cand = q.n_cand;
        for (int c = 0; c < 6; c++) b.cand[c] = q.cand[c];
        b.slot = (uint16_t)slot;
        b.ctu = i;
        blocks.push_back(b);
      }
    }
  }
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_search_reqs.reserve(sizeof(CostReq) * blocks.size()), "cudaMalloc");
  CK(ctx->d_search_ctus.reserve(sizeof(vvcg_ctu_search_req) * num_reqs), "cudaMalloc");
  CK(ctx->d_search_cost.reserve(sizeof(uint32_t) * 15 * (size_t)num_reqs), "cudaMalloc");
  CK(ctx->d_search_mode.reserve(15 * (size_t)num_reqs), "cudaMalloc");
  // pageable sources: the copies have read them when cudaMemcpyAsync returns
  CK(cudaMemcpyAsync(ctx->d_search_reqs.p, blocks.data(), sizeof(CostReq) * blocks.size(), cudaMemcpyHostToDevice,
                     ctx->stream),
     "upload");
  CK(cudaMemcpyAsync(ctx->d_search_ctus.p, reqs, sizeof(vvcg_ctu_search_req) * num_reqs, cudaMemcpyHostToDevice,
                     ctx->stream),
     "upload");
  CostArgs A{src, (int64_t)stride, (int32_t)width, (int32_t)height, bit_depth, (int32_t)blocks.size(), lambda_q8,
             (const CostReq*)ctx->d_search_reqs.p, (uint32_t*)ctx->d_search_cost.p,
             (uint8_t*)ctx->d_search_mode.p};
  const uint32_t grid = (uint32_t)std::min<size_t>(blocks.size(), (size_t)ctx->num_sms * 8);
  k_cost_search<<<grid, kIsrWarps * 32, 0, ctx->stream>>>(A);
  CK(cudaGetLastError(), "search launch");
  k_ctu_search_combine<<<(num_reqs + 127) / 128, 128, 0, ctx->stream>>>(
      (const vvcg_ctu_search_req*)ctx->d_search_ctus.p, (int)num_reqs, lambda_q8,
      (const uint32_t*)ctx->d_search_cost.p, (const uint8_t*)ctx->d_search_mode.p, res);
  CK(cudaGetLastError(), "search launch");
  ctx->launches += 2;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// CTU search from device positions, full or CNN-pruned (vvcg_ctu_search_pruned_dev).
// ---------------------------------------------------------------------------
static vvcg_status ctu_search_xy(vvcg_ctx* ctx, const uint16_t* src, uint64_t stride, uint32_t width,
                                 uint32_t height, uint8_t bit_depth, uint32_t lambda_q8, const uint32_t* ctu_xy,
                                 uint32_t num_ctus, const float* logits, uint32_t top_modes, uint32_t top_splits,
                                 float threshold, uint32_t rule, vvcg_ctu_search_res* res, uint32_t* mode_costs);

extern "C" vvcg_status vvcg_ctu_search_pruned_dev(vvcg_ctx* ctx, const uint16_t* src, uint64_t stride,
                                                  uint32_t width, uint32_t height, uint8_t bit_depth,
                                                  uint32_t lambda_q8, const uint32_t* ctu_xy, uint32_t num_ctus,
                                                  const float* logits, uint32_t top_modes, uint32_t top_splits,
                                                  float threshold, vvcg_ctu_search_res* res) {
  return ctu_search_xy(ctx, src, stride, width, height, bit_depth, lambda_q8, ctu_xy, num_ctus, logits, top_modes,
                       top_splits, threshold, VVCG_PRUNE_MASS, res, nullptr);
}

extern "C" vvcg_status vvcg_ctu_search_pruned_rule_dev(vvcg_ctx* ctx, const uint16_t* src, uint64_t stride,
                                                       uint32_t width, uint32_t height, uint8_t bit_depth,
                                                       uint32_t lambda_q8, const uint32_t* ctu_xy, uint32_t num_ctus,
                                                       const float* logits, uint32_t top_modes, uint32_t top_splits,
                                                       float threshold, uint32_t rule, vvcg_ctu_search_res* res) {
  if (ctx && rule > VVCG_PRUNE_MAX_PROB) return fail(ctx, VVCG_INVALID_INPUT, "unknown fallback rule");
  return ctu_search_xy(ctx, src, stride, width, height, bit_depth, lambda_q8, ctu_xy, num_ctus, logits, top_modes,
                       top_splits, threshold, rule, res, nullptr);
}

extern "C" vvcg_status vvcg_ctu_search_costs_dev(vvcg_ctx* ctx, const uint16_t* src, uint64_t stride, uint32_t width,
                                                 uint32_t height, uint8_t bit_depth, uint32_t lambda_q8,
                                                 const uint32_t* ctu_xy, uint32_t num_ctus, vvcg_ctu_search_res* res,
                                                 uint32_t* mode_costs) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (num_ctus && !mode_costs) return fail(ctx, VVCG_INVALID_INPUT, "missing mode costs");
  return ctu_search_xy(ctx, src, stride, width, height, bit_depth, lambda_q8, ctu_xy, num_ctus, nullptr, 6, 2, 0.0f,
                       VVCG_PRUNE_MASS, res, mode_costs);
}

static vvcg_status ctu_search_xy(vvcg_ctx* ctx, const uint16_t* src, uint64_t stride, uint32_t width,
                                 uint32_t height, uint8_t bit_depth, uint32_t lambda_q8, const uint32_t* ctu_xy,
                                 uint32_t num_ctus, const float* logits, uint32_t top_modes, uint32_t top_splits,
                                 float threshold, uint32_t rule, vvcg_ctu_search_res* res, uint32_t* mode_costs) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_ctus) return VVCG_OK;
  if (!src || !ctu_xy || !res) return fail(ctx, VVCG_INVALID_INPUT, "missing plane, positions or results");
  if (stride < width || bit_depth < 8 || bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "plane geometry");
  if (top_modes < 1 || top_modes > 6 || top_splits < 1 || top_splits > 6)
    return fail(ctx, VVCG_INVALID_INPUT, "top_modes and top_splits must be 1..6");
  if (width > (1u << 20) || height > (1u << 20) || num_ctus > (1u << 24))
    return fail(ctx, VVCG_LIMIT_EXCEEDED, "plane or CTU count too large");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  const size_t nb = (size_t)num_ctus * 15;
  CK(ctx->d_search_reqs.reserve(sizeof(CostReq) * nb), "cudaMalloc");
  CK(ctx->d_search_ctus.reserve(sizeof(vvcg_ctu_search_req) * num_ctus), "cudaMalloc");
  CK(ctx->d_search_cost.reserve(sizeof(uint32_t) * nb), "cudaMalloc");
  CK(ctx->d_search_mode.reserve(nb), "cudaMalloc");
  k_prune_requests<<<(num_ctus + 127) / 128, 128, 0, ctx->stream>>>(
      logits, ctu_xy, (int)num_ctus, (int)width, (int)height, (int)top_modes, (int)top_splits, threshold,
      rule == VVCG_PRUNE_MAX_PROB, (vvcg_ctu_search_req*)ctx->d_search_ctus.p, (CostReq*)ctx->d_search_reqs.p);
  CK(cudaGetLastError(), "prune launch");
  CostArgs A{src, (int64_t)stride, (int32_t)width, (int32_t)height, bit_depth, (int32_t)nb, lambda_q8,
             (const CostReq*)ctx->d_search_reqs.p, (uint32_t*)ctx->d_search_cost.p,
             (uint8_t*)ctx->d_search_mode.p, mode_costs};
  k_cost_search<<<(uint32_t)std::min<size_t>(nb, (size_t)ctx->num_sms * 8), kIsrWarps * 32, 0, ctx->stream>>>(A);
  CK(cudaGetLastError(), "search launch");
  k_ctu_search_combine<<<(num_ctus + 127) / 128, 128, 0, ctx->stream>>>(
      (const vvcg_ctu_search_req*)ctx->d_search_ctus.p, (int)num_ctus, lambda_q8,
      (const uint32_t*)ctx->d_search_cost.p, (const uint8_t*)ctx->d_search_mode.p, res);
  CK(cudaGetLastError(), "search launch");
  ctx->launches += 3;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// CNN pruner forward pass (vvcg_cnn_forward_dev).
// ---------------------------------------------------------------------------
static_assert(kCnnParams == VVCG_CNN_PARAMS && kCnnOut == VVCG_CNN_OUT, "CNN layout");
static_assert(sizeof(vvcg_split_req) == 16, "split request layout");
static_assert(sizeof(vvcg_mv_cand) == 24 && sizeof(vvcg_me_req) == 28 && sizeof(vvcg_me_res) == 40,
              "motion-estimation layouts");
static float cnn_qp_input(uint32_t qp) {  // QP / 63 rounded to bf16 (nearest even)
  float f = (float)qp / 63.0f;
  uint32_t u;
  memcpy(&u, &f, 4);
  u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
  memcpy(&f, &u, 4);
  return f;
}

extern "C" vvcg_status vvcg_cnn_forward_dev(vvcg_ctx* ctx, const uint16_t* plane, uint64_t stride, uint32_t width,
                                            uint32_t height, uint8_t bit_depth, uint8_t qp, const uint32_t* ctu_xy,
                                            uint32_t num_blocks, const float* params, float* logits, float* gap,
                                            uint16_t* acts, uint32_t* status) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_blocks) return VVCG_OK;
  if (!plane || !ctu_xy || !params || !logits || !status)
    return fail(ctx, VVCG_INVALID_INPUT, "missing plane, positions, parameters, logits or status");
  if (stride < width || bit_depth < 8 || bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "plane geometry");
  if (width > (1u << 20) || height > (1u << 20) || num_blocks > (1u << 24))
    return fail(ctx, VVCG_LIMIT_EXCEEDED, "plane or block count too large");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  static bool attr_set[64] = {};
  if (ctx->device < 64 && !attr_set[ctx->device]) {
    CK(cudaFuncSetAttribute(k_cnn_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, kCnnSmem), "smem attribute");
    attr_set[ctx->device] = true;
  }
  CK(ctx->d_cnn_pack.reserve(3 * kPackL), "cudaMalloc");
  k_cnn_pack<<<(3 * kCnnConvW + 255) / 256, 256, 0, ctx->stream>>>(params, (uint16_t*)ctx->d_cnn_pack.p, false);
  CK(cudaGetLastError(), "cnn pack launch");
  if (qp > 63) return fail(ctx, VVCG_INVALID_INPUT, "QP above 63");
  CnnFwdArgs A{plane, (int64_t)stride, (int32_t)width, (int32_t)height, (1 << bit_depth) - 1, (int32_t)num_blocks,
               cnn_qp_input(qp), ctu_xy, params, (const uint16_t*)ctx->d_cnn_pack.p, logits, gap, acts, status};
  const uint32_t grid = std::min<uint32_t>(num_blocks, (uint32_t)ctx->num_sms);
  k_cnn_forward<<<grid, kCnnThreads, kCnnSmem, ctx->stream>>>(A);
  CK(cudaGetLastError(), "cnn launch");
  ctx->launches += 2;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// CNN pruner training step (vvcg_cnn_train_step_dev).
// ---------------------------------------------------------------------------
static vvcg_status cnn_train_step(vvcg_ctx* ctx, const uint16_t* plane, uint64_t stride, uint32_t width,
                                  uint32_t height, uint8_t bit_depth, uint8_t qp, const uint32_t* ctu_xy,
                                  const uint8_t* labels, const float* soft, uint32_t num_blocks, float* params,
                                  float* adam_m, float* adam_v, uint32_t step, float lr, float* grads, float* loss,
                                  uint32_t* status);

extern "C" vvcg_status vvcg_cnn_train_step_dev(vvcg_ctx* ctx, const uint16_t* plane, uint64_t stride,
                                               uint32_t width, uint32_t height, uint8_t bit_depth, uint8_t qp,
                                               const uint32_t* ctu_xy, const uint8_t* labels, uint32_t num_blocks,
                                               float* params, float* adam_m, float* adam_v, uint32_t step, float lr,
                                               float* grads, float* loss, uint32_t* status) {
  return cnn_train_step(ctx, plane, stride, width, height, bit_depth, qp, ctu_xy, labels, nullptr, num_blocks, params,
                        adam_m, adam_v, step, lr, grads, loss, status);
}

extern "C" vvcg_status vvcg_cnn_train_step_soft_dev(vvcg_ctx* ctx, const uint16_t* plane, uint64_t stride,
                                                    uint32_t width, uint32_t height, uint8_t bit_depth, uint8_t qp,
                                                    const uint32_t* ctu_xy, const uint8_t* labels,
                                                    const float* soft_modes, uint32_t num_blocks, float* params,
                                                    float* adam_m, float* adam_v, uint32_t step, float lr,
                                                    float* grads, float* loss, uint32_t* status) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (num_blocks && !soft_modes) return fail(ctx, VVCG_INVALID_INPUT, "missing mode targets");
  return cnn_train_step(ctx, plane, stride, width, height, bit_depth, qp, ctu_xy, labels, soft_modes, num_blocks,
                        params, adam_m, adam_v, step, lr, grads, loss, status);
}

static vvcg_status cnn_train_step(vvcg_ctx* ctx, const uint16_t* plane, uint64_t stride, uint32_t width,
                                  uint32_t height, uint8_t bit_depth, uint8_t qp, const uint32_t* ctu_xy,
                                  const uint8_t* labels, const float* soft, uint32_t num_blocks, float* params,
                                  float* adam_m, float* adam_v, uint32_t step, float lr, float* grads, float* loss,
                                  uint32_t* status) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_blocks) return VVCG_OK;
  if (!plane || !ctu_xy || !labels || !params || !grads || !loss || !status)
    return fail(ctx, VVCG_INVALID_INPUT, "missing buffers");
  if (lr > 0.0f && (!adam_m || !adam_v || step == 0))
    return fail(ctx, VVCG_INVALID_INPUT, "an update needs the Adam moments and a step count from 1");
  if (stride < width || bit_depth < 8 || bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "plane geometry");
  if (num_blocks > 65536) return fail(ctx, VVCG_LIMIT_EXCEEDED, "more than 65536 blocks in one step");
  if (qp > 63) return fail(ctx, VVCG_INVALID_INPUT, "QP above 63");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  static bool attr_set[64] = {};
  if (ctx->device < 64 && !attr_set[ctx->device]) {
    CK(cudaFuncSetAttribute(k_cnn_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, kCnnSmem), "smem attribute");
    CK(cudaFuncSetAttribute(k_cnn_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, kCnnBwdSmem),
       "smem attribute");
    attr_set[ctx->device] = true;
  }
  const uint32_t grid = std::min<uint32_t>(num_blocks, (uint32_t)ctx->num_sms);
  CK(ctx->d_cnn_pack.reserve(3 * kPackL), "cudaMalloc");
  CK(ctx->d_cnn_packT.reserve(3 * kPackL), "cudaMalloc");
  CK(ctx->d_cnn_acts.reserve((size_t)num_blocks * 4 * 1024 * 32 * 2), "cudaMalloc");
  CK(ctx->d_cnn_logits.reserve((size_t)num_blocks * kCnnOut * 4), "cudaMalloc");
  CK(ctx->d_cnn_gap.reserve((size_t)num_blocks * 32 * 4), "cudaMalloc");
  CK(ctx->d_cnn_partial.reserve((size_t)grid * (kCnnParams + 1) * 4), "cudaMalloc");
  k_cnn_pack<<<(3 * kCnnConvW + 255) / 256, 256, 0, ctx->stream>>>(params, (uint16_t*)ctx->d_cnn_pack.p, false);
  k_cnn_pack<<<(3 * kCnnConvW + 255) / 256, 256, 0, ctx->stream>>>(params, (uint16_t*)ctx->d_cnn_packT.p, true);
  CK(cudaGetLastError(), "cnn pack launch");
  CnnFwdArgs F{plane, (int64_t)stride, (int32_t)width, (int32_t)height, (1 << bit_depth) - 1, (int32_t)num_blocks,
               cnn_qp_input(qp), ctu_xy, params, (const uint16_t*)ctx->d_cnn_pack.p, (float*)ctx->d_cnn_logits.p,
               (float*)ctx->d_cnn_gap.p, (uint16_t*)ctx->d_cnn_acts.p, status};
  k_cnn_forward<<<grid, kCnnThreads, kCnnSmem, ctx->stream>>>(F);
  CK(cudaGetLastError(), "cnn forward launch");
  CnnBwdArgs B{plane, (int64_t)stride, (int32_t)width, (int32_t)height, (1 << bit_depth) - 1, (int32_t)num_blocks,
               cnn_qp_input(qp), ctu_xy, labels, params, soft, (const uint16_t*)ctx->d_cnn_packT.p,
               (const float*)ctx->d_cnn_logits.p,
               (const float*)ctx->d_cnn_gap.p, (const uint16_t*)ctx->d_cnn_acts.p, (float*)ctx->d_cnn_partial.p,
               1.0f / (float)num_blocks, status};
  k_cnn_backward<<<grid, kCnnThreads, kCnnBwdSmem, ctx->stream>>>(B);
  CK(cudaGetLastError(), "cnn backward launch");
  k_cnn_reduce<<<(kCnnParams + 1 + 255) / 256, 256, 0, ctx->stream>>>((const float*)ctx->d_cnn_partial.p, (int)grid,
                                                                      grads, loss);
  CK(cudaGetLastError(), "cnn reduce launch");
  ctx->launches += 5;
  if (lr > 0.0f) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_cnn_adam<<<(kCnnParams + 255) / 256, 256, 0, ctx->stream>>>(params, grads, adam_m, adam_v, lr, b1, b2, 1e-8f,
                                                                   c1, c2);
    CK(cudaGetLastError(), "adam launch");
    ctx->launches++;
  }
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// Tensor-core self-test (vvcg_tc_selftest_dev).
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_tc_selftest_dev(vvcg_ctx* ctx, const uint16_t* a, const uint16_t* b, float* d,
                                            uint32_t* status) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!a || !b || !d || !status) return fail(ctx, VVCG_INVALID_INPUT, "missing buffers");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  k_umma_selftest<<<1, 128, 0, ctx->stream>>>(a, b, d, status);
  CK(cudaGetLastError(), "self-test launch");
  ctx->launches++;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// General-decoder intra prediction (vvcg_gen_intra_predict_dev).
// ---------------------------------------------------------------------------
static bool pow2_in(uint32_t v, uint32_t lo, uint32_t hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; }

extern "C" vvcg_status vvcg_gen_intra_predict_dev(vvcg_ctx* ctx, const vvcg_gen_intra_state* st,
                                                  const vvcg_gen_intra_req* reqs, uint32_t num_reqs, int16_t* out,
                                                  uint64_t out_count) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!st || !reqs || !out) return fail(ctx, VVCG_INVALID_INPUT, "missing state, requests or output");
  if (!st->plane[0] || !st->plane[1] || !st->plane[2] || !st->dec_y || !st->dec_c)
    return fail(ctx, VVCG_INVALID_INPUT, "missing planes or decoded maps");
  if (!st->width || !st->height || (st->width & 7) || (st->height & 7))
    return fail(ctx, VVCG_INVALID_INPUT, "picture size must be a multiple of 8");
  if (st->width > 16384 || st->height > 16384) return fail(ctx, VVCG_LIMIT_EXCEEDED, "picture larger than 16384");
  if (st->stride[0] < st->width || st->stride[1] < st->width / 2 || st->stride[2] < st->width / 2)
    return fail(ctx, VVCG_INVALID_INPUT, "stride smaller than the plane width");
  if (st->bit_depth < 8 || st->bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "bit depth");
  if (st->ctu_size && !pow2_in(st->ctu_size, 16, 128)) return fail(ctx, VVCG_INVALID_INPUT, "CTU size");
  for (uint32_t i = 0; i < num_reqs; i++) {
    const vvcg_gen_intra_req& r = reqs[i];
    if (r.comp > 2) return fail(ctx, VVCG_INVALID_INPUT, "request %u: component", i);
    if ((uint64_t)r.out_off + (uint64_t)r.w * r.h > out_count)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: output past the buffer", i);
    if (r.comp == 0) {
      if (!pow2_in(r.w, 1, 64) || !pow2_in(r.h, 1, 64) || r.x + r.w > st->width || r.y + r.h > st->height)
        return fail(ctx, VVCG_INVALID_INPUT, "request %u: luma block", i);
      if (r.mrl > 2 || r.isp > VVCG_ISP_VER || r.bdpcm > VVCG_BDPCM_VER)
        return fail(ctx, VVCG_INVALID_INPUT, "request %u: mrl / isp / bdpcm", i);
      if (r.isp != VVCG_ISP_NONE) {
        if (!pow2_in(r.cu_w, 4, 64) || !pow2_in(r.cu_h, 4, 64) || r.x < r.cu_x || r.y < r.cu_y ||
            r.x + r.w > r.cu_x + r.cu_w || r.y + r.h > r.cu_y + r.cu_h)
          return fail(ctx, VVCG_INVALID_INPUT, "request %u: ISP sub-partition outside its CU", i);
        if (r.isp == VVCG_ISP_VER && (r.cu_w == 4 || (r.cu_w == 8 && r.cu_h > 4)) && (r.cu_x & 3))
          return fail(ctx, VVCG_INVALID_INPUT, "request %u: ISP region off the 4-sample grid", i);
      } else if (r.mrl && (r.w < 4 || r.h < 4)) {
        return fail(ctx, VVCG_INVALID_INPUT, "request %u: MRL on a block below 4x4", i);
      }
    } else {
      if (!pow2_in(r.w, 2, 32) || !pow2_in(r.h, 2, 32) || r.x + r.w > st->width / 2 || r.y + r.h > st->height / 2)
        return fail(ctx, VVCG_INVALID_INPUT, "request %u: chroma block", i);
      if (r.mode > 66 && (r.mode < 81 || r.mode > 83)) return fail(ctx, VVCG_INVALID_INPUT, "request %u: mode", i);
      if (r.mode >= 81 && ((r.x | r.y) & 1)) return fail(ctx, VVCG_INVALID_INPUT, "request %u: CCLM position", i);
    }
  }
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_tu_recs.reserve(sizeof(vvcg_gen_intra_req) * num_reqs), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_tu_recs.p, reqs, sizeof(vvcg_gen_intra_req) * num_reqs, cudaMemcpyHostToDevice,
                     ctx->stream),
     "upload");
  GenIntraArgs A{*st, (const vvcg_gen_intra_req*)ctx->d_tu_recs.p, (int32_t)num_reqs, out};
  const uint32_t grid = std::min<uint32_t>((num_reqs + kGiWarps - 1) / kGiWarps, (uint32_t)ctx->num_sms * 8);
  k_gen_intra<<<grid, kGiWarps * 32, 0, ctx->stream>>>(A);
  CK(cudaGetLastError(), "intra launch");
  ctx->launches++;
  return VVCG_OK;
}

// Checks one general intra request against the picture (shared by the
// prediction and the reconstruction entry points); null when valid.
static const char* gen_intra_req_error(const vvcg_gen_intra_state* st, const vvcg_gen_intra_req& r,
                                       uint64_t out_count) {
  if (r.comp > 2) return "component";
  if ((uint64_t)r.out_off + (uint64_t)r.w * r.h > out_count) return "output past the buffer";
  if (r.comp == 0) {
    if (!pow2_in(r.w, 1, 64) || !pow2_in(r.h, 1, 64) || r.x + r.w > st->width || r.y + r.h > st->height)
      return "luma block";
    if (r.mrl > 2 || r.isp > VVCG_ISP_VER || r.bdpcm > VVCG_BDPCM_VER) return "mrl / isp / bdpcm";
    if (r.isp != VVCG_ISP_NONE) {
      if (!pow2_in(r.cu_w, 4, 64) || !pow2_in(r.cu_h, 4, 64) || r.x < r.cu_x || r.y < r.cu_y ||
          r.x + r.w > r.cu_x + r.cu_w || r.y + r.h > r.cu_y + r.cu_h)
        return "ISP sub-partition outside its CU";
      if (r.isp == VVCG_ISP_VER && (r.cu_w == 4 || (r.cu_w == 8 && r.cu_h > 4)) && (r.cu_x & 3))
        return "ISP region off the 4-sample grid";
    } else if (r.mrl && (r.w < 4 || r.h < 4)) {
      return "MRL on a block below 4x4";
    }
  } else {
    if (!pow2_in(r.w, 2, 32) || !pow2_in(r.h, 2, 32) || r.x + r.w > st->width / 2 || r.y + r.h > st->height / 2)
      return "chroma block";
    if (r.mode > 66 && (r.mode < 81 || r.mode > 83)) return "mode";
    if (r.mode >= 81 && ((r.x | r.y) & 1)) return "CCLM position";
  }
  return nullptr;
}

// ---------------------------------------------------------------------------
// General-decoder sequential reconstruction (vvcg_gen_intra_recon_dev).
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_gen_intra_recon_dev(vvcg_ctx* ctx, const vvcg_gen_intra_state* st,
                                                const vvcg_gen_intra_req* reqs, uint32_t num_reqs,
                                                const uint32_t* group_start, uint32_t num_groups,
                                                const int16_t* residual, int16_t* pred, uint64_t out_count) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_groups) return VVCG_OK;
  if (!st || !reqs || !group_start || !pred) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  if (!st->plane[0] || !st->plane[1] || !st->plane[2] || !st->dec_y || !st->dec_c)
    return fail(ctx, VVCG_INVALID_INPUT, "missing planes or decoded maps");
  if (!st->width || !st->height || (st->width & 7) || (st->height & 7))
    return fail(ctx, VVCG_INVALID_INPUT, "picture size must be a multiple of 8");
  if (st->width > 16384 || st->height > 16384) return fail(ctx, VVCG_LIMIT_EXCEEDED, "picture larger than 16384");
  if (st->stride[0] < st->width || st->stride[1] < st->width / 2 || st->stride[2] < st->width / 2)
    return fail(ctx, VVCG_INVALID_INPUT, "stride smaller than the plane width");
  if (st->bit_depth < 8 || st->bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "bit depth");
  if (st->ctu_size && !pow2_in(st->ctu_size, 16, 128)) return fail(ctx, VVCG_INVALID_INPUT, "CTU size");
  if (group_start[0] != 0 || group_start[num_groups] != num_reqs)
    return fail(ctx, VVCG_INVALID_INPUT, "groups must cover the requests from 0 to num_reqs");
  for (uint32_t g = 0; g < num_groups; g++)
    if (group_start[g + 1] < group_start[g]) return fail(ctx, VVCG_INVALID_INPUT, "group %u: decreasing start", g);
  for (uint32_t i = 0; i < num_reqs; i++)
    if (const char* e = gen_intra_req_error(st, reqs[i], out_count))
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: %s", i, e);
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  const size_t rb = sizeof(vvcg_gen_intra_req) * num_reqs, gb = sizeof(uint32_t) * (num_groups + 1);
  CK(ctx->d_tu_recs.reserve(rb + 256 + gb), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_tu_recs.p, reqs, rb, cudaMemcpyHostToDevice, ctx->stream), "upload");
  uint32_t* d_groups = (uint32_t*)((char*)ctx->d_tu_recs.p + ((rb + 255) & ~(size_t)255));
  CK(cudaMemcpyAsync(d_groups, group_start, gb, cudaMemcpyHostToDevice, ctx->stream), "upload");
  GenReconArgs A{*st, (const vvcg_gen_intra_req*)ctx->d_tu_recs.p, d_groups, (int32_t)num_groups, residual, pred};
  const uint32_t grid = std::min<uint32_t>((num_groups + kGiWarps - 1) / kGiWarps, (uint32_t)ctx->num_sms * 8);
  k_gen_intra_recon<<<grid, kGiWarps * 32, 0, ctx->stream>>>(A);
  CK(cudaGetLastError(), "intra reconstruction launch");
  ctx->launches++;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// General-decoder deblocking (vvcg_deblock_general_dev).
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_deblock_general_dev(vvcg_ctx* ctx, uint16_t* const planes[3], const uint32_t stride[3],
                                                uint32_t vis_width, uint32_t vis_height, uint8_t bit_depth,
                                                uint32_t ctu_size, const vvcg_dbk_cell* cells, uint32_t cell_cols,
                                                uint32_t cell_rows, const vvcg_dbk_ccell* ccells,
                                                uint32_t ccell_cols, uint32_t ccell_rows,
                                                const vvcg_dbk_params* params) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!planes || !stride || !cells || !ccells || !params) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  if (!vis_width || !vis_height) return VVCG_OK;
  if (vis_width > 32768 || vis_height > 32768) return fail(ctx, VVCG_LIMIT_EXCEEDED, "picture larger than 32768");
  const uint32_t cw = (vis_width + 1) / 2, ch = (vis_height + 1) / 2;
  for (int c = 0; c < 3; c++)
    if (!planes[c] || stride[c] < (c ? cw : vis_width))
      return fail(ctx, VVCG_INVALID_INPUT, "plane %d: missing or stride too small", c);
  if (bit_depth < 8 || bit_depth > 12) return fail(ctx, VVCG_INVALID_INPUT, "bit depth");
  if (ctu_size < 16 || ctu_size > 128 || (ctu_size & (ctu_size - 1)))
    return fail(ctx, VVCG_INVALID_INPUT, "CTU size must be a power of two in 16..128");
  if (cell_cols < (vis_width + 3) / 4 || cell_rows < (vis_height + 3) / 4)
    return fail(ctx, VVCG_INVALID_INPUT, "luma cell map smaller than the picture");
  if (ccell_cols < (cw + 1) / 2 || ccell_rows < (ch + 1) / 2)
    return fail(ctx, VVCG_INVALID_INPUT, "chroma cell map smaller than the picture");
  if (params->num_ref[0] < 0 || params->num_ref[0] > 16 || params->num_ref[1] < 0 || params->num_ref[1] > 16)
    return fail(ctx, VVCG_INVALID_INPUT, "reference list length must be 0..16");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  DbkGenArgs A;
  for (int c = 0; c < 3; c++) {
    A.plane[c] = planes[c];
    A.stride[c] = (int32_t)stride[c];
  }
  A.vis_w = (int32_t)vis_width;
  A.vis_h = (int32_t)vis_height;
  A.cw = (int32_t)cw;
  A.ch = (int32_t)ch;
  A.bd = bit_depth;
  A.ctu = (int32_t)ctu_size;
  A.cells = cells;
  A.cols = (int32_t)cell_cols;
  A.rows = (int32_t)cell_rows;
  A.cc = ccells;
  A.ccols = (int32_t)ccell_cols;
  A.crows = (int32_t)ccell_rows;
  A.prm = *params;
  const uint64_t n = (uint64_t)((vis_width + 3) / 4) * ((vis_height + 3) / 4);
  const dim3 grid((uint32_t)std::min<uint64_t>((n + 127) / 128, (uint64_t)ctx->num_sms * 16), 3);
  k_dbk_general<true><<<grid, 128, 0, ctx->stream>>>(A);
  CK(cudaGetLastError(), "deblock launch");
  k_dbk_general<false><<<grid, 128, 0, ctx->stream>>>(A);
  CK(cudaGetLastError(), "deblock launch");
  ctx->launches += 2;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// Inter-prediction tools (BDOF, DMVR, affine / PROF, CIIP, GPM).
// ---------------------------------------------------------------------------
static_assert(sizeof(vvcg_bdof_req) == 8 && sizeof(vvcg_dmvr_req) == 28 && sizeof(vvcg_affine_req) == 36 &&
                  sizeof(vvcg_prof_req) == 16 && sizeof(vvcg_ciip_req) == 12 && sizeof(vvcg_gpm_req) == 12,
              "inter tool request layouts");

namespace {

// Copies n host requests into the context's request buffer; the device copy.
template <class T>
vvcg_status upload_reqs(vvcg_ctx* ctx, const T* reqs, uint32_t n, const T** dev) {
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_tu_recs.reserve(sizeof(T) * n), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_tu_recs.p, reqs, sizeof(T) * n, cudaMemcpyHostToDevice, ctx->stream), "upload");
  *dev = (const T*)ctx->d_tu_recs.p;
  return VVCG_OK;
}

}  // namespace

extern "C" vvcg_status vvcg_bdof_dev(vvcg_ctx* ctx, const vvcg_bdof_req* reqs, uint32_t num_reqs, const int32_t* pred0,
                                     const int32_t* pred1, int32_t* out, uint64_t count) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!reqs || !pred0 || !pred1 || !out) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  for (uint32_t i = 0; i < num_reqs; i++) {
    const vvcg_bdof_req& r = reqs[i];
    if (r.w < 4 || r.h < 4 || (r.w & 3) || (r.h & 3) || r.w > 128 || r.h > 128)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: block must be 4..128 and a multiple of 4", i);
    if ((uint64_t)r.off + (uint64_t)r.w * r.h > count) return fail(ctx, VVCG_INVALID_INPUT, "request %u: past the arrays", i);
  }
  const vvcg_bdof_req* d;
  vvcg_status st = upload_reqs(ctx, reqs, num_reqs, &d);
  if (st != VVCG_OK) return st;
  k_bdof<<<num_reqs, 128, 0, ctx->stream>>>(d, pred0, pred1, out);
  CK(cudaGetLastError(), "bdof launch");
  ctx->launches++;
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_dmvr_dev(vvcg_ctx* ctx, const uint8_t* ref0, const uint8_t* ref1, uint32_t width,
                                     uint32_t height, uint32_t stride, const vvcg_dmvr_req* reqs, uint32_t num_reqs,
                                     int32_t* mv_out) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!ref0 || !ref1 || !reqs || !mv_out) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  if (!width || !height || stride < width || width > 16384 || height > 16384)
    return fail(ctx, VVCG_INVALID_INPUT, "reference plane geometry");
  for (uint32_t i = 0; i < num_reqs; i++)
    if (!reqs[i].dx || !reqs[i].dy || reqs[i].dx > 16 || reqs[i].dy > 16)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: subblock must be 1..16 x 1..16", i);
  const vvcg_dmvr_req* d;
  vvcg_status st = upload_reqs(ctx, reqs, num_reqs, &d);
  if (st != VVCG_OK) return st;
  DmvrArgs A{ref0, ref1, (int32_t)width, (int32_t)height, (int32_t)stride, (int32_t)num_reqs, d, mv_out};
  k_dmvr<<<(num_reqs + 3) / 4, 128, 0, ctx->stream>>>(A);
  CK(cudaGetLastError(), "dmvr launch");
  ctx->launches++;
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_affine_mvs_dev(vvcg_ctx* ctx, const vvcg_affine_req* reqs, uint32_t num_reqs,
                                           int32_t* sub_mv, uint64_t sub_count, int32_t* prof) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!reqs || !sub_mv || !prof) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  for (uint32_t i = 0; i < num_reqs; i++) {
    const vvcg_affine_req& r = reqs[i];
    if (!pow2_in(r.w, 8, 128) || !pow2_in(r.h, 8, 128) || r.inter_dir < 1 || r.inter_dir > 3)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: size or prediction type", i);
    if ((uint64_t)r.sub_off + (uint64_t)(r.w / 4) * (r.h / 4) > sub_count)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: subblock MVs past the array", i);
  }
  const vvcg_affine_req* d;
  vvcg_status st = upload_reqs(ctx, reqs, num_reqs, &d);
  if (st != VVCG_OK) return st;
  k_affine_mvs<<<(num_reqs + 127) / 128, 128, 0, ctx->stream>>>(d, (int)num_reqs, sub_mv, prof);
  CK(cudaGetLastError(), "affine launch");
  ctx->launches++;
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_prof_dev(vvcg_ctx* ctx, const vvcg_prof_req* reqs, uint32_t num_reqs, const int32_t* src,
                                     uint64_t src_count, const int32_t* dmv, uint64_t dmv_count, int32_t* out,
                                     uint64_t out_count) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!reqs || !src || !dmv || !out) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  for (uint32_t i = 0; i < num_reqs; i++)
    if ((uint64_t)reqs[i].src_off + 36 > src_count || (uint64_t)reqs[i].dmv_off + 32 > dmv_count ||
        (uint64_t)reqs[i].out_off + 16 > out_count)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: past the arrays", i);
  const vvcg_prof_req* d;
  vvcg_status st = upload_reqs(ctx, reqs, num_reqs, &d);
  if (st != VVCG_OK) return st;
  k_prof<<<(16 * num_reqs + 127) / 128, 128, 0, ctx->stream>>>(d, (int)num_reqs, src, dmv, out);
  CK(cudaGetLastError(), "prof launch");
  ctx->launches++;
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_ciip_blend_dev(vvcg_ctx* ctx, const vvcg_ciip_req* reqs, uint32_t num_reqs,
                                           const int32_t* inter, const int32_t* intra, int32_t* out, uint64_t count) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!reqs || !inter || !intra || !out) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  for (uint32_t i = 0; i < num_reqs; i++)
    if ((uint64_t)reqs[i].off + reqs[i].n > count) return fail(ctx, VVCG_INVALID_INPUT, "request %u: past the arrays", i);
  const vvcg_ciip_req* d;
  vvcg_status st = upload_reqs(ctx, reqs, num_reqs, &d);
  if (st != VVCG_OK) return st;
  k_ciip<<<num_reqs, 128, 0, ctx->stream>>>(d, inter, intra, out);
  CK(cudaGetLastError(), "ciip launch");
  ctx->launches++;
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_gpm_blend_dev(vvcg_ctx* ctx, const vvcg_gpm_req* reqs, uint32_t num_reqs,
                                          const int32_t* pred0, const int32_t* pred1, int32_t* out, uint64_t count) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!num_reqs) return VVCG_OK;
  if (!reqs || !pred0 || !pred1 || !out) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  for (uint32_t i = 0; i < num_reqs; i++) {
    const vvcg_gpm_req& r = reqs[i];
    if (!r.w || !r.h || r.w > 128 || r.h > 128 || r.split_dir > 63 || r.scale_x > 1 || r.scale_y > 1)
      return fail(ctx, VVCG_INVALID_INPUT, "request %u: size, split direction or subsampling", i);
    if ((uint64_t)r.off + (uint64_t)r.w * r.h > count) return fail(ctx, VVCG_INVALID_INPUT, "request %u: past the arrays", i);
  }
  const vvcg_gpm_req* d;
  vvcg_status st = upload_reqs(ctx, reqs, num_reqs, &d);
  if (st != VVCG_OK) return st;
  k_gpm<<<num_reqs, 128, 0, ctx->stream>>>(d, pred0, pred1, out);
  CK(cudaGetLastError(), "gpm launch");
  ctx->launches++;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// CTU-boundary deblocking of inter pictures (vvcg_deblock_ctu_edges_dev).
// ---------------------------------------------------------------------------
static_assert(sizeof(vvcg_ctu_motion) == 40, "CTU motion layout");

extern "C" vvcg_status vvcg_deblock_ctu_edges_dev(vvcg_ctx* ctx, uint16_t* const planes[3], const uint32_t stride[3],
                                                  uint32_t width, uint32_t height, uint32_t ctu, uint8_t qp,
                                                  const vvcg_ctu_motion* cells) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!planes || !stride || !cells) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  if (ctu != 32 && ctu != 64 && ctu != 128) return fail(ctx, VVCG_INVALID_INPUT, "CTU size must be 32, 64 or 128");
  if (!width || !height || width % ctu || height % ctu)
    return fail(ctx, VVCG_INVALID_INPUT, "picture size must be a nonzero multiple of the CTU size");
  if ((uint64_t)width * height > kMaxLumaSamples) return fail(ctx, VVCG_LIMIT_EXCEEDED, "picture too large");
  if (qp > 63) return fail(ctx, VVCG_INVALID_INPUT, "QP above 63");
  const int w = (int)width, h = (int)height, cw = w / 2, ch = h / 2, c = (int)ctu, cc = c / 2;
  for (int k = 0; k < 3; k++)
    if (!planes[k] || stride[k] < (uint32_t)(k ? cw : w) || (stride[k] & 7) ||
        (reinterpret_cast<uintptr_t>(planes[k]) & 15))
      return fail(ctx, VVCG_INVALID_INPUT,
                  "plane %d: needs a 16-byte aligned pointer and a stride >= the width that is a multiple of 8", k);
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  // slice.rs:2305-2311: SliceQpY, derived_chroma_qp, lengths of min(ctu, 32)
  // luma and ctu/2 chroma transform sides
  const int cqp = std::min(63, std::max(0, (int)qp <= 26 ? (int)qp : (int)qp - 1));
  const int lml = std::min(c, 32) >= 32 ? 7 : 3;
  const int cols = w / c, rows = h / c;
  auto& v = ctx->dbf_ctu;
  v.clear();
  // luma V, Cb V, Cr V, luma H, Cb H, Cr H
  v.push_back(DbfPass{planes[0], (int32_t)stride[0], w, h, 8, c, c, (int)qp, 0, 0, 0, lml, lml, 1, cols - 1, h / 4,
                      cells, cols, 0, c});
  for (int k = 1; k <= 2; k++)
    v.push_back(DbfPass{planes[k], (int32_t)stride[k], cw, ch, 8, cc, cc, cqp, 0, 0, 0, 3, 3, 2, cols - 1, ch / 2,
                        cells, cols, k, cc});
  v.push_back(DbfPass{planes[0], (int32_t)stride[0], w, h, 8, c, c, (int)qp, 0, 0, 0, lml, lml, 1, rows - 1, w / 4,
                      cells, cols, 0, c});
  for (int k = 1; k <= 2; k++)
    v.push_back(DbfPass{planes[k], (int32_t)stride[k], cw, ch, 8, cc, cc, cqp, 0, 0, 0, 3, 3, 2, rows - 1, cw / 2,
                        cells, cols, k, cc});
  CK(ctx->d_dbf_ctu.reserve(sizeof(DbfPass) * v.size()), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_dbf_ctu.p, v.data(), sizeof(DbfPass) * v.size(), cudaMemcpyHostToDevice, ctx->stream),
     "upload");
  const DbfPass* d = (const DbfPass*)ctx->d_dbf_ctu.p;
  auto blocks = [](const DbfPass& p) { return (unsigned)((std::max(0, p.n_edges * p.n_segs) + 127) / 128); };
  if (cols > 1) {
    k_deblock_luma<true><<<dim3(blocks(v[0]), 1), 128, 0, ctx->stream>>>(d, 1);
    k_deblock_chroma<true><<<dim3(blocks(v[1]), 2), 128, 0, ctx->stream>>>(d + 1, 2);
    ctx->launches += 2;
  }
  if (rows > 1) {
    k_deblock_luma<false><<<dim3(blocks(v[3]), 1), 128, 0, ctx->stream>>>(d + 3, 1);
    k_deblock_chroma<false><<<dim3(blocks(v[4]), 2), 128, 0, ctx->stream>>>(d + 4, 2);
    ctx->launches += 2;
  }
  CK(cudaGetLastError(), "deblock launch");
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// General-decoder SAO of one plane (vvcg_sao_bounded_16_dev).
// ---------------------------------------------------------------------------
extern "C" vvcg_status vvcg_sao_bounded_16_dev(vvcg_ctx* ctx, const uint16_t* src, uint16_t* dst, uint32_t stride,
                                               uint32_t width, uint32_t height, uint32_t vis_width,
                                               uint32_t vis_height, uint8_t bit_depth, uint32_t ctu_size,
                                               uint32_t ctu_cols, const vvcg_sao* params) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!width || !height) return VVCG_OK;
  if (!src || !dst || !params || stride < width || !ctu_size || bit_depth < 8 || bit_depth > 12)
    return fail(ctx, VVCG_INVALID_INPUT, "invalid SAO arguments");
  if (vis_width > width || vis_height > height) return fail(ctx, VVCG_INVALID_INPUT, "visible size");
  if (ctu_cols < (vis_width + ctu_size - 1) / ctu_size) return fail(ctx, VVCG_INVALID_INPUT, "CTU columns");
  if (src == dst) return fail(ctx, VVCG_INVALID_INPUT, "SAO reads an unfiltered copy: src and dst must differ");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  SaoBoundedPass S{src, dst, params, (int32_t)stride, (int32_t)width, (int32_t)height, (int32_t)vis_width,
                   (int32_t)vis_height, bit_depth, (int32_t)ctu_size, (int32_t)ctu_cols};
  const uint64_t n = (uint64_t)width * height;
  const uint32_t grid = (uint32_t)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->num_sms * 16);
  k_sao_bounded<<<grid, 256, 0, ctx->stream>>>(S);
  CK(cudaGetLastError(), "sao launch");
  ctx->launches++;
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// Plane metrics (vvcg_plane_metrics_8_dev / vvcg_plane_metrics_16_dev).
// ---------------------------------------------------------------------------
namespace {

template <typename T>
vvcg_status plane_metrics(vvcg_ctx* ctx, const T* ref, uint64_t ref_stride, const T* dist, uint64_t dist_stride,
                          uint32_t w, uint32_t h, uint64_t* out) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!out) return fail(ctx, VVCG_INVALID_INPUT, "missing output");
  if (w && h && (!ref || !dist)) return fail(ctx, VVCG_INVALID_INPUT, "missing plane");
  if (w && h && (ref_stride < w || dist_stride < w))
    return fail(ctx, VVCG_INVALID_INPUT, "plane view exceeds its backing buffer");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  // out[0] SSE, out[1] SAD, out[2] samples (accelerator.rs:258-292)
  CK(cudaMemsetAsync(out, 0, 2 * sizeof(uint64_t), ctx->stream), "memset");
  const uint64_t samples = (uint64_t)w * h;
  CK(cudaMemcpyAsync(out + 2, &samples, sizeof(samples), cudaMemcpyHostToDevice, ctx->stream), "samples");
  if (samples == 0) return VVCG_OK;
  const uint64_t work = samples / (16 / sizeof(T)) + h;
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((work + 255) / 256, (uint64_t)ctx->num_sms * 8));
  k_plane_metrics<T><<<grid, 256, 0, ctx->stream>>>(ref, ref_stride, dist, dist_stride, w, h,
                                                    reinterpret_cast<unsigned long long*>(out));
  CK(cudaGetLastError(), "metrics launch");
  ctx->launches++;
  return VVCG_OK;
}

}  // namespace

extern "C" vvcg_status vvcg_plane_metrics_8_dev(vvcg_ctx* ctx, const uint8_t* ref, uint64_t ref_stride,
                                                const uint8_t* dist, uint64_t dist_stride, uint32_t width,
                                                uint32_t height, uint64_t* out) {
  return plane_metrics(ctx, ref, ref_stride, dist, dist_stride, width, height, out);
}

extern "C" vvcg_status vvcg_plane_metrics_16_dev(vvcg_ctx* ctx, const uint16_t* ref, uint64_t ref_stride,
                                                 const uint16_t* dist, uint64_t dist_stride, uint32_t width,
                                                 uint32_t height, uint64_t* out) {
  return plane_metrics(ctx, ref, ref_stride, dist, dist_stride, width, height, out);
}

// ---------------------------------------------------------------------------
// Encoder (vvcg_encode_batch).
// ---------------------------------------------------------------------------
namespace {

// hls.rs:796-802 derived_chroma_qp_bd with a zero chroma QP offset.
int derived_chroma_qp_bd_host(int qpy, int bd) {
  const int off = 6 * (bd - 8);
  const int qpi = std::min(63, std::max(-off, qpy));
  const int mapped = qpi <= 26 ? qpi : qpi - 1;
  const int base = std::min(63, std::max(-off, mapped)) + off;
  return std::min(63 + off, std::max(0, base));
}

// CU records and level-pool entries of one picture (one slot of
// tb*tb + 2*tb_cw*tb_ch levels per CU); false for a geometry the frame path
// rejects (slice.rs:129-160).
bool encode_geometry(const vvcg_pic_desc& d, uint32_t* cus, uint64_t* levels) {
  if (d.ctu_log2 < 5 || d.ctu_log2 > 7 || d.chroma_format > 3) return false;
  const uint32_t ctu = 1u << d.ctu_log2;
  if (d.width < ctu || d.height < ctu || d.width % ctu || d.height % ctu) return false;
  const int tb = std::min<int>(ctu, 32), cf = d.chroma_format;
  const int sw = (cf == 1 || cf == 2) ? 2 : 1, sh = cf == 1 ? 2 : 1;
  const int tcw = cf ? std::max(tb / sw, 2) : 0, tch = cf ? std::max(tb / sh, 2) : 0;
  *cus = (d.width / tb) * (d.height / tb);
  *levels = (uint64_t)*cus * (uint64_t)(tb * tb + 2 * tcw * tch);
  return true;
}

}  // namespace

extern "C" vvcg_status vvcg_encode_sizes(const vvcg_pic_desc* pics, uint32_t num_pics, uint32_t* num_cus,
                                         uint64_t* num_levels) {
  if (!pics || !num_cus || !num_levels) return VVCG_INVALID_INPUT;
  uint64_t c = 0, l = 0;
  for (uint32_t i = 0; i < num_pics; i++) {
    uint32_t pc;
    uint64_t pl;
    if (!encode_geometry(pics[i], &pc, &pl)) return VVCG_INVALID_INPUT;
    c += pc;
    l += pl;
  }
  if (c > 0xffffffffull || l > 0x7fffffffull) return VVCG_LIMIT_EXCEEDED;
  *num_cus = (uint32_t)c;
  *num_levels = l;
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_encode_batch(vvcg_ctx* ctx, const vvcg_pic_desc* pics, uint32_t num_pics,
                                         const vvcg_plane_in* src, vvcg_cu_rec* cus, uint32_t cus_cap,
                                         int16_t* levels, uint64_t levels_cap) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!pics || !num_pics || !src || !cus || !levels) return fail(ctx, VVCG_INVALID_INPUT, "missing arguments");
  uint32_t total_cus = 0;
  uint64_t total_levels = 0;
  vvcg_status st = vvcg_encode_sizes(pics, num_pics, &total_cus, &total_levels);
  if (st != VVCG_OK) return fail(ctx, st, "picture geometry outside the frame path or too many levels");
  if (cus_cap < total_cus || levels_cap < total_levels)
    return fail(ctx, VVCG_INVALID_INPUT, "outputs need %u records and %llu levels", total_cus,
                (unsigned long long)total_levels);
  std::vector<vvcg_pic_desc> d(pics, pics + num_pics);
  std::vector<uint32_t> lv_base(num_pics);
  uint32_t cu_at = 0;
  uint64_t lv_at = 0;
  for (uint32_t i = 0; i < num_pics; i++) {
    if (d[i].tools & (VVCG_TOOL_SAO | VVCG_TOOL_ALF))
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: the encoder does not apply SAO or ALF", i);
    if (d[i].tools & VVCG_TOOL_SPARSE_LEVELS)
      return fail(ctx, VVCG_INVALID_INPUT, "picture %u: the encoder writes dense levels", i);
    if (d[i].slice_qp > 63) return fail(ctx, VVCG_INVALID_INPUT, "picture %u: slice QP above 63", i);
    for (int c = 0; c < (d[i].chroma_format ? 3 : 1); c++)
      if (!src[i * 3 + c].data) return fail(ctx, VVCG_INVALID_INPUT, "picture %u: missing source plane %d", i, c);
    uint32_t pc;
    uint64_t pl;
    encode_geometry(d[i], &pc, &pl);
    d[i].chroma_qp_scaled = (uint8_t)derived_chroma_qp_bd_host(d[i].slice_qp, d[i].bit_depth);
    d[i].cu_offset = cu_at;
    d[i].ctu_offset = 0;
    d[i].alf_aps = -1;
    lv_base[i] = (uint32_t)lv_at;
    cu_at += pc;
    lv_at += pl;
  }
  std::vector<vvcg_cu_rec> none(total_cus);
  for (auto& r : none) r = vvcg_cu_rec{0, 0, 0, 0, {-1, -1, -1}};
  vvcg_batch b{d.data(), num_pics, total_cus, none.data(), nullptr, 0, nullptr, 0, 0, nullptr};
  if ((st = vvcg_batch_prepare(ctx, &b)) != VVCG_OK) return st;
  ctx->prepared = false;  // until the encode has finished
  CK(ctx->d_levels.reserve(std::max<uint64_t>(1, total_levels) * sizeof(int16_t)), "cudaMalloc levels");
  ctx->num_levels = total_levels;
  for (uint32_t i = 0; i < num_pics; i++) {
    ctx->pics[i].lv_pool = (int16_t*)ctx->d_levels.p;
    ctx->pics[i].lv_base = (int32_t)lv_base[i];
  }
  if ((st = upload_vec(ctx, ctx->d_pics, ctx->pics)) != VVCG_OK) return st;
  CK(cudaMemsetAsync(ctx->d_levels.p, 0, total_levels * sizeof(int16_t), ctx->stream), "memset levels");
  for (uint32_t i = 0; i < num_pics; i++) {
    const DevPic& P = ctx->pics[i];
    for (int c = 0; c < (P.cf ? 3 : 1); c++) {
      // the mode decisions read not-yet-coded samples as 0 (zeroed planes)
      CK(cudaMemsetAsync(P.plane[c], 0, (size_t)P.stride[c] * P.ph[c] * sizeof(uint16_t), ctx->stream), "memset");
      const vvcg_plane_in& in = src[i * 3 + c];
      if (in.stride < (uint32_t)P.pw[c]) return fail(ctx, VVCG_INVALID_INPUT, "picture %u: source stride", i);
      CK(cudaMemcpy2DAsync(P.scratch[c], (size_t)P.stride[c] * 2, in.data, (size_t)in.stride * 2,
                           (size_t)P.pw[c] * 2, P.ph[c], cudaMemcpyDefault, ctx->stream),
         "source upload");
    }
  }
  uint32_t* ctrl = (uint32_t*)ctx->d_ctrl.p;
  CK(cudaMemsetAsync(ctrl, 0, 2 * sizeof(uint32_t), ctx->stream), "memset");
  ctx->epoch++;
  const uint32_t n = (uint32_t)ctx->items.size();
  const size_t smem = kEncWarps * sizeof(EncWs);
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_encode_rows, kEncWarps * 32, smem), "occupancy");
  const uint32_t warps = (uint32_t)ctx->num_sms * std::max(1, per_sm) * kEncWarps;
  const uint32_t grid = (std::min<uint32_t>(n, warps) + kEncWarps - 1) / kEncWarps;
  k_encode_rows<<<grid, kEncWarps * 32, smem, ctx->stream>>>((const DevPic*)ctx->d_pics.p,
                                                            (const RowItem*)ctx->d_items.p, n, ctrl, ctx->epoch,
                                                            ctx->spin_limit, ctrl + 1);
  CK(cudaGetLastError(), "encode launch");
  ctx->launches++;
  ctx->prepared = true;
  if ((st = vvcg_batch_sync(ctx)) != VVCG_OK) return st;
  if ((st = vvcg_batch_run(ctx, VVCG_STAGE_DEBLOCK)) != VVCG_OK) return st;
  CK(cudaMemcpyAsync(cus, ctx->d_cus.p, sizeof(vvcg_cu_rec) * total_cus, cudaMemcpyDefault, ctx->stream),
     "records download");
  CK(cudaMemcpyAsync(levels, ctx->d_levels.p, sizeof(int16_t) * total_levels, cudaMemcpyDefault, ctx->stream),
     "levels download");
  return vvcg_batch_sync(ctx);
}

// ---------------------------------------------------------------------------
// Transform-unit batches (vvcg_tu_inverse_batch / vvcg_tu_forward_batch).
// ---------------------------------------------------------------------------
namespace {

// Size bins of the transform-unit batches (at most 256, 1024 and 4096
// coefficients) and the CTA widths each can launch with: one unit per warp,
// kTuTable[bin][variant] warps per CTA. Wider CTAs share fewer, larger
// launches; narrower ones spread a small bin over more SMs. The results do
// not depend on the width (every warp transforms its own unit), so
// vvcg_tu_autotune can pick the fastest per bin by timing alone.
using TuKernel = void (*)(const vvcg_tu_rec*, const uint32_t*, uint32_t, const int16_t*, int16_t*);
struct TuVariant {
  TuKernel inv, fwd;
  int warps;
  size_t smem;
};
constexpr int kTuBins = 3, kTuVariants = 3;
template <int kEl, int kW>
TuVariant tu_variant() {
  return TuVariant{k_tu<kEl, kW, false>, k_tu<kEl, kW, true>, kW, tu_smem_bytes<kEl, kW>()};
}
const TuVariant kTuTable[kTuBins][kTuVariants] = {
    {tu_variant<256, 2>(), tu_variant<256, 4>(), tu_variant<256, 8>()},
    {tu_variant<1024, 2>(), tu_variant<1024, 4>(), tu_variant<1024, 8>()},
    {tu_variant<4096, 1>(), tu_variant<4096, 2>(), tu_variant<4096, 4>()}};
static_assert(sizeof(((vvcg_ctx*)nullptr)->tu_pick[0]) == kTuBins, "one choice per bin");

bool tu_set_smem_limits() {
  for (int b = 0; b < kTuBins; b++)
    for (int v = 0; v < kTuVariants; v++) {
      const TuVariant& V = kTuTable[b][v];
      if (cudaFuncSetAttribute(V.inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)V.smem) != cudaSuccess ||
          cudaFuncSetAttribute(V.fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)V.smem) != cudaSuccess)
        return false;
    }
  return true;
}

int tu_bin(const vvcg_tu_rec& r) {
  const uint32_t el = 1u << (r.log2_w + r.log2_h);
  return el <= 256 ? 0 : (el <= 1024 ? 1 : 2);
}

// Why the reference would reject a unit (dct.rs matrix_for_any / zero-out
// checks, lfnst.rs parameters_rect, slice.rs:701 MTS with LFNST), or nullptr.
const char* tu_reject(const vvcg_tu_rec& r, bool forward, uint64_t in_count, uint64_t out_count) {
  if (r.log2_w > 6 || r.log2_h > 6 || r.log2_w + r.log2_h == 0) return "size outside 1x2..64x64";
  const uint32_t n = 1u << (r.log2_w + r.log2_h);
  if (r.bit_depth < 8 || r.bit_depth > 12) return "bit depth outside 8..=12";
  if (r.qp > 87) return "Qp' above 87";
  if ((uint64_t)r.in_off + n > in_count) return "input range past the buffer";
  if ((uint64_t)r.out_off + n > out_count) return "output range past the buffer";
  if (forward && (r.flags & (VVCG_TU_BDPCM_HOR | VVCG_TU_BDPCM_VER))) return "BDPCM is inverse only";
  if ((r.flags & VVCG_TU_BDPCM_HOR) && (r.flags & VVCG_TU_BDPCM_VER)) return "two BDPCM directions";
  if (r.flags & VVCG_TU_TRANSFORM_SKIP) return nullptr;
  if (r.mts_idx > 4) return "mts_idx above 4";
  if (r.lfnst_idx > 2) return "lfnst_idx above 2";
  if (forward && r.lfnst_idx && r.mts_idx) return "MTS combined with LFNST";
  TuShape S;
  tu_shape(r, S);
  auto has = [](int tr, int lg) { return tr == 0 ? (lg >= 1 && lg <= 6) : (lg >= 2 && lg <= 5); };
  if (S.w > 1 && (!has(S.th, S.lw) || S.sw >= S.w)) return "unsupported horizontal transform";
  if (S.h > 1 && (!has(S.tv, S.lh) || S.sh >= S.h)) return "unsupported vertical transform";
  if (r.lfnst_idx > 0 && r.mts_idx == 0 && (S.w < 4 || S.h < 4 || r.lfnst_mode >= 95)) return "unsupported LFNST";
  return nullptr;
}

// Validates the units, groups them by size bin (count[b] units of bin b, in
// that order in d_tu_idx) and uploads records and order to the device.
vvcg_status tu_stage(vvcg_ctx* ctx, const vvcg_tu_rec* recs, uint32_t n, uint64_t in_count, uint64_t out_count,
                     bool forward, uint32_t count[kTuBins]) {
  for (int b = 0; b < kTuBins; b++) count[b] = 0;
  for (uint32_t i = 0; i < n; i++) {
    if (const char* why = tu_reject(recs[i], forward, in_count, out_count))
      return fail(ctx, VVCG_INVALID_INPUT, "transform unit %u: %s", i, why);
    count[tu_bin(recs[i])]++;
  }
  // units grouped by size bin
  ctx->tu_idx.resize(n);
  uint32_t at[kTuBins] = {0, count[0], count[0] + count[1]};
  for (uint32_t i = 0; i < n; i++) ctx->tu_idx[at[tu_bin(recs[i])]++] = i;
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(ctx->d_tu_recs.reserve(sizeof(vvcg_tu_rec) * n), "cudaMalloc");
  CK(ctx->d_tu_idx.reserve(sizeof(uint32_t) * n), "cudaMalloc");
  CK(cudaMemcpyAsync(ctx->d_tu_recs.p, recs, sizeof(vvcg_tu_rec) * n, cudaMemcpyHostToDevice, ctx->stream), "upload");
  CK(cudaMemcpyAsync(ctx->d_tu_idx.p, ctx->tu_idx.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, ctx->stream),
     "upload");
  return VVCG_OK;
}

// Launches the staged units of size bin b with CTA width variant v.
vvcg_status tu_launch(vvcg_ctx* ctx, const uint32_t count[kTuBins], int b, int v, bool forward, const int16_t* in,
                      int16_t* out) {
  const TuVariant& V = kTuTable[b][v];
  uint32_t first = 0;
  for (int k = 0; k < b; k++) first += count[k];
  const TuKernel k = forward ? V.fwd : V.inv;
  k<<<(count[b] + V.warps - 1) / V.warps, V.warps * 32, V.smem, ctx->stream>>>(
      (const vvcg_tu_rec*)ctx->d_tu_recs.p, (const uint32_t*)ctx->d_tu_idx.p + first, count[b], in, out);
  CK(cudaGetLastError(), "transform-unit launch");
  ctx->launches++;
  return VVCG_OK;
}

vvcg_status tu_batch(vvcg_ctx* ctx, const vvcg_tu_rec* recs, uint32_t n, const int16_t* in,
                     uint64_t in_count, int16_t* out, uint64_t out_count, bool forward) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (n == 0) return VVCG_OK;
  if (!recs || !in || !out) return fail(ctx, VVCG_INVALID_INPUT, "missing records or buffers");
  uint32_t count[kTuBins];
  vvcg_status st = tu_stage(ctx, recs, n, in_count, out_count, forward, count);
  for (int b = 0; b < kTuBins && st == VVCG_OK; b++)
    if (count[b]) st = tu_launch(ctx, count, b, ctx->tu_pick[forward ? 1 : 0][b], forward, in, out);
  return st;
}

}  // namespace

extern "C" vvcg_status vvcg_tu_inverse_batch(vvcg_ctx* ctx, const vvcg_tu_rec* recs, uint32_t num_recs,
                                             const int16_t* in, uint64_t in_count, int16_t* out,
                                             uint64_t out_count) {
  return tu_batch(ctx, recs, num_recs, in, in_count, out, out_count, false);
}

extern "C" vvcg_status vvcg_tu_forward_batch(vvcg_ctx* ctx, const vvcg_tu_rec* recs, uint32_t num_recs,
                                             const int16_t* in, uint64_t in_count, int16_t* out,
                                             uint64_t out_count) {
  return tu_batch(ctx, recs, num_recs, in, in_count, out, out_count, true);
}

// Times every CTA width of each non-empty size bin on the caller's batch
// (one warm-up launch, then kTuTuneReps launches between two events on the
// context's stream) and keeps the fastest in the context.
extern "C" vvcg_status vvcg_tu_autotune(vvcg_ctx* ctx, const vvcg_tu_rec* recs, uint32_t num_recs,
                                        const int16_t* in, uint64_t in_count, int16_t* out, uint64_t out_count,
                                        uint32_t forward, uint32_t warps[3]) {
  constexpr int kTuTuneReps = 3;
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!warps) return fail(ctx, VVCG_INVALID_INPUT, "missing result array");
  for (int b = 0; b < kTuBins; b++) warps[b] = 0;
  if (num_recs == 0) return VVCG_OK;
  if (!recs || !in || !out) return fail(ctx, VVCG_INVALID_INPUT, "missing records or buffers");
  const bool fwd = forward != 0;
  uint32_t count[kTuBins];
  vvcg_status st = tu_stage(ctx, recs, num_recs, in_count, out_count, fwd, count);
  if (st != VVCG_OK) return st;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  struct Events {
    cudaEvent_t* e;
    ~Events() {
      for (int i = 0; i < 2; i++)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } guard{ev};
  CK(cudaEventCreate(&ev[0]), "cudaEventCreate");
  CK(cudaEventCreate(&ev[1]), "cudaEventCreate");
  for (int b = 0; b < kTuBins; b++) {
    if (!count[b]) continue;
    int best = ctx->tu_pick[fwd ? 1 : 0][b];
    float best_ms = 0.0f;
    for (int v = 0; v < kTuVariants; v++) {
      if ((st = tu_launch(ctx, count, b, v, fwd, in, out)) != VVCG_OK) return st;
      CK(cudaEventRecord(ev[0], ctx->stream), "cudaEventRecord");
      for (int r = 0; r < kTuTuneReps; r++)
        if ((st = tu_launch(ctx, count, b, v, fwd, in, out)) != VVCG_OK) return st;
      CK(cudaEventRecord(ev[1], ctx->stream), "cudaEventRecord");
      CK(cudaEventSynchronize(ev[1]), "transform-unit timing");
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, ev[0], ev[1]), "cudaEventElapsedTime");
      if (v == 0 || ms < best_ms) {
        best_ms = ms;
        best = v;
      }
    }
    ctx->tu_pick[fwd ? 1 : 0][b] = (uint8_t)best;
    warps[b] = (uint32_t)kTuTable[b][best].warps;
  }
  CK(cudaStreamSynchronize(ctx->stream), "transform-unit timing");
  return VVCG_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free single-picture reconstruction (vvcg_recon_picture_static).
//
// The context entry points above grow their device buffers with cudaMalloc.
// This one takes records, levels and planes in the caller's device memory and
// keeps its own bookkeeping in the fixed array g_static_scratch below, which
// is part of the library's module image: nothing is allocated per call. The
// residuals go into the caller's planes (DevPic::scratch aliases
// DevPic::plane): the wavefront kernel reads each sample's residual in the
// same lane, just before it stores that sample's reconstruction, and
// neighbouring blocks only read samples that are already reconstructed.
// ---------------------------------------------------------------------------
namespace {

constexpr uint32_t kStaticMaxCtuRows = VVCG_STATIC_MAX_CTU_ROWS;

// Written from the host on every call.
struct StaticHeader {
  DevPic pic;
  DbfPass dbf[6];  // luma V, luma H, Cb V, Cr V, Cb H, Cr H
  RowItem rows[kStaticMaxCtuRows];
};

// Byte layout of the array: [0, 256) control words ([0] row queue counter,
// [1] status word), then one 128-byte progress line per CTU row, then the
// header. The control words and the progress lines must start at zero.
constexpr size_t kStaticFlagsOff = 256;
constexpr size_t kStaticFlagsBytes = (size_t)kStaticMaxCtuRows * kRowFlagStride * sizeof(uint64_t);
constexpr size_t kStaticHeaderOff = kStaticFlagsOff + kStaticFlagsBytes;
constexpr size_t kStaticScratchBytes = 40960;
static_assert(kStaticHeaderOff % 256 == 0, "header alignment");
static_assert(kStaticHeaderOff + sizeof(StaticHeader) <= kStaticScratchBytes, "scratch array too small");

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct StaticDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_static_scratch
  int num_sms = 0;
  int recon_ctas_per_sm = 0;
};

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
StaticDevice g_static_dev[kStaticMaxDevices];

vvcg_status static_fail(char* err, size_t cap, vvcg_status st, const char* fmt, ...) {
  if (err && cap) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, cap, fmt, ap);
    va_end(ap);
  }
  return st;
}

#define SCK(call, what)                                                                 \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e != cudaSuccess)                                                              \
      return static_fail(err, err_cap, VVCG_EXECUTION, "%s: %s", what, cudaGetErrorString(_e)); \
  } while (0)

// Once per device, with that device current: tables, kernel attributes, the
// array's device address and the wavefront grid size.
vvcg_status static_setup(int dev, const StaticDevice** out, char* err, size_t err_cap) {
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (dev < 0 || dev >= kStaticMaxDevices)
    return static_fail(err, err_cap, VVCG_UNAVAILABLE, "device %d is beyond the %d this entry point tracks",
                       dev, kStaticMaxDevices);
  StaticDevice& S = g_static_dev[dev];
  if (!S.ready) {
    vvcg_ctx tables_ctx;  // host-side only: carries the device number and an error message
    tables_ctx.device = dev;
    if (upload_tables(&tables_ctx) != VVCG_OK)
      return static_fail(err, err_cap, VVCG_UNAVAILABLE, "%s", tables_ctx.err.c_str());
    const int wave_smem = (int)(kWarpsPerCta * sizeof(WaveWs));
    SCK(cudaFuncSetAttribute(k_recon_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, wave_smem),
        "cudaFuncSetAttribute");
    void* p = nullptr;
    SCK(cudaGetSymbolAddress(&p, g_static_scratch), "cudaGetSymbolAddress");
    SCK(cudaDeviceGetAttribute(&S.num_sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    SCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&S.recon_ctas_per_sm, k_recon_rows,
                                                      kWarpsPerCta * 32, wave_smem),
        "occupancy");
    S.scratch = (unsigned char*)p;
    S.ready = true;
  }
  *out = &S;
  return VVCG_OK;
}

}  // namespace

extern "C" vvcg_status vvcg_recon_picture_static(const vvcg_pic_desc* pic, const vvcg_cu_rec* cus,
                                                 uint32_t num_cus, const int16_t* levels,
                                                 uint64_t num_levels, const vvcg_plane_out* planes,
                                                 void* cuda_stream, char* err, size_t err_cap) {
  if (err && err_cap) err[0] = 0;
  if (!pic || !planes || !cus) return static_fail(err, err_cap, VVCG_INVALID_INPUT, "missing picture, records or planes");
  const vvcg_pic_desc& d = *pic;
  if (d.ctu_log2 < 5 || d.ctu_log2 > 7)
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "CTU size outside 32..=128");
  const uint32_t ctu = 1u << d.ctu_log2;
  if (d.width < ctu || d.height < ctu || d.width % ctu || d.height % ctu)
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "coded size not aligned to the CTU grid");
  if ((uint64_t)d.width * d.height > kMaxLumaSamples)
    return static_fail(err, err_cap, VVCG_LIMIT_EXCEEDED, "%ux%u exceeds %llu luma samples", d.width,
                       d.height, (unsigned long long)kMaxLumaSamples);
  if (d.height / ctu > kStaticMaxCtuRows)
    return static_fail(err, err_cap, VVCG_LIMIT_EXCEEDED,
                       "%u CTU rows; this entry point holds at most %u (use vvcg_decode_batch)",
                       d.height / ctu, kStaticMaxCtuRows);
  if (d.bit_depth < 8 || d.bit_depth > 12 || d.chroma_format > 3)
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "bit depth or chroma format");
  if (d.tools & (VVCG_TOOL_SAO | VVCG_TOOL_ALF))
    return static_fail(err, err_cap, VVCG_INVALID_INPUT,
                       "SAO and ALF need a second set of planes (use vvcg_decode_batch)");
  const int tb = std::min<int>(ctu, 32);
  const int cf = d.chroma_format;
  const int sw = (cf == 1 || cf == 2) ? 2 : 1, sh = cf == 1 ? 2 : 1;
  const uint32_t gw = d.width / tb, gh = d.height / tb;
  if ((uint64_t)d.cu_offset + (uint64_t)gw * gh > num_cus)
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "CU records out of range");
  if (num_levels && !levels) return static_fail(err, err_cap, VVCG_INVALID_INPUT, "missing levels");
  const int ncomp = cf ? 3 : 1;

  StaticHeader h;
  memset(&h, 0, sizeof(h));
  DevPic& P = h.pic;
  for (int c = 0; c < 3; c++) {
    P.pw[c] = c == 0 ? d.width : (cf ? (d.width + sw - 1) / sw : 0);
    P.ph[c] = c == 0 ? d.height : (cf ? (d.height + sh - 1) / sh : 0);
    if (c >= ncomp) continue;
    const vvcg_plane_out& o = planes[c];
    if (!o.data || (reinterpret_cast<uintptr_t>(o.data) & 15) || (o.stride & 7) || o.stride < (uint32_t)P.pw[c])
      return static_fail(err, err_cap, VVCG_INVALID_INPUT,
                         "plane %d: needs a 16-byte aligned pointer and a stride >= %d that is a multiple of 8",
                         c, P.pw[c]);
    P.plane[c] = o.data;
    P.scratch[c] = o.data;  // residuals first, reconstruction over them
    P.stride[c] = (int32_t)o.stride;
  }
  P.bd = d.bit_depth;
  P.cf = cf;
  P.ctu_log2 = d.ctu_log2;
  P.ctu = ctu;
  P.tb = tb;
  P.tb_cw = cf ? std::max(tb / sw, 2) : 0;
  P.tb_ch = cf ? std::max(tb / sh, 2) : 0;
  P.sub_w = sw;
  P.sub_h = sh;
  P.grid_w = gw;
  P.grid_h = gh;
  P.ctu_w = d.width / ctu;
  P.ctu_h = d.height / ctu;
  // slice.rs:4681-4682 Qp'Y and Qp'C, both at least 4
  const int off = 6 * (d.bit_depth - 8);
  P.lqp = std::max(std::min(63 + off, std::max(0, (int)d.slice_qp + off)), 4);
  P.cqp = std::max((int)d.chroma_qp_scaled, 4);
  P.slice_qp = d.slice_qp;
  P.tools = d.tools;
  P.aps = -1;
  P.cus = cus + d.cu_offset;
  P.ctus = nullptr;
  for (int cy = 0; cy < P.ctu_h; cy++) h.rows[cy] = RowItem{0, (uint32_t)cy};

  // Deblocking passes: the same lattice, CTB and QP rules as vvcg_batch_prepare
  // (slice.rs:4990-5020).
  int n_dbf[4] = {0, 0, 0, 0};  // luma V, luma H, chroma V, chroma H
  if (d.tools & VVCG_TOOL_DEBLOCK) {
    const int step = std::max(P.tb, 8), ctb = std::max(P.ctu, step);
    const int lml = step <= 4 ? 1 : (step >= 32 ? 7 : 3);
    DbfPass v{P.plane[0], P.stride[0], P.pw[0], P.ph[0], P.bd, step, ctb, (int)d.slice_qp, 2, 0, 0,
              lml, lml, 1, 0, 0};
    v.n_edges = (P.pw[0] - 8) / step;
    v.n_segs = P.ph[0] / 4;
    DbfPass hz = v;
    hz.n_edges = (P.ph[0] - 8) / step;
    hz.n_segs = P.pw[0] / 4;
    if (v.n_edges > 0 && v.n_segs > 0) h.dbf[n_dbf[0]++] = v;
    if (hz.n_edges > 0 && hz.n_segs > 0) h.dbf[1 + n_dbf[1]++] = hz;
    if (cf) {
      const int cqp = std::min(63, std::max(0, (int)d.slice_qp <= 26 ? (int)d.slice_qp : (int)d.slice_qp - 1));
      const int cstep = std::max(P.tb_cw, 8);
      const int cctb = std::max(P.ctu / P.sub_h, cstep);
      const int clen = cstep >= 8 ? 3 : 1;
      for (int c = 1; c <= 2; c++) {
        DbfPass cv{P.plane[c], P.stride[c], P.pw[c], P.ph[c], P.bd, cstep, cctb, cqp, 2, 0, 0,
                   clen, clen, P.sub_h, 0, 0};
        cv.n_edges = P.pw[c] >= 8 ? (P.pw[c] - 4) / cstep : 0;
        cv.n_segs = P.ph[c] / (P.sub_h == 1 ? 4 : 2);
        DbfPass ch = cv;
        ch.sub = P.sub_w;
        ch.n_edges = P.ph[c] >= 8 ? (P.ph[c] - 4) / cstep : 0;
        ch.n_segs = P.pw[c] / (P.sub_w == 1 ? 4 : 2);
        if (cv.n_edges > 0 && cv.n_segs > 0) h.dbf[2 + n_dbf[2]++] = cv;
        if (ch.n_edges > 0 && ch.n_segs > 0) h.dbf[4 + n_dbf[3]++] = ch;
      }
    }
  }

  int dev = 0;
  SCK(cudaGetDevice(&dev), "cudaGetDevice");
  const StaticDevice* S = nullptr;
  vvcg_status st = static_setup(dev, &S, err, err_cap);
  if (st != VVCG_OK) return st;
  cudaStream_t s = (cudaStream_t)cuda_stream;
  unsigned char* base = S->scratch;
  uint32_t* ctrl = reinterpret_cast<uint32_t*>(base);
  P.row_done = reinterpret_cast<uint64_t*>(base + kStaticFlagsOff);
  const DevPic* d_pic = reinterpret_cast<const DevPic*>(base + kStaticHeaderOff + offsetof(StaticHeader, pic));
  const DbfPass* d_dbf = reinterpret_cast<const DbfPass*>(base + kStaticHeaderOff + offsetof(StaticHeader, dbf));
  const RowItem* d_rows = reinterpret_cast<const RowItem*>(base + kStaticHeaderOff + offsetof(StaticHeader, rows));

  // control words and this picture's progress lines start at zero; the header
  // is rewritten whole up to the last row item in use
  SCK(cudaMemsetAsync(base, 0, kStaticFlagsOff + (size_t)P.ctu_h * kRowFlagStride * sizeof(uint64_t), s),
      "clear scratch");
  SCK(cudaMemcpyAsync(base + kStaticHeaderOff, &h, offsetof(StaticHeader, rows) + sizeof(RowItem) * P.ctu_h,
                      cudaMemcpyHostToDevice, s),
      "header upload");
  const uint32_t ncus = gw * gh;
  k_residual<<<dim3((ncus + kWarpsPerCta - 1) / kWarpsPerCta, 1), kWarpsPerCta * 32, 0, s>>>(
      d_pic, levels, num_levels, ctrl + 1);
  SCK(cudaGetLastError(), "residual launch");
  if (d.tools & VVCG_TOOL_TU_TOOLS) {
    k_residual_tools<<<dim3((ncus + kResToolWarps - 1) / kResToolWarps, 1), kResToolWarps * 32, 0, s>>>(
        d_pic, levels, num_levels, ctrl + 1);
    SCK(cudaGetLastError(), "residual (TU tools) launch");
  }
  const uint32_t warps = (uint32_t)S->num_sms * std::max(1, S->recon_ctas_per_sm) * kWarpsPerCta;
  const uint32_t grid = (std::min<uint32_t>((uint32_t)P.ctu_h, warps) + kWarpsPerCta - 1) / kWarpsPerCta;
  const uint32_t epoch = 1;  // progress lines were cleared above
  k_recon_rows<<<grid, kWarpsPerCta * 32, kWarpsPerCta * sizeof(WaveWs), s>>>(
      d_pic, d_rows, (uint32_t)P.ctu_h, ctrl, epoch, kDefaultSpinLimit, ctrl + 1);
  SCK(cudaGetLastError(), "recon launch");
  for (int k = 0; k < 4; k++) {
    const int n = n_dbf[k];
    if (!n) continue;
    const int first = k == 0 ? 0 : (k == 1 ? 1 : (k == 2 ? 2 : 4));
    uint32_t maxw = 0;
    for (int i = 0; i < n; i++) maxw = std::max<uint32_t>(maxw, (uint32_t)(h.dbf[first + i].n_edges * h.dbf[first + i].n_segs));
    dim3 g((maxw + 127) / 128, (unsigned)n);
    if (k == 0) k_deblock_luma<true><<<g, 128, 0, s>>>(d_dbf + first, n);
    if (k == 1) k_deblock_luma<false><<<g, 128, 0, s>>>(d_dbf + first, n);
    if (k == 2) k_deblock_chroma<true><<<g, 128, 0, s>>>(d_dbf + first, n);
    if (k == 3) k_deblock_chroma<false><<<g, 128, 0, s>>>(d_dbf + first, n);
    SCK(cudaGetLastError(), "deblock launch");
  }
  uint32_t status = 0;
  SCK(cudaMemcpyAsync(&status, ctrl + 1, sizeof(status), cudaMemcpyDeviceToHost, s), "status");
  SCK(cudaStreamSynchronize(s), "synchronize");
  if (status & kStatusTimeout)
    return static_fail(err, err_cap, VVCG_TIMEOUT, "a wavefront wait gave up after %u polls", kDefaultSpinLimit);
  if (status & kStatusBadRecord) return static_fail(err, err_cap, VVCG_INVALID_INPUT, "a level offset or sparse level entry was out of range");
  return VVCG_OK;
}

#include "gen_picture.cuh"
#include "p_picture.cuh"

// ---------------------------------------------------------------------------
// CABAC parse of strict-profile pictures on the host (vvcg_parse_strict).
// ---------------------------------------------------------------------------
#include <atomic>
#include <thread>

#include "cabac_parse.h"
#include "mt_parse.h"

namespace {

// Runs parse(i, &levels_used[i]) for every picture on `threads` host
// threads (pictures taken in turn from a shared counter) and reports the
// first picture that failed.
template <class F>
vvcg_status parse_pictures(uint32_t num_pics, uint32_t threads, uint64_t* levels_used, char* err, size_t err_cap,
                           F parse) {
  std::atomic<uint32_t> next{0};
  std::vector<int> code(num_pics, 0);
  auto work = [&]() {
    for (uint32_t i; (i = next.fetch_add(1)) < num_pics;) code[i] = parse(i, &levels_used[i]);
  };
  const uint32_t n = std::max<uint32_t>(1, std::min<uint32_t>(threads ? threads : 1, num_pics));
  std::vector<std::thread> pool;
  for (uint32_t t = 1; t < n; t++) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  static const char* kWhy[] = {"",
                               "last position outside the block",
                               "level outside 16 bits",
                               "syntax",
                               "level capacity exceeded",
                               "no end of slice or alignment",
                               "intra coding unit inside an inter slice"};
  for (uint32_t i = 0; i < num_pics; i++)
    if (code[i])
      return static_fail(err, err_cap, code[i] == vvcg_parse::kTruncated ? VVCG_LIMIT_EXCEEDED : VVCG_INVALID_INPUT,
                         "picture %u: %s", i, kWhy[std::min(code[i], 6)]);
  return VVCG_OK;
}

}  // namespace

extern "C" vvcg_status vvcg_parse_strict(const vvcg_strict_substream* pics, uint32_t num_pics, uint32_t sparse,
                                         uint32_t threads, vvcg_cu_rec* cus, uint64_t num_cus, int16_t* levels,
                                         uint64_t num_levels, uint64_t* levels_used, char* err, size_t err_cap) {
  if (err && err_cap) err[0] = 0;
  if (!num_pics) return VVCG_OK;
  if (!pics || !cus || !levels || !levels_used)
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "missing pictures, records, levels or counts");
  for (uint32_t i = 0; i < num_pics; i++) {
    const vvcg_strict_substream& p = pics[i];
    if (!p.data && p.size) return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: missing data", i);
    if (!p.width || !p.height || p.width % 32 || p.height % 32 || p.width > 16384 || p.height > 16384)
      return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: coded size not a multiple of 32", i);
    if (p.qp > 63) return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: slice QP above 63", i);
    if ((uint64_t)p.cu_offset + (uint64_t)(p.width / 32) * (p.height / 32) > num_cus)
      return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: records past the array", i);
    if (p.level_offset + p.level_cap > num_levels || (sparse && (p.level_offset & 1)))
      return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: level range", i);
  }
  return parse_pictures(num_pics, threads, levels_used, err, err_cap, [&](uint32_t i, uint64_t* used) {
    const vvcg_strict_substream& p = pics[i];
    vvcg_parse::LevelSink sink{levels + p.level_offset, p.level_cap, 0, sparse != 0};
    const int code = vvcg_parse::parse_strict_picture(p.data, p.size, p.qp, (int)p.width, (int)p.height,
                                                      cus + p.cu_offset, sink, (int64_t)p.level_offset);
    *used = sink.at;
    return code;
  });
}

namespace {

// Checks of one multi-tool substream: CTU 32, options, record and level ranges.
vvcg_status check_slice_substream(const vvcg_slice_substream& p, uint32_t i, uint32_t sparse, uint64_t num_cus,
                                  uint64_t num_levels, uint32_t allowed, char* err, size_t err_cap) {
  if (!p.data && p.size) return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: missing data", i);
  if (p.ctu_log2 != 5) return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: CTU size must be 32", i);
  if (!p.width || !p.height || p.width % 32 || p.height % 32 || p.width > 16384 || p.height > 16384)
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: coded size not a multiple of 32", i);
  if (p.qp > 63) return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: slice QP above 63", i);
  if (p.options & ~allowed)
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: unsupported slice options 0x%x", i, p.options);
  if ((uint64_t)p.cu_offset + (uint64_t)(p.width / 32) * (p.height / 32) > num_cus)
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: records past the array", i);
  if (p.level_offset + p.level_cap > num_levels || (sparse && (p.level_offset & 1)))
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "picture %u: level range", i);
  return VVCG_OK;
}

}  // namespace

extern "C" vvcg_status vvcg_parse_multitool_idr(const vvcg_slice_substream* pics, uint32_t num_pics, uint32_t sparse,
                                                uint32_t threads, vvcg_cu_rec* cus, uint64_t num_cus, int16_t* levels,
                                                uint64_t num_levels, uint64_t* levels_used, char* err,
                                                size_t err_cap) {
  if (err && err_cap) err[0] = 0;
  if (!num_pics) return VVCG_OK;
  if (!pics || !cus || !levels || !levels_used)
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "missing pictures, records, levels or counts");
  const uint32_t allowed =
      VVCG_SLICE_DEP_QUANT | VVCG_SLICE_SIGN_HIDING | VVCG_SLICE_FULL_INTRA_MODES | VVCG_SLICE_DEBLOCK;
  for (uint32_t i = 0; i < num_pics; i++) {
    vvcg_status st = check_slice_substream(pics[i], i, sparse, num_cus, num_levels, allowed, err, err_cap);
    if (st != VVCG_OK) return st;
  }
  return parse_pictures(num_pics, threads, levels_used, err, err_cap, [&](uint32_t i, uint64_t* used) {
    const vvcg_slice_substream& p = pics[i];
    vvcg_parse::LevelSink sink{levels + p.level_offset, p.level_cap, 0, sparse != 0};
    const int code = vvcg_parse::parse_mt_idr_picture(
        p.data, p.size, p.qp, (int)p.width, (int)p.height, (p.options & VVCG_SLICE_DEP_QUANT) != 0,
        (p.options & VVCG_SLICE_SIGN_HIDING) != 0, cus + p.cu_offset, sink, (int64_t)p.level_offset);
    *used = sink.at;
    return code;
  });
}

extern "C" vvcg_status vvcg_parse_multitool_p(const vvcg_slice_substream* pics, uint32_t num_pics, uint32_t sparse,
                                              uint32_t threads, vvcg_inter_cu* cus, uint64_t num_cus, int16_t* levels,
                                              uint64_t num_levels, uint64_t* levels_used, char* err, size_t err_cap) {
  if (err && err_cap) err[0] = 0;
  if (!num_pics) return VVCG_OK;
  if (!pics || !cus || !levels || !levels_used)
    return static_fail(err, err_cap, VVCG_INVALID_INPUT, "missing pictures, records, levels or counts");
  const uint32_t allowed =
      VVCG_SLICE_DEP_QUANT | VVCG_SLICE_SIGN_HIDING | VVCG_SLICE_FULL_INTRA_MODES | VVCG_SLICE_DEBLOCK;
  for (uint32_t i = 0; i < num_pics; i++) {
    vvcg_status st = check_slice_substream(pics[i], i, sparse, num_cus, num_levels, allowed, err, err_cap);
    if (st != VVCG_OK) return st;
  }
  return parse_pictures(num_pics, threads, levels_used, err, err_cap, [&](uint32_t i, uint64_t* used) {
    const vvcg_slice_substream& p = pics[i];
    vvcg_parse::LevelSink sink{levels + p.level_offset, p.level_cap, 0, sparse != 0};
    const int code = vvcg_parse::parse_mt_p_picture(
        p.data, p.size, p.qp, (int)p.width, (int)p.height, (p.options & VVCG_SLICE_DEP_QUANT) != 0,
        (p.options & VVCG_SLICE_SIGN_HIDING) != 0, cus + p.cu_offset, sink, (int64_t)p.level_offset);
    *used = sink.at;
    return code;
  });
}

extern "C" vvcg_status vvcg_parse_residual_block(const uint8_t* data, uint64_t size, uint32_t w, uint32_t h,
                                                 uint32_t flags, uint32_t qp, int32_t* out) {
  if (!out || (!data && size)) return VVCG_INVALID_INPUT;
  if (w < 1 || h < 1 || w > 64 || h > 64 || (w & (w - 1)) || (h & (h - 1)) || w * h < 2 || qp > 63)
    return VVCG_INVALID_INPUT;
  if ((flags & VVCG_PARSE_TRANSFORM_SKIP) && (w > 32 || h > 32)) return VVCG_INVALID_INPUT;
  const vvcg_parse::Scan s = vvcg_parse::make_scan((int)w, (int)h);
  vvcg_parse::Reader r;
  r.start(data, size);
  vvcg_parse::Models m;
  m.init_i_slice((int)qp);
  if (flags & VVCG_PARSE_TRANSFORM_SKIP) {
    vvcg_parse::decode_ts_residual(r, m, s, out);
  } else if (vvcg_parse::decode_residual(r, m, s, out, (flags & VVCG_PARSE_LUMA) != 0,
                                         (flags & VVCG_PARSE_DEP_QUANT) != 0,
                                         (flags & VVCG_PARSE_SIGN_HIDING) != 0) != vvcg_parse::kOk) {
    return VVCG_INVALID_INPUT;
  }
  if (!r.terminate() || !r.aligned_end()) return VVCG_INVALID_INPUT;
  return VVCG_OK;
}


// ---- Annex-B access units (host only) ----------------------------------------

static vvcg_status copy_out(const std::vector<uint8_t>& v, uint8_t* out, size_t cap, size_t* size) {
  if (size) *size = v.size();
  if (v.size() > cap) return VVCG_LIMIT_EXCEEDED;
  if (!v.empty()) {
    if (!out) return VVCG_INVALID_INPUT;
    memcpy(out, v.data(), v.size());
  }
  return VVCG_OK;
}

extern "C" vvcg_status vvcg_hls_rbsp(const vvcg_stream_cfg* cfg, uint32_t kind, int32_t arg, uint8_t* out,
                                     size_t cap, size_t* size) {
  namespace ab = vvcg::annexb;
  if (!cfg || !size) return VVCG_INVALID_INPUT;
  if (cfg->ctu_log2 < 5 || cfg->ctu_log2 > 7 || (cfg->crop_right & 1) || (cfg->crop_bottom & 1) ||
      cfg->min_cb_log2 < 2 || cfg->ts_log2 < 2)
    return VVCG_INVALID_INPUT;
  const ab::StreamCfg c{cfg->width,    cfg->height,    cfg->crop_right,  cfg->crop_bottom, cfg->qp,
                        cfg->level_idc, cfg->ctu_log2, cfg->min_cb_log2, cfg->ts_log2};
  switch (kind) {
    case VVCG_HLS_AUD: return copy_out(ab::aud_rbsp((uint8_t)arg), out, cap, size);
    case VVCG_HLS_VPS: return copy_out(ab::vps_rbsp(c), out, cap, size);
    case VVCG_HLS_SPS: return copy_out(ab::sps_rbsp(c), out, cap, size);
    case VVCG_HLS_PPS: return copy_out(ab::pps_rbsp(c), out, cap, size);
    case VVCG_HLS_PH: return copy_out(ab::ph_rbsp((uint32_t)arg), out, cap, size);
    case VVCG_HLS_SLICE_HEADER: return copy_out(ab::slice_header(arg), out, cap, size);
    default: return VVCG_INVALID_INPUT;
  }
}

extern "C" vvcg_status vvcg_annexb_idr(uint32_t width, uint32_t height, uint8_t qp, const uint8_t* slice_data,
                                       size_t n, uint8_t* out, size_t cap, size_t* size) {
  if (!size || !width || !height || width > (1u << 16) || height > (1u << 16) || qp > 63 || (n && !slice_data))
    return VVCG_INVALID_INPUT;
  const vvcg::annexb::StreamCfg c = vvcg::annexb::encoder_cfg(width, height, qp);
  return copy_out(vvcg::annexb::idr_access_unit(c, slice_data, n), out, cap, size);
}

extern "C" vvcg_status vvcg_annexb_read_idr(const uint8_t* au, size_t n, vvcg_annexb_info* info,
                                            uint8_t* slice_data, size_t cap, size_t* size) {
  namespace ab = vvcg::annexb;
  if (!au || !info || !size) return VVCG_INVALID_INPUT;
  const std::vector<ab::Nal> nals = ab::split(au, n);
  memset(info, 0, sizeof(*info));
  info->num_nals = (uint32_t)nals.size();
  bool have_pps = false;
  int32_t init_qp = 0;
  for (const ab::Nal& x : nals) {
    if (x.type == ab::kNalPps) {  // hls.rs:529-564
      const std::vector<uint8_t> r = ab::unescape(au + x.begin, x.end - x.begin);
      ab::Reader b(r.data(), r.size());
      b.u(6); b.u(4); b.u(1);  // PPS id, SPS id, mixed NALU types
      info->width = b.ue();
      info->height = b.ue();
      b.u(1); b.u(1); b.u(1);  // conformance window, scaling window, output flag (0 in this layout)
      if (b.u(1) != 1) return VVCG_INVALID_INPUT;  // pps_no_pic_partition_flag
      b.u(1); b.u(1);          // subpic id mapping, CABAC init present
      b.ue(); b.ue();          // default active ref idx L0 / L1
      b.u(1); b.u(1); b.u(1); b.u(1);
      init_qp = 26 + b.se();
      if (!b.ok()) return VVCG_INVALID_INPUT;
      have_pps = true;
    } else if (x.type == 7 || x.type == ab::kNalIdrNLp) {  // hls.rs:598-637
      if (!have_pps) return VVCG_INVALID_INPUT;
      const std::vector<uint8_t> r = ab::unescape(au + x.begin, x.end - x.begin);
      ab::Reader b(r.data(), r.size());
      if (b.u(1) != 0) return VVCG_INVALID_INPUT;  // sh_picture_header_in_slice_header_flag
      b.u(1);                                      // sh_no_output_of_prior_pics_flag
      const int32_t qp_delta = b.se();
      b.u(1);                                      // sh_ts_residual_coding_disabled_flag
      if (b.u(1) != 1) return VVCG_INVALID_INPUT;  // byte_alignment(): the one bit ...
      while (b.ok() && (b.pos() & 7))
        if (b.u(1) != 0) return VVCG_INVALID_INPUT;  // ... then zeros
      if (!b.ok()) return VVCG_INVALID_INPUT;
      info->qp = init_qp + qp_delta;
      info->slice_nal_type = x.type;
      const std::vector<uint8_t> data(r.begin() + (ptrdiff_t)(b.pos() >> 3), r.end());
      return copy_out(data, slice_data, cap, size);
    }
  }
  return VVCG_INVALID_INPUT;
}
