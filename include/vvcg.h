/*
 * vvcg.h - C ABI of the B200 (sm_100a) VVC reconstruction, in-loop filter and
 * candidate-cost library (libvvcg.so).
 *
 * The library replaces the sample-domain half of rustmpeg-video's VVC
 * decoder and encoder (crates/rustmpeg-video/src/vvc/). The CPU keeps CABAC
 * parsing and syntax; after a picture has been parsed, its coding-unit
 * records and transform levels cross this boundary and the GPU performs
 * dequantisation, the inverse transform, intra prediction (a CTU wavefront),
 * reconstruction, deblocking, SAO and ALF. Motion-compensation interpolation
 * and encoder candidate-cost evaluation are exposed as batched kernels.
 *
 * Conventions
 *  - Plain C types only; all sizes in samples unless stated otherwise.
 *  - Functions named *_dev take device pointers and run asynchronously on the
 *    context's stream; all others take host pointers and return once their
 *    results are in host memory.
 *  - Every function returns a vvcg_status. A failed call leaves caller output
 *    buffers untouched; vvcg_last_error() gives a one-line reason.
 *  - A context is bound to one CUDA device and one stream. It is not
 *    re-entrant: one thread at a time may use it. Separate contexts are
 *    independent.
 *  - There is no CPU fallback inside the library: without a usable CUDA
 *    device every call returns VVCG_UNAVAILABLE.
 *  - Results are bit-identical to the reference CPU code for every input
 *    the reference accepts.
 */
#ifndef VVCG_H
#define VVCG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VVCG_ABI_VERSION 1

/* Status codes. They map one-to-one onto the reference's AcceleratorError
 * (crates/rustmpeg-video/src/accelerator.rs:17-31): UNAVAILABLE ->
 * Unavailable, INVALID_INPUT -> InvalidInput, LIMIT_EXCEEDED ->
 * LimitExceeded, EXECUTION / TIMEOUT / MISMATCH -> Execution. */
typedef enum vvcg_status {
  VVCG_OK = 0,
  VVCG_INVALID_INPUT = 1,
  VVCG_LIMIT_EXCEEDED = 2,
  VVCG_UNAVAILABLE = 3,
  VVCG_EXECUTION = 4,
  VVCG_TIMEOUT = 5,  /* a bounded device-side wait gave up */
  VVCG_MISMATCH = 6  /* a device self-check disagreed */
} vvcg_status;

typedef struct vvcg_ctx vvcg_ctx;

typedef struct vvcg_config {
  int32_t device;              /* CUDA device ordinal */
  uint32_t flags;              /* reserved, 0 */
  uint64_t reserve_bytes;      /* device arena to reserve up front (0 = grow on demand) */
  uint32_t spin_limit;         /* wavefront wait limit in polls (0 = library default) */
  uint32_t reserved;
} vvcg_config;

/* Chroma format (ChromaFormatIdc, crates/rustmpeg-video/src/vvc/predict.rs:2806). */
enum { VVCG_CHROMA_400 = 0, VVCG_CHROMA_420 = 1, VVCG_CHROMA_422 = 2, VVCG_CHROMA_444 = 3 };

/* Picture tool switches that change reconstruction (SliceCodingOptions,
 * crates/rustmpeg-video/src/vvc/slice.rs:1472-1510). */
enum {
  VVCG_TOOL_DEP_QUANT = 1u << 0, /* dependent quantisation (dep_quant) */
  VVCG_TOOL_DEBLOCK = 1u << 1,   /* enable_deblock */
  VVCG_TOOL_SAO = 1u << 2,       /* enable_sao */
  VVCG_TOOL_ALF = 1u << 3,       /* enable_alf */
  /* encoder only (vvcg_encode_batch): */
  VVCG_TOOL_ENC_FULL_INTRA = 1u << 4, /* all 7 searched luma modes, not only Planar / DC */
  VVCG_TOOL_ENC_CCLM = 1u << 5,       /* chroma mode by SAD among DM and the 3 CCLM modes */
  /* decoder: the picture's level_off values index sparse TBs (see vvcg_cu_rec) */
  VVCG_TOOL_SPARSE_LEVELS = 1u << 6,
  /* decoder: the CU records carry per-TB transform choices in tu_tools (the
   * strict 8-bit decoder's transform skip, mts_idx and lfnst_idx,
   * slice.rs:458-627) */
  VVCG_TOOL_TU_TOOLS = 1u << 7
};

/* vvcg_cu_rec.tu_tools of a picture with VVCG_TOOL_TU_TOOLS (ignored
 * otherwise): transform skip per component, and the luma TB's explicit MTS
 * index (mts_types, slice.rs:647-656) or LFNST index (LFNST set from the
 * CU's luma mode). mts_idx and lfnst_idx are not both nonzero, and neither
 * is with luma transform skip. */
enum {
  VVCG_CU_TS_Y = 1u << 0,
  VVCG_CU_TS_CB = 1u << 1,
  VVCG_CU_TS_CR = 1u << 2,
  VVCG_CU_MTS_SHIFT = 3,   /* bits 3..5: mts_idx 0..4 */
  VVCG_CU_LFNST_SHIFT = 6  /* bits 6..7: lfnst_idx 0..2 */
};

/* One picture of the 8..12-bit frame path: the inputs of
 * slice::decode_vvc_frame_picture_with_chroma_qp (slice.rs:4659) once CABAC
 * has been parsed. The coding units form a uniform grid of tb x tb luma
 * blocks, tb = min(CTU size, 32) (slice.rs:4675), coded CTU by CTU in raster
 * order with quadtree z-order inside a CTU (slice.rs:164-187). */
typedef struct vvcg_pic_desc {
  uint32_t width;            /* coded width, a multiple of the CTU size */
  uint32_t height;           /* coded height, a multiple of the CTU size */
  uint32_t visible_width;    /* cropped output width (<= width) */
  uint32_t visible_height;   /* cropped output height (<= height) */
  uint8_t bit_depth;         /* 8..12 */
  uint8_t chroma_format;     /* VVCG_CHROMA_* */
  uint8_t ctu_log2;          /* 5..7 */
  uint8_t slice_qp;          /* SliceQpY, 0..63 */
  uint8_t chroma_qp_scaled;  /* Qp'C including QpBdOffset (slice.rs:4662) */
  uint8_t tools;             /* VVCG_TOOL_* */
  int16_t alf_aps;           /* index into vvcg_batch.aps, -1 = fixed filters */
  uint32_t cu_offset;        /* first record of this picture in vvcg_batch.cus */
  uint32_t ctu_offset;       /* first record of this picture in vvcg_batch.ctus */
} vvcg_pic_desc;

/* One coding unit. Records of a picture are stored in raster order of its
 * tb grid (index gy * (width / tb) + gx), not in coding order. */
typedef struct vvcg_cu_rec {
  uint8_t luma_mode;    /* IntraPredModeY, 0..66 */
  uint8_t chroma_mode;  /* 0..66, or 81 / 82 / 83 for CCLM LM / LM-L / LM-T */
  uint8_t cbf;          /* bit0 Y, bit1 Cb, bit2 Cr */
  uint8_t tu_tools;     /* VVCG_TU_* with VVCG_TOOL_TU_TOOLS, else 0 */
  int32_t level_off[3]; /* start of each TB's raster-order levels in the level
                           pool (int16), -1 when the TB has no levels. With
                           VVCG_TOOL_SPARSE_LEVELS the TB is sparse: at
                           level_off (even) the count n of its coded levels,
                           one unused int16, then n pairs (raster index,
                           level) with strictly rising indices; an index
                           outside the TB or out of order fails the batch
                           with VVCG_INVALID_INPUT */
} vvcg_cu_rec;

/* SAO parameters of one colour component of one CTU (filter.rs:1229 SaoType). */
typedef struct vvcg_sao {
  uint8_t type;          /* 0 off, 1 band offset, 2 edge offset */
  uint8_t band_or_class; /* band position 0..31, or edge class 0..3 */
  int8_t offsets[4];
} vvcg_sao;

/* Per-CTU filter switches, in raster CTU order per picture. */
typedef struct vvcg_ctu_filter {
  vvcg_sao sao[3];
  uint8_t alf_luma;      /* alf_ctb_flag of the luma CTB */
  uint8_t reserved;
} vvcg_ctu_filter;

/* Luma ALF parameters (hls.rs:2699 VvcAlfAps, luma part). */
typedef struct vvcg_alf_aps {
  uint8_t num_luma_filters;    /* 0 = fixed filter of each class */
  uint8_t luma_clip;           /* alf_luma_clip_flag */
  uint8_t coeff_delta_idx[25]; /* class -> filter */
  uint8_t reserved;
  int16_t coeff[25][12];
  uint8_t clip_idx[25][12];
} vvcg_alf_aps;

/* A batch of independent pictures (frames of one or many streams). */
typedef struct vvcg_batch {
  const vvcg_pic_desc* pics;
  uint32_t num_pics;
  uint32_t num_cus;
  const vvcg_cu_rec* cus;
  const int16_t* levels;
  uint64_t num_levels;
  const vvcg_ctu_filter* ctus;
  uint32_t num_ctus;
  uint32_t num_aps;
  const vvcg_alf_aps* aps;
} vvcg_batch;

/* Destination of one output plane; stride in samples. */
typedef struct vvcg_plane_out {
  uint16_t* data;
  uint32_t stride;
  uint32_t reserved;
} vvcg_plane_out;

/* Stages of vvcg_batch_run. */
enum {
  VVCG_STAGE_RECON = 1u << 0,   /* dequant + inverse transform + intra + add/clip */
  VVCG_STAGE_DEBLOCK = 1u << 1, /* pictures with VVCG_TOOL_DEBLOCK */
  VVCG_STAGE_SAO = 1u << 2,     /* pictures with VVCG_TOOL_SAO; where luma ALF also applies, the
                                   luma plane's SAO and ALF run fused in this stage */
  VVCG_STAGE_ALF = 1u << 3,     /* luma ALF of pictures with VVCG_TOOL_ALF, an enabled CTU and no SAO */
  VVCG_STAGE_ALL = 0xFu
};

/* ---- context ------------------------------------------------------------ */

/* Replaces: constructing the reference's accelerator provider
 * (accelerator.rs:155-200 trait objects). */
vvcg_status vvcg_ctx_create(const vvcg_config* cfg, vvcg_ctx** out);
void vvcg_ctx_destroy(vvcg_ctx* ctx);
const char* vvcg_last_error(const vvcg_ctx* ctx);
/* Use a caller-owned cudaStream_t (NULL = the context's own stream). */
vvcg_status vvcg_set_stream(vvcg_ctx* ctx, void* cuda_stream);
/* Number of this library's kernels launched since the context was created. */
uint64_t vvcg_kernel_launches(const vvcg_ctx* ctx);

/* ---- picture batches (frame path) ---------------------------------------- */

/* Whole call with host buffers: upload, reconstruct, filter, download.
 * `out` holds 3 planes (Y, Cb, Cr) per picture, num_pics * 3 entries; the
 * visible area of each plane is written.
 * Replaces: the per-CU reconstruction loop and the picture-level loop
 * filters of slice::decode_vvc_frame_picture_with_chroma_qp
 * (slice.rs:4834-4988 and :4990-5072). */
vvcg_status vvcg_decode_batch(vvcg_ctx* ctx, const vvcg_batch* batch, const vvcg_plane_out* out);

/* vvcg_decode_batch without the final wait: uploads, kernels and the copies
 * into `out` are queued on the context's stream and the call returns;
 * vvcg_batch_sync waits for them and reports the batch's status. The next
 * call on the same context first waits for the previous batch, so a caller
 * that streams batches alternates two contexts: one batch's download then
 * overlaps the next batch's upload and kernels. Host buffers (records,
 * levels, `out`) must be pinned for the copies to be asynchronous and must
 * stay valid until vvcg_batch_sync returns. */
vvcg_status vvcg_decode_batch_async(vvcg_ctx* ctx, const vvcg_batch* batch, const vvcg_plane_out* out);

/* vvcg_decode_batch with the host copies overlapped: the batch is split into
 * chunks of chunk_pictures pictures, processed round robin on num_lanes
 * internal sub-contexts (own streams and device arenas; 0 = 3), so that one
 * chunk's upload and another's download run while a third is reconstructed.
 * Host buffers should be pinned for the copies to overlap. The caller's
 * buffers must stay valid until the call returns; results equal
 * vvcg_decode_batch's. chunk_pictures 0 or >= num_pics is vvcg_decode_batch. */
vvcg_status vvcg_decode_batch_pipelined(vvcg_ctx* ctx, const vvcg_batch* batch, const vvcg_plane_out* out,
                                        uint32_t chunk_pictures, uint32_t num_lanes);

/* Split form of vvcg_decode_batch, for callers that keep pictures on the GPU:
 * prepare (validate, schedule, size the device arena), upload (records and
 * levels to the device), run (kernels only, asynchronous on the stream),
 * sync (wait and read the device status word), download (visible planes). */
vvcg_status vvcg_batch_prepare(vvcg_ctx* ctx, const vvcg_batch* batch);
vvcg_status vvcg_batch_upload(vvcg_ctx* ctx, const vvcg_batch* batch);
vvcg_status vvcg_batch_run(vvcg_ctx* ctx, uint32_t stage_mask);
/* vvcg_batch_run replayed from a CUDA graph: the first call for a prepared
 * batch and stage mask captures the stages into a graph (the progress words
 * of the wavefront are cleared inside it), later calls launch the graph.
 * vvcg_batch_prepare drops the graph. Same results as vvcg_batch_run. */
vvcg_status vvcg_batch_run_graph(vvcg_ctx* ctx, uint32_t stage_mask);
vvcg_status vvcg_batch_sync(vvcg_ctx* ctx);
vvcg_status vvcg_batch_download(vvcg_ctx* ctx, const vvcg_plane_out* out);
/* Device address and stride (samples) of one reconstructed plane. */
vvcg_status vvcg_batch_plane(vvcg_ctx* ctx, uint32_t pic, uint32_t comp, void** dev_ptr,
                             uint32_t* stride);

/* ---- motion compensation (batched blocks, device pointers) --------------- */

enum {
  VVCG_MC_BI = 1u << 0,      /* emit 14-bit bi-prediction intermediates */
  VVCG_MC_AFFINE = 1u << 1,  /* 6-tap affine luma filters */
  VVCG_MC_ALT_HPEL = 1u << 2 /* alternative half-pel luma filter */
};

typedef struct vvcg_mc_block {
  int32_t x, y;        /* block position in the reference plane's sample grid */
  uint16_t w, h;       /* block size, 1..128 */
  int32_t mv_x, mv_y;  /* motion vector in 1/16 luma sample units */
  uint32_t flags;      /* VVCG_MC_* */
  uint32_t reserved;
  uint64_t out_offset; /* first int32 output element; outputs are w*h, raster */
} vvcg_mc_block;

/* Batched luma interpolation. Replaces: inter::interpolate_luma_block_16
 * (crates/rustmpeg-video/src/vvc/inter.rs:2010). Outputs clipped samples
 * (uni-prediction) or 14-bit intermediates (VVCG_MC_BI). */
vvcg_status vvcg_mc_luma_16_dev(vvcg_ctx* ctx, const uint16_t* ref, uint32_t width,
                                uint32_t height, uint32_t stride, uint8_t bit_depth,
                                const vvcg_mc_block* blocks, uint32_t num_blocks, int32_t* out);
/* Batched chroma interpolation (chroma_format 1..3). Replaces:
 * inter::interpolate_chroma_block_format_16 (inter.rs:2543). Block positions
 * are in chroma samples; motion vectors stay in 1/16 luma units. */
vvcg_status vvcg_mc_chroma_16_dev(vvcg_ctx* ctx, const uint16_t* ref, uint32_t width,
                                  uint32_t height, uint32_t stride, uint8_t bit_depth,
                                  uint8_t chroma_format, const vvcg_mc_block* blocks,
                                  uint32_t num_blocks, int32_t* out);
/* 8-bit planes (the strict / multitool 8-bit encoders and decoders):
 * interpolate_luma_block (inter.rs:896-1051) and interpolate_chroma_block_420
 * (inter.rs:1056-1182, 4:2:0, MV in 1/16 luma = 1/32 chroma units). Flags and
 * outputs as in the 16-bit functions; uni-prediction outputs are 0..255. */
vvcg_status vvcg_mc_luma_8_dev(vvcg_ctx* ctx, const uint8_t* ref, uint32_t width, uint32_t height,
                               uint32_t stride, const vvcg_mc_block* blocks, uint32_t num_blocks,
                               int32_t* out);
vvcg_status vvcg_mc_chroma_420_8_dev(vvcg_ctx* ctx, const uint8_t* ref, uint32_t width, uint32_t height,
                                     uint32_t stride, const vvcg_mc_block* blocks, uint32_t num_blocks,
                                     int32_t* out);
/* BCW weighted bi-prediction average. Replaces: inter::weighted_average_bi_16
 * (inter.rs:2676); with bit_depth 8 it is also weighted_average_bi
 * (inter.rs:1189-1201). */
vvcg_status vvcg_mc_bi_average_16_dev(vvcg_ctx* ctx, const int32_t* pred0, const int32_t* pred1,
                                      uint64_t count, uint8_t bcw_idx, uint8_t bit_depth,
                                      uint16_t* out);

/* ---- encoder (frame path) ------------------------------------------------ */

/* Source planes of one picture for vvcg_encode_batch: coded size, host or
 * device memory (the copy direction is inferred). */
typedef struct vvcg_plane_in {
  const uint16_t* data;
  uint32_t stride; /* samples */
  uint32_t reserved;
} vvcg_plane_in;

/* Encodes a batch of pictures: per CU the 7-mode SAD intra decision, the
 * prediction, forward DCT-2, regular or dependent quantisation and the
 * encoder's own reconstruction, in CTU wavefront order, then deblocking when
 * the picture asks for it. Replaces: slice::encode_vvc_frame_picture
 * (crates/rustmpeg-video/src/vvc/slice.rs:4171-4634) without the CABAC
 * writes. pics[i].chroma_qp_scaled is derived from slice_qp here
 * (hls.rs:796 derived_chroma_qp_bd); tools may hold DEP_QUANT, DEBLOCK,
 * ENC_FULL_INTRA and ENC_CCLM. `src` holds 3 planes per picture.
 * Outputs (host or device memory): one record per tb-grid cell (cu_offset is
 * assigned in picture order; level_off indexes `levels`, -1 when the TB has no
 * nonzero level) and the level pool, where each CU owns a slot of
 * tb*tb + 2*tb_cw*tb_ch levels (see vvcg_encode_levels_size). The
 * reconstructed pictures stay in the context: vvcg_batch_plane and
 * vvcg_batch_download read them, and vvcg_batch_run(VVCG_STAGE_RECON) decodes
 * the emitted records again. Synchronous. */
vvcg_status vvcg_encode_batch(vvcg_ctx* ctx, const vvcg_pic_desc* pics, uint32_t num_pics,
                              const vvcg_plane_in* src, vvcg_cu_rec* cus, uint32_t cus_cap,
                              int16_t* levels, uint64_t levels_cap);
/* Records and level-pool entries vvcg_encode_batch writes for these pictures. */
vvcg_status vvcg_encode_sizes(const vvcg_pic_desc* pics, uint32_t num_pics, uint32_t* num_cus,
                              uint64_t* num_levels);

/* ---- transform units (function level, batched, device buffers) ---------- */

enum {
  VVCG_TU_DEP_QUANT = 1u << 0,      /* dependent quantisation (4-state) */
  VVCG_TU_TRANSFORM_SKIP = 1u << 1, /* transform skip: per-sample (de)quantisation */
  VVCG_TU_BDPCM_HOR = 1u << 2,      /* inverse only: BDPCM accumulation along rows */
  VVCG_TU_BDPCM_VER = 1u << 3,      /* inverse only: BDPCM accumulation along columns */
  VVCG_TU_IMPLICIT_MTS = 1u << 4,   /* DST-7 for a dimension in 4..16 when mts_idx and
                                       lfnst_idx are 0 (luma, no MIP) */
  VVCG_TU_INTER = 1u << 5           /* forward only: inter rounding offset (85, not 171) */
};

typedef struct vvcg_tu_rec {
  uint8_t log2_w, log2_h; /* 0..6 each, w * h >= 2 */
  uint8_t bit_depth;      /* 8..12 */
  uint8_t qp;             /* Qp' = QP + QpBdOffset, 0..87 */
  uint8_t flags;          /* VVCG_TU_* */
  uint8_t mts_idx;        /* 0, or 1..4: (DST7,DST7) (DCT8,DST7) (DST7,DCT8) (DCT8,DCT8) */
  uint8_t lfnst_idx;      /* 0..2 (ignored by the inverse when mts_idx != 0) */
  uint8_t lfnst_mode;     /* LFNST intra mode index 0..94 (lfnst::get_lfnst_intra_mode of the
                             wide-angle mode) */
  uint32_t in_off;        /* first int16 input element (raster, w*h) */
  uint32_t out_off;       /* first int16 output element (raster, w*h) */
} vvcg_tu_rec;            /* 16 bytes */

/* Levels -> residual of each transform unit: transform-skip or regular /
 * dependent dequantisation, inverse LFNST, inverse DCT-2 / DST-7 / DCT-8 with
 * the zero-out rules, then BDPCM. Replaces: residual_of + inverse_residual
 * (crates/rustmpeg-video/src/vvc/decode_general.rs:4100-4199) and the BDPCM
 * step of reconstruct_tu (decode_general.rs:4055-4060, predict.rs:4224). `recs`
 * is host memory; `in`/`out` are device buffers of in_count / out_count int16.
 * Asynchronous on the context's stream. */
vvcg_status vvcg_tu_inverse_batch(vvcg_ctx* ctx, const vvcg_tu_rec* recs, uint32_t num_recs,
                                  const int16_t* in, uint64_t in_count, int16_t* out,
                                  uint64_t out_count);
/* Residual -> levels: forward transform, forward LFNST and regular / dependent
 * / transform-skip quantisation. Replaces: the level side of plan_primary and
 * plan_transform_skip (slice.rs:690-760) over dct::forward_transform_rect_bd
 * (dct.rs:865), lfnst::forward_lfnst_rect (lfnst.rs:131), quantize_rect_bd
 * (dct.rs:1113), quantize_dep_quant_bd (dct.rs:1252), quantize_ts
 * (transform.rs:214). */
vvcg_status vvcg_tu_forward_batch(vvcg_ctx* ctx, const vvcg_tu_rec* recs, uint32_t num_recs,
                                  const int16_t* in, uint64_t in_count, int16_t* out,
                                  uint64_t out_count);
/* Block-size-binning autotuner of the two functions above (no counterpart in
 * the reference, which transforms one unit at a time). The units are grouped
 * by size (at most 256, 1024 and 4096 coefficients); for each non-empty group
 * every CTA width the library has for it (2, 4 or 8 warps; 1, 2 or 4 for the
 * largest group; one unit per warp) is timed on this batch, and the fastest
 * stays in the context for later vvcg_tu_inverse_batch (forward = 0) or
 * vvcg_tu_forward_batch (forward = 1) calls. warps[g] receives the chosen
 * width of group g, 0 for an empty group (whose choice is kept). Arguments
 * and checks as in those functions; out receives the batch's results, which
 * never depend on the width. Synchronous: returns after the timings. */
vvcg_status vvcg_tu_autotune(vvcg_ctx* ctx, const vvcg_tu_rec* recs, uint32_t num_recs, const int16_t* in,
                             uint64_t in_count, int16_t* out, uint64_t out_count, uint32_t forward,
                             uint32_t warps[3]);

/* ---- encoder candidate cost: luma transform search ----------------------- */

enum {
  VVCG_TXS_TRANSFORM_SKIP = 1u << 0, /* code the block with transform skip only (QP 4 path) */
  VVCG_TXS_LFNST = 1u << 1           /* also try LFNST 1 and 2 (chroma_can_lfnst) */
};

typedef struct vvcg_tx_search_req {
  uint8_t log2_size; /* 2..5: square blocks 4x4 .. 32x32 */
  uint8_t qp;        /* QP of the 8-bit strict encoder, 0..63 */
  uint8_t mode;      /* the block's intra mode: 0 Planar, 1 DC, 2..66 (LFNST set) */
  uint8_t flags;     /* VVCG_TXS_* */
  uint32_t in_off;   /* first of the n*n prediction / source samples (int16 raster) */
  uint32_t out_off;  /* first of the n*n output levels / samples (int16 raster) */
  uint32_t reserved;
} vvcg_tx_search_req; /* 16 bytes */

typedef struct vvcg_tx_search_res {
  uint64_t sse;           /* reconstruction SSE of the chosen candidate */
  uint8_t mts_idx;        /* 0..4 */
  uint8_t lfnst_idx;      /* 0..2 */
  uint8_t transform_skip; /* 1 when coded with transform skip */
  uint8_t cbf;            /* any nonzero level */
  uint32_t reserved;
} vvcg_tx_search_res; /* 16 bytes */

/* Transform choice of each 8-bit luma block by reconstruction SSE: DCT-2,
 * then MTS 1..4, then (VVCG_TXS_LFNST) LFNST 1..2, each replacing the best
 * only when it can be signalled and its SSE is strictly lower; writes the
 * winner's levels and reconstructed samples. Replaces: slice::encode_luma
 * after the prediction (crates/rustmpeg-video/src/vvc/slice.rs:810-874, with
 * plan_primary :699, plan_transform_skip :671, mts_candidate_ok /
 * lfnst_candidate_ok :877-896, block_sse :908). `reqs` is host memory; pred,
 * src, levels, samples (int16, counts in_count / out_count) and `res`
 * (num_reqs entries) are device memory. Asynchronous on the stream. */
vvcg_status vvcg_luma_tx_search_dev(vvcg_ctx* ctx, const vvcg_tx_search_req* reqs, uint32_t num_reqs,
                                    const int16_t* pred, const int16_t* src, uint64_t in_count,
                                    int16_t* levels, int16_t* samples, uint64_t out_count,
                                    vvcg_tx_search_res* res);

/* ---- LMCS and joint chroma residuals (general decoding path) ------------- */

/* LMCS APS (hls.rs:2723 VvcLmcsAps). */
typedef struct vvcg_lmcs_aps {
  int16_t bin_cw_delta[16];          /* LmcsDeltaCW[i] */
  uint8_t min_bin_idx;               /* lmcs_min_bin_idx, 0..15 */
  uint8_t max_bin_idx;               /* 15 - lmcs_delta_max_bin_idx */
  int8_t chroma_res_scaling_offset;  /* LmcsDeltaCrs, -7..7 */
  uint8_t reserved;
} vvcg_lmcs_aps; /* 36 bytes */

/* Reshaper tables of one APS at one bit depth (LmcsReshaper16, filter.rs:2604). */
typedef struct vvcg_lmcs_tables {
  uint8_t bit_depth, min_bin_idx, max_bin_idx, reserved;
  int32_t reshape_pivot[17];
  int32_t chroma_adj_lut[16];
  uint16_t fwd_lut[4096]; /* 1 << bit_depth entries used */
  uint16_t inv_lut[4096];
} vvcg_lmcs_tables;

/* Builds the reshaper tables on the host. Replaces: LmcsReshaper16::from_aps
 * (crates/rustmpeg-video/src/vvc/filter.rs:2628-2705). */
vvcg_status vvcg_lmcs_build(const vvcg_lmcs_aps* aps, uint8_t bit_depth, vvcg_lmcs_tables* out);
/* Maps a 16-bit luma plane through the inverse (inverse != 0) or forward LUT in
 * place (device plane). Replaces: apply_inverse_plane_16 / apply_forward_plane_16
 * (filter.rs:2708-2722). */
vvcg_status vvcg_lmcs_map_plane_16_dev(vvcg_ctx* ctx, const vvcg_lmcs_tables* tables, int inverse,
                                       uint16_t* plane, uint32_t stride, uint32_t width, uint32_t height);
/* Chroma residual scale factor (cScale) of the VPDU containing each luma
 * position pos_xy[2i], pos_xy[2i+1] (device), from the average reconstructed
 * luma left of and above the VPDU. Replaces: chroma_adj_luma
 * (decode_general.rs:4803-4835) + chroma_scale_for_luma (filter.rs:2725). */
vvcg_status vvcg_lmcs_chroma_scales_dev(vvcg_ctx* ctx, const vvcg_lmcs_tables* tables, const uint16_t* luma,
                                        uint32_t stride, uint32_t pic_width, uint32_t pic_height,
                                        uint32_t ctu_size, const uint32_t* pos_xy, uint32_t num,
                                        int32_t* scale_out);

enum {
  VVCG_CRES_SCALE = 1u << 0, /* apply the LMCS chroma residual scaling with `scale` */
  VVCG_CRES_SINGLE = 1u << 1 /* one component only (cb_off); no joint combination */
};

typedef struct vvcg_cres_rec {
  uint8_t log2_w, log2_h; /* chroma TB size */
  uint8_t bit_depth;      /* 8..12 */
  int8_t joint;           /* JCCR mode with the picture's sign: -3..3, 0 = none */
  uint32_t flags;         /* VVCG_CRES_* */
  int32_t scale;          /* cScale (vvcg_lmcs_chroma_scales_dev) */
  uint32_t cb_off, cr_off;/* int16 residual blocks (raster) in the buffer, in place */
} vvcg_cres_rec; /* 20 bytes */

/* Joint Cb-Cr residual derivation and LMCS chroma residual scaling of
 * residual pairs in place. Replaces: the residual part of
 * reconstruct_joint_cbcr (decode_general.rs:3932-3966) and of reconstruct_tu
 * (:4075-4080) with LmcsReshaper16::scale_chroma_residual (filter.rs:2740).
 * `recs` host memory, `res` device memory of `count` int16. */
vvcg_status vvcg_chroma_residuals_dev(vvcg_ctx* ctx, const vvcg_cres_rec* recs, uint32_t num, int16_t* res,
                                      uint64_t count);

/* ---- matrix-based intra prediction (function level, batched) ------------- */

#define VVCG_MIP_SEARCH 0xFFu /* vvcg_mip_req.mode: search every (transposed, mode) */

typedef struct vvcg_mip_req {
  uint8_t log2_w, log2_h; /* 2..6: blocks 4x4 .. 64x64 */
  uint8_t bit_depth;      /* 8..12 */
  uint8_t mode;           /* MIP mode (taken modulo the size class's mode count), or VVCG_MIP_SEARCH */
  uint8_t transposed;     /* intra_mip_transposed_flag (ignored when searching) */
  uint8_t reserved[3];
  uint32_t ref_off;       /* first of the w above then h left reference samples (int16) in `refs` */
  uint32_t out_off;       /* first of the w*h prediction samples (int16, raster) in `pred`; the
                             source block of a search sits at the same offset in `src` */
} vvcg_mip_req; /* 16 bytes */

typedef struct vvcg_mip_res {
  uint64_t sad;        /* SAD of the chosen candidate against the source */
  uint8_t mode, transposed;
  uint8_t reserved[6];
} vvcg_mip_res; /* 16 bytes */

/* MIP predictions of a batch of blocks from their reference samples; with
 * VVCG_MIP_SEARCH, the (transposed, mode) of least SAD against `src` (a later
 * candidate wins only when strictly lower; transposed 0 first), its SAD in
 * `res` and its prediction in `pred`. Replaces: predict_mip_16 /
 * predict_mip_bd (crates/rustmpeg-video/src/vvc/predict.rs:4109, :2461-2611)
 * and choose_best_mip_mode_16 (predict.rs:4166-4199). `reqs` host memory;
 * refs, src, pred (int16, counts ref_count / count) and res (device, one per
 * request, needed only when searching) device memory. */
vvcg_status vvcg_mip_predict_dev(vvcg_ctx* ctx, const vvcg_mip_req* reqs, uint32_t num_reqs, const int16_t* refs,
                                 uint64_t ref_count, const int16_t* src, int16_t* pred, uint64_t count,
                                 vvcg_mip_res* res);

/* ---- general-decoder ALF (luma with virtual boundaries, chroma, CCALF) --- */

enum { VVCG_ALF_OFF = 0, VVCG_ALF_FIXED = 1, VVCG_ALF_APS = 2 };

/* One CTU's ALF switches (the general decoder's alf_luma / alf_cb / alf_cr /
 * ccalf_cb / ccalf_cr per CTU). */
typedef struct vvcg_alf_ctu {
  uint8_t luma_mode;     /* VVCG_ALF_OFF / _FIXED / _APS */
  uint8_t luma_set;      /* fixed filter set 0..15 (VVCG_ALF_FIXED) */
  uint8_t cb_alt, cr_alt;/* chroma filter alternative, 0xFF = off */
  uint8_t cc_cb, cc_cr;  /* CCALF filter index + 1, 0 = off */
  uint8_t reserved[2];
} vvcg_alf_ctu; /* 8 bytes */

/* ALF parameters of a picture: the luma, chroma and CCALF parts of the APSs
 * its slice refers to (hls.rs:2699 VvcAlfAps). */
typedef struct vvcg_alf_params {
  uint8_t num_luma_filters, luma_clip, num_chroma_filters, chroma_clip;
  uint8_t num_cc_cb, num_cc_cr, reserved[2];
  uint8_t coeff_delta_idx[25];
  uint8_t reserved2[3];
  int16_t luma_coeff[25][12];
  uint8_t luma_clip_idx[25][12];
  int16_t chroma_coeff[8][6];
  uint8_t chroma_clip_idx[8][6];
  int16_t cc_cb[4][7];
  int16_t cc_cr[4][7];
} vvcg_alf_params;

/* ALF of a 4:2:0 picture as the general decoder applies it: per CTU, the luma
 * 7x7 filter (fixed set or APS) with the CTU-row virtual boundary 4 rows above
 * each CTU bottom, the chroma 5x5 filter (virtual boundary 2 rows above), and
 * CCALF from the unfiltered luma added to the filtered chroma. src / dst are
 * device planes (Y at width x height, Cb / Cr at half size, the given
 * strides); CTUs without a switch copy src. ctus (one per CTU of the visible
 * picture, ctu_cols per row) and params are host memory; a CTU in
 * VVCG_ALF_APS mode needs num_luma_filters >= 1. Replaces:
 * apply_alf (decode_general.rs:5225-5345) with alf_luma_block (:5411),
 * alf_chroma_block (:5568), ccalf_block (:5348) and
 * derive_alf_class_4x4_vb_16 (filter.rs:1558). */
vvcg_status vvcg_alf_general_dev(vvcg_ctx* ctx, const uint16_t* const src[3], uint16_t* const dst[3],
                                 const uint32_t stride[3], uint32_t width, uint32_t height, uint32_t vis_width,
                                 uint32_t vis_height, uint8_t bit_depth, uint32_t ctu_size, uint32_t ctu_cols,
                                 const vvcg_alf_ctu* ctus, const vvcg_alf_params* params);

/* ---- 8-bit luma intra mode search ---------------------------------------- */

enum { VVCG_ISR_MPM_ONLY = 1, VVCG_ISR_MRL = 2 };

/* One luma block of an 8-bit picture to choose an intra mode for. */
typedef struct vvcg_intra_search_req {
  uint32_t x, y;           /* top-left sample; the block lies inside the plane */
  uint8_t log2_w, log2_h;  /* 2..6 */
  uint8_t flags;           /* VVCG_ISR_MPM_ONLY: the 6 MPMs instead of all 67 modes;
                              VVCG_ISR_MRL: then reference lines 1 and 2 for mpm[1..5] */
  uint8_t log2_ctu;        /* 4..7: CTU size (a block on a CTU's first row keeps line 0) */
  uint8_t mpm[6];          /* most probable modes, 0..66 */
  uint8_t reserved[2];
} vvcg_intra_search_req; /* 20 bytes */

typedef struct vvcg_intra_search_res {
  uint64_t sad;            /* sum of |source - prediction| of the winner */
  uint8_t mode, mrl_idx;   /* winning mode 0..66 and reference line */
  uint8_t reserved[6];
} vvcg_intra_search_res; /* 16 bytes */

/* Luma intra mode decision of the 8-bit multi-tool encoder for a batch of
 * blocks: Planar, DC and the 65 angular modes (or the MPMs) predicted from
 * recon, compared with src by SAD, the first lowest winning (Planar on a
 * tie); with VVCG_ISR_MRL the lines 1 and 2 predictions of mpm[1..5] then
 * replace it when strictly lower. recon / src are device 8-bit planes of
 * width x height with the given strides (in bytes), reqs host memory, res
 * device memory (one per request). Replaces: choose_luma_intra_pred_mode
 * (predict.rs:2737-2801) with predict_block_full (:2655-2699) and the MRL
 * candidate loop of encode_picture_multitool (slice.rs:2698-2731). */
vvcg_status vvcg_luma_intra_search_8_dev(vvcg_ctx* ctx, const uint8_t* recon, uint64_t recon_stride,
                                         const uint8_t* src, uint64_t src_stride, uint32_t width, uint32_t height,
                                         const vvcg_intra_search_req* reqs, uint32_t num_reqs,
                                         vvcg_intra_search_res* res);

/* ---- CTU full search of the GPU encoder ------------------------------------ */

/* Split types of a 32x32 CTU: none, quad (4 x 16x16), binary with a
 * horizontal / vertical split line (2 x 32x16 / 2 x 16x32), ternary with
 * horizontal / vertical lines (32x8 + 32x16 + 32x8 / 8x32 + 16x32 + 8x32). */
enum {
  VVCG_SPLIT_NONE = 0, VVCG_SPLIT_QT = 1, VVCG_SPLIT_BT_H = 2, VVCG_SPLIT_BT_V = 3,
  VVCG_SPLIT_TT_H = 4, VVCG_SPLIT_TT_V = 5
};

/* ---- partition hook of the reference encoders -------------------------------- */

typedef struct vvcg_split_req {
  uint32_t x, y;    /* top-left luma sample of the region (it may reach past the plane) */
  uint16_t w, h;    /* region size, 1..4096 each */
  uint16_t min_cb;  /* minimum coding-block size: w or h <= max(min_cb, 8) means no split */
  uint8_t qp;       /* slice QP, 0..63 */
  uint8_t reserved;
} vvcg_split_req;   /* 16 bytes */

/* Quadrant-mean split decision of each region: res[i] (device) becomes
 * VVCG_SPLIT_NONE, _QT, _BT_H or _BT_V. Replaces choose_qt_mtt_partition_rdo_16
 * and choose_qt_mtt_partition_rdo (crates/rustmpeg-video/src/vvc/slice.rs:
 * 4111-4167), hooks that no encoder of the reference calls: samples are
 * rounded to 8 bits as Plane16::to_plane_8bit does (predict.rs:2914-2926); a
 * quadrant's mean is the sum of its samples inside the plane over the full
 * quadrant area; mean differences across the two midlines against
 * max(qp, 4) / 2 + 8 decide. plane: device luma, bit_depth 8..12 in uint16
 * (8-bit samples as they are); reqs: host. Asynchronous on the context's
 * stream. */
vvcg_status vvcg_qt_mtt_split_dev(vvcg_ctx* ctx, const uint16_t* plane, uint64_t stride, uint32_t width,
                                  uint32_t height, uint8_t bit_depth, const vvcg_split_req* reqs,
                                  uint32_t num_reqs, uint8_t* res);

/* ---- motion-estimation hook of the reference encoders ------------------------ */

typedef struct vvcg_mv_cand {  /* InterMergeCand (crates/rustmpeg-video/src/vvc/inter.rs:274) */
  int32_t mv[2][2];            /* per list L0 / L1: (horizontal, vertical) in 1/16 luma samples */
  int8_t ref_idx[2];           /* per list: reference index, < 0 = list unused */
  uint8_t inter_dir;           /* bit 0: L0, bit 1: L1 */
  uint8_t bcw_idx;             /* BCW weight index (values above 4 act as 4; 2 = equal weights) */
  uint8_t alt_hpel;            /* alternative half-sample luma filter */
  uint8_t reserved[3];
} vvcg_mv_cand;                /* 24 bytes */

typedef struct vvcg_me_req {
  uint32_t x, y;               /* top-left luma sample; the block lies inside the plane */
  uint16_t w, h;               /* block size, 1..128 each */
  uint32_t cand_off;           /* first merge candidate of this block in the candidate array */
  uint16_t num_cands;          /* merge list length (may be 0) */
  uint16_t search_range;       /* diamond iterations at most (0 acts as 1) */
  int32_t amvp[2];             /* the L0 AMVP predictor, 1/16 luma samples */
} vvcg_me_req;                 /* 28 bytes */

typedef struct vvcg_me_res {
  uint64_t sad;                /* luma SAD of the choice; UINT64_MAX when nothing was evaluated */
  vvcg_mv_cand cand;           /* the chosen merge candidate, or L0 uni-prediction at the searched MV */
  uint16_t merge_idx;          /* merge list index when is_merge */
  uint8_t is_merge;
  uint8_t reserved[5];
} vvcg_me_res;                 /* 40 bytes */

/* Motion estimation of each block on 8-bit luma planes. Replaces
 * estimate_inter_block (crates/rustmpeg-video/src/vvc/inter.rs:1866-2003), a
 * hook that no encoder of the reference calls: the SAD of every merge
 * candidate's luma prediction (predict_inter_pu, inter.rs:1733-1847, with BDOF
 * and DMVR off: 8-tap interpolation, BCW average for bi-prediction, 128 without
 * a usable list), then, when L0 has a reference, an integer diamond search on
 * L0 reference 0 from the AMVP predictor and a quarter-sample refinement; the
 * lowest SAD wins, the merge candidate on a tie. src and the references are
 * device planes of one size and stride; ref_l0 / ref_l1 are host arrays of at
 * most 16 device pointers each; cands and reqs are host arrays; res is device
 * memory. Asynchronous on the context's stream. */
vvcg_status vvcg_inter_search_8_dev(vvcg_ctx* ctx, const uint8_t* src, uint64_t stride, uint32_t width,
                                    uint32_t height, const uint8_t* const* ref_l0, uint32_t num_l0,
                                    const uint8_t* const* ref_l1, uint32_t num_l1, const vvcg_mv_cand* cands,
                                    uint32_t num_cands, const vvcg_me_req* reqs, uint32_t num_reqs,
                                    vvcg_me_res* res);

typedef struct vvcg_ctu_search_req {
  uint32_t x, y;       /* top-left luma sample of a 32x32 CTU inside the plane */
  uint8_t split_mask;  /* bit s: evaluate split type s (0x3F: all six) */
  uint8_t n_cand;      /* 0: all 67 modes for every block, else cand[0..n_cand) */
  uint8_t cand[6];
} vvcg_ctu_search_req; /* 16 bytes */

typedef struct vvcg_ctu_search_res {
  uint32_t cost;           /* cost of the chosen split */
  uint32_t split_cost[6];  /* per split type, UINT32_MAX where not evaluated */
  uint8_t split;           /* chosen split type */
  uint8_t cu_mode;         /* best mode of the unsplit CU (0xFF when not evaluated) */
  uint8_t modes[4];        /* modes of the chosen split's blocks, 0xFF past its count */
  uint8_t reserved[2];
} vvcg_ctu_search_res; /* 36 bytes */

/* Mode and split decision of 32x32 CTUs of a luma plane (device, 8..12-bit
 * samples in uint16, stride in samples) by full search: for every evaluated
 * split type, each block takes the mode of lowest cost among all 67 (or the
 * candidates) with predictions from the source plane's own samples (the
 * predictors of predict_block_16, predict.rs:3079-3410); cost = sum over 8x8
 * tiles of (sum |Hadamard(source - prediction)| + 2) >> 2 plus
 * (lambda_q8 * bits) >> 8, with 8 header bits per block plus mode bits
 * 2 + i for the i-th default MPM (Planar, DC, 50, 18, 46, 54) and 7 for any
 * other mode, and split bits 1 / 2 / 3 / 3 / 4 / 4 added per split type. The first lowest cost wins, blocks
 * and splits alike. reqs host memory, res device memory. This is the GPU
 * encoder's candidate-cost stage; the reference's encoders evaluate a
 * single 32x32 CU per CTU (slice.rs:2575-2800). */
vvcg_status vvcg_ctu_search_dev(vvcg_ctx* ctx, const uint16_t* src, uint64_t stride, uint32_t width, uint32_t height,
                                uint8_t bit_depth, uint32_t lambda_q8, const vvcg_ctu_search_req* reqs,
                                uint32_t num_reqs, vvcg_ctu_search_res* res);

/* ---- CNN pruner ------------------------------------------------------------- */

/* Number of fp32 parameters of the CNN pruner and their layout: conv1 W
 * [32 out][2 in][9 taps] and b[32]; conv2..4 W [32 out][32 in][9 taps] and
 * b[32]; intra head W [67][32] and b[67]; split head W [6][32] and b[6].
 * Taps are row-major over (dy, dx) in -1..1. */
#define VVCG_CNN_PARAMS 30761
#define VVCG_CNN_OUT 73 /* 67 intra-mode logits, then 6 split logits */

/* Forward pass of the CNN pruner on 32x32 luma blocks of a device plane
 * (8..12-bit samples in uint16, stride in samples) at the (x, y) positions
 * ctu_xy (device, num_blocks pairs), coded at qp (0..63): input samples /
 * (2^bit_depth - 1) rounded to bf16, and a constant plane qp / 63 (bf16);
 * conv 3x3 2->32 + ReLU (fp32, CUDA cores); 3 x conv 3x3
 * 32->32 + ReLU on the tensor cores (bf16 operands, fp32 accumulation in
 * TMEM, bf16 activations); global average; the two linear heads (fp32).
 * logits: device, num_blocks x VVCG_CNN_OUT. gap (num_blocks x 32 fp32) and
 * acts (num_blocks x 4 layers x 1024 pixels x 32 channels, bf16) are
 * optional device outputs for training. status (device, one word) gets bit
 * 0 when a completion wait gave up and bit 1 when a block lay outside the
 * plane (its logits are NaN). This is the GPU encoder's pruning network;
 * the reference has none. */
vvcg_status vvcg_cnn_forward_dev(vvcg_ctx* ctx, const uint16_t* plane, uint64_t stride, uint32_t width,
                                 uint32_t height, uint8_t bit_depth, uint8_t qp, const uint32_t* ctu_xy,
                                 uint32_t num_blocks,
                                 const float* params, float* logits, float* gap, uint16_t* acts, uint32_t* status);

/* One training step of the CNN pruner on num_blocks 32x32 blocks (the batch,
 * all coded at qp) with labels (device, num_blocks x (intra mode 0..66, split type 0..5)):
 * the forward pass, the mean softmax cross-entropy of both heads, the
 * backward pass (input gradients of the 3x3 32->32 layers on the tensor
 * cores, weight gradients on the CUDA cores), written to grads (device,
 * VVCG_CNN_PARAMS fp32) and loss (device, one fp32); then, when lr > 0, an
 * Adam update (beta 0.9 / 0.999, eps 1e-8, bias correction for `step`,
 * counted from 1) of params with the moments adam_m / adam_v (device,
 * VVCG_CNN_PARAMS fp32 each). status as for vvcg_cnn_forward_dev; blocks
 * outside the plane or with a label out of range are skipped and flag bit
 * 1. Asynchronous on the context's stream. */
vvcg_status vvcg_cnn_train_step_dev(vvcg_ctx* ctx, const uint16_t* plane, uint64_t stride, uint32_t width,
                                    uint32_t height, uint8_t bit_depth, uint8_t qp, const uint32_t* ctu_xy,
                                    const uint8_t* labels, uint32_t num_blocks, float* params, float* adam_m,
                                    float* adam_v, uint32_t step, float lr, float* grads, float* loss,
                                    uint32_t* status);
/* vvcg_cnn_train_step_dev with a target distribution for the mode head
 * (soft_modes: device memory, num_blocks x 67 fp32, each row summing to 1):
 * its cross-entropy loss and gradient p - target; the split head keeps the
 * labels' split type. */
vvcg_status vvcg_cnn_train_step_soft_dev(vvcg_ctx* ctx, const uint16_t* plane, uint64_t stride, uint32_t width,
                                         uint32_t height, uint8_t bit_depth, uint8_t qp, const uint32_t* ctu_xy,
                                         const uint8_t* labels, const float* soft_modes, uint32_t num_blocks,
                                         float* params, float* adam_m, float* adam_v, uint32_t step, float lr,
                                         float* grads, float* loss, uint32_t* status);

/* ---- tensor-core self-test ---------------------------------------------------- */

/* One 128 x 32 x 16 bf16 tcgen05 MMA with fp32 accumulation in TMEM:
 * d (128 x 32, row-major fp32) = a (128 x 16, row-major bf16 bits) times the
 * transpose of b (32 x 16, row-major bf16 bits); device pointers. status
 * (device, one word) becomes 1 if the completion wait gave up. Checks the
 * descriptor, TMEM and completion plumbing that the CNN kernels share. */
vvcg_status vvcg_tc_selftest_dev(vvcg_ctx* ctx, const uint16_t* a, const uint16_t* b, float* d, uint32_t* status);

/* The CTU search of vvcg_ctu_search_dev with device-resident positions
 * (ctu_xy: num_ctus (x, y) pairs) and, with logits (device, num_ctus x
 * VVCG_CNN_OUT from vvcg_cnn_forward_dev), pruned by the CNN: the top_modes
 * most probable intra modes are the candidates of every block and the
 * top_splits most probable split types are evaluated; a head whose chosen
 * entries hold less than threshold of its softmax probability mass keeps its
 * full set (threshold 0: never). logits = NULL
 * is the full search. A CTU outside the plane gets cost UINT32_MAX and
 * split 0xFF. All on the context's stream, no host round trip. */
vvcg_status vvcg_ctu_search_pruned_dev(vvcg_ctx* ctx, const uint16_t* src, uint64_t stride, uint32_t width,
                                       uint32_t height, uint8_t bit_depth, uint32_t lambda_q8,
                                       const uint32_t* ctu_xy, uint32_t num_ctus, const float* logits,
                                       uint32_t top_modes, uint32_t top_splits, float threshold,
                                       vvcg_ctu_search_res* res);

/* Fallback rules of vvcg_ctu_search_pruned_rule_dev: a head keeps its full
 * set when its chosen entries hold less than the threshold of its softmax
 * mass (VVCG_PRUNE_MASS, the rule of vvcg_ctu_search_pruned_dev), or when
 * its most probable entry does (VVCG_PRUNE_MAX_PROB: "full-search fallback
 * when max softmax < threshold"). */
enum { VVCG_PRUNE_MASS = 0, VVCG_PRUNE_MAX_PROB = 1 };
vvcg_status vvcg_ctu_search_pruned_rule_dev(vvcg_ctx* ctx, const uint16_t* src, uint64_t stride, uint32_t width,
                                            uint32_t height, uint8_t bit_depth, uint32_t lambda_q8,
                                            const uint32_t* ctu_xy, uint32_t num_ctus, const float* logits,
                                            uint32_t top_modes, uint32_t top_splits, float threshold, uint32_t rule,
                                            vvcg_ctu_search_res* res);

/* The full CTU search of vvcg_ctu_search_pruned_dev (no pruning) that also
 * writes, per CTU, the cost (SATD + lambda * mode bits) of each of the 67
 * luma modes for the unsplit 32x32 coding unit: mode_costs, device memory,
 * num_ctus x 67 uint32. The training targets of the pruner's mode head are
 * built from them (a near-tie between modes costs little to miss). No
 * counterpart in the reference, whose encoder keeps only the best mode. */
vvcg_status vvcg_ctu_search_costs_dev(vvcg_ctx* ctx, const uint16_t* src, uint64_t stride, uint32_t width,
                                      uint32_t height, uint8_t bit_depth, uint32_t lambda_q8, const uint32_t* ctu_xy,
                                      uint32_t num_ctus, vvcg_ctu_search_res* res, uint32_t* mode_costs);

/* ---- general-decoder intra prediction -------------------------------------- */

enum { VVCG_ISP_NONE = 0, VVCG_ISP_HOR = 1, VVCG_ISP_VER = 2 };
enum { VVCG_BDPCM_NONE = 0, VVCG_BDPCM_HOR = 1, VVCG_BDPCM_VER = 2 };

/* One transform block to predict. Luma: Planar / DC / angular with reference
 * line mrl, ISP sub-partitions (references over the CU width / height plus
 * the block's, and the shared 4-wide prediction region of narrow vertical
 * sub-partitions) or BDPCM. Chroma (4:2:0): Planar / DC / angular or CCLM
 * (mode 81 LM, 82 LM-L, 83 LM-T). */
typedef struct vvcg_gen_intra_req {
  uint16_t x, y, w, h;          /* the block in its component's samples */
  uint16_t cu_x, cu_y, cu_w, cu_h; /* its coding unit in luma samples (ISP) */
  uint8_t comp;                 /* 0 Y, 1 Cb, 2 Cr */
  uint8_t mode;                 /* 0..66 (larger luma values act as 66), or 81..83 for chroma */
  uint8_t mrl;                  /* luma reference line 0..2 */
  uint8_t isp;                  /* VVCG_ISP_* (luma) */
  uint8_t bdpcm;                /* VVCG_BDPCM_* (luma) */
  uint8_t reserved[3];
  uint32_t out_off;             /* first of the w x h int16 predictions in the output */
} vvcg_gen_intra_req; /* 28 bytes */

/* The general decoder's state the predictions read: the Y / Cb / Cr planes
 * (device, 16-bit samples, strides in samples, luma width x height = the
 * picture padded to whole CTUs) and its decoded-sample maps (device): one
 * byte per 4x4 luma cell (dec_y, width / 4 x height / 4) and one per chroma
 * sample (dec_c, width / 2 x height / 2), nonzero where reconstructed. */
typedef struct vvcg_gen_intra_state {
  const uint16_t* plane[3];
  uint32_t stride[3];
  uint32_t width, height;
  const uint8_t* dec_y;
  const uint8_t* dec_c;
  uint8_t bit_depth;            /* 8..12 */
  uint8_t vert_collocated;      /* sps_chroma_vertical_collocated_flag */
  uint8_t reserved[2];
  uint32_t ctu_size;
} vvcg_gen_intra_state;

/* Intra prediction of independent transform blocks as the general decoder
 * forms it (no residual, no reconstruction): reference samples with its
 * availability and substitution (Gen::gather_len, decode_general.rs:
 * 4260-4341; gather_mrl :4542-4632; isp_refs :4634-4648), predict_luma
 * (:4650-4732) and predict_chroma (:4734-4793) with cclm_predict
 * (:4372-4537), and the 4-wide ISP region of reconstruct_tu (:4001-4024).
 * Blocks of one call must not read each other's samples (the caller orders
 * calls along the decode order). reqs host memory, out device memory
 * (int16). MIP coding units use vvcg_mip_predict_dev. */
vvcg_status vvcg_gen_intra_predict_dev(vvcg_ctx* ctx, const vvcg_gen_intra_state* state,
                                       const vvcg_gen_intra_req* reqs, uint32_t num_reqs, int16_t* out,
                                       uint64_t out_count);


/* Reconstruction of transform blocks in decode order, for blocks that read
 * each other's samples, such as the ISP sub-partitions of a coding unit:
 * reqs are split into groups (group_start: num_groups + 1 indices into reqs,
 * host memory); the blocks of a group are reconstructed one after the other
 * by one warp, different groups in parallel (groups of one call must not read
 * each other's samples). Each block is predicted as vvcg_gen_intra_predict_dev
 * predicts it (into pred, device, at out_off), residual (device, int16, w x h
 * at out_off, the inverse-transformed and BDPCM-accumulated residual of
 * vvcg_tu_inverse_batch; NULL for none) is added, the sum clipped to the bit
 * depth and stored into the block's plane of the state, and the block marked
 * decoded in the state's maps (luma: every 4x4 cell it touches; chroma: every
 * sample), which the next block's reference gathering reads. The state's
 * planes and maps are written (device memory).
 * Replaces: reconstruct_tu (decode_general.rs:3985-4096) for each transform
 * unit of a coding unit, in order, with mark_tu's decoded maps (:4891-4906);
 * for ISP the loop over sub-partitions of :4009-4024. */
vvcg_status vvcg_gen_intra_recon_dev(vvcg_ctx* ctx, const vvcg_gen_intra_state* state,
                                     const vvcg_gen_intra_req* reqs, uint32_t num_reqs,
                                     const uint32_t* group_start, uint32_t num_groups,
                                     const int16_t* residual, int16_t* pred, uint64_t out_count);
/* ---- general-decoder deblocking ------------------------------------------- */

enum { VVCG_DBK_CODED = 1, VVCG_DBK_INTRA = 2, VVCG_DBK_CBF = 4 };
#define VVCG_DBK_NO_TU 0xFFFFFFFFu

/* One 4x4 luma cell of the general decoder's deblocking state: the
 * transform block marked there (mark_tu, decode_general.rs:4837-4907: id,
 * width, height, luma cbf) and the coding-unit fields the boundary strength
 * reads (LumaCell, decode_general.rs:114: valid, intra, ref_idx, mv). */
typedef struct vvcg_dbk_cell {
  uint32_t tu_id;      /* VVCG_DBK_NO_TU where no luma transform block is marked */
  uint16_t tu_w, tu_h; /* luma samples */
  int32_t mv[2][2];    /* [list][horizontal, vertical], 1/16 sample */
  int8_t ref_idx[2];   /* -1 = list unused */
  uint8_t flags;       /* VVCG_DBK_CODED | VVCG_DBK_INTRA | VVCG_DBK_CBF */
  uint8_t reserved;
} vvcg_dbk_cell; /* 28 bytes */

/* One 2x2 chroma cell (4:2:0): the Cb and Cr transform blocks marked there
 * and their size in chroma samples. */
typedef struct vvcg_dbk_ccell {
  uint32_t tu_cb, tu_cr; /* VVCG_DBK_NO_TU where none */
  uint16_t tu_w, tu_h;
} vvcg_dbk_ccell; /* 12 bytes */

/* Slice-level deblocking parameters: QP and beta / tC offsets (div2) of Y,
 * Cb, Cr, and the POC of each reference index of lists 0 and 1 (an index at
 * or beyond num_ref reads POC 0, as the reference's unwrap_or(0) does). */
typedef struct vvcg_dbk_params {
  int32_t qp[3];
  int32_t beta_offset_div2[3];
  int32_t tc_offset_div2[3];
  int32_t num_ref[2];
  int32_t ref_poc[2][16];
} vvcg_dbk_params;

/* Deblocking of a 4:2:0 picture as the general decoder applies it, in place
 * on device planes: luma transform-block edges on the 4-sample grid with the
 * filter lengths of the transform sizes (1 / 3 / 7) and the intra / cbf /
 * motion boundary strength; chroma transform-block edges on the 8-sample
 * grid in 2-line groups with bS 2. Vertical edges, then horizontal edges.
 * cells (cell_cols x cell_rows, raster, device memory) covers the picture
 * padded to whole CTUs; ccells likewise covers its chroma at one cell per 2x2
 * chroma samples. The maps must be what mark_tu leaves for a coding tree
 * (transform blocks of 4 or more samples start on the 4-sample grid), which
 * keeps the segments of one direction from touching each other's samples.
 * Replaces: apply_deblock (decode_general.rs:4977-5187) with luma_lens
 * (:4916), chroma_lens (:4929), deblock_bs (:4939), over
 * deblock_luma_edge_normative_bd (filter.rs:718) and deblock_chroma_edge
 * (filter.rs:935-1007). */
vvcg_status vvcg_deblock_general_dev(vvcg_ctx* ctx, uint16_t* const planes[3], const uint32_t stride[3],
                                     uint32_t vis_width, uint32_t vis_height, uint8_t bit_depth, uint32_t ctu_size,
                                     const vvcg_dbk_cell* cells, uint32_t cell_cols, uint32_t cell_rows,
                                     const vvcg_dbk_ccell* ccells, uint32_t ccell_cols, uint32_t ccell_rows,
                                     const vvcg_dbk_params* params);

/* ---- general-decoder intra pictures, batched ------------------------------ */

/* One transform block of a general-decoder intra picture, in decode order:
 * its prediction (vvcg_gen_intra_req: block, coding unit, component, mode,
 * MRL, ISP, BDPCM; out_off indexes the batch's residual / prediction slots)
 * and, when coded, its residual (vvcg_tu_rec with the block's log2 sizes,
 * the picture's bit depth, levels at in_off of the level pool and
 * out_off = pred.out_off; the rules of vvcg_tu_inverse_batch). */
typedef struct vvcg_gen_tb {
  vvcg_gen_intra_req pred;
  vvcg_tu_rec tu;
  uint32_t coded; /* 0: no residual, the block is its prediction */
} vvcg_gen_tb;    /* 48 bytes */

/* One 4:2:0 picture of the general decoder (decode_general.rs), coded as a
 * tree of intra coding units. Its transform blocks form groups in decode
 * order (vvcg_gen_batch.group_first): a group is reconstructed block after
 * block (a coding unit's luma blocks or ISP sub-partitions, then its chroma
 * blocks; or the chroma blocks of a node whose luma was split below 8x8),
 * and groups that do not read each other's samples run in parallel. */
typedef struct vvcg_gen_pic {
  uint32_t width, height;            /* coded size: whole CTUs, multiples of 8 */
  uint32_t vis_width, vis_height;    /* cropped size (<= coded) */
  uint8_t bit_depth;                 /* 8..12 */
  uint8_t ctu_log2;                  /* 4..7 */
  uint8_t vert_collocated;           /* sps_chroma_vertical_collocated_flag */
  uint8_t tools;                     /* VVCG_TOOL_DEBLOCK | VVCG_TOOL_SAO | VVCG_TOOL_ALF */
  uint32_t group_offset, num_groups; /* its groups: group_first[group_offset .. + num_groups] */
  uint32_t sao_offset;               /* with SAO: 3 x CTUs vvcg_sao at sao[sao_offset] (Y, Cb, Cr per CTU,
                                        CTUs of the visible picture in raster order) */
  uint32_t alf_offset;               /* with ALF: CTUs vvcg_alf_ctu at alf_ctus[alf_offset] */
  int32_t alf_params;                /* with ALF: index into vvcg_gen_batch.alf_params */
  vvcg_dbk_params dbk;               /* with deblocking: QPs and offsets (reference lists unused) */
} vvcg_gen_pic;

typedef struct vvcg_gen_batch {
  const vvcg_gen_pic* pics;
  uint32_t num_pics;
  uint32_t num_groups;               /* all pictures' groups */
  const vvcg_gen_tb* tbs;            /* all pictures' blocks, each picture's in decode order */
  const uint32_t* group_first;       /* num_groups + 1 block indices, nondecreasing */
  uint64_t num_tbs;
  const int16_t* levels;             /* level pool of the coded blocks */
  uint64_t num_levels;
  uint64_t slot_count;               /* residual / prediction slots (int16) the blocks' out_off index */
  const vvcg_sao* sao;
  uint64_t num_sao;
  const vvcg_alf_ctu* alf_ctus;
  uint64_t num_alf_ctus;
  const vvcg_alf_params* alf_params;
  uint32_t num_alf_params;
  uint32_t reserved;
} vvcg_gen_batch;

/* The general decoder's picture pass over a batch of intra pictures, the
 * reconstruction and loop filters of decode_general_picture
 * (decode_general.rs:1134-1150 after the parse): residuals of every coded
 * block (the size-binned TU kernels), intra reconstruction in decode order
 * (reconstruct_tus :3885 / reconstruct_tu :3985 with mark_tu's decoded maps),
 * deblocking with the transform-block maps mark_tu leaves (apply_deblock
 * :4977), SAO (apply_sao :5189) and ALF (apply_alf :5225). The groups of all
 * pictures are put in dependency levels on the host: a group runs after
 * every earlier group whose samples it may read and every earlier group that
 * may read its samples, so each block sees the decoded maps of the
 * picture's sequential decode. prepare validates and uploads the batch (host
 * memory) and derives the levels and deblocking maps; run enqueues the pass
 * (graph != 0: as one CUDA graph, captured on the first run of the prepared
 * batch); download synchronises and copies the visible planes to out (3 per
 * picture, host, 16-bit samples). vvcg_decode_general_batch does all three. */
vvcg_status vvcg_gen_prepare(vvcg_ctx* ctx, const vvcg_gen_batch* b);
vvcg_status vvcg_gen_run(vvcg_ctx* ctx, uint32_t graph);
vvcg_status vvcg_gen_download(vvcg_ctx* ctx, const vvcg_plane_out* out);
vvcg_status vvcg_decode_general_batch(vvcg_ctx* ctx, const vvcg_gen_batch* b, const vvcg_plane_out* out);
/* Dependency levels of the prepared batch (the intra kernel's launches per run). */
uint32_t vvcg_gen_levels(const vvcg_ctx* ctx);

/* ---- CABAC parse of strict-profile pictures (host) ------------------------ */

/* One IDR picture of the strict 8-bit 4:2:0 intra profile: its slice data
 * (the CABAC substream the reference's encode_picture writes, slice.rs:325),
 * coded size (multiples of 32, CTU 32) and slice QP, and where its records
 * and levels go. */
typedef struct vvcg_strict_substream {
  const uint8_t* data;
  uint64_t size;
  uint32_t width, height;
  uint8_t qp;
  uint8_t reserved[3];
  uint32_t cu_offset;     /* first of its (width / 32) * (height / 32) records in cus */
  uint64_t level_offset;  /* first level it writes (even with sparse) */
  uint64_t level_cap;     /* levels it may write */
} vvcg_strict_substream;

/* Parses each picture's slice data on the host as decode_picture does
 * (slice.rs:458-575: luma and chroma modes, cbfs, transform_skip_flag,
 * residual_coding / residual_ts_coding, lfnst_idx and mts_idx where present,
 * end_of_slice_one_bit) into frame-path CU records (VVCG_TOOL_TU_TOOLS
 * tu_tools; level_off absolute in `levels`) and levels, dense or, with
 * sparse != 0, in the VVCG_TOOL_SPARSE_LEVELS form. Pictures are parsed in
 * parallel on `threads` host threads (0: one). levels_used[i] receives the
 * levels picture i wrote. VVCG_LIMIT_EXCEEDED when a picture's level_cap is
 * too small, VVCG_INVALID_INPUT for a malformed substream; err (optional)
 * receives the reason. No device work. */
vvcg_status vvcg_parse_strict(const vvcg_strict_substream* pics, uint32_t num_pics, uint32_t sparse,
                              uint32_t threads, vvcg_cu_rec* cus, uint64_t num_cus, int16_t* levels,
                              uint64_t num_levels, uint64_t* levels_used, char* err, size_t err_cap);

enum { VVCG_PARSE_LUMA = 1, VVCG_PARSE_DEP_QUANT = 2, VVCG_PARSE_SIGN_HIDING = 4, VVCG_PARSE_TRANSFORM_SKIP = 8 };

/* One block's CABAC substream (its residual_coding, or with
 * VVCG_PARSE_TRANSFORM_SKIP its residual_ts_coding, on fresh I-slice
 * contexts at qp, then end_of_slice_one_bit and the byte alignment) into w x
 * h raster levels (out, host int32): the parser's residual decoding alone
 * (residual.rs:534-881 decode_residual_with_options, slice.rs:1323-1435
 * decode_ts_block). VVCG_INVALID_INPUT for a malformed substream. */
vvcg_status vvcg_parse_residual_block(const uint8_t* data, uint64_t size, uint32_t w, uint32_t h, uint32_t flags,
                                      uint32_t qp, int32_t* out);

/* ---- the multi-tool stream: IDR and P pictures, picture buffer ------------ */

/* Slice coding options of the multi-tool stream (SliceCodingOptions,
 * slice.rs:1471-1507) this library's multi-tool entries take; the other
 * tools (CCLM, MIP, MRL, ISP, BDPCM, joint Cb-Cr, SAO, ALF, LMCS, palette,
 * IBC, ACT) are not supported by them and rejected. */
enum {
  VVCG_SLICE_DEP_QUANT = 1u << 0,        /* dep_quant */
  VVCG_SLICE_SIGN_HIDING = 1u << 1,      /* sign_data_hiding (syntax only) */
  VVCG_SLICE_DEBLOCK = 1u << 2,          /* enable_deblock (IDR: the frame path's deblocking; P: CTU boundaries) */
  VVCG_SLICE_FULL_INTRA_MODES = 1u << 3  /* full_intra_modes (an encoder decision; no syntax change) */
};

/* One slice-data substream of the multi-tool stream: an IDR picture
 * (encode_picture_multitool, slice.rs:2575) or a P picture
 * (encode_inter_picture, slice.rs:3307), coded size (multiples of the CTU
 * size), slice QP, CTU size, options, and where its records and levels go. */
typedef struct vvcg_slice_substream {
  const uint8_t* data;
  uint64_t size;
  uint32_t width, height;
  uint8_t qp;
  uint8_t ctu_log2;       /* 5: CTU 32, one coding unit per CTU */
  uint8_t options;        /* VVCG_SLICE_* */
  uint8_t reserved;
  uint32_t cu_offset;     /* first record of the picture in the output array */
  uint64_t level_offset;  /* first level it writes (even with sparse) */
  uint64_t level_cap;     /* levels it may write */
} vvcg_slice_substream;

/* Parses IDR pictures of the multi-tool stream on the host as
 * decode_picture_multitool does (slice.rs:3012-3190: per coding unit the luma
 * mode against the MPM list of the left neighbour, the chroma mode, the cbfs,
 * transform_skip_flag and the residuals; end_of_slice_one_bit) into
 * frame-path records (VVCG_TOOL_TU_TOOLS with transform-skip flags only;
 * (width / 32) * (height / 32) records, raster order), dense or sparse
 * levels, pictures on `threads` host threads. The pictures decode on the
 * frame path (vvcg_decode_batch) with tools TU_TOOLS, plus DEP_QUANT and
 * DEBLOCK as the substream's options ask, at SliceQpY max(qp, 4) (the QP
 * decode_picture_multitool reconstructs and deblocks with). Errors as
 * vvcg_parse_strict. */
vvcg_status vvcg_parse_multitool_idr(const vvcg_slice_substream* pics, uint32_t num_pics, uint32_t sparse,
                                     uint32_t threads, vvcg_cu_rec* cus, uint64_t num_cus, int16_t* levels,
                                     uint64_t num_levels, uint64_t* levels_used, char* err, size_t err_cap);

enum {
  VVCG_INTER_CU_MERGE = 1,   /* merge (or skip) coding unit: motion of merge candidate 0 */
  VVCG_INTER_CU_SKIP = 2,    /* cu_skip_flag */
  VVCG_INTER_CU_ALT_HPEL = 4 /* the alternative half-sample luma filter */
};

/* One coding unit (a whole CTU) of a P picture: its motion as
 * decode_inter_picture derives it (merge candidate 0, or the AMVP predictor
 * plus the coded difference), the cbfs, transform-skip flags and levels
 * (level_off as in vvcg_cu_rec). mvd and mvp_idx are the parsed AMVP syntax;
 * the GPU reads only the motion. */
typedef struct vvcg_inter_cu {
  int32_t mv[2][2];  /* [L0, L1][horizontal, vertical], 1/16 luma sample */
  int32_t mvd[2];    /* AMVP: coded motion vector difference */
  int8_t ref_idx[2]; /* per list; -1 = list unused */
  uint8_t inter_dir; /* 1 = L0 (P pictures take L0 only) */
  uint8_t bcw_idx;   /* 2 = equal weights */
  uint8_t flags;     /* VVCG_INTER_CU_* */
  uint8_t mvp_idx;   /* AMVP: predictor index */
  uint8_t cbf;       /* bit0 Y, bit1 Cb, bit2 Cr */
  uint8_t tu_tools;  /* bit c: transform skip of component c */
  int32_t level_off[3];
  uint32_t reserved;
} vvcg_inter_cu; /* 48 bytes */

/* Parses P pictures of the multi-tool stream on the host as
 * decode_inter_picture does (slice.rs:3552-3677: cu_skip_flag with its
 * neighbour context, pred_mode_flag, general_merge_flag, mvd_coding and
 * mvp_l0_flag, rqt_root_cbf, the cbfs with tu_y_coded_flag inferred,
 * transform_skip_flag and the residuals on P-slice contexts) and derives
 * each coding unit's motion (derive_merge_candidates candidate 0 or
 * derive_amvp_candidates plus the difference, the HMVP table reset per CTU
 * row). One record per CTU, raster order. Intra coding units in a P picture
 * are rejected as the reference rejects them. Errors as vvcg_parse_strict. */
vvcg_status vvcg_parse_multitool_p(const vvcg_slice_substream* pics, uint32_t num_pics, uint32_t sparse,
                                   uint32_t threads, vvcg_inter_cu* cus, uint64_t num_cus, int16_t* levels,
                                   uint64_t num_levels, uint64_t* levels_used, char* err, size_t err_cap);

/* The context's picture buffer: device pictures of 8-bit 4:2:0 samples in
 * 16-bit planes (stride a multiple of 64 samples), the reference pictures of
 * P pictures (the reference decoder's DecodedPictureBuffer, inter.rs:446,
 * kept on the device). vvcg_dpb_reserve makes `slots` (1..1024) slots of width x
 * height (contents undefined; earlier slots are released). */
vvcg_status vvcg_dpb_reserve(vvcg_ctx* ctx, uint32_t slots, uint32_t width, uint32_t height);
/* Copies picture `pic` of the last frame-path batch (vvcg_decode_batch or
 * vvcg_batch_run; same coded size, 8-bit 4:2:0) into a slot, on the device. */
vvcg_status vvcg_dpb_store(vvcg_ctx* ctx, uint32_t pic, uint32_t slot);
/* Host or device planes (copy direction inferred) into / out of a slot. */
vvcg_status vvcg_dpb_upload(vvcg_ctx* ctx, uint32_t slot, const vvcg_plane_in planes[3]);
vvcg_status vvcg_dpb_download(vvcg_ctx* ctx, uint32_t slot, const vvcg_plane_out planes[3]);
/* Device pointer and stride (samples) of one plane of a slot. */
vvcg_status vvcg_dpb_plane(vvcg_ctx* ctx, uint32_t slot, uint32_t comp, void** dev_ptr, uint32_t* stride);

/* One P picture of the multi-tool stream for vvcg_decode_p_batch: 8-bit
 * 4:2:0, CTU 32 (one coding unit per CTU). */
typedef struct vvcg_p_pic {
  uint32_t width, height; /* the picture buffer's size */
  uint8_t qp;             /* SliceQpY */
  uint8_t options;        /* VVCG_SLICE_DEP_QUANT, VVCG_SLICE_DEBLOCK */
  uint8_t num_refs;       /* L0 entries, 1..4 */
  uint8_t sparse;         /* levels in the VVCG_TOOL_SPARSE_LEVELS form */
  int32_t ref_slot[4];    /* picture-buffer slot of L0 reference index i */
  int32_t out_slot;       /* slot of the reconstruction; not one of its references */
  uint32_t cu_offset;     /* first of its (width / 32) * (height / 32) records */
} vvcg_p_pic; /* 36 bytes */

/* Decodes P pictures in the given order into their picture-buffer slots:
 * per coding unit the luma 8-tap and chroma 4-tap motion compensation from
 * the reference slot (8-bit uni-prediction, clamped reference reads), the
 * dequantised and inverse DCT-2 (or transform-skip) residual, add and clip,
 * then with VVCG_SLICE_DEBLOCK the CTU-boundary deblocking. Pictures whose
 * slots do not depend on each other run in the same launches. Records and
 * levels are host memory. Replaces: decode_inter_picture's reconstruction
 * (slice.rs:3677-3834) over predict_inter_pu (inter.rs:1734),
 * reconstruct_component_full (slice.rs:1920) and apply_inter_loop_filters
 * (slice.rs:2291). Synchronous; VVCG_INVALID_INPUT for bad records. */
vvcg_status vvcg_decode_p_batch(vvcg_ctx* ctx, const vvcg_p_pic* pics, uint32_t num_pics, const vvcg_inter_cu* cus,
                                uint32_t num_cus, const int16_t* levels, uint64_t num_levels);

/* ---- inter-prediction tools (BDOF, DMVR, affine / PROF, CIIP, GPM) -------- */

/* A block of the batched inter tools: w x h samples at `off` of the tool's
 * int32 input and output arrays (row-major). */
typedef struct vvcg_bdof_req {
  uint16_t w, h;  /* multiples of 4 */
  uint32_t off;
} vvcg_bdof_req;

/* BDOF of bi-predicted luma blocks: pred0 / pred1 are the two 14-bit
 * intermediate predictions, out the 8-bit result (device, int32).
 * Replaces: apply_bdof_luma (inter.rs:1218-1339). */
vvcg_status vvcg_bdof_dev(vvcg_ctx* ctx, const vvcg_bdof_req* reqs, uint32_t num_reqs, const int32_t* pred0,
                          const int32_t* pred1, int32_t* out, uint64_t count);

/* A DMVR subblock: position and size (luma samples) and the bi-prediction's
 * motion vectors [list][horizontal, vertical] (1/16 sample). */
typedef struct vvcg_dmvr_req {
  int32_t bx, by;
  uint16_t dx, dy; /* at most 16 x 16 */
  int32_t mv[2][2];
} vvcg_dmvr_req;

/* DMVR refinement of each subblock against 8-bit reference planes ref0 /
 * ref1 (device, width x height, stride; samples outside read the nearest
 * edge): the refined pair goes to mv_out (device, 4 int32 per request).
 * Replaces: refine_dmvr_subblock (inter.rs:1371-1471). */
vvcg_status vvcg_dmvr_dev(vvcg_ctx* ctx, const uint8_t* ref0, const uint8_t* ref1, uint32_t width, uint32_t height,
                          uint32_t stride, const vvcg_dmvr_req* reqs, uint32_t num_reqs, int32_t* mv_out);

/* An affine coding unit: control-point MVs [top-left, top-right,
 * bottom-left][horizontal, vertical], size, model and prediction type. */
typedef struct vvcg_affine_req {
  int32_t cp[3][2];
  uint16_t w, h;      /* multiples of 4, 8..128 */
  uint8_t six_param;  /* 1: 6-parameter model, 0: 4-parameter */
  uint8_t inter_dir;  /* 1 / 2 uni-prediction, 3 bi-prediction */
  uint8_t reserved[2];
  uint32_t sub_off;   /* first subblock MV of this CU in sub_mv (pairs) */
} vvcg_affine_req;

/* Affine subblock motion: the (w/4) x (h/4) 4x4-subblock MVs of each CU
 * (sub_mv, device, int32 pairs from sub_off), and its PROF deltas (prof,
 * device, 33 int32 per request: 16 horizontal, 16 vertical, 1 when PROF
 * applies). Replaces: derive_affine_subblock_mvs (inter.rs:1502-1579). */
vvcg_status vvcg_affine_mvs_dev(vvcg_ctx* ctx, const vvcg_affine_req* reqs, uint32_t num_reqs, int32_t* sub_mv,
                                uint64_t sub_count, int32_t* prof);

/* A PROF subblock: its 6x6 14-bit intermediate window (36 int32 at src_off),
 * deltas (16 horizontal then 16 vertical at dmv_off), 16 outputs at out_off. */
typedef struct vvcg_prof_req {
  uint32_t src_off, dmv_off, out_off;
  uint8_t bi; /* 1: keep the refined intermediate, 0: round to 8 bits */
  uint8_t reserved[3];
} vvcg_prof_req;

/* PROF of 4x4 subblocks (device arrays). Replaces: apply_prof_4x4
 * (inter.rs:1581-1609). */
vvcg_status vvcg_prof_dev(vvcg_ctx* ctx, const vvcg_prof_req* reqs, uint32_t num_reqs, const int32_t* src,
                          uint64_t src_count, const int32_t* dmv, uint64_t dmv_count, int32_t* out, uint64_t out_count);

/* A CIIP block: n samples at off; whether the left / above neighbours are intra. */
typedef struct vvcg_ciip_req {
  uint32_t n, off;
  uint8_t left_intra, above_intra, reserved[2];
} vvcg_ciip_req;

/* CIIP blending of inter and Planar intra predictions (device int32).
 * Replaces: apply_ciip_blend (inter.rs:1615-1630). */
vvcg_status vvcg_ciip_blend_dev(vvcg_ctx* ctx, const vvcg_ciip_req* reqs, uint32_t num_reqs, const int32_t* inter,
                                const int32_t* intra, int32_t* out, uint64_t count);

/* A GPM block: size in its component's samples, split direction 0..63 and
 * the component's subsampling (0 luma, 1 for 4:2:0 chroma). */
typedef struct vvcg_gpm_req {
  uint16_t w, h;
  uint8_t split_dir, scale_x, scale_y, reserved;
  uint32_t off;
} vvcg_gpm_req;

/* GPM blending of two uni-predictions (device int32).
 * Replaces: derive_gpm_params_table + predict_gpm_block (inter.rs:1641-1731). */
vvcg_status vvcg_gpm_blend_dev(vvcg_ctx* ctx, const vvcg_gpm_req* reqs, uint32_t num_reqs, const int32_t* pred0,
                               const int32_t* pred1, int32_t* out, uint64_t count);

/* ---- CTU-boundary deblocking of inter pictures ---------------------------- */

/* One CTU of an inter picture of the 8-bit multi-tool path as its CTU-boundary
 * deblocking reads it (slice.rs:2319-2326, :2438-2444): mv_field[0] of the
 * prediction unit at the CTU's top-left, top-right and bottom-left luma
 * samples (what get_at_luma returns on the Q side of an edge, the P side of
 * a vertical edge and the P side of a horizontal edge), and the CTU's
 * coded-residual flags (the cbf grids). */
typedef struct vvcg_ctu_motion {
  int32_t mv[3][2]; /* [top-left, top-right, bottom-left][horizontal, vertical], 1/16 sample */
  int32_t ref[3];   /* ref_idx of the same three */
  uint8_t cbf;      /* bit0 Y, bit1 Cb, bit2 Cr */
  uint8_t reserved[3];
} vvcg_ctu_motion; /* 40 bytes */

/* Deblocking of an 8-bit 4:2:0 inter picture in place on device planes, on
 * CTU boundaries only: every vertical CTU boundary, then every horizontal
 * one, each CTU-long edge with its own boundary strength
 * (derive_boundary_strength, filter.rs:202-226, of the two CTUs' cbf of the
 * plane and motion; not intra), SliceQpY `qp` for luma and derived_chroma_qp
 * for chroma, maximum filter lengths of min(ctu, 32)-sample luma and
 * ctu/2-sample chroma transforms, the P side of a horizontal chroma edge
 * limited to 1 (CTB-row boundary). Samples are 8-bit values in 16-bit
 * planes (the reference's u8 planes); width and height are multiples of ctu
 * (32, 64 or 128); cells: (width/ctu) x (height/ctu) records in raster order,
 * device memory.
 * Replaces: the deblocking part of apply_inter_loop_filters
 * (slice.rs:2291-2554), over deblock_luma_edge_normative (filter.rs:689) and
 * deblock_chroma_edge_region (filter.rs:1069). */
vvcg_status vvcg_deblock_ctu_edges_dev(vvcg_ctx* ctx, uint16_t* const planes[3], const uint32_t stride[3],
                                       uint32_t width, uint32_t height, uint32_t ctu, uint8_t qp,
                                       const vvcg_ctu_motion* cells);

/* ---- general-decoder SAO -------------------------------------------------- */

/* SAO of one plane as the general decoder applies it: every CTU region,
 * cropped to the visible size, with its vvcg_sao (params: device memory, one
 * per CTU, ctu_cols per row; ctu_size in this plane's samples). Edge class 3
 * uses the (-1, 1) / (1, -1) pair and edge neighbours outside the visible
 * picture leave a sample unchanged. Reads src, writes every sample of dst
 * (device planes, same stride). Replaces: apply_sao (decode_general.rs:5189)
 * over apply_sao_region_bounded_16 (filter.rs:1954-2033). */
vvcg_status vvcg_sao_bounded_16_dev(vvcg_ctx* ctx, const uint16_t* src, uint16_t* dst, uint32_t stride,
                                    uint32_t width, uint32_t height, uint32_t vis_width, uint32_t vis_height,
                                    uint8_t bit_depth, uint32_t ctu_size, uint32_t ctu_cols,
                                    const vvcg_sao* params);

/* ---- plane metrics ---------------------------------------------------------- */

/* Sum of squared errors, sum of absolute differences and sample count of one
 * plane pair (device pointers, strides in samples), written to out[0..2]
 * (device memory, 3 x uint64). Replaces: CpuFrameMetrics::plane_metrics
 * (crates/rustmpeg-video/src/accelerator.rs:258-292); PSNR and MSE follow
 * from these on the host (PlaneMetrics::psnr, accelerator.rs:111-118).
 * Asynchronous on the context's stream. */
vvcg_status vvcg_plane_metrics_8_dev(vvcg_ctx* ctx, const uint8_t* ref, uint64_t ref_stride,
                                     const uint8_t* dist, uint64_t dist_stride, uint32_t width,
                                     uint32_t height, uint64_t* out);
/* The same sums for 16-bit planes (the library's 8..12-bit sample planes). */
vvcg_status vvcg_plane_metrics_16_dev(vvcg_ctx* ctx, const uint16_t* ref, uint64_t ref_stride,
                                      const uint16_t* dist, uint64_t dist_stride, uint32_t width,
                                      uint32_t height, uint64_t* out);

/* ---- allocation-free single picture --------------------------------------- */

/* Largest picture height, in CTU rows, that vvcg_recon_picture_static takes
 * (8192 luma rows with 32x32 CTUs). */
#define VVCG_STATIC_MAX_CTU_ROWS 256u

/* Reconstructs one picture, and deblocks it when its tools ask for that,
 * without allocating any memory. No counterpart in the reference: it is a
 * variant of vvcg_decode_batch for callers that must not allocate, such as a
 * decoder whose device memory is fixed when it starts, code that must not let
 * cudaMalloc/cudaFree stall other work queued on the device, or a host whose
 * own allocator owns all device memory.
 *
 * Inputs and outputs are the caller's device memory: `cus` holds the
 * picture's records from pic->cu_offset on (num_cus entries in all), `levels`
 * the level pool (num_levels int16 values), and planes[0..2] the Y, Cb and Cr
 * planes at coded size (width x height, 4:0:0 uses planes[0] only), each
 * 16-byte aligned with a stride of at least the plane width that is a
 * multiple of 8 samples. The planes
 * are also the work space: they first receive the residuals, then the
 * reconstructed samples. pic is host memory. SAO and ALF are rejected
 * (VVCG_INVALID_INPUT): they need a second set of planes.
 *
 * The library's bookkeeping (queue counter, status word, row progress words,
 * the picture's descriptor and deblocking passes) lives in one fixed array of
 * 40 KB in device memory, one per device, which holds up to
 * VVCG_STATIC_MAX_CTU_ROWS CTU rows; taller pictures return
 * VVCG_LIMIT_EXCEEDED. The call runs on the calling thread's current device
 * and on `cuda_stream` (NULL = the legacy default stream), and returns after
 * the stream has finished the picture.
 *
 * The first call on a device does the set-up (it loads the tables, finds the
 * array's address and sets the kernels' attributes). Every call copies the picture's header
 * from host memory into the array, reads the status word back and waits for
 * `cuda_stream` before it returns. Every call shares the array and leaves the previous call's
 * contents in it; each call clears the parts that must start at zero. Calls
 * that overlap in time on one device, from several host threads, race on the
 * array: serialise them. `err` (may be NULL) receives a message on failure. */
vvcg_status vvcg_recon_picture_static(const vvcg_pic_desc* pic, const vvcg_cu_rec* cus,
                                      uint32_t num_cus, const int16_t* levels,
                                      uint64_t num_levels, const vvcg_plane_out* planes,
                                      void* cuda_stream, char* err, size_t err_cap);

/* ---- Annex-B access units around the slice data -----------------------
 *
 * Host-side bitstream assembly of the reference encoder's default stream
 * (8-bit 4:2:0, 32x32 CTUs; MTS, LFNST and transform skip enabled, every
 * other tool off) and its reverse, so that slice data parsed by
 * vvcg_parse_strict can come from, and go to, an H.266 Annex-B byte stream.
 * No GPU is involved. */

/* The stream configuration the parameter sets describe (replaces hls.rs
 * VvcStreamConfig, crates/rustmpeg-video/src/vvc/hls.rs:94-107). */
typedef struct vvcg_stream_cfg {
  uint32_t width, height;            /* coded size in luma samples */
  uint32_t crop_right, crop_bottom;  /* conformance-window crop in luma samples, even */
  uint8_t qp, level_idc, ctu_log2, min_cb_log2, ts_log2;
  uint8_t reserved[3];
} vvcg_stream_cfg;

typedef enum vvcg_hls_kind {
  VVCG_HLS_AUD = 0,          /* hls.rs:756 build_aud_rbsp_pic_type; arg = aud_pic_type */
  VVCG_HLS_VPS = 1,          /* hls.rs:353 build_vps_rbsp */
  VVCG_HLS_SPS = 2,          /* hls.rs:373 build_sps_rbsp */
  VVCG_HLS_PPS = 3,          /* hls.rs:529 build_pps_rbsp */
  VVCG_HLS_PH = 4,           /* hls.rs:571 build_ph_rbsp; arg = POC LSB */
  VVCG_HLS_SLICE_HEADER = 5  /* hls.rs:598 build_slice_header_bits; arg = sh_qp_delta */
} vvcg_hls_kind;

/* One RBSP (before emulation prevention) of the default stream into `out`
 * (cap bytes). *size receives its length; VVCG_LIMIT_EXCEEDED when it does
 * not fit (nothing written), VVCG_INVALID_INPUT for an unknown kind or a
 * configuration the syntax cannot carry (ctu_log2 outside 5..7, odd crop,
 * min_cb_log2 or ts_log2 below 2). */
vvcg_status vvcg_hls_rbsp(const vvcg_stream_cfg* cfg, uint32_t kind, int32_t arg, uint8_t* out, size_t cap,
                          size_t* size);

/* The IDR access unit VvcEncoder::encode_i420 emits for a picture of
 * width x height visible luma samples coded at qp (mod.rs:582-616): AUD,
 * VPS, SPS, PPS, picture header, then one IDR_N_LP slice NAL unit holding
 * the slice header and `slice_data` (what vvcg_parse_strict reads), each
 * behind a 4-byte start code with emulation prevention. The coded size is
 * the visible size rounded up to whole CTUs (mod.rs:300-318), the level the
 * smallest whose picture size holds it (hls.rs:182). *size receives the
 * length; VVCG_LIMIT_EXCEEDED when it exceeds cap (nothing written). */
vvcg_status vvcg_annexb_idr(uint32_t width, uint32_t height, uint8_t qp, const uint8_t* slice_data, size_t n,
                            uint8_t* out, size_t cap, size_t* size);

typedef struct vvcg_annexb_info {
  uint32_t width, height;  /* coded size (from the PPS) */
  int32_t qp;              /* slice QP: 26 + pps_init_qp_minus26 + sh_qp_delta */
  uint32_t num_nals;       /* NAL units in the access unit */
  uint32_t slice_nal_type; /* nal_unit_type of the slice (7 or 8: IDR) */
  uint32_t reserved;
} vvcg_annexb_info;

/* The reverse for one access unit of that stream: splits the byte stream at
 * its start codes, reads the coded size and initial QP from the PPS, then
 * the IDR slice's header, and writes the slice data after it (emulation
 * prevention removed) to `slice_data`; *size receives its length.
 * VVCG_INVALID_INPUT when no PPS or IDR slice is present, or a syntax
 * element differs from the default stream's layout (pps_no_pic_partition,
 * a picture header in the slice header, an unterminated slice header);
 * VVCG_LIMIT_EXCEEDED when the slice data exceeds cap. */
vvcg_status vvcg_annexb_read_idr(const uint8_t* au, size_t n, vvcg_annexb_info* info, uint8_t* slice_data,
                                 size_t cap, size_t* size);

#ifdef __cplusplus
}
#endif

#endif /* VVCG_H */
