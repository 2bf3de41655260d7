// CPU oracle for the VVC reconstruction / loop-filter / candidate-cost path.
//
// TEST INFRASTRUCTURE ONLY. This is a plain C++ restatement of the reference
// codec's single-threaded CPU code (rustmpeg-video, crates/rustmpeg-video/src/vvc/),
// function by function, each citing the reference file:line it follows. It is
// the checker that the CUDA path is compared against, and the timed CPU
// baseline in bench.py. Nothing in the product library links, loads or calls
// it: only tests/, __graft_entry__.smoke() and bench.py's CPU legs use it.
//
// Parity pinning: the reference is Rust and no Rust toolchain is available,
// so the reference itself cannot be run to produce golden outputs. The
// restatement is pinned by the reference's own known-answer and property
// tests, ported in tests/test_oracle_kats.py (see the header of that file for
// the list); anything those tests do not reach is "parity unpinned".
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <vector>

#include "../include/vvcg.h"

namespace orc {

enum TrType { kDct2 = 0, kDst7 = 1, kDct8 = 2 };

// ---- dct.rs -----------------------------------------------------------------
const int8_t* matrix_for_any(int tr, int size);
int forward_transform_rect_bd(int w, int h, const int32_t* residual, int tr_hor, int tr_ver,
                              int extra_skip_w, int extra_skip_h, int bd, int32_t* out);
int inverse_transform_rect_bd(int w, int h, const int32_t* coeffs, int tr_hor, int tr_ver,
                              int extra_skip_w, int extra_skip_h, int bd, int32_t* out);
int quantize_rect_bd(int w, int h, const int32_t* coeffs, int qp_scaled, int bd, bool is_intra,
                     int32_t* out);
int dequantize_rect_bd(int w, int h, const int32_t* levels, int qp_scaled, int bd, int32_t* out);
int dequantize_dep_quant_bd(int w, int h, const int32_t* levels, const int32_t* scan_raster,
                            int qp_scaled, int bd, int32_t* out);
int quantize_dep_quant_bd(int w, int h, const int32_t* coeffs, const int32_t* scan_raster,
                          int qp_scaled, int bd, int32_t* out);

// ---- transform.rs -------------------------------------------------------------
// Grouped diagonal scan; returns the number of scan positions written.
int coeff_scan_raster(int w, int h, int32_t* raster);
int32_t quantize_ts(int32_t residual, int qp);
int32_t dequantize_ts(int32_t level, int qp);

// ---- lfnst.rs -----------------------------------------------------------------
int get_lfnst_intra_mode(int mode);
int inverse_lfnst_rect(int32_t* coeffs, int w, int h, int lfnst_idx, int intra_mode);
int forward_lfnst_rect(int32_t* coeffs, int w, int h, int lfnst_idx, int intra_mode);

// ---- predict.rs (16-bit sample planes) ----------------------------------------
struct Plane16 {
  uint16_t* data;
  int width;
  int height;
  int bd;
  uint16_t get(int x, int y) const { return data[(size_t)y * width + x]; }
  void set(int x, int y, int v) {
    int mx = (1 << bd) - 1;
    data[(size_t)y * width + x] = (uint16_t)(v > mx ? mx : v);
  }
};

// predict.rs:987-1030 Plane: row-major 8-bit samples, stride = width
struct Plane8 {
  const uint8_t* data;
  int width;
  int height;
  int get(int x, int y) const { return data[(size_t)y * width + x]; }
};

struct Refs16 {
  int top_left;
  std::vector<int> above;  // 2 * width
  std::vector<int> left;   // 2 * height
  int bd;
};

// Coded-unit availability map of the 10-bit frame path (slice.rs CodedUnits).
struct CodedMap {
  const uint8_t* coded;
  int grid_w, grid_h, tb;
  bool is_coded_luma(int x, int y) const {
    int gx = x / tb, gy = y / tb;
    return gx < grid_w && gy < grid_h && coded[gy * grid_w + gx];
  }
};

Refs16 gather_references_16(const Plane16& p, int x, int y, int w, int h);
void predict_from_refs_16(const Refs16& refs, int w, int h, bool is_luma, int mode, uint16_t* out);
void predict_block_16(const Plane16& p, int x, int y, int w, int h, bool is_luma, int mode,
                      uint16_t* out);
void predict_coded_block_16(const Plane16& p, int x, int y, int w, int h, bool is_luma, int mode,
                            int scale_x, int scale_y, const CodedMap& cm, uint16_t* out);
// cclm_mode: 0 = LM (LT), 1 = LM-L, 2 = LM-T; chroma_format 1 = 4:2:0, 2 = 4:2:2, 3 = 4:4:4
void predict_cclm_with_format_16(const Plane16& luma, const Plane16& chroma, int bxc, int byc,
                                 int cw, int ch, int cclm_mode, int chroma_format, int ctu_size,
                                 uint16_t* out);
int choose_intra_mode_16(const Plane16& recon, const Plane16& src, int bx, int by, int w, int h,
                         bool is_luma);

struct AngularParams {
  int pred_mode;
  bool is_mode_ver;
  int intra_pred_angle;
  int abs_inv_angle;
  bool ref_filter_flag;
  bool interpolation_flag;
  bool apply_pdpc;
  int angular_scale;
  int ref_w, ref_h;  // refW / refH (H.266 8.4.5.2.6)
};
AngularParams init_angular_params(int dir_mode, int pu_w, int pu_h, int cu_w, int cu_h,
                                  bool is_luma, int mrl_idx, bool use_isp);
int get_modified_wide_angle(int w, int h, int mode);

// ---- filter.rs (16-bit) ---------------------------------------------------------
void deblock_luma_plane_16(Plane16& p, int cu_step, int ctb_size, int qp, int bs, int beta_off,
                           int tc_off);
void deblock_chroma_plane_16(Plane16& p, int cu_step, int ctb_height_c, int qp_c, int bs,
                             int beta_off, int tc_off, int sub_w, int sub_h);
struct Sao {
  int type;  // 0 off, 1 band offset, 2 edge offset
  int band_pos_or_class;
  int offsets[4];
};
// Returns -1 (without writing) where the reference aborts: see orc_filter.cpp.
int apply_sao_region_16(const Plane16& src, Plane16& dst, int bx, int by, int w, int h,
                        const Sao& sao);
// filter.rs:1954-2033 / decode_general.rs:5189-5223: the general decoder's SAO of one plane.
void sao_plane_bounded_16(const uint16_t* src, uint16_t* dst, int stride, int pw, int ph, int vis_w, int vis_h,
                          int bd, int ctu, int ctu_cols, const Sao* params);
// predict.rs:2088-2177 derive_cclm_params_from_4_samples (sl / sc reordered in place).
void cclm_params(int sl[4], int sc[4], int cnt, int bd, int* a_out, int* b_out, int* shift_out);
// decode_general.rs:4001-4024 / :4260-4793: the general decoder's intra prediction of one block.
void gen_intra_predict(const vvcg_gen_intra_state& st, const vvcg_gen_intra_req& r, int16_t* out);
// predict.rs:2737-2801 choose_luma_intra_pred_mode (+ the multi-tool encoder's
// MRL candidates, slice.rs:2698-2731) and predict_block_full (:2655) on 8-bit planes.
void luma_intra_search_8(const Plane8& recon, const Plane8& src, int bx, int by, int w, int h, const uint8_t mpm[6],
                         bool mpm_only, bool mrl, int ctu_size, int* best_mode, int* best_mrl, uint64_t* best_sad);
void predict_luma_8(const Plane8& recon, int bx, int by, int w, int h, int mode, int mrl, int ctu_size, int32_t* out);
// predict.rs:2619 predict_block: Planar / DC / angular of one component block on an 8-bit plane.
void predict_block_8(const Plane8& recon, int bx, int by, int w, int h, bool is_luma, int mode, int32_t* out);
// slice.rs:325-455 encode_picture (decisions and reconstruction; no CABAC) and
// slice.rs:458-627 decode_picture (reconstruction from parsed syntax) of the
// strict 8-bit 4:2:0 intra profile (orc_strict.cpp). Records as vvcg_cu_rec
// documents for VVCG_TOOL_TU_TOOLS pictures; planes row-major, stride = width.
int strict_encode(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h, int qp, int ctu_log2,
                  vvcg_cu_rec* cus, int16_t* levels, uint64_t* num_levels, uint8_t* ry, uint8_t* ru, uint8_t* rv);
int strict_decode(const vvcg_cu_rec* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                  int ctu_log2, uint8_t* ry, uint8_t* ru, uint8_t* rv);
// orc_cabac.cpp: the encoder side of CABAC (cabac.rs BinEncoder, residual.rs
// encode_residual_with_options, slice.rs encode_ts_block and encode_picture's
// syntax writes) for records as strict_encode returns them, and for one block.
int strict_write(const vvcg_cu_rec* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                 std::vector<uint8_t>* out);
int block_write(const int32_t* c, int w, int h, bool luma, bool dq, bool sdh, bool ts, int qp,
                std::vector<uint8_t>* out);
// orc_multitool.cpp: the multi-tool stream (VvcMultiToolEncoder): IDR
// pictures (encode_picture_multitool slice.rs:2575 / decode_picture_multitool
// :3012) as vvcg_cu_rec records, P pictures (encode_inter_picture :3307 /
// decode_inter_picture :3552) as vvcg_inter_cu records; opts VVCG_SLICE_*;
// refs: num_refs L0 pictures of three 8-bit planes each.
void derive_intra_mpms(int left_dir, int above_dir, uint8_t mpm[6]);
int mt_encode(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h, int qp, int ctu_log2,
              uint32_t opts, vvcg_cu_rec* cus, int16_t* levels, uint64_t* num_levels, uint8_t* ry, uint8_t* ru,
              uint8_t* rv);
int mt_decode(const vvcg_cu_rec* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp, int ctu_log2,
              uint32_t opts, uint8_t* ry, uint8_t* ru, uint8_t* rv);
int inter_encode(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h, int qp, int ctu_log2,
                 uint32_t opts, const uint8_t* const* refs, int num_refs, vvcg_inter_cu* cus, int16_t* levels,
                 uint64_t* num_levels, uint8_t* ry, uint8_t* ru, uint8_t* rv);
int inter_resolve_motion(vvcg_inter_cu* cus, int w, int h, int ctu_log2);
int inter_decode(const vvcg_inter_cu* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                 int ctu_log2, uint32_t opts, const uint8_t* const* refs, int num_refs, uint8_t* ry, uint8_t* ru,
                 uint8_t* rv);
void inter_ctu_cells(const vvcg_inter_cu* cus, int w, int h, int ctu, vvcg_ctu_motion* cells);
// orc_cabac.cpp: the slice data encode_picture_multitool and
// encode_inter_picture write for such records.
int mt_write(const vvcg_cu_rec* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
             uint32_t opts, std::vector<uint8_t>* out);
int p_write(const vvcg_inter_cu* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
            uint32_t opts, std::vector<uint8_t>* out);
// The GPU encoder's CTU full search (orc_search.cpp; no reference counterpart).
void ctu_search(const Plane16& src, int cx, int cy, int split_mask, int n_cand, const uint8_t* cand,
                uint32_t lambda_q8, uint32_t* cost, uint32_t split_cost[6], int* split, int* cu_mode, int modes[4]);
// slice.rs:4111-4167: the quadrant-mean partition hook (orc_search.cpp).
int qt_mtt_split(const Plane16& src, int64_t bx, int64_t by, int64_t w, int64_t h, int qp, int64_t min_cb);
// decode_general.rs:4916-4975 / filter.rs:202-226: general-decoder deblocking helpers.
void dbk_luma_lens(int size_p, int size_q, int* lp, int* lq);
void dbk_chroma_lens(int size_p, int size_q, bool ctb_boundary, int* lp, int* lq);
int dbk_boundary_strength(bool p_intra, bool q_intra, bool p_cbf, bool q_cbf, bool tu_edge, int pmv_h,
                          int pmv_v, int qmv_h, int qmv_v, int pref, int qref);
// decode_general.rs:4977-5187 apply_deblock on a 4:2:0 picture, in place.
void inter_ctu_deblock(uint16_t* const planes[3], const int stride[3], int w, int h, int ctu, int qp,
                       const vvcg_ctu_motion* cells);
void deblock_general(uint16_t* const planes[3], const int stride[3], int vis_w, int vis_h, int bd, int ctu,
                     const vvcg_dbk_cell* cells, int cols, int rows, const vvcg_dbk_ccell* cc, int ccols,
                     int crows, const vvcg_dbk_params& prm);
struct AlfAps {
  int num_luma_filters;  // 0 = fixed filters of the class
  bool luma_clip;
  uint8_t coeff_delta_idx[25];
  int16_t coeff[25][12];
  uint8_t clip_idx[25][12];
};
// Sets g_alf_status to -1 where the reference would abort (see orc_filter.cpp).
extern int g_alf_status;
void apply_alf_luma_plane_16(Plane16& p, const AlfAps& aps);
void classify_alf_4x4_16(const Plane16& p, int bx, int by, int* class_idx, int* transpose_idx);

// ---- inter.rs (16-bit) ----------------------------------------------------------
void interpolate_luma_block_16(const Plane16& ref, int bx, int by, int w, int h, int mv_x,
                               int mv_y, bool bi, bool affine, bool alt_hpel, int32_t* out);
void interpolate_chroma_block_format_16(const Plane16& ref, int bxc, int byc, int cw, int ch,
                                        int mv_x, int mv_y, bool bi, int chroma_format,
                                        int32_t* out);
void weighted_average_bi_16(const int32_t* p0, const int32_t* p1, int n, int bcw_idx, int bd,
                            uint16_t* out);
// ---- inter.rs (8-bit planes) ------------------------------------------------------
void interpolate_luma_block_8(const uint8_t* ref, int pw, int ph, int stride, int bx, int by, int w, int h,
                              int mv_x, int mv_y, bool bi, bool alt_hpel, bool affine, int32_t* out);
void interpolate_chroma_block_420_8(const uint8_t* ref, int pw, int ph, int stride, int cx, int cy, int cw,
                                    int ch, int mv_x, int mv_y, bool bi, int32_t* out);
void weighted_average_bi_8(const int32_t* p0, const int32_t* p1, int n, int bcw_idx, int32_t* out);
// inter.rs:1866-2003 estimate_inter_block on 8-bit planes of one size and stride.
void estimate_inter_block_8(const uint8_t* src, const uint8_t* const* l0, int n0, const uint8_t* const* l1, int n1,
                            int pw, int ph, int stride, const vvcg_mv_cand* cands, int ncand, int amvp_x, int amvp_y,
                            int bx, int by, int w, int h, int range, vvcg_me_res* res);

// ---- transform units (orc_tu.cpp) ------------------------------------------------
// Same layout and flag values as vvcg_tu_rec / VVCG_TU_* of the C ABI.
enum : uint8_t {
  kTuDepQuant = 1,
  kTuTransformSkip = 2,
  kTuBdpcmHor = 4,
  kTuBdpcmVer = 8,
  kTuImplicitMts = 16,
  kTuInter = 32,
};
struct TuRec {
  uint8_t log2_w, log2_h, bit_depth, qp, flags, mts_idx, lfnst_idx, lfnst_mode;
  uint32_t in_off, out_off;
};
static_assert(sizeof(TuRec) == 16, "TuRec layout");
// Return 0, or a negative code where the reference returns an error.
int tu_inverse(const TuRec& r, const int16_t* in, int16_t* out);
int tu_forward(const TuRec& r, const int16_t* in, int16_t* out);

// ---- hls.rs ---------------------------------------------------------------------
int scaled_luma_qp_bd(int qpy, int bd);
int derived_chroma_qp_bd(int qpy, int bd, int chroma_qp_offset);
int derived_chroma_qp(int qp);

}  // namespace orc
