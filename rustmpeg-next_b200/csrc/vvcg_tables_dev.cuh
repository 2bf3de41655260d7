// Device copies of the normative H.266 tables (vvc_tables.h) used by the
// kernels. Small tables live in constant memory (warp-uniform indices); the
// transform matrices live in global memory and are staged into shared memory.
// They are filled once per device by upload_tables() (vvcg.cu).
#pragma once
#include <stdint.h>

namespace vvcg {

__constant__ int c_ang_table[32];
__constant__ int c_inv_ang_table[32];
__constant__ int c_intra_filter_thr[8];
__constant__ int8_t c_chroma_taps4[128];
__constant__ uint8_t c_cclm_div_sig[16];
__constant__ int c_inv_quant_scale[2][6];
__constant__ int c_quant_scale[2][6];
__constant__ int16_t c_dbf_tc[66];
__constant__ int16_t c_dbf_beta[64];
__constant__ int8_t c_luma_taps8[128];
__constant__ int8_t c_affine_taps8[128];
__constant__ int c_luma_alt_hpel[8];
__constant__ int c_bcw_weights[5];
__constant__ int c_alf_clip[3][4];
__constant__ int8_t c_alf_fixed[64 * 13];
__constant__ uint8_t c_alf_class_to_filter[16 * 25];
__constant__ uint8_t c_alf_transpose_perm[48];

// DCT-II / DST-VII / DCT-VIII matrices, row k = basis function k.
__device__ int8_t g_dct2_m[6][64 * 64];  // N = 2, 4, 8, 16, 32, 64
__device__ int8_t g_dst7_m[4][32 * 32];  // N = 4, 8, 16, 32
__device__ int8_t g_dct8_m[4][32 * 32];
// Grouped diagonal scans (raster index per scan position) for every
// (log2 w, log2 h) in 1..6 x 1..6, and their offsets into g_scan.
__device__ int16_t g_scan[36 * 1024];
__device__ int32_t g_scan_off[36];
// Inverse of g_scan for TBs of at most 32x32: scan position of each raster
// index (same offsets as g_scan).
__device__ int16_t g_scan_pos[36 * 1024];

}  // namespace vvcg
