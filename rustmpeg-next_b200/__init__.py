"""rustmpeg-next_b200: B200 (sm_100a) VVC reconstruction, loop filtering and
motion compensation behind the C ABI of include/vvcg.h (libvvcg.so).

This module is the Python binding of that ABI (ctypes): the record layouts as
numpy dtypes, a context class, and typed errors that mirror the reference's
AcceleratorError (crates/rustmpeg-video/src/accelerator.rs:17-31). All
computation happens in the CUDA library; there is no CPU fallback, and every
call raises when the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libvvcg.so")
CSRC = os.path.join(HERE, "csrc")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]

# ------------------------------------------------------------------ records --
CU_DTYPE = np.dtype([("luma_mode", "u1"), ("chroma_mode", "u1"), ("cbf", "u1"),
                     ("tu_tools", "u1"), ("level_off", "<i4", (3,))])
SAO_DTYPE = np.dtype([("type", "u1"), ("band_or_class", "u1"), ("offsets", "i1", (4,))])
CTU_DTYPE = np.dtype([("sao", SAO_DTYPE, (3,)), ("alf_luma", "u1"), ("reserved", "u1")])
PIC_DTYPE = np.dtype([("width", "<u4"), ("height", "<u4"), ("visible_width", "<u4"),
                      ("visible_height", "<u4"), ("bit_depth", "u1"), ("chroma_format", "u1"),
                      ("ctu_log2", "u1"), ("slice_qp", "u1"), ("chroma_qp_scaled", "u1"),
                      ("tools", "u1"), ("alf_aps", "<i2"), ("cu_offset", "<u4"),
                      ("ctu_offset", "<u4")])
APS_DTYPE = np.dtype([("num_luma_filters", "u1"), ("luma_clip", "u1"),
                      ("coeff_delta_idx", "u1", (25,)), ("reserved", "u1"),
                      ("coeff", "<i2", (25, 12)), ("clip_idx", "u1", (25, 12))])
MC_BLOCK_DTYPE = np.dtype([("x", "<i4"), ("y", "<i4"), ("w", "<u2"), ("h", "<u2"),
                           ("mv_x", "<i4"), ("mv_y", "<i4"), ("flags", "<u4"),
                           ("reserved", "<u4"), ("out_offset", "<u8")], align=True)

LMCS_APS_DTYPE = np.dtype([("bin_cw_delta", "<i2", (16,)), ("min_bin_idx", "u1"), ("max_bin_idx", "u1"),
                           ("chroma_res_scaling_offset", "i1"), ("reserved", "u1")])
LMCS_TABLES_DTYPE = np.dtype([("bit_depth", "u1"), ("min_bin_idx", "u1"), ("max_bin_idx", "u1"),
                              ("reserved", "u1"), ("reshape_pivot", "<i4", (17,)), ("chroma_adj_lut", "<i4", (16,)),
                              ("fwd_lut", "<u2", (4096,)), ("inv_lut", "<u2", (4096,))])
CRES_DTYPE = np.dtype([("log2_w", "u1"), ("log2_h", "u1"), ("bit_depth", "u1"), ("joint", "i1"),
                       ("flags", "<u4"), ("scale", "<i4"), ("cb_off", "<u4"), ("cr_off", "<u4")])
CRES_SCALE, CRES_SINGLE = 1, 2
ALF_CTU_DTYPE = np.dtype([("luma_mode", "u1"), ("luma_set", "u1"), ("cb_alt", "u1"), ("cr_alt", "u1"),
                          ("cc_cb", "u1"), ("cc_cr", "u1"), ("reserved", "u1", (2,))])
ALF_PARAMS_DTYPE = np.dtype([("num_luma_filters", "u1"), ("luma_clip", "u1"), ("num_chroma_filters", "u1"),
                             ("chroma_clip", "u1"), ("num_cc_cb", "u1"), ("num_cc_cr", "u1"),
                             ("reserved", "u1", (2,)), ("coeff_delta_idx", "u1", (25,)), ("reserved2", "u1", (3,)),
                             ("luma_coeff", "<i2", (25, 12)), ("luma_clip_idx", "u1", (25, 12)),
                             ("chroma_coeff", "<i2", (8, 6)), ("chroma_clip_idx", "u1", (8, 6)),
                             ("cc_cb", "<i2", (4, 7)), ("cc_cr", "<i2", (4, 7))])
ALF_OFF, ALF_FIXED, ALF_APS = 0, 1, 2
ISR_REQ_DTYPE = np.dtype([("x", "<u4"), ("y", "<u4"), ("log2_w", "u1"), ("log2_h", "u1"), ("flags", "u1"),
                          ("log2_ctu", "u1"), ("mpm", "u1", (6,)), ("reserved", "u1", (2,))])
ISR_RES_DTYPE = np.dtype([("sad", "<u8"), ("mode", "u1"), ("mrl_idx", "u1"), ("reserved", "u1", (6,))])
ISR_MPM_ONLY, ISR_MRL = 1, 2
CTU_SEARCH_REQ_DTYPE = np.dtype([("x", "<u4"), ("y", "<u4"), ("split_mask", "u1"), ("n_cand", "u1"),
                                 ("cand", "u1", (6,))])
CTU_SEARCH_RES_DTYPE = np.dtype([("cost", "<u4"), ("split_cost", "<u4", (6,)), ("split", "u1"), ("cu_mode", "u1"),
                                 ("modes", "u1", (4,)), ("reserved", "u1", (2,))])
SPLIT_NONE, SPLIT_QT, SPLIT_BT_H, SPLIT_BT_V, SPLIT_TT_H, SPLIT_TT_V = range(6)
MV_CAND_DTYPE = np.dtype([("mv", "<i4", (2, 2)), ("ref_idx", "i1", (2,)), ("inter_dir", "u1"), ("bcw_idx", "u1"),
                          ("alt_hpel", "u1"), ("reserved", "u1", (3,))])
ME_REQ_DTYPE = np.dtype([("x", "<u4"), ("y", "<u4"), ("w", "<u2"), ("h", "<u2"), ("cand_off", "<u4"),
                         ("num_cands", "<u2"), ("search_range", "<u2"), ("amvp", "<i4", (2,))])
ME_RES_DTYPE = np.dtype([("sad", "<u8"), ("cand", MV_CAND_DTYPE), ("merge_idx", "<u2"), ("is_merge", "u1"),
                         ("reserved", "u1", (5,))])
SPLIT_REQ_DTYPE = np.dtype([("x", "<u4"), ("y", "<u4"), ("w", "<u2"), ("h", "<u2"), ("min_cb", "<u2"), ("qp", "u1"),
                            ("reserved", "u1")])
CNN_PARAMS, CNN_OUT, CNN_MODES, CNN_SPLITS = 30761, 73, 67, 6
GEN_INTRA_REQ_DTYPE = np.dtype([("x", "<u2"), ("y", "<u2"), ("w", "<u2"), ("h", "<u2"), ("cu_x", "<u2"),
                                ("cu_y", "<u2"), ("cu_w", "<u2"), ("cu_h", "<u2"), ("comp", "u1"), ("mode", "u1"),
                                ("mrl", "u1"), ("isp", "u1"), ("bdpcm", "u1"), ("reserved", "u1", (3,)),
                                ("out_off", "<u4")])
ISP_NONE, ISP_HOR, ISP_VER = 0, 1, 2
BDPCM_NONE, BDPCM_HOR, BDPCM_VER = 0, 1, 2


class _GenIntraState(C.Structure):
    _fields_ = [("plane", C.c_void_p * 3), ("stride", C.c_uint32 * 3), ("width", C.c_uint32),
                ("height", C.c_uint32), ("dec_y", C.c_void_p), ("dec_c", C.c_void_p), ("bit_depth", C.c_uint8),
                ("vert_collocated", C.c_uint8), ("reserved", C.c_uint8 * 2), ("ctu_size", C.c_uint32)]


DBK_CELL_DTYPE = np.dtype([("tu_id", "<u4"), ("tu_w", "<u2"), ("tu_h", "<u2"), ("mv", "<i4", (2, 2)),
                           ("ref_idx", "i1", (2,)), ("flags", "u1"), ("reserved", "u1")])
DBK_CCELL_DTYPE = np.dtype([("tu_cb", "<u4"), ("tu_cr", "<u4"), ("tu_w", "<u2"), ("tu_h", "<u2")])
DBK_PARAMS_DTYPE = np.dtype([("qp", "<i4", (3,)), ("beta_offset_div2", "<i4", (3,)), ("tc_offset_div2", "<i4", (3,)),
                             ("num_ref", "<i4", (2,)), ("ref_poc", "<i4", (2, 16))])
DBK_CODED, DBK_INTRA, DBK_CBF = 1, 2, 4
CTU_MOTION_DTYPE = np.dtype([("mv", "<i4", (3, 2)), ("ref", "<i4", (3,)), ("cbf", "u1"), ("reserved", "u1", (3,))])
BDOF_REQ_DTYPE = np.dtype([("w", "<u2"), ("h", "<u2"), ("off", "<u4")])
DMVR_REQ_DTYPE = np.dtype([("bx", "<i4"), ("by", "<i4"), ("dx", "<u2"), ("dy", "<u2"), ("mv", "<i4", (2, 2))])
AFFINE_REQ_DTYPE = np.dtype([("cp", "<i4", (3, 2)), ("w", "<u2"), ("h", "<u2"), ("six_param", "u1"),
                             ("inter_dir", "u1"), ("reserved", "u1", (2,)), ("sub_off", "<u4")])
PROF_REQ_DTYPE = np.dtype([("src_off", "<u4"), ("dmv_off", "<u4"), ("out_off", "<u4"), ("bi", "u1"),
                           ("reserved", "u1", (3,))])
CIIP_REQ_DTYPE = np.dtype([("n", "<u4"), ("off", "<u4"), ("left_intra", "u1"), ("above_intra", "u1"),
                           ("reserved", "u1", (2,))])
GPM_REQ_DTYPE = np.dtype([("w", "<u2"), ("h", "<u2"), ("split_dir", "u1"), ("scale_x", "u1"), ("scale_y", "u1"),
                          ("reserved", "u1"), ("off", "<u4")])
DBK_NO_TU = 0xFFFFFFFF
MIP_REQ_DTYPE = np.dtype([("log2_w", "u1"), ("log2_h", "u1"), ("bit_depth", "u1"), ("mode", "u1"),
                          ("transposed", "u1"), ("reserved", "u1", (3,)), ("ref_off", "<u4"), ("out_off", "<u4")])
MIP_RES_DTYPE = np.dtype([("sad", "<u8"), ("mode", "u1"), ("transposed", "u1"), ("reserved", "u1", (6,))])
MIP_SEARCH = 0xFF
TXS_REQ_DTYPE = np.dtype([("log2_size", "u1"), ("qp", "u1"), ("mode", "u1"), ("flags", "u1"),
                          ("in_off", "<u4"), ("out_off", "<u4"), ("reserved", "<u4")])
TXS_RES_DTYPE = np.dtype([("sse", "<u8"), ("mts_idx", "u1"), ("lfnst_idx", "u1"), ("transform_skip", "u1"),
                          ("cbf", "u1"), ("reserved", "<u4")])
TXS_TRANSFORM_SKIP, TXS_LFNST = 1, 2
TU_DTYPE = np.dtype([("log2_w", "u1"), ("log2_h", "u1"), ("bit_depth", "u1"), ("qp", "u1"),
                     ("flags", "u1"), ("mts_idx", "u1"), ("lfnst_idx", "u1"),
                     ("lfnst_mode", "u1"), ("in_off", "<u4"), ("out_off", "<u4")])

GEN_TB_DTYPE = np.dtype([("pred", GEN_INTRA_REQ_DTYPE), ("tu", TU_DTYPE), ("coded", "<u4")])
GEN_PIC_DTYPE = np.dtype([("width", "<u4"), ("height", "<u4"), ("vis_width", "<u4"), ("vis_height", "<u4"),
                          ("bit_depth", "u1"), ("ctu_log2", "u1"), ("vert_collocated", "u1"), ("tools", "u1"),
                          ("group_offset", "<u4"), ("num_groups", "<u4"), ("sao_offset", "<u4"),
                          ("alf_offset", "<u4"), ("alf_params", "<i4"), ("dbk", DBK_PARAMS_DTYPE)])

TOOL_DEP_QUANT, TOOL_DEBLOCK, TOOL_SAO, TOOL_ALF = 1, 2, 4, 8
TOOL_ENC_FULL_INTRA, TOOL_ENC_CCLM, TOOL_SPARSE_LEVELS, TOOL_TU_TOOLS = 16, 32, 64, 128
CU_TS_Y, CU_TS_CB, CU_TS_CR, CU_MTS_SHIFT, CU_LFNST_SHIFT = 1, 2, 4, 3, 6
# the multi-tool stream (vvcg.h VVCG_SLICE_*, VVCG_INTER_CU_*, vvcg_inter_cu, vvcg_p_pic)
SLICE_DEP_QUANT, SLICE_SIGN_HIDING, SLICE_DEBLOCK, SLICE_FULL_INTRA_MODES = 1, 2, 4, 8
INTER_CU_MERGE, INTER_CU_SKIP, INTER_CU_ALT_HPEL = 1, 2, 4
INTER_CU_DTYPE = np.dtype([("mv", "<i4", (2, 2)), ("mvd", "<i4", (2,)), ("ref_idx", "i1", (2,)), ("inter_dir", "u1"),
                           ("bcw_idx", "u1"), ("flags", "u1"), ("mvp_idx", "u1"), ("cbf", "u1"), ("tu_tools", "u1"),
                           ("level_off", "<i4", (3,)), ("reserved", "<u4")])
P_PIC_DTYPE = np.dtype([("width", "<u4"), ("height", "<u4"), ("qp", "u1"), ("options", "u1"), ("num_refs", "u1"),
                        ("sparse", "u1"), ("ref_slot", "<i4", (4,)), ("out_slot", "<i4"), ("cu_offset", "<u4")])
assert INTER_CU_DTYPE.itemsize == 48 and P_PIC_DTYPE.itemsize == 36
TU_DEP_QUANT, TU_TRANSFORM_SKIP, TU_BDPCM_HOR, TU_BDPCM_VER, TU_IMPLICIT_MTS, TU_INTER = 1, 2, 4, 8, 16, 32
STAGE_RECON, STAGE_DEBLOCK, STAGE_SAO, STAGE_ALF, STAGE_ALL = 1, 2, 4, 8, 15
MC_BI, MC_AFFINE, MC_ALT_HPEL = 1, 2, 4
CHROMA_400, CHROMA_420, CHROMA_422, CHROMA_444 = 0, 1, 2, 3

OK, INVALID_INPUT, LIMIT_EXCEEDED, UNAVAILABLE, EXECUTION, TIMEOUT, MISMATCH = range(7)


class AcceleratorError(RuntimeError):
    """Base of the typed errors (reference AcceleratorError)."""

    status = EXECUTION


class Unavailable(AcceleratorError):
    status = UNAVAILABLE


class InvalidInput(AcceleratorError):
    status = INVALID_INPUT


class LimitExceeded(AcceleratorError):
    status = LIMIT_EXCEEDED


class Execution(AcceleratorError):
    status = EXECUTION


class Timeout(Execution):
    status = TIMEOUT


class Mismatch(Execution):
    status = MISMATCH


_ERRORS = {INVALID_INPUT: InvalidInput, LIMIT_EXCEEDED: LimitExceeded, UNAVAILABLE: Unavailable,
           EXECUTION: Execution, TIMEOUT: Timeout, MISMATCH: Mismatch}


class _Batch(C.Structure):
    _fields_ = [("pics", C.c_void_p), ("num_pics", C.c_uint32), ("num_cus", C.c_uint32),
                ("cus", C.c_void_p), ("levels", C.c_void_p), ("num_levels", C.c_uint64),
                ("ctus", C.c_void_p), ("num_ctus", C.c_uint32), ("num_aps", C.c_uint32),
                ("aps", C.c_void_p)]


class _GenBatch(C.Structure):
    _fields_ = [("pics", C.c_void_p), ("num_pics", C.c_uint32), ("num_groups", C.c_uint32),
                ("tbs", C.c_void_p), ("group_first", C.c_void_p), ("num_tbs", C.c_uint64),
                ("levels", C.c_void_p), ("num_levels", C.c_uint64), ("slot_count", C.c_uint64),
                ("sao", C.c_void_p), ("num_sao", C.c_uint64), ("alf_ctus", C.c_void_p),
                ("num_alf_ctus", C.c_uint64), ("alf_params", C.c_void_p), ("num_alf_params", C.c_uint32),
                ("reserved", C.c_uint32)]


class _StrictSubstream(C.Structure):
    _fields_ = [("data", C.c_void_p), ("size", C.c_uint64), ("width", C.c_uint32), ("height", C.c_uint32),
                ("qp", C.c_uint8), ("reserved", C.c_uint8 * 3), ("cu_offset", C.c_uint32),
                ("level_offset", C.c_uint64), ("level_cap", C.c_uint64)]


class _SliceSubstream(C.Structure):
    _fields_ = [("data", C.c_void_p), ("size", C.c_uint64), ("width", C.c_uint32), ("height", C.c_uint32),
                ("qp", C.c_uint8), ("ctu_log2", C.c_uint8), ("options", C.c_uint8), ("reserved", C.c_uint8),
                ("cu_offset", C.c_uint32), ("level_offset", C.c_uint64), ("level_cap", C.c_uint64)]


class _PlaneOut(C.Structure):
    _fields_ = [("data", C.c_void_p), ("stride", C.c_uint32), ("reserved", C.c_uint32)]


class _PlaneIn(C.Structure):
    _fields_ = [("data", C.c_void_p), ("stride", C.c_uint32), ("reserved", C.c_uint32)]


class _Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("flags", C.c_uint32), ("reserve_bytes", C.c_uint64),
                ("spin_limit", C.c_uint32), ("reserved", C.c_uint32)]


assert C.sizeof(_Batch) == 64 and CU_DTYPE.itemsize == 16 and PIC_DTYPE.itemsize == 32
assert CTU_DTYPE.itemsize == 20 and MC_BLOCK_DTYPE.itemsize == 40 and TU_DTYPE.itemsize == 16
assert TXS_REQ_DTYPE.itemsize == 16 and TXS_RES_DTYPE.itemsize == 16
assert MIP_REQ_DTYPE.itemsize == 16 and MIP_RES_DTYPE.itemsize == 16
assert ALF_CTU_DTYPE.itemsize == 8 and ALF_PARAMS_DTYPE.itemsize == 1192
assert ISR_REQ_DTYPE.itemsize == 20 and ISR_RES_DTYPE.itemsize == 16
assert CTU_SEARCH_REQ_DTYPE.itemsize == 16 and CTU_SEARCH_RES_DTYPE.itemsize == 36
assert GEN_INTRA_REQ_DTYPE.itemsize == 28
assert DBK_CELL_DTYPE.itemsize == 28 and DBK_CCELL_DTYPE.itemsize == 12 and DBK_PARAMS_DTYPE.itemsize == 172
assert CTU_MOTION_DTYPE.itemsize == 40 and BDOF_REQ_DTYPE.itemsize == 8 and DMVR_REQ_DTYPE.itemsize == 28
assert AFFINE_REQ_DTYPE.itemsize == 36 and PROF_REQ_DTYPE.itemsize == 16 and CIIP_REQ_DTYPE.itemsize == 12
assert GPM_REQ_DTYPE.itemsize == 12
assert GEN_TB_DTYPE.itemsize == 48 and GEN_PIC_DTYPE.itemsize == 212
assert LMCS_APS_DTYPE.itemsize == 36 and LMCS_TABLES_DTYPE.itemsize == 16520 and CRES_DTYPE.itemsize == 20


def build(force: bool = False) -> str:
    """Compile csrc/vvcg.cu for sm_100a into lib/libvvcg.so (nvcc cross-compiles without a GPU)."""
    srcs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    newest = max(os.path.getmtime(s) for s in srcs + [os.path.join(HERE, "..", "include", "vvcg.h")])
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= newest:
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = ["nvcc", *NVCC_FLAGS, "-o", LIB_PATH, os.path.join(CSRC, "vvcg.cu")]
    subprocess.run(cmd, check=True)
    return LIB_PATH


_lib = None


def lib():
    """Load libvvcg.so (raises Unavailable when it was never built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise Unavailable(f"libvvcg.so is not built ({LIB_PATH}); run build()")
        L = C.CDLL(LIB_PATH)
        vp, u32, u64, u8 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint8
        L.vvcg_ctx_create.argtypes = [vp, C.POINTER(vp)]
        L.vvcg_ctx_destroy.argtypes = [vp]
        L.vvcg_ctx_destroy.restype = None
        L.vvcg_last_error.argtypes = [vp]
        L.vvcg_last_error.restype = C.c_char_p
        L.vvcg_set_stream.argtypes = [vp, vp]
        L.vvcg_kernel_launches.argtypes = [vp]
        L.vvcg_kernel_launches.restype = u64
        for n in ("vvcg_batch_prepare", "vvcg_batch_upload"):
            getattr(L, n).argtypes = [vp, vp]
        L.vvcg_decode_batch.argtypes = [vp, vp, vp]
        L.vvcg_decode_batch_pipelined.argtypes = [vp, vp, vp, u32, u32]
        L.vvcg_decode_batch_async.argtypes = [vp, vp, vp]
        L.vvcg_batch_run.argtypes = [vp, u32]
        L.vvcg_batch_run_graph.argtypes = [vp, u32]
        L.vvcg_batch_sync.argtypes = [vp]
        L.vvcg_batch_download.argtypes = [vp, vp]
        L.vvcg_batch_plane.argtypes = [vp, u32, u32, C.POINTER(vp), C.POINTER(u32)]
        L.vvcg_mc_luma_16_dev.argtypes = [vp, vp, u32, u32, u32, u8, vp, u32, vp]
        L.vvcg_mc_chroma_16_dev.argtypes = [vp, vp, u32, u32, u32, u8, u8, vp, u32, vp]
        L.vvcg_mc_bi_average_16_dev.argtypes = [vp, vp, vp, u64, u8, u8, vp]
        L.vvcg_mc_luma_8_dev.argtypes = [vp, vp, u32, u32, u32, vp, u32, vp]
        L.vvcg_mc_chroma_420_8_dev.argtypes = [vp, vp, u32, u32, u32, vp, u32, vp]
        for n in ("vvcg_tu_inverse_batch", "vvcg_tu_forward_batch"):
            getattr(L, n).argtypes = [vp, vp, u32, vp, u64, vp, u64]
        L.vvcg_tu_autotune.argtypes = [vp, vp, u32, vp, u64, vp, u64, u32, vp]
        L.vvcg_qt_mtt_split_dev.argtypes = [vp, vp, u64, u32, u32, u8, vp, u32, vp]
        L.vvcg_inter_search_8_dev.argtypes = [vp, vp, u64, u32, u32, vp, u32, vp, u32, vp, u32, vp, u32, vp]
        L.vvcg_encode_sizes.argtypes = [vp, u32, C.POINTER(u32), C.POINTER(u64)]
        L.vvcg_encode_batch.argtypes = [vp, vp, u32, vp, vp, u32, vp, u64]
        for n in ("vvcg_plane_metrics_8_dev", "vvcg_plane_metrics_16_dev"):
            getattr(L, n).argtypes = [vp, vp, u64, vp, u64, u32, u32, vp]
        L.vvcg_luma_tx_search_dev.argtypes = [vp, vp, u32, vp, vp, u64, vp, vp, u64, vp]
        L.vvcg_lmcs_build.argtypes = [vp, u8, vp]
        L.vvcg_lmcs_map_plane_16_dev.argtypes = [vp, vp, C.c_int, vp, u32, u32, u32]
        L.vvcg_lmcs_chroma_scales_dev.argtypes = [vp, vp, vp, u32, u32, u32, u32, vp, u32, vp]
        L.vvcg_chroma_residuals_dev.argtypes = [vp, vp, u32, vp, u64]
        L.vvcg_sao_bounded_16_dev.argtypes = [vp, vp, vp, u32, u32, u32, u32, u32, u8, u32, u32, vp]
        L.vvcg_mip_predict_dev.argtypes = [vp, vp, u32, vp, u64, vp, vp, u64, vp]
        L.vvcg_alf_general_dev.argtypes = [vp, vp, vp, vp, u32, u32, u32, u32, u8, u32, u32, vp, vp]
        L.vvcg_luma_intra_search_8_dev.argtypes = [vp, vp, u64, vp, u64, u32, u32, vp, u32, vp]
        L.vvcg_ctu_search_dev.argtypes = [vp, vp, u64, u32, u32, u8, u32, vp, u32, vp]
        L.vvcg_ctu_search_pruned_dev.argtypes = [vp, vp, u64, u32, u32, u8, u32, vp, u32, vp, u32, u32, C.c_float, vp]
        L.vvcg_ctu_search_pruned_rule_dev.argtypes = [vp, vp, u64, u32, u32, u8, u32, vp, u32, vp, u32, u32,
                                                      C.c_float, u32, vp]
        L.vvcg_ctu_search_costs_dev.argtypes = [vp, vp, u64, u32, u32, u8, u32, vp, u32, vp, vp]
        L.vvcg_tc_selftest_dev.argtypes = [vp, vp, vp, vp, vp]
        L.vvcg_cnn_forward_dev.argtypes = [vp, vp, u64, u32, u32, u8, u8, vp, u32, vp, vp, vp, vp, vp]
        L.vvcg_cnn_train_step_dev.argtypes = [vp, vp, u64, u32, u32, u8, u8, vp, vp, u32, vp, vp, vp, u32, C.c_float,
                                              vp, vp, vp]
        L.vvcg_cnn_train_step_soft_dev.argtypes = [vp, vp, u64, u32, u32, u8, u8, vp, vp, vp, u32, vp, vp, vp, u32,
                                                   C.c_float, vp, vp, vp]
        L.vvcg_gen_intra_predict_dev.argtypes = [vp, vp, vp, u32, vp, u64]
        L.vvcg_gen_intra_recon_dev.argtypes = [vp, vp, vp, u32, vp, u32, vp, vp, u64]
        L.vvcg_deblock_general_dev.argtypes = [vp, vp, vp, u32, u32, u8, u32, vp, u32, u32, vp, u32, u32, vp]
        L.vvcg_deblock_ctu_edges_dev.argtypes = [vp, vp, vp, u32, u32, u32, u8, vp]
        L.vvcg_bdof_dev.argtypes = [vp, vp, u32, vp, vp, vp, u64]
        L.vvcg_dmvr_dev.argtypes = [vp, vp, vp, u32, u32, u32, vp, u32, vp]
        L.vvcg_affine_mvs_dev.argtypes = [vp, vp, u32, vp, u64, vp]
        L.vvcg_prof_dev.argtypes = [vp, vp, u32, vp, u64, vp, u64, vp, u64]
        L.vvcg_ciip_blend_dev.argtypes = [vp, vp, u32, vp, vp, vp, u64]
        L.vvcg_gpm_blend_dev.argtypes = [vp, vp, u32, vp, vp, vp, u64]
        L.vvcg_recon_picture_static.argtypes = [vp, vp, u32, vp, u64, vp, vp, C.c_char_p, C.c_size_t]
        L.vvcg_gen_prepare.argtypes = [vp, vp]
        L.vvcg_gen_run.argtypes = [vp, u32]
        L.vvcg_gen_download.argtypes = [vp, vp]
        L.vvcg_decode_general_batch.argtypes = [vp, vp, vp]
        L.vvcg_gen_levels.argtypes = [vp]
        L.vvcg_gen_levels.restype = u32
        L.vvcg_parse_strict.argtypes = [vp, u32, u32, u32, vp, u64, vp, u64, vp, C.c_char_p, C.c_size_t]
        L.vvcg_parse_residual_block.argtypes = [vp, u64, u32, u32, u32, u32, vp]
        L.vvcg_parse_multitool_idr.argtypes = [vp, u32, u32, u32, vp, u64, vp, u64, vp, C.c_char_p, C.c_size_t]
        L.vvcg_parse_multitool_p.argtypes = [vp, u32, u32, u32, vp, u64, vp, u64, vp, C.c_char_p, C.c_size_t]
        L.vvcg_dpb_reserve.argtypes = [vp, u32, u32, u32]
        L.vvcg_dpb_store.argtypes = [vp, u32, u32]
        L.vvcg_dpb_upload.argtypes = [vp, u32, vp]
        L.vvcg_dpb_download.argtypes = [vp, u32, vp]
        L.vvcg_dpb_plane.argtypes = [vp, u32, u32, vp, vp]
        L.vvcg_decode_p_batch.argtypes = [vp, vp, u32, vp, u32, vp, u64]
        L.vvcg_hls_rbsp.argtypes = [vp, u32, C.c_int32, vp, C.c_size_t, C.POINTER(C.c_size_t)]
        L.vvcg_annexb_idr.argtypes = [u32, u32, u8, vp, C.c_size_t, vp, C.c_size_t, C.POINTER(C.c_size_t)]
        L.vvcg_annexb_read_idr.argtypes = [vp, C.c_size_t, vp, vp, C.c_size_t, C.POINTER(C.c_size_t)]
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def chroma_dims(w, h, cf):
    if cf == CHROMA_400:
        return 0, 0
    sw = 2 if cf in (CHROMA_420, CHROMA_422) else 1
    sh = 2 if cf == CHROMA_420 else 1
    return (w + sw - 1) // sw, (h + sh - 1) // sh


class Batch:
    """Host-side records of a picture batch (the inputs of vvcg_batch)."""

    def __init__(self, pics, cus, levels, ctus=None, aps=None):
        self.pics = np.ascontiguousarray(pics, dtype=PIC_DTYPE)
        self.cus = np.ascontiguousarray(cus, dtype=CU_DTYPE)
        self.levels = levels if hasattr(levels, "data_ptr") else np.ascontiguousarray(levels, dtype=np.int16)
        self.ctus = None if ctus is None else np.ascontiguousarray(ctus, dtype=CTU_DTYPE)
        self.aps = None if aps is None else np.ascontiguousarray(aps, dtype=APS_DTYPE)

    def as_struct(self):
        nlev = self.levels.numel() if hasattr(self.levels, "numel") else self.levels.size
        return _Batch(_ptr(self.pics), len(self.pics), len(self.cus), _ptr(self.cus),
                      _ptr(self.levels), nlev,
                      _ptr(self.ctus) if self.ctus is not None else None,
                      0 if self.ctus is None else len(self.ctus),
                      0 if self.aps is None else len(self.aps),
                      _ptr(self.aps) if self.aps is not None else None)

    def output_planes(self):
        """Allocate visible-size output planes: list of (y, u, v) uint16 arrays."""
        outs = []
        for p in self.pics:
            w, h, cf = int(p["visible_width"]), int(p["visible_height"]), int(p["chroma_format"])
            cw, ch = chroma_dims(w, h, cf)
            outs.append((np.zeros((h, w), np.uint16),
                         np.zeros((ch, cw), np.uint16) if cf else None,
                         np.zeros((ch, cw), np.uint16) if cf else None))
        return outs


class GenBatch:
    """Host-side records of a batch of general-decoder intra pictures (the
    inputs of vvcg_gen_batch): GEN_PIC_DTYPE pictures, GEN_TB_DTYPE blocks in
    decode order, group_first (num_groups + 1 block indices), the int16 level
    pool, the residual / prediction slot count, and the SAO (SAO_DTYPE, 3 per
    CTU), ALF CTU (ALF_CTU_DTYPE) and ALF parameter (ALF_PARAMS_DTYPE) arrays."""

    def __init__(self, pics, tbs, group_first, levels, slot_count, sao=None, alf_ctus=None, alf_params=None):
        self.pics = np.ascontiguousarray(pics, dtype=GEN_PIC_DTYPE)
        self.tbs = np.ascontiguousarray(tbs, dtype=GEN_TB_DTYPE)
        self.group_first = np.ascontiguousarray(group_first, dtype=np.uint32)
        self.levels = np.ascontiguousarray(levels, dtype=np.int16)
        self.slot_count = int(slot_count)
        self.sao = None if sao is None else np.ascontiguousarray(sao, dtype=SAO_DTYPE)
        self.alf_ctus = None if alf_ctus is None else np.ascontiguousarray(alf_ctus, dtype=ALF_CTU_DTYPE)
        self.alf_params = None if alf_params is None else np.ascontiguousarray(alf_params, dtype=ALF_PARAMS_DTYPE)

    def as_struct(self):
        n = lambda a: 0 if a is None else len(a)  # noqa: E731
        return _GenBatch(_ptr(self.pics), len(self.pics), len(self.group_first) - 1, _ptr(self.tbs),
                         _ptr(self.group_first), len(self.tbs), _ptr(self.levels), self.levels.size,
                         self.slot_count, _ptr(self.sao), n(self.sao), _ptr(self.alf_ctus), n(self.alf_ctus),
                         _ptr(self.alf_params), n(self.alf_params), 0)

    def output_planes(self):
        outs = []
        for p in self.pics:
            w, h = int(p["vis_width"]), int(p["vis_height"])
            outs.append((np.zeros((h, w), np.uint16), np.zeros(((h + 1) // 2, (w + 1) // 2), np.uint16),
                         np.zeros(((h + 1) // 2, (w + 1) // 2), np.uint16)))
        return outs


class Context:
    """One libvvcg context: a CUDA device, a stream and the device arena."""

    def __init__(self, device: int = 0, spin_limit: int = 0, reserve_bytes: int = 0):
        L = lib()
        cfg = _Config(device, 0, reserve_bytes, spin_limit, 0)
        h = C.c_void_p()
        st = L.vvcg_ctx_create(C.byref(cfg), C.byref(h))
        if st != OK:
            raise _ERRORS.get(st, Execution)(f"vvcg_ctx_create failed with status {st}")
        self._h = h
        self._L = L
        self._keep = None

    def close(self):
        if self._h:
            self._L.vvcg_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st != OK:
            msg = self._L.vvcg_last_error(self._h).decode()
            raise _ERRORS.get(st, Execution)(msg)

    @property
    def kernel_launches(self) -> int:
        return int(self._L.vvcg_kernel_launches(self._h))

    def set_stream(self, stream=None):
        """Use a torch.cuda.Stream (or raw handle) for every launch; None = own stream."""
        raw = None if stream is None else getattr(stream, "cuda_stream", stream)
        self._check(self._L.vvcg_set_stream(self._h, C.c_void_p(raw) if raw else None))
        self.torch_stream = stream if hasattr(stream, "cuda_stream") and raw else None

    def torch_stream_scope(self):
        """A `with` scope in which torch's current stream is this context's
        stream (a new torch stream is bound to the context when it has none),
        so that tensors made for a call are ordered with its kernels."""
        import torch

        if getattr(self, "torch_stream", None) is None:
            self.set_stream(torch.cuda.Stream())
        return torch.cuda.stream(self.torch_stream)

    # -- picture batches --
    def decode_batch(self, batch: Batch, outs=None):
        """Whole call with host buffers; returns [(y, u, v)] visible planes."""
        outs = outs if outs is not None else batch.output_planes()
        po = self._plane_outs(outs)
        self._keep = (batch, outs, po)
        self._check(self._L.vvcg_decode_batch(self._h, C.byref(batch.as_struct()), po))
        return outs

    # -- general-decoder intra pictures --
    def gen_prepare(self, batch: GenBatch):
        self._gen_keep = (batch, batch.as_struct())
        self._check(self._L.vvcg_gen_prepare(self._h, C.byref(self._gen_keep[1])))

    def gen_run(self, graph=False):
        self._check(self._L.vvcg_gen_run(self._h, 1 if graph else 0))

    def gen_download(self, outs):
        po = self._plane_outs(outs)
        self._check(self._L.vvcg_gen_download(self._h, po))
        return outs

    @property
    def gen_levels(self) -> int:
        return int(self._L.vvcg_gen_levels(self._h))

    def decode_general(self, batch: GenBatch, outs=None):
        """Whole call with host buffers; returns [(y, u, v)] visible planes."""
        outs = outs if outs is not None else batch.output_planes()
        po = self._plane_outs(outs)
        st = batch.as_struct()
        self._keep = (batch, outs, po, st)
        self._check(self._L.vvcg_decode_general_batch(self._h, C.byref(st), po))
        return outs

    # -- the multi-tool stream: picture buffer and P pictures --
    def dpb_reserve(self, slots, width, height):
        """Device picture buffer of `slots` 8-bit 4:2:0 pictures (vvcg_dpb_reserve)."""
        self._check(self._L.vvcg_dpb_reserve(self._h, slots, width, height))
        self._dpb_size = (width, height)
        self._dpb_slots = slots

    def dpb_store(self, pic, slot):
        """Picture `pic` of the last frame-path batch into a slot (on the device)."""
        self._check(self._L.vvcg_dpb_store(self._h, pic, slot))

    def dpb_upload(self, slot, planes):
        """(y, u, v) host planes (uint8 or uint16 samples) into a slot."""
        arrs = [np.ascontiguousarray(a, dtype=np.uint16) for a in planes]
        pin = (_PlaneIn * 3)(*[_PlaneIn(_ptr(a), a.shape[1], 0) for a in arrs])
        self._check(self._L.vvcg_dpb_upload(self._h, slot, pin))

    def dpb_download(self, slot, outs=None):
        """A slot's (y, u, v) planes as host uint16 arrays."""
        w, h = self._dpb_size
        if outs is None:
            outs = (np.zeros((h, w), np.uint16), np.zeros((h // 2, w // 2), np.uint16),
                    np.zeros((h // 2, w // 2), np.uint16))
        self._check(self._L.vvcg_dpb_download(self._h, slot, self._plane_outs([outs])))
        return outs

    def decode_p_batch(self, pics, cus, levels):
        """P pictures (P_PIC_DTYPE) with their INTER_CU_DTYPE records and levels
        into their picture-buffer slots, in order (vvcg_decode_p_batch)."""
        pics = np.ascontiguousarray(pics, dtype=P_PIC_DTYPE)
        cus = np.ascontiguousarray(cus, dtype=INTER_CU_DTYPE)
        levels = np.ascontiguousarray(levels, dtype=np.int16)
        self._check(self._L.vvcg_decode_p_batch(self._h, _ptr(pics), len(pics), _ptr(cus), len(cus), _ptr(levels),
                                                levels.size))

    def decode_multitool_stream(self, streams, sparse=False, threads=0, stream_ids=None, download=True):
        """Decode the multi-tool stream's pictures (VvcMultiToolEncoder: IDR
        and P pictures, each P picture predicting from the picture before it
        in its stream, the DPB's build_ref_lists, inter.rs:481) from their
        slice data.

        streams: [(kind "I" / "P", bytes, width, height, qp, options)] in
        decoding order, one size; stream_ids (optional) tells the pictures of
        independent streams apart. The IDR pictures are parsed and decoded on
        the frame path in one batch, the P pictures parsed in parallel and
        decoded in one call from the picture buffer (slot k holds picture k).
        Returns [(y, u, v)] uint16 planes, or None with download=False."""
        if not streams:
            return []
        w, h = streams[0][2], streams[0][3]
        if any((s[2], s[3]) != (w, h) for s in streams):
            raise InvalidInput("the pictures of a stream share one size")
        sid = list(stream_ids) if stream_ids is not None else [0] * len(streams)
        idx_i = [k for k, s in enumerate(streams) if s[0] == "I"]
        idx_p = [k for k, s in enumerate(streams) if s[0] != "I"]
        prev, ref_of = {}, {}
        for k, s in enumerate(streams):
            if s[0] != "I":
                if sid[k] not in prev:
                    raise InvalidInput("a P picture needs a picture before it")
                ref_of[k] = prev[sid[k]]
            prev[sid[k]] = k
        if getattr(self, "_dpb_size", None) != (w, h) or getattr(self, "_dpb_slots", 0) < len(streams):
            self.dpb_reserve(len(streams), w, h)
        if idx_i:
            pics, cus, levels, _ = parse_multitool([streams[k] for k in idx_i], "I", sparse, threads)
            ctus = np.zeros(len(idx_i) * (w // 32) * (h // 32), CTU_DTYPE)
            pics["ctu_offset"] = np.arange(len(idx_i)) * (w // 32) * (h // 32)
            batch = Batch(pics, cus, levels, ctus)
            self.decode_batch(batch)
            for j, k in enumerate(idx_i):
                self.dpb_store(j, k)
        if idx_p:
            pp, pcus, plevels, _ = parse_multitool([streams[k] for k in idx_p], "P", sparse, threads)
            for j, k in enumerate(idx_p):
                pp[j]["ref_slot"][:] = ref_of[k]
                pp[j]["num_refs"] = 1
                pp[j]["out_slot"] = k
            self.decode_p_batch(pp, pcus, plevels)
        if not download:
            return None
        return [self.dpb_download(k) for k in range(len(streams))]

    def decode_batch_async(self, batch: Batch, outs):
        """decode_batch without the wait: sync() waits and reports the status.
        `batch` and `outs` (pinned host memory) must stay alive until then."""
        po = self._plane_outs(outs)
        self._keep_async = (batch, outs, po, batch.as_struct())
        self._check(self._L.vvcg_decode_batch_async(self._h, C.byref(self._keep_async[3]), po))
        return outs

    def decode_batch_pipelined(self, batch: Batch, outs=None, chunk_pictures: int = 32, lanes: int = 3):
        """decode_batch with host copies overlapped over picture chunks."""
        outs = outs if outs is not None else batch.output_planes()
        po = self._plane_outs(outs)
        self._keep = (batch, outs, po)
        self._check(self._L.vvcg_decode_batch_pipelined(self._h, C.byref(batch.as_struct()), po,
                                                        chunk_pictures, lanes))
        return outs

    def prepare(self, batch: Batch):
        self._keep = batch
        self._check(self._L.vvcg_batch_prepare(self._h, C.byref(batch.as_struct())))

    def upload(self, batch: Batch):
        self._check(self._L.vvcg_batch_upload(self._h, C.byref(batch.as_struct())))

    def run(self, stages: int = STAGE_ALL, graph: bool = False):
        """Run the prepared batch's stages (graph=True: replay a captured CUDA graph)."""
        fn = self._L.vvcg_batch_run_graph if graph else self._L.vvcg_batch_run
        self._check(fn(self._h, stages))

    def sync(self):
        self._check(self._L.vvcg_batch_sync(self._h))

    def download(self, outs):
        po = self._plane_outs(outs)
        self._check(self._L.vvcg_batch_download(self._h, po))
        return outs

    def plane(self, pic: int, comp: int):
        p = C.c_void_p()
        s = C.c_uint32()
        self._check(self._L.vvcg_batch_plane(self._h, pic, comp, C.byref(p), C.byref(s)))
        return p.value, s.value

    @staticmethod
    def _plane_outs(outs):
        arr = (_PlaneOut * (3 * len(outs)))()
        for i, planes in enumerate(outs):
            for c in range(3):
                a = planes[c]
                if a is None:
                    arr[i * 3 + c] = _PlaneOut(None, 0, 0)
                else:
                    stride = a.stride(0) if hasattr(a, "stride") and callable(a.stride) else a.strides[0] // 2
                    arr[i * 3 + c] = _PlaneOut(_ptr(a), stride, 0)
        return arr

    # -- motion compensation (torch CUDA tensors) --
    def mc_luma(self, ref, bit_depth, blocks, out):
        """ref: (H, W) uint16-as-int16 CUDA tensor; blocks: CUDA uint8 tensor of MC_BLOCK_DTYPE bytes."""
        h, w = ref.shape
        n = blocks.numel() // MC_BLOCK_DTYPE.itemsize
        self._check(self._L.vvcg_mc_luma_16_dev(self._h, _ptr(ref), w, h, ref.stride(0), bit_depth,
                                                _ptr(blocks), n, _ptr(out)))

    def mc_chroma(self, ref, bit_depth, chroma_format, blocks, out):
        h, w = ref.shape
        n = blocks.numel() // MC_BLOCK_DTYPE.itemsize
        self._check(self._L.vvcg_mc_chroma_16_dev(self._h, _ptr(ref), w, h, ref.stride(0),
                                                  bit_depth, chroma_format, _ptr(blocks), n,
                                                  _ptr(out)))

    # -- encoder --
    def encode_batch(self, pics, srcs):
        """Encode pictures (PIC_DTYPE; srcs: [(y, u, v)] coded-size uint16 arrays
        or CUDA tensors). Returns (cus, levels) as host arrays; the
        reconstruction stays in the context (download / plane)."""
        pics = np.ascontiguousarray(pics, dtype=PIC_DTYPE)
        nc, nl = C.c_uint32(), C.c_uint64()
        st = self._L.vvcg_encode_sizes(_ptr(pics), len(pics), C.byref(nc), C.byref(nl))
        if st != OK:
            raise _ERRORS.get(st, Execution)("invalid picture geometry")
        arr = (_PlaneIn * (3 * len(pics)))()
        keep = []
        for i, planes in enumerate(srcs):
            for c in range(3):
                a = planes[c] if c < len(planes) else None
                if a is None:
                    arr[i * 3 + c] = _PlaneIn(None, 0, 0)
                    continue
                if not hasattr(a, "data_ptr"):
                    a = np.ascontiguousarray(a, dtype=np.uint16)
                keep.append(a)
                stride = a.stride(0) if hasattr(a, "data_ptr") else a.strides[0] // 2
                arr[i * 3 + c] = _PlaneIn(_ptr(a), stride, 0)
        cus = np.zeros(nc.value, CU_DTYPE)
        levels = np.zeros(max(1, nl.value), np.int16)
        self._keep = (pics, keep, arr)
        self._check(self._L.vvcg_encode_batch(self._h, _ptr(pics), len(pics), arr, _ptr(cus), nc.value,
                                              _ptr(levels), nl.value))
        return cus, levels[:nl.value]

    # -- luma transform search --
    def luma_tx_search(self, reqs, pred, src, levels, samples):
        """TXS_REQ_DTYPE requests (host) over int16 CUDA tensors; returns the
        TXS_RES_DTYPE results (synchronises)."""
        import torch

        reqs = np.ascontiguousarray(reqs, dtype=TXS_REQ_DTYPE)
        res = torch.zeros(len(reqs) * TXS_RES_DTYPE.itemsize, dtype=torch.uint8, device=pred.device)
        self._keep = reqs
        self._check(self._L.vvcg_luma_tx_search_dev(self._h, _ptr(reqs), len(reqs), _ptr(pred), _ptr(src),
                                                    pred.numel(), _ptr(levels), _ptr(samples), levels.numel(),
                                                    _ptr(res)))
        torch.cuda.synchronize(pred.device)
        return res.cpu().numpy().view(TXS_RES_DTYPE)

    # -- LMCS / joint chroma residuals --
    def lmcs_map_plane(self, tables, plane, inverse=True):
        """Map a (H, W) int16 CUDA tensor of 16-bit luma samples in place."""
        t = np.asarray(tables, dtype=LMCS_TABLES_DTYPE).reshape(1).copy()
        h, w = plane.shape
        self._check(self._L.vvcg_lmcs_map_plane_16_dev(self._h, _ptr(t), int(inverse), _ptr(plane),
                                                       plane.stride(0), w, h))

    def lmcs_chroma_scales(self, tables, luma, ctu, pos, out):
        """cScale per luma position; pos: (N, 2) uint32-as-int32 CUDA tensor, out int32 CUDA tensor."""
        t = np.asarray(tables, dtype=LMCS_TABLES_DTYPE).reshape(1).copy()
        h, w = luma.shape
        self._check(self._L.vvcg_lmcs_chroma_scales_dev(self._h, _ptr(t), _ptr(luma), luma.stride(0), w, h, ctu,
                                                        _ptr(pos), pos.shape[0], _ptr(out)))

    def chroma_residuals(self, recs, res):
        recs = np.ascontiguousarray(recs, dtype=CRES_DTYPE)
        self._keep = recs
        self._check(self._L.vvcg_chroma_residuals_dev(self._h, _ptr(recs), len(recs), _ptr(res), res.numel()))

    # -- matrix-based intra prediction --
    def mip_predict(self, reqs, refs, pred, src=None):
        """MIP_REQ_DTYPE requests (host) over int16 CUDA tensors; returns the
        MIP_RES_DTYPE results of searching requests (synchronises)."""
        import torch

        reqs = np.ascontiguousarray(reqs, dtype=MIP_REQ_DTYPE)
        res = torch.zeros(len(reqs) * MIP_RES_DTYPE.itemsize, dtype=torch.uint8, device=refs.device)
        self._keep = reqs
        self._check(self._L.vvcg_mip_predict_dev(self._h, _ptr(reqs), len(reqs), _ptr(refs), refs.numel(),
                                                 _ptr(src), _ptr(pred), pred.numel(), _ptr(res)))
        torch.cuda.synchronize(refs.device)
        return res.cpu().numpy().view(MIP_RES_DTYPE)

    # -- general-decoder ALF --
    def alf_general(self, src, dst, vis_w, vis_h, bit_depth, ctu, ctu_cols, ctus, params):
        """src / dst: (Y, Cb, Cr) int16 CUDA tensors of a 4:2:0 picture; ctus
        (ALF_CTU_DTYPE) and params (ALF_PARAMS_DTYPE) host arrays."""
        ctus = np.ascontiguousarray(ctus, dtype=ALF_CTU_DTYPE)
        params = np.ascontiguousarray(params, dtype=ALF_PARAMS_DTYPE).reshape(1)
        sp = (C.c_void_p * 3)(*[t.data_ptr() for t in src])
        dp = (C.c_void_p * 3)(*[t.data_ptr() for t in dst])
        st = (C.c_uint32 * 3)(*[t.stride(0) for t in src])
        h, w = src[0].shape
        self._keep = (ctus, params)
        self._check(self._L.vvcg_alf_general_dev(self._h, sp, dp, st, w, h, vis_w, vis_h, bit_depth, ctu, ctu_cols,
                                                 _ptr(ctus), _ptr(params)))

    # -- 8-bit luma intra mode search --
    def luma_intra_search_8(self, recon, src, reqs):
        """recon / src: (H, W) uint8 CUDA tensors; reqs: ISR_REQ_DTYPE host
        records. Returns the ISR_RES_DTYPE results (synchronises)."""
        import torch

        reqs = np.ascontiguousarray(reqs, dtype=ISR_REQ_DTYPE)
        h, w = recon.shape
        if tuple(src.shape) != (h, w):
            raise InvalidInput("recon and source planes differ in size")
        out = torch.empty(max(len(reqs), 1) * ISR_RES_DTYPE.itemsize, dtype=torch.uint8, device=recon.device)
        self._keep = reqs
        self._check(self._L.vvcg_luma_intra_search_8_dev(self._h, _ptr(recon), recon.stride(0), _ptr(src),
                                                         src.stride(0), w, h, _ptr(reqs), len(reqs), _ptr(out)))
        torch.cuda.synchronize(recon.device)
        return out.cpu().numpy().view(ISR_RES_DTYPE)[:len(reqs)]

    # -- CTU full search of the GPU encoder --
    def ctu_search(self, src, bit_depth, lambda_q8, reqs, out=None, sync=True):
        """src: (H, W) int16 CUDA tensor of 16-bit luma samples; reqs:
        CTU_SEARCH_REQ_DTYPE host records. Returns the CTU_SEARCH_RES_DTYPE
        results (or fills the CUDA uint8 tensor out without synchronising)."""
        import torch

        reqs = np.ascontiguousarray(reqs, dtype=CTU_SEARCH_REQ_DTYPE)
        h, w = src.shape
        dst = out if out is not None else torch.empty(max(len(reqs), 1) * CTU_SEARCH_RES_DTYPE.itemsize,
                                                      dtype=torch.uint8, device=src.device)
        self._keep = reqs
        self._check(self._L.vvcg_ctu_search_dev(self._h, _ptr(src), src.stride(0), w, h, bit_depth, lambda_q8,
                                                _ptr(reqs), len(reqs), _ptr(dst)))
        if out is not None and not sync:
            return None
        torch.cuda.synchronize(src.device)
        return dst.cpu().numpy().view(CTU_SEARCH_RES_DTYPE)[:len(reqs)]

    # -- CNN pruner --
    def cnn_forward(self, plane, bit_depth, xy, params, qp, want_acts=False, sync=True):
        """plane: (H, W) int16 CUDA tensor of 16-bit luma samples; xy: (n, 2)
        int32 CUDA tensor of 32x32 block positions; params: CNN_PARAMS fp32
        CUDA tensor; qp: the QP the blocks are coded at. Returns (logits (n, 73), gap (n, 32), acts (n, 4, 1024,
        32) bf16 or None) as CUDA tensors."""
        import torch

        n = int(xy.shape[0])
        dev = plane.device
        logits = torch.empty((n, CNN_OUT), dtype=torch.float32, device=dev)
        gap = torch.empty((n, 32), dtype=torch.float32, device=dev)
        acts = torch.empty((n, 4, 1024, 32), dtype=torch.bfloat16, device=dev) if want_acts else None
        st = torch.zeros(1, dtype=torch.int32, device=dev)
        h, w = plane.shape
        self._check(self._L.vvcg_cnn_forward_dev(self._h, _ptr(plane), plane.stride(0), w, h, bit_depth, qp,
                                                 _ptr(xy.contiguous()), n, _ptr(params), _ptr(logits), _ptr(gap),
                                                 _ptr(acts), _ptr(st)))
        if sync:
            torch.cuda.synchronize(dev)
            code = int(st.item())
            if code & 1:
                raise Execution("CNN forward: a tensor-core completion wait gave up")
            if code & 2:
                raise InvalidInput("CNN forward: a block lies outside the plane")
        return logits, gap, acts

    def cnn_train_step(self, plane, bit_depth, qp, xy, labels, params, adam_m=None, adam_v=None, step=0, lr=0.0,
                       sync=True, soft=None):
        """One training step on the blocks xy ((n, 2) int32 CUDA) with labels
        ((n, 2) uint8 CUDA: intra mode, split type), or with soft ((n, 67)
        fp32 CUDA) the mode head's target distribution. Updates params (and
        the Adam moments) in place when lr > 0. Returns (loss, grads) CUDA
        tensors (one fp32; CNN_PARAMS fp32)."""
        import torch

        dev = plane.device
        grads = torch.empty(CNN_PARAMS, dtype=torch.float32, device=dev)
        loss = torch.empty(1, dtype=torch.float32, device=dev)
        st = torch.zeros(1, dtype=torch.int32, device=dev)
        h, w = plane.shape
        if soft is None:
            self._check(self._L.vvcg_cnn_train_step_dev(
                self._h, _ptr(plane), plane.stride(0), w, h, bit_depth, qp, _ptr(xy.contiguous()),
                _ptr(labels.contiguous()), int(xy.shape[0]), _ptr(params), _ptr(adam_m), _ptr(adam_v), step, lr,
                _ptr(grads), _ptr(loss), _ptr(st)))
        else:
            soft = soft.contiguous()
            self._check(self._L.vvcg_cnn_train_step_soft_dev(
                self._h, _ptr(plane), plane.stride(0), w, h, bit_depth, qp, _ptr(xy.contiguous()),
                _ptr(labels.contiguous()), _ptr(soft), int(xy.shape[0]), _ptr(params), _ptr(adam_m), _ptr(adam_v),
                step, lr, _ptr(grads), _ptr(loss), _ptr(st)))
        if sync:
            torch.cuda.synchronize(dev)
            code = int(st.item())
            if code & 1:
                raise Execution("CNN training: a tensor-core completion wait gave up")
            if code & 2:
                raise InvalidInput("CNN training: a block outside the plane or a label out of range")
        return loss, grads

    # -- tensor-core self-test --
    def tc_selftest(self, a, b):
        """a: (128, 16), b: (32, 16) bfloat16 CUDA tensors; returns the fp32
        (128, 32) product a @ b.T from one tcgen05 MMA, or raises Execution
        when its completion wait gave up."""
        import torch

        d = torch.zeros((128, 32), dtype=torch.float32, device=a.device)
        st = torch.zeros(1, dtype=torch.int32, device=a.device)
        self._check(self._L.vvcg_tc_selftest_dev(self._h, _ptr(a.contiguous()), _ptr(b.contiguous()), _ptr(d),
                                                 _ptr(st)))
        torch.cuda.synchronize(a.device)
        if int(st.item()):
            raise Execution("tensor-core self-test: completion wait gave up")
        return d

    def ctu_search_xy(self, src, bit_depth, lambda_q8, xy, logits=None, top_modes=6, top_splits=2,
                      threshold=0.7, out=None, sync=True, rule=0):
        """The CTU search over device positions xy ((n, 2) int32 CUDA), full
        (logits None) or pruned by the CNN's logits ((n, 73) fp32 CUDA): the
        top_modes / top_splits most probable entries of each head, or its full
        set when they hold less than threshold of its softmax mass (rule
        PRUNE_MASS) or when its most probable entry does (PRUNE_MAX_PROB).
        Returns CTU_SEARCH_RES_DTYPE results, or fills the CUDA uint8 tensor
        out (n x 36 bytes) without synchronising when sync is False."""
        import torch

        n = int(xy.shape[0])
        h, w = src.shape
        dst = out if out is not None else torch.empty(max(n, 1) * CTU_SEARCH_RES_DTYPE.itemsize, dtype=torch.uint8,
                                                      device=src.device)
        self._check(self._L.vvcg_ctu_search_pruned_rule_dev(
            self._h, _ptr(src), src.stride(0), w, h, bit_depth, lambda_q8, _ptr(xy.contiguous()), n, _ptr(logits),
            top_modes, top_splits, threshold, rule, _ptr(dst)))
        if not sync:
            return None
        torch.cuda.synchronize(src.device)
        return dst.cpu().numpy().view(CTU_SEARCH_RES_DTYPE)[:n]

    def ctu_search_costs(self, src, bit_depth, lambda_q8, xy):
        """The full CTU search over device positions xy with every luma mode's
        cost of each unsplit 32x32 CU (vvcg_ctu_search_costs_dev): returns
        (CTU_SEARCH_RES_DTYPE results, (n, 67) int64 CUDA tensor of costs)."""
        import torch

        n = int(xy.shape[0])
        h, w = src.shape
        dst = torch.empty(max(n, 1) * CTU_SEARCH_RES_DTYPE.itemsize, dtype=torch.uint8, device=src.device)
        costs = torch.empty((max(n, 1), 67), dtype=torch.int32, device=src.device)
        self._check(self._L.vvcg_ctu_search_costs_dev(self._h, _ptr(src), src.stride(0), w, h, bit_depth, lambda_q8,
                                                      _ptr(xy.contiguous()), n, _ptr(dst), _ptr(costs)))
        torch.cuda.synchronize(src.device)
        return dst.cpu().numpy().view(CTU_SEARCH_RES_DTYPE)[:n], costs[:n].to(torch.int64)

    # -- general-decoder intra prediction --
    def gen_intra_predict(self, planes, dec_y, dec_c, bit_depth, ctu, reqs, out_count, vert_collocated=False):
        """planes: (Y, Cb, Cr) int16 CUDA tensors (Y at the padded picture
        size); dec_y / dec_c: uint8 CUDA tensors (one byte per 4x4 luma cell /
        per chroma sample); reqs: GEN_INTRA_REQ_DTYPE host records. Returns
        the int16 CUDA output of out_count samples (synchronises)."""
        import torch

        reqs = np.ascontiguousarray(reqs, dtype=GEN_INTRA_REQ_DTYPE)
        st = _GenIntraState()
        for c in range(3):
            st.plane[c] = planes[c].data_ptr()
            st.stride[c] = planes[c].stride(0)
        st.height, st.width = planes[0].shape
        st.dec_y, st.dec_c = dec_y.data_ptr(), dec_c.data_ptr()
        st.bit_depth, st.vert_collocated, st.ctu_size = bit_depth, int(vert_collocated), ctu
        out = torch.zeros(max(out_count, 1), dtype=torch.int16, device=planes[0].device)
        self._keep = (reqs, st)
        self._check(self._L.vvcg_gen_intra_predict_dev(self._h, C.byref(st), _ptr(reqs), len(reqs), _ptr(out),
                                                       out_count))
        torch.cuda.synchronize(planes[0].device)
        return out

    def gen_intra_recon(self, planes, dec_y, dec_c, bit_depth, ctu, reqs, group_start, residual, out_count,
                        vert_collocated=False):
        """Sequential reconstruction (vvcg_gen_intra_recon_dev), in place on
        planes and the decoded maps (CUDA tensors as for gen_intra_predict).
        group_start: num_groups + 1 request indices; residual: int16 CUDA
        tensor of out_count samples or None. Returns the predictions
        (synchronises)."""
        import torch

        reqs = np.ascontiguousarray(reqs, dtype=GEN_INTRA_REQ_DTYPE)
        groups = np.ascontiguousarray(group_start, dtype=np.uint32)
        st = _GenIntraState()
        for c in range(3):
            st.plane[c] = planes[c].data_ptr()
            st.stride[c] = planes[c].stride(0)
        st.height, st.width = planes[0].shape
        st.dec_y, st.dec_c = dec_y.data_ptr(), dec_c.data_ptr()
        st.bit_depth, st.vert_collocated, st.ctu_size = bit_depth, int(vert_collocated), ctu
        pred = torch.zeros(max(out_count, 1), dtype=torch.int16, device=planes[0].device)
        self._keep = (reqs, groups, st)
        self._check(self._L.vvcg_gen_intra_recon_dev(self._h, C.byref(st), _ptr(reqs), len(reqs), _ptr(groups),
                                                     len(groups) - 1, _ptr(residual), _ptr(pred), out_count))
        torch.cuda.synchronize(planes[0].device)
        return pred

    # -- inter-prediction tools (device int32 arrays; requests are host records) --
    # The context's stream does not wait for torch's: each call synchronises
    # the device before (tensors just made or filled by torch) and after
    # (results read through torch).
    def _inter_tool(self, fn, reqs, dtype, dev, *args):
        import torch

        reqs = np.ascontiguousarray(reqs, dtype=dtype)
        self._keep = reqs
        torch.cuda.synchronize(dev)
        self._check(fn(self._h, _ptr(reqs), len(reqs), *args))
        torch.cuda.synchronize(dev)

    def bdof(self, reqs, pred0, pred1, out):
        """BDOF_REQ_DTYPE requests over int32 CUDA tensors (14-bit intermediates in, 8-bit out)."""
        self._inter_tool(self._L.vvcg_bdof_dev, reqs, BDOF_REQ_DTYPE, out.device, _ptr(pred0), _ptr(pred1), _ptr(out),
                         out.numel())

    def dmvr(self, ref0, ref1, reqs, mv_out):
        """ref0 / ref1: (H, W) uint8 CUDA tensors; mv_out: int32 CUDA tensor of 4 per request."""
        import torch

        h, w = ref0.shape
        reqs = np.ascontiguousarray(reqs, dtype=DMVR_REQ_DTYPE)
        self._keep = reqs
        torch.cuda.synchronize(mv_out.device)
        self._check(self._L.vvcg_dmvr_dev(self._h, _ptr(ref0), _ptr(ref1), w, h, ref0.stride(0), _ptr(reqs),
                                          len(reqs), _ptr(mv_out)))
        torch.cuda.synchronize(mv_out.device)

    def affine_mvs(self, reqs, sub_mv, prof):
        self._inter_tool(self._L.vvcg_affine_mvs_dev, reqs, AFFINE_REQ_DTYPE, sub_mv.device, _ptr(sub_mv),
                         sub_mv.numel() // 2, _ptr(prof))

    def prof(self, reqs, src, dmv, out):
        self._inter_tool(self._L.vvcg_prof_dev, reqs, PROF_REQ_DTYPE, out.device, _ptr(src), src.numel(), _ptr(dmv),
                         dmv.numel(), _ptr(out), out.numel())

    def ciip_blend(self, reqs, inter, intra, out):
        self._inter_tool(self._L.vvcg_ciip_blend_dev, reqs, CIIP_REQ_DTYPE, out.device, _ptr(inter), _ptr(intra),
                         _ptr(out), out.numel())

    def gpm_blend(self, reqs, pred0, pred1, out):
        self._inter_tool(self._L.vvcg_gpm_blend_dev, reqs, GPM_REQ_DTYPE, out.device, _ptr(pred0), _ptr(pred1),
                         _ptr(out), out.numel())

    # -- general-decoder deblocking --
    def deblock_ctu_edges(self, planes, ctu, qp, cells):
        """CTU-boundary deblocking of an 8-bit 4:2:0 inter picture, in place on
        planes, (Y, Cb, Cr) int16 CUDA tensors (8-bit sample values); cells:
        (rows, cols) CTU_MOTION_DTYPE records (numpy, uploaded here)."""
        import torch

        cells = np.ascontiguousarray(cells, dtype=CTU_MOTION_DTYPE)
        h, w = planes[0].shape
        if cells.shape != (h // ctu, w // ctu):
            raise InvalidInput(f"cells are {cells.shape}; the picture needs {(h // ctu, w // ctu)}")
        dc = torch.from_numpy(cells.view(np.uint8).reshape(-1).copy()).to(planes[0].device)
        pp = (C.c_void_p * 3)(*[t.data_ptr() for t in planes])
        st = (C.c_uint32 * 3)(*[t.stride(0) for t in planes])
        self._keep = dc
        torch.cuda.synchronize(planes[0].device)
        self._check(self._L.vvcg_deblock_ctu_edges_dev(self._h, pp, st, w, h, ctu, qp, _ptr(dc)))
        torch.cuda.synchronize(planes[0].device)

    def deblock_general(self, planes, vis_w, vis_h, bit_depth, ctu, cells, ccells, params):
        """In place on planes, (Y, Cb, Cr) int16 CUDA tensors of a 4:2:0
        picture. cells / ccells: 2-D CUDA uint8 tensors or numpy arrays of
        DBK_CELL_DTYPE / DBK_CCELL_DTYPE records (rows x cols, numpy arrays are
        uploaded); params: one DBK_PARAMS_DTYPE record."""
        import torch

        def dev(a, dt):
            if isinstance(a, np.ndarray):
                a = np.ascontiguousarray(a, dtype=dt)
                rows, cols = a.shape
                t = torch.from_numpy(a.view(np.uint8).reshape(rows, cols * dt.itemsize).copy())
                return t.to(planes[0].device), rows, cols
            rows, nb = a.shape
            return a, rows, nb // dt.itemsize

        dc, rows, cols = dev(cells, DBK_CELL_DTYPE)
        dcc, crows, ccols = dev(ccells, DBK_CCELL_DTYPE)
        params = np.ascontiguousarray(params, dtype=DBK_PARAMS_DTYPE).reshape(1)
        pp = (C.c_void_p * 3)(*[t.data_ptr() for t in planes])
        st = (C.c_uint32 * 3)(*[t.stride(0) for t in planes])
        self._keep = (dc, dcc, params)
        self._check(self._L.vvcg_deblock_general_dev(self._h, pp, st, vis_w, vis_h, bit_depth, ctu, _ptr(dc), cols,
                                                     rows, _ptr(dcc), ccols, crows, _ptr(params)))

    # -- general-decoder SAO --
    def sao_bounded(self, src, dst, vis_w, vis_h, bit_depth, ctu, ctu_cols, params):
        """src / dst: (H, W) int16 CUDA tensors of 16-bit samples; params: CUDA
        uint8 tensor of SAO_DTYPE records (one per CTU)."""
        h, w = src.shape
        self._check(self._L.vvcg_sao_bounded_16_dev(self._h, _ptr(src), _ptr(dst), src.stride(0), w, h, vis_w, vis_h,
                                                    bit_depth, ctu, ctu_cols, _ptr(params)))

    # -- metrics --
    def plane_metrics(self, ref, dist):
        """(sse, sad, samples) of two equally shaped 2-D CUDA tensors (uint8, or
        int16 holding 16-bit samples); synchronises the stream."""
        import torch

        if tuple(ref.shape) != tuple(dist.shape):
            raise InvalidInput(f"plane dimensions differ: {tuple(ref.shape)} and {tuple(dist.shape)}")
        out = torch.zeros(3, dtype=torch.int64, device=ref.device)
        h, w = ref.shape
        fn = self._L.vvcg_plane_metrics_8_dev if ref.element_size() == 1 else self._L.vvcg_plane_metrics_16_dev
        self._check(fn(self._h, _ptr(ref), ref.stride(0), _ptr(dist), dist.stride(0), w, h, _ptr(out)))
        torch.cuda.synchronize(ref.device)
        return tuple(int(v) for v in out.cpu())

    @staticmethod
    def psnr(sse, samples, bit_depth):
        """PlaneMetrics::psnr (accelerator.rs:111-118): 100 dB for a zero error."""
        import math

        mse = sse / samples if samples else 0.0
        if mse <= 1e-12:
            return 100.0
        peak = float((1 << min(bit_depth, 16)) - 1)
        return 10.0 * math.log10(peak * peak / mse)

    # -- transform units (records on the host, int16 CUDA tensors) --
    def tu_inverse(self, recs, data, out):
        """Levels -> residual for every TU_DTYPE record (asynchronous on the stream)."""
        recs = np.ascontiguousarray(recs, dtype=TU_DTYPE)
        self._keep = recs
        self._check(self._L.vvcg_tu_inverse_batch(self._h, _ptr(recs), len(recs), _ptr(data),
                                                  data.numel(), _ptr(out), out.numel()))

    def tu_forward(self, recs, data, out):
        """Residual -> levels for every TU_DTYPE record (asynchronous on the stream)."""
        recs = np.ascontiguousarray(recs, dtype=TU_DTYPE)
        self._keep = recs
        self._check(self._L.vvcg_tu_forward_batch(self._h, _ptr(recs), len(recs), _ptr(data),
                                                  data.numel(), _ptr(out), out.numel()))

    def inter_search_8(self, src, refs_l0, refs_l1, cands, reqs):
        """Motion estimation (estimate_inter_block) of each ME_REQ_DTYPE block on
        a (H, W) uint8 CUDA plane against lists of same-size uint8 CUDA
        references, with MV_CAND_DTYPE merge candidates; returns ME_RES_DTYPE."""
        import torch

        cands = np.ascontiguousarray(cands, dtype=MV_CAND_DTYPE)
        reqs = np.ascontiguousarray(reqs, dtype=ME_REQ_DTYPE)
        h, w = src.shape
        for r in list(refs_l0) + list(refs_l1):
            if tuple(r.shape) != (h, w) or r.stride(0) != src.stride(0):
                raise InvalidInput("references must have the source plane's size and stride")
        l0 = (C.c_void_p * max(len(refs_l0), 1))(*[r.data_ptr() for r in refs_l0])
        l1 = (C.c_void_p * max(len(refs_l1), 1))(*[r.data_ptr() for r in refs_l1])
        out = torch.empty(max(len(reqs), 1) * ME_RES_DTYPE.itemsize, dtype=torch.uint8, device=src.device)
        self._check(self._L.vvcg_inter_search_8_dev(self._h, _ptr(src), src.stride(0), w, h, l0, len(refs_l0), l1,
                                                    len(refs_l1), _ptr(cands) if len(cands) else None, len(cands),
                                                    _ptr(reqs), len(reqs), _ptr(out)))
        torch.cuda.synchronize(src.device)
        return out.cpu().numpy().view(ME_RES_DTYPE)[:len(reqs)]

    def qt_mtt_split(self, plane, bit_depth, reqs):
        """Quadrant-mean split decision (choose_qt_mtt_partition_rdo_16) of each
        SPLIT_REQ_DTYPE region of a (H, W) 16-bit CUDA luma plane; returns uint8
        SPLIT_NONE / SPLIT_QT / SPLIT_BT_H / SPLIT_BT_V per region."""
        import torch

        reqs = np.ascontiguousarray(reqs, dtype=SPLIT_REQ_DTYPE)
        h, w = plane.shape
        out = torch.empty(max(len(reqs), 1), dtype=torch.uint8, device=plane.device)
        self._check(self._L.vvcg_qt_mtt_split_dev(self._h, _ptr(plane), plane.stride(0), w, h, bit_depth, _ptr(reqs),
                                                  len(reqs), _ptr(out)))
        torch.cuda.synchronize(plane.device)
        return out.cpu().numpy()[:len(reqs)]

    def tu_autotune(self, recs, data, out, forward):
        """Times each CTA width of every size group of this batch and keeps the
        fastest for later tu_inverse (forward False) / tu_forward (True) calls;
        returns the chosen warps per CTA of the 256 / 1024 / 4096-coefficient
        groups (0: no unit of that size). out receives the batch's results."""
        recs = np.ascontiguousarray(recs, dtype=TU_DTYPE)
        warps = np.zeros(3, np.uint32)
        self._check(self._L.vvcg_tu_autotune(self._h, _ptr(recs), len(recs), _ptr(data), data.numel(), _ptr(out),
                                             out.numel(), int(bool(forward)), _ptr(warps)))
        return tuple(int(w) for w in warps)

    def mc_luma_8(self, ref, blocks, out):
        """ref: (H, W) uint8 CUDA tensor (the 8-bit functions of inter.rs)."""
        h, w = ref.shape
        n = blocks.numel() // MC_BLOCK_DTYPE.itemsize
        self._check(self._L.vvcg_mc_luma_8_dev(self._h, _ptr(ref), w, h, ref.stride(0), _ptr(blocks), n, _ptr(out)))

    def mc_chroma_420_8(self, ref, blocks, out):
        h, w = ref.shape
        n = blocks.numel() // MC_BLOCK_DTYPE.itemsize
        self._check(self._L.vvcg_mc_chroma_420_8_dev(self._h, _ptr(ref), w, h, ref.stride(0), _ptr(blocks), n,
                                                     _ptr(out)))

    def mc_bi_average(self, p0, p1, bcw_idx, bit_depth, out):
        self._check(self._L.vvcg_mc_bi_average_16_dev(self._h, _ptr(p0), _ptr(p1), p0.numel(),
                                                      bcw_idx, bit_depth, _ptr(out)))


def recon_picture_static(pic, cus, levels, planes, stream=None):
    """Allocation-free reconstruction (+ deblocking) of one picture in place.

    `pic` is one PIC_DTYPE record; `cus` a CUDA uint8 tensor of CU_DTYPE
    records; `levels` a CUDA int16 tensor; `planes` the coded-size (Y, Cb, Cr)
    CUDA int16 tensors the library writes (None for absent chroma). Runs on
    the current device and `stream` (a torch.cuda.Stream, a raw handle, or
    None for the legacy default stream) and returns when it has finished.
    """
    import torch

    L = lib()
    desc = np.asarray(pic, dtype=PIC_DTYPE).reshape(1).copy()
    # The C side sees raw pointers only: every size, type and layout the
    # kernels rely on is checked here, before anything is launched.
    dev = torch.cuda.current_device()

    def on_device(t, what):
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.device.index != dev:
            raise InvalidInput(f"{what} must be a CUDA tensor on the current device (cuda:{dev})")

    on_device(cus, "cus")
    on_device(levels, "levels")
    if cus.dtype != torch.uint8 or not cus.is_contiguous():
        raise InvalidInput("cus must be a contiguous uint8 tensor of CU_DTYPE records")
    if cus.numel() % CU_DTYPE.itemsize:
        raise InvalidInput(f"cus holds {cus.numel()} bytes, not a whole number of {CU_DTYPE.itemsize}-byte records")
    if levels.dtype != torch.int16 or not levels.is_contiguous():
        raise InvalidInput("levels must be a contiguous int16 tensor")
    w, h, cf = int(desc[0]["width"]), int(desc[0]["height"]), int(desc[0]["chroma_format"])
    cw, ch = chroma_dims(w, h, cf)
    dims = [(h, w), (ch, cw), (ch, cw)]
    arr = (_PlaneOut * 3)()
    for c in range(3):
        a = planes[c] if c < len(planes) else None
        if c > 0 and cf == CHROMA_400:
            a = None
        elif a is None:
            raise InvalidInput(f"plane {c} is missing")
        if a is not None:
            on_device(a, f"plane {c}")
            if a.dtype not in (torch.int16, torch.uint16) or a.dim() != 2 or a.stride(1) != 1:
                raise InvalidInput(f"plane {c} must be a 2-D 16-bit tensor with unit column stride")
            if a.shape[0] < dims[c][0] or a.shape[1] < dims[c][1]:
                raise InvalidInput(f"plane {c} is {tuple(a.shape)}; the coded size needs {dims[c]}")
        arr[c] = _PlaneOut(None, 0, 0) if a is None else _PlaneOut(_ptr(a), a.stride(0), 0)
    raw = None if stream is None else getattr(stream, "cuda_stream", stream)
    err = C.create_string_buffer(512)
    st = L.vvcg_recon_picture_static(_ptr(desc), _ptr(cus), cus.numel() // CU_DTYPE.itemsize,
                                     _ptr(levels), levels.numel(), arr,
                                     C.c_void_p(raw) if raw else None, err, len(err))
    if st != OK:
        raise _ERRORS.get(st, Execution)(err.value.decode())


def lmcs_build(aps, bit_depth):
    """Reshaper tables (LMCS_TABLES_DTYPE) of an LMCS APS (host function of the library)."""
    a = np.asarray(aps, dtype=LMCS_APS_DTYPE).reshape(1).copy()
    t = np.zeros(1, LMCS_TABLES_DTYPE)
    st = lib().vvcg_lmcs_build(_ptr(a), bit_depth, _ptr(t))
    if st != OK:
        raise _ERRORS.get(st, Execution)("invalid LMCS APS")
    return t[0]


PARSE_LUMA, PARSE_DEP_QUANT, PARSE_SIGN_HIDING, PARSE_TRANSFORM_SKIP = 1, 2, 4, 8


# -- Annex-B access units (include/vvcg.h "Annex-B access units") --
STREAM_CFG_DTYPE = np.dtype([("width", "<u4"), ("height", "<u4"), ("crop_right", "<u4"), ("crop_bottom", "<u4"),
                             ("qp", "u1"), ("level_idc", "u1"), ("ctu_log2", "u1"), ("min_cb_log2", "u1"),
                             ("ts_log2", "u1"), ("reserved", "u1", (3,))])
ANNEXB_INFO_DTYPE = np.dtype([("width", "<u4"), ("height", "<u4"), ("qp", "<i4"), ("num_nals", "<u4"),
                              ("slice_nal_type", "<u4"), ("reserved", "<u4")])
HLS_AUD, HLS_VPS, HLS_SPS, HLS_PPS, HLS_PH, HLS_SLICE_HEADER = range(6)
PRUNE_MASS, PRUNE_MAX_PROB = 0, 1  # fallback rules of vvcg_ctu_search_pruned_rule_dev


def _sized_call(fn, *args):
    """Calls fn(*args, out, cap, &size) twice: once for the size, once into a
    buffer of that size; returns the bytes."""
    size = C.c_size_t(0)
    st = fn(*args, None, 0, C.byref(size))
    if st not in (OK, LIMIT_EXCEEDED):
        raise _ERRORS.get(st, Execution)(f"{fn.__name__} rejected its input")
    out = np.zeros(max(1, size.value), np.uint8)
    st = fn(*args, _ptr(out), out.size, C.byref(size))
    if st != OK:
        raise _ERRORS.get(st, Execution)(f"{fn.__name__} rejected its input")
    return out[:size.value].tobytes()


def hls_rbsp(kind, width, height, qp, level_idc, ctu_log2=5, min_cb_log2=5, ts_log2=5, crop_right=0,
             crop_bottom=0, arg=0):
    """One RBSP of the default stream's parameter sets or headers
    (vvcg_hls_rbsp): kind HLS_AUD / VPS / SPS / PPS / PH / SLICE_HEADER, arg
    the AUD picture type, the POC LSB or the slice QP delta; bytes."""
    cfg = np.zeros(1, STREAM_CFG_DTYPE)
    for k, v in dict(width=width, height=height, crop_right=crop_right, crop_bottom=crop_bottom, qp=qp,
                     level_idc=level_idc, ctu_log2=ctu_log2, min_cb_log2=min_cb_log2, ts_log2=ts_log2).items():
        cfg[k] = v
    return _sized_call(lib().vvcg_hls_rbsp, _ptr(cfg), kind, arg)


def annexb_idr(slice_data, width, height, qp):
    """The reference encoder's IDR access unit (AUD, VPS, SPS, PPS, picture
    header, IDR slice) around strict-profile slice data, for a picture of
    width x height visible samples at qp (vvcg_annexb_idr); bytes."""
    buf = np.frombuffer(bytes(slice_data), np.uint8)
    return _sized_call(lib().vvcg_annexb_idr, width, height, qp, _ptr(buf) if buf.size else None, buf.size)


def annexb_read_idr(au):
    """The slice data of an IDR access unit of the default stream and what
    the PPS and slice header say (vvcg_annexb_read_idr): returns (slice
    data bytes, width, height, qp), ready for parse_strict."""
    buf = np.frombuffer(bytes(au), np.uint8)
    info = np.zeros(1, ANNEXB_INFO_DTYPE)
    data = _sized_call(lib().vvcg_annexb_read_idr, _ptr(buf) if buf.size else None, buf.size, _ptr(info))
    return data, int(info["width"][0]), int(info["height"][0]), int(info["qp"][0])


def parse_strict(streams, sparse=False, threads=0):
    """Parse strict-profile slice data on the host (vvcg_parse_strict).

    streams: [(bytes, width, height, qp)]. Returns (pics, cus, levels): a
    PIC_DTYPE batch (8-bit 4:2:0, CTU 32, VVCG_TOOL_TU_TOOLS, plus
    VVCG_TOOL_SPARSE_LEVELS when sparse), the CU records and the level pool,
    ready for Batch / decode_batch, and the levels each picture used."""
    L = lib()
    n = len(streams)
    subs = (_StrictSubstream * max(1, n))()
    bufs, cu_at, lv_at = [], 0, 0
    for i, (data, w, h, qp) in enumerate(streams):
        buf = np.frombuffer(bytes(data), np.uint8)
        bufs.append(buf)
        ncu = (w // 32) * (h // 32)
        cap = (w * h * 3) // 2 * (2 if sparse else 1) + 8 * ncu
        subs[i] = _StrictSubstream(_ptr(buf) if buf.size else None, buf.size, w, h, qp, (C.c_uint8 * 3)(), cu_at,
                                   lv_at, cap)
        cu_at += ncu
        lv_at += cap + (cap & 1)
    cus = np.zeros(cu_at, CU_DTYPE)
    levels = np.zeros(max(1, lv_at), np.int16)
    used = np.zeros(max(1, n), np.uint64)
    err = C.create_string_buffer(256)
    st = L.vvcg_parse_strict(subs, n, int(sparse), threads, _ptr(cus), len(cus), _ptr(levels), levels.size,
                             _ptr(used), err, 256)
    if st != OK:
        raise _ERRORS.get(st, Execution)(err.value.decode())
    # one compact pool: each picture's levels moved next to the previous
    # picture's (even offsets for the sparse form), its records rebased
    pool_n, starts = 0, []
    for i in range(n):
        pool_n += pool_n & 1
        starts.append(pool_n)
        pool_n += int(used[i])
    pool = np.zeros(max(1, pool_n), np.int16)
    for i in range(n):
        a, m = int(subs[i].level_offset), int(used[i])
        pool[starts[i]:starts[i] + m] = levels[a:a + m]
        c0, w, h = int(subs[i].cu_offset), streams[i][1], streams[i][2]
        rec = cus[c0:c0 + (w // 32) * (h // 32)]
        lo = rec["level_off"].astype(np.int64)
        rec["level_off"] = np.where(lo >= 0, lo - a + starts[i], -1).astype(np.int32)
    levels = pool
    pics = np.zeros(n, PIC_DTYPE)
    for i, (_, w, h, qp) in enumerate(streams):
        p = pics[i:i + 1]
        p["width"], p["height"], p["visible_width"], p["visible_height"] = w, h, w, h
        p["bit_depth"], p["chroma_format"], p["ctu_log2"], p["slice_qp"] = 8, CHROMA_420, 5, qp
        qpc = min(63, max(0, qp if qp <= 26 else qp - 1))  # derived_chroma_qp (hls.rs:778) at 8 bits
        p["chroma_qp_scaled"] = qpc
        p["tools"] = TOOL_TU_TOOLS | (TOOL_SPARSE_LEVELS if sparse else 0)
        p["alf_aps"] = -1
        p["cu_offset"] = subs[i].cu_offset
    return pics, cus, levels, used[:n].copy()


def parse_multitool(streams, kind, sparse=False, threads=0):
    """Parse the multi-tool stream's slice data on the host.

    streams: [(kind, bytes, width, height, qp, options)] (kind is ignored;
    every entry is parsed as `kind`: "I" with vvcg_parse_multitool_idr, "P"
    with vvcg_parse_multitool_p). Returns (pics, cus, levels, used): for "I"
    a PIC_DTYPE batch for the frame path (8-bit 4:2:0, CTU 32, TU_TOOLS, plus
    DEP_QUANT / SPARSE_LEVELS as the options ask) with CU_DTYPE records; for
    "P" P_PIC_DTYPE pictures (slots to fill in) with INTER_CU_DTYPE records.
    Each picture's levels are compacted into one pool."""
    L = lib()
    is_p = kind != "I"
    n = len(streams)
    subs = (_SliceSubstream * max(1, n))()
    bufs, cu_at, lv_at = [], 0, 0
    for i, (_, data, w, h, qp, opts) in enumerate(streams):
        buf = np.frombuffer(bytes(data), np.uint8)
        bufs.append(buf)
        ncu = (w // 32) * (h // 32)
        cap = (w * h * 3) // 2 * (2 if sparse else 1) + 8 * ncu
        subs[i] = _SliceSubstream(_ptr(buf) if buf.size else None, buf.size, w, h, qp, 5, opts, 0, cu_at, lv_at, cap)
        cu_at += ncu
        lv_at += cap + (cap & 1)
    cus = np.zeros(cu_at, INTER_CU_DTYPE if is_p else CU_DTYPE)
    levels = np.zeros(max(1, lv_at), np.int16)
    used = np.zeros(max(1, n), np.uint64)
    err = C.create_string_buffer(256)
    fn = L.vvcg_parse_multitool_p if is_p else L.vvcg_parse_multitool_idr
    st = fn(subs, n, int(sparse), threads, _ptr(cus), len(cus), _ptr(levels), levels.size, _ptr(used), err, 256)
    if st != OK:
        raise _ERRORS.get(st, Execution)(err.value.decode())
    pool_n, starts = 0, []
    for i in range(n):
        pool_n += pool_n & 1
        starts.append(pool_n)
        pool_n += int(used[i])
    pool = np.zeros(max(1, pool_n), np.int16)
    for i in range(n):
        a, m = int(subs[i].level_offset), int(used[i])
        pool[starts[i]:starts[i] + m] = levels[a:a + m]
        c0, w, h = int(subs[i].cu_offset), streams[i][2], streams[i][3]
        rec = cus[c0:c0 + (w // 32) * (h // 32)]
        lo = rec["level_off"].astype(np.int64)
        rec["level_off"] = np.where(lo >= 0, lo - a + starts[i], -1).astype(np.int32)
    if is_p:
        pics = np.zeros(n, P_PIC_DTYPE)
        for i, (_, _, w, h, qp, opts) in enumerate(streams):
            pics[i]["width"], pics[i]["height"], pics[i]["qp"] = w, h, qp
            pics[i]["options"], pics[i]["sparse"] = opts & (SLICE_DEP_QUANT | SLICE_DEBLOCK), int(sparse)
            pics[i]["num_refs"], pics[i]["cu_offset"] = 1, subs[i].cu_offset
    else:
        pics = np.zeros(n, PIC_DTYPE)
        for i, (_, _, w, h, qp, opts) in enumerate(streams):
            p = pics[i:i + 1]
            p["width"], p["height"], p["visible_width"], p["visible_height"] = w, h, w, h
            # decode_picture_multitool reconstructs and deblocks at max(QP, 4)
            # and max(derived_chroma_qp, 4) (slice.rs:3029-3031, :3290-3297)
            lqp = max(qp, 4)
            p["bit_depth"], p["chroma_format"], p["ctu_log2"], p["slice_qp"] = 8, CHROMA_420, 5, lqp
            p["chroma_qp_scaled"] = min(63, lqp if lqp <= 26 else lqp - 1)  # derived_chroma_qp (hls.rs:778)
            p["tools"] = (TOOL_TU_TOOLS | (TOOL_SPARSE_LEVELS if sparse else 0) |
                          (TOOL_DEP_QUANT if opts & SLICE_DEP_QUANT else 0) |
                          (TOOL_DEBLOCK if opts & SLICE_DEBLOCK else 0))
            p["alf_aps"] = -1
            p["cu_offset"] = subs[i].cu_offset
    return pics, cus, pool, used[:n].copy()


def parse_residual_block(data, w, h, flags, qp):
    """One block's substream into (h, w) int32 levels (vvcg_parse_residual_block)."""
    buf = np.frombuffer(bytes(data), np.uint8)
    out = np.zeros((h, w), np.int32)
    st = lib().vvcg_parse_residual_block(_ptr(buf) if buf.size else None, buf.size, w, h, flags, qp, _ptr(out))
    if st != OK:
        raise _ERRORS.get(st, Execution)("malformed residual substream")
    return out

