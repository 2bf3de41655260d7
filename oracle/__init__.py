"""CPU oracle for the VVC reconstruction / loop-filter / candidate-cost path.

TEST INFRASTRUCTURE ONLY: a C++ restatement of the reference codec's CPU code
(rustmpeg-video, crates/rustmpeg-video/src/vvc/), loaded with ctypes. Only the
tests, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` may use it,
and only as the checker or the timed CPU baseline; the product library never
links or calls it.

Parity pinning: the reference is Rust and cannot be built here, so the
restatement is pinned by the reference's own known-answer and property tests
(ported in tests/test_oracle_kats.py). Paths those tests do not reach are
"parity unpinned".
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborc_vvc.so")
_lib = None

DCT2, DST7, DCT8 = 0, 1, 2
CHROMA_400, CHROMA_420, CHROMA_422, CHROMA_444 = 0, 1, 2, 3
OPT_FULL_INTRA, OPT_CCLM, OPT_DEP_QUANT, OPT_DEBLOCK = 1, 2, 4, 8


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -O2, scalar)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    else:
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _declare(L):
    vp, i = C.c_void_p, C.c_int
    for name in ("orc_forward_transform", "orc_inverse_transform"):
        getattr(L, name).argtypes = [i, i, vp, i, i, i, i, i, vp]
    L.orc_quantize.argtypes = [i, i, vp, i, i, i, vp]
    L.orc_dequantize.argtypes = [i, i, vp, i, i, vp]
    L.orc_quantize_dq.argtypes = [i, i, vp, i, i, vp]
    L.orc_dequantize_dq.argtypes = [i, i, vp, i, i, vp]
    L.orc_coeff_scan.argtypes = [i, i, vp]
    L.orc_quantize_ts.argtypes = [i, i]
    L.orc_dequantize_ts.argtypes = [i, i]
    L.orc_scaled_luma_qp.argtypes = [i, i]
    L.orc_chroma_qp.argtypes = [i, i, i]
    L.orc_wide_angle.argtypes = [i, i, i]
    L.orc_angular_params.argtypes = [i, i, i, i, vp]
    L.orc_angular_params.restype = None
    L.orc_predict_block.argtypes = [vp, i, i, i, i, i, i, i, i, i, vp]
    L.orc_predict_block.restype = None
    L.orc_predict_coded_block.argtypes = [vp, i, i, i, i, i, i, i, i, i, i, i, vp, i, i, i, vp]
    L.orc_predict_coded_block.restype = None
    L.orc_predict_cclm.argtypes = [vp, i, i, vp, i, i, i, i, i, i, i, i, i, i, vp]
    L.orc_predict_cclm.restype = None
    L.orc_choose_intra_mode.argtypes = [vp, vp, i, i, i, i, i, i, i]
    L.orc_deblock_luma.argtypes = [vp, i, i, i, i, i, i, i, i, i]
    L.orc_deblock_luma.restype = None
    L.orc_deblock_chroma.argtypes = [vp, i, i, i, i, i, i, i, i, i, i, i]
    L.orc_deblock_chroma.restype = None
    L.orc_sao_region.argtypes = [vp, vp, i, i, i, i, i, i, i, i, i, vp]
    L.orc_alf_luma.argtypes = [vp, i, i, i, i, i, vp, vp, vp]
    L.orc_alf_classify.argtypes = [vp, i, i, i, i, i, vp]
    L.orc_alf_classify.restype = None
    L.orc_mc_luma.argtypes = [vp, i, i, i, i, i, i, i, i, i, i, i, i, vp]
    L.orc_mc_luma.restype = None
    L.orc_mc_chroma.argtypes = [vp, i, i, i, i, i, i, i, i, i, i, i, vp]
    L.orc_mc_chroma.restype = None
    L.orc_bi_average.argtypes = [vp, vp, i, i, i, vp]
    L.orc_bi_average.restype = None
    L.orc_encode_frame.argtypes = [vp, vp, vp, i, i, i, i, i, i, i, vp, vp, C.c_uint64,
                                   C.POINTER(C.c_uint64), vp, vp, vp]
    L.orc_recon_frame.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    L.orc_tu_batch.argtypes = [i, vp, i, vp, vp]
    L.orc_alf_general.argtypes = [vp, vp, vp, vp, vp, vp, i, i, i, i, i, i, i, vp, vp]
    L.orc_alf_general.restype = None
    L.orc_mip_predict.argtypes = [vp, vp, i, i, i, i, i, vp]
    L.orc_mip_predict.restype = None
    L.orc_mip_search.argtypes = [vp, vp, vp, i, i, i, vp, C.POINTER(C.c_uint64)]
    L.orc_sao_bounded.argtypes = [vp, vp, i, i, i, i, i, i, i, vp, i]
    L.orc_luma_intra_search_8.argtypes = [vp, vp, i, i, i, i, i, i, vp, i, i, i, vp]
    L.orc_luma_intra_search_8.restype = None
    L.orc_predict_luma_8.argtypes = [vp, i, i, i, i, i, i, i, i, i, vp]
    L.orc_predict_luma_8.restype = None
    L.orc_ctu_search.argtypes = [vp, i, i, i, i, i, i, i, vp, C.c_uint32, vp]
    L.orc_ctu_search.restype = None
    L.orc_lfnst.argtypes = [i, vp, i, i, i, i]
    L.orc_lfnst.restype = i
    L.orc_inter_search_8.argtypes = [vp, i, i, vp, i, i, vp, vp, i, vp]
    L.orc_inter_search_8.restype = None
    L.orc_qt_mtt_split.argtypes = [vp, i, i, i, vp, i, vp]
    L.orc_qt_mtt_split.restype = None
    L.orc_gen_intra_predict.argtypes = [vp, vp, vp, i, i, i, i, vp, vp, i, i, i, vp, i, vp]
    L.orc_gen_intra_predict.restype = None
    L.orc_deblock_general.argtypes = [vp, vp, vp, i, i, i, i, i, i, vp, i, i, vp, i, i, vp]
    L.orc_deblock_general.restype = None
    L.orc_inter_ctu_deblock.argtypes = [vp, vp, vp, i, i, i, i, i, i, vp]
    L.orc_inter_ctu_deblock.restype = None
    L.orc_strict_encode.argtypes = [vp, vp, vp, i, i, i, i, vp, vp, vp, vp, vp, vp]
    L.orc_strict_decode.argtypes = [vp, vp, C.c_uint64, i, i, i, i, vp, vp, vp]
    L.orc_strict_write.argtypes = [vp, vp, C.c_uint64, i, i, i, vp, C.c_uint64, vp]
    L.orc_block_write.argtypes = [vp, i, i, i, i, i, i, i, vp, C.c_uint64, vp]
    u32 = C.c_uint32
    L.orc_mt_encode.argtypes = [vp, vp, vp, i, i, i, i, u32, vp, vp, vp, vp, vp, vp]
    L.orc_mt_decode.argtypes = [vp, vp, C.c_uint64, i, i, i, i, u32, vp, vp, vp]
    L.orc_inter_encode.argtypes = [vp, vp, vp, i, i, i, i, u32, vp, i, vp, vp, vp, vp, vp, vp]
    L.orc_inter_resolve_motion.argtypes = [vp, i, i, i]
    L.orc_inter_decode.argtypes = [vp, vp, C.c_uint64, i, i, i, i, u32, vp, i, vp, vp, vp]
    L.orc_derive_intra_mpms.argtypes = [i, i, vp]
    L.orc_derive_intra_mpms.restype = None
    L.orc_mt_write.argtypes = [vp, vp, C.c_uint64, i, i, i, u32, vp, C.c_uint64, vp]
    L.orc_p_write.argtypes = [vp, vp, C.c_uint64, i, i, i, u32, vp, C.c_uint64, vp]
    L.orc_bdof.argtypes = [vp, vp, i, i, vp]
    L.orc_bdof.restype = None
    L.orc_dmvr.argtypes = [vp, vp, i, i, i, i, i, i, i, vp]
    L.orc_dmvr.restype = None
    L.orc_affine_mvs.argtypes = [vp, i, i, i, i, vp, vp, vp]
    L.orc_affine_mvs.restype = i
    L.orc_prof.argtypes = [vp, vp, vp, i, vp]
    L.orc_prof.restype = None
    L.orc_ciip.argtypes = [vp, vp, i, i, i, vp]
    L.orc_ciip.restype = None
    L.orc_gpm.argtypes = [vp, vp, i, i, i, i, i, vp]
    L.orc_gpm.restype = None
    L.orc_dbk_lens.argtypes = [i, i, i, i, vp]
    L.orc_dbk_lens.restype = None
    L.orc_dbk_bs.argtypes = [i] * 11
    L.orc_sao_bounded.restype = None
    L.orc_mc_luma_8.argtypes = [vp, i, i, i, i, i, i, i, i, i, i, i, i, vp]
    L.orc_mc_luma_8.restype = None
    L.orc_mc_chroma_420_8.argtypes = [vp, i, i, i, i, i, i, i, i, i, i, vp]
    L.orc_mc_chroma_420_8.restype = None
    L.orc_bi_average_8.argtypes = [vp, vp, i, i, vp]
    L.orc_bi_average_8.restype = None
    L.orc_lmcs_build.argtypes = [vp, i, vp]
    L.orc_lmcs_map_plane.argtypes = [vp, i, vp, i]
    L.orc_lmcs_map_plane.restype = None
    L.orc_lmcs_chroma_scale.argtypes = [vp, vp, i, i, i, i, i, i]
    L.orc_chroma_residuals.argtypes = [vp, vp]
    L.orc_chroma_residuals.restype = None
    L.orc_luma_tx_search.argtypes = [i, vp, vp, i, i, i, i, vp, vp, C.POINTER(C.c_uint64)]
    L.orc_plane_metrics.argtypes = [vp, C.c_uint64, vp, C.c_uint64, C.c_uint32, C.c_uint32, i, vp]


# ---------------------------------------------------------------- transforms --

def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def forward_transform(res, tr_hor=DCT2, tr_ver=DCT2, skip_w=0, skip_h=0, bd=8):
    res = _i32(res)
    h, w = res.shape
    out = np.zeros_like(res)
    rc = lib().orc_forward_transform(w, h, _p(res), tr_hor, tr_ver, skip_w, skip_h, bd, _p(out))
    if rc:
        raise ValueError(f"forward transform rejected ({rc})")
    return out


def inverse_transform(co, tr_hor=DCT2, tr_ver=DCT2, skip_w=0, skip_h=0, bd=8):
    co = _i32(co)
    h, w = co.shape
    out = np.zeros_like(co)
    rc = lib().orc_inverse_transform(w, h, _p(co), tr_hor, tr_ver, skip_w, skip_h, bd, _p(out))
    if rc:
        raise ValueError(f"inverse transform rejected ({rc})")
    return out


def quantize(co, qp, bd=8, intra=True):
    co = _i32(co)
    h, w = co.shape
    out = np.zeros_like(co)
    if lib().orc_quantize(w, h, _p(co), qp, bd, int(intra), _p(out)):
        raise ValueError("quantize rejected")
    return out


def dequantize(lv, qp, bd=8):
    lv = _i32(lv)
    h, w = lv.shape
    out = np.zeros_like(lv)
    if lib().orc_dequantize(w, h, _p(lv), qp, bd, _p(out)):
        raise ValueError("dequantize rejected")
    return out


def quantize_dq(co, qp, bd=8):
    co = _i32(co)
    h, w = co.shape
    out = np.zeros_like(co)
    if lib().orc_quantize_dq(w, h, _p(co), qp, bd, _p(out)):
        raise ValueError("dep quant rejected")
    return out


def dequantize_dq(lv, qp, bd=8):
    lv = _i32(lv)
    h, w = lv.shape
    out = np.zeros_like(lv)
    if lib().orc_dequantize_dq(w, h, _p(lv), qp, bd, _p(out)):
        raise ValueError("dep dequant rejected")
    return out


def coeff_scan(w, h):
    out = np.zeros(w * h, dtype=np.int32)
    n = lib().orc_coeff_scan(w, h, _p(out))
    return out[:n]


def quantize_ts(r, qp):
    return lib().orc_quantize_ts(int(r), qp)


def dequantize_ts(level, qp):
    return lib().orc_dequantize_ts(int(level), qp)


def scaled_luma_qp(qp, bd):
    return lib().orc_scaled_luma_qp(qp, bd)


def chroma_qp(qp, bd, offset=0):
    return lib().orc_chroma_qp(qp, bd, offset)


def wide_angle(w, h, mode):
    return lib().orc_wide_angle(w, h, mode)


def angular_params(mode, w, h, is_luma=True):
    out = np.zeros(8, dtype=np.int32)
    lib().orc_angular_params(mode, w, h, int(is_luma), _p(out))
    keys = ("pred_mode", "is_mode_ver", "intra_pred_angle", "abs_inv_angle",
            "ref_filter_flag", "interpolation_flag", "apply_pdpc", "angular_scale")
    return dict(zip(keys, out.tolist()))


# --------------------------------------------------------------------- intra --

def _u16(a):
    return np.ascontiguousarray(a, dtype=np.uint16)


def predict_block(plane, bd, x, y, w, h, mode, is_luma=True):
    plane = _u16(plane)
    out = np.zeros((h, w), dtype=np.uint16)
    lib().orc_predict_block(_p(plane), plane.shape[1], plane.shape[0], bd, x, y, w, h,
                            int(is_luma), mode, _p(out))
    return out


def predict_coded_block(plane, bd, x, y, w, h, mode, coded, tb, is_luma=True, sx=1, sy=1):
    plane = _u16(plane)
    coded = np.ascontiguousarray(coded, dtype=np.uint8)
    out = np.zeros((h, w), dtype=np.uint16)
    lib().orc_predict_coded_block(_p(plane), plane.shape[1], plane.shape[0], bd, x, y, w, h,
                                  int(is_luma), mode, sx, sy, _p(coded), coded.shape[1],
                                  coded.shape[0], tb, _p(out))
    return out


def predict_cclm(luma, chroma, bd, bxc, byc, cw, ch, mode, cf=CHROMA_420, ctu=32):
    luma, chroma = _u16(luma), _u16(chroma)
    out = np.zeros((ch, cw), dtype=np.uint16)
    lib().orc_predict_cclm(_p(luma), luma.shape[1], luma.shape[0], _p(chroma), chroma.shape[1],
                           chroma.shape[0], bd, bxc, byc, cw, ch, mode, cf, ctu, _p(out))
    return out


def predict_luma_8(recon, x, y, w, h, mode, mrl=0, ctu=32):
    """predict_block_full (predict.rs:2655) of one luma Planar / DC / angular
    mode on an 8-bit plane; int32 (h, w)."""
    recon = np.ascontiguousarray(recon, dtype=np.uint8)
    out = np.zeros((h, w), dtype=np.int32)
    lib().orc_predict_luma_8(_p(recon), recon.shape[1], recon.shape[0], x, y, w, h, mode, mrl, ctu, _p(out))
    return out


def luma_intra_search_8(recon, src, x, y, w, h, mpm, mpm_only=False, mrl=False, ctu=32):
    """choose_luma_intra_pred_mode (predict.rs:2737) on 8-bit planes, with the
    multi-tool encoder's MRL candidates (slice.rs:2698-2731) when mrl;
    returns (mode, mrl_idx, sad)."""
    recon = np.ascontiguousarray(recon, dtype=np.uint8)
    src = np.ascontiguousarray(src, dtype=np.uint8)
    m = np.ascontiguousarray(mpm, dtype=np.uint8)
    out = np.zeros(4, np.uint32)
    lib().orc_luma_intra_search_8(_p(recon), _p(src), recon.shape[1], recon.shape[0], x, y, w, h, _p(m),
                                  int(mpm_only), int(mrl), ctu, _p(out))
    return int(out[0]), int(out[1]), int(out[2]) | (int(out[3]) << 32)


def ctu_search(src, bd, x, y, lambda_q8, split_mask=0x3F, cand=()):
    """The GPU encoder's CTU full search on a 16-bit luma plane (no reference
    counterpart); returns a dict with the fields of vvcg_ctu_search_res."""
    src = _u16(src)
    c = np.zeros(6, np.uint8)
    c[:len(cand)] = cand
    out = np.zeros(10, np.uint32)
    lib().orc_ctu_search(_p(src), src.shape[1], src.shape[0], bd, x, y, split_mask, len(cand), _p(c), lambda_q8,
                         _p(out))
    m = int(out[9])
    return dict(cost=int(out[0]), split_cost=[int(v) for v in out[1:7]], split=int(out[7]), cu_mode=int(out[8]),
                modes=[(m >> (8 * k)) & 0xFF for k in range(4)])


def lfnst(coeffs, w, h, idx, mode, forward):
    """forward_lfnst_rect / inverse_lfnst_rect (lfnst.rs) on a copy of the
    w x h raster coefficients; returns (status, coefficients), status 0 = ok."""
    c = np.ascontiguousarray(np.asarray(coeffs, dtype=np.int32).reshape(-1)).copy()
    rc = lib().orc_lfnst(int(bool(forward)), _p(c), w, h, idx, mode)
    return rc, c


def inter_search_8(src, refs_l0, refs_l1, cands, reqs, res_dtype):
    """estimate_inter_block (inter.rs:1866-2003) of each request on 8-bit
    planes of one size: cands / reqs are structured arrays in the
    vvcg_mv_cand / vvcg_me_req layouts; returns res_dtype (vvcg_me_res) results."""
    src = np.ascontiguousarray(src, dtype=np.uint8)
    planes = [np.ascontiguousarray(r, dtype=np.uint8) for r in list(refs_l0) + list(refs_l1)]
    refs = np.ascontiguousarray(np.stack(planes)) if planes else np.zeros(1, np.uint8)
    cands = np.ascontiguousarray(cands)
    reqs = np.ascontiguousarray(reqs)
    out = np.zeros(len(reqs), res_dtype)
    lib().orc_inter_search_8(_p(src), src.shape[1], src.shape[0], _p(refs), len(refs_l0), len(refs_l1),
                             _p(cands) if len(cands) else None, _p(reqs), len(reqs), _p(out))
    return out


def qt_mtt_split(src, bd, regions):
    """choose_qt_mtt_partition_rdo_16 (slice.rs:4111-4167) of each region
    (x, y, w, h, qp, min_cb) of a 16-bit luma plane of bit depth bd; returns
    uint8 splits: 0 none, 1 quad, 2 binary horizontal, 3 binary vertical."""
    src = _u16(src)
    r = np.ascontiguousarray(np.asarray(regions, dtype=np.int64).reshape(-1, 6))
    out = np.zeros(len(r), np.uint8)
    lib().orc_qt_mtt_split(_p(src), src.shape[1], src.shape[0], bd, _p(r), len(r), _p(out))
    return out


def search_lambda_q8(qp, bit_depth=10):
    """lambda of the CTU search (SATD domain) in 1/256 units:
    sqrt(0.57 * 2^((qp - 12) / 3)) * 2^(bit_depth - 8)."""
    return int(round(256.0 * np.sqrt(0.57 * 2.0 ** ((qp - 12) / 3.0)) * 2.0 ** (bit_depth - 8)))


def gen_intra_predict(y, u, v, dec_y, dec_c, bd, ctu, reqs, out_count, vert_collocated=False):
    """The general decoder's intra prediction (decode_general.rs:3983-4793)
    of each request (vvcg_gen_intra_req layout) from the planes (Y at the
    padded picture size, Cb / Cr at half) and the decoded maps (one byte per
    4x4 luma cell, one per chroma sample). Returns the int16 output buffer."""
    y, u, v = _u16(y), _u16(u), _u16(v)
    dy = np.ascontiguousarray(dec_y, dtype=np.uint8)
    dc = np.ascontiguousarray(dec_c, dtype=np.uint8)
    r = np.ascontiguousarray(reqs)
    out = np.zeros(out_count, np.int16)
    lib().orc_gen_intra_predict(_p(y), _p(u), _p(v), y.shape[1], u.shape[1], y.shape[1], y.shape[0], _p(dy), _p(dc),
                                bd, int(vert_collocated), ctu, _p(r), len(r), _p(out))
    return out


def gen_intra_recon(y, u, v, dec_y, dec_c, bd, ctu, reqs, group_start, residual, out_count, vert_collocated=False):
    """Transform blocks reconstructed in decode order, as reconstruct_tu
    (decode_general.rs:3985-4096) does for each transform unit of a coding
    unit (for ISP, its sub-partitions, :4009-4024): the prediction of the
    block from the current planes and decoded maps (gen_intra_predict), plus
    the residual (int16, w x h at out_off; None = zero), clipped to the bit
    depth (:4087-4093) and stored, then the block marked decoded as mark_tu
    does (:4891-4906: every 4x4 luma cell it touches, every chroma sample).
    Groups are processed one after another. Returns the new (y, u, v, dec_y,
    dec_c) and the predictions."""
    planes = [_u16(p).copy() for p in (y, u, v)]
    dy = np.ascontiguousarray(dec_y, dtype=np.uint8).copy()
    dc = np.ascontiguousarray(dec_c, dtype=np.uint8).copy()
    reqs = np.ascontiguousarray(reqs)
    pred = np.zeros(out_count, np.int16)
    maxv = (1 << bd) - 1
    h_pic, w_pic = planes[0].shape
    for g in range(len(group_start) - 1):
        for q in range(int(group_start[g]), int(group_start[g + 1])):
            r = reqs[q:q + 1]
            w, h, x0, y0, comp = int(r["w"][0]), int(r["h"][0]), int(r["x"][0]), int(r["y"][0]), int(r["comp"][0])
            off = int(r["out_off"][0])
            one = r.copy()
            one["out_off"] = 0
            p = gen_intra_predict(planes[0], planes[1], planes[2], dy, dc, bd, ctu, one, w * h,
                                  vert_collocated)[:w * h].astype(np.int32)
            pred[off:off + w * h] = p
            res = np.zeros(w * h, np.int32) if residual is None else residual[off:off + w * h].astype(np.int32)
            planes[comp][y0:y0 + h, x0:x0 + w] = np.clip(p + res, 0, maxv).reshape(h, w).astype(np.uint16)
            if comp == 0:
                cw = w_pic // 4
                rows = slice(y0 // 4, min((y0 + h + 3) // 4, h_pic // 4))
                cols = slice(x0 // 4, min((x0 + w + 3) // 4, cw))
                dy.reshape(-1, cw)[rows, cols] = 1
            else:
                dc.reshape(-1, w_pic // 2)[y0:y0 + h, x0:x0 + w] = 1
    return planes[0], planes[1], planes[2], dy, dc, pred


def choose_intra_mode(recon, src, bd, bx, by, w, h):
    recon, src = _u16(recon), _u16(src)
    return lib().orc_choose_intra_mode(_p(recon), _p(src), recon.shape[1], recon.shape[0], bd,
                                       bx, by, w, h)


# ------------------------------------------------------------------- filters --

def deblock_luma(plane, bd, cu_step, ctb, qp, bs=2, beta_off=0, tc_off=0):
    p = _u16(plane).copy()
    lib().orc_deblock_luma(_p(p), p.shape[1], p.shape[0], bd, cu_step, ctb, qp, bs, beta_off,
                           tc_off)
    return p


def deblock_chroma(plane, bd, cu_step, ctb_h, qp, bs=2, beta_off=0, tc_off=0, sub_w=2, sub_h=2):
    p = _u16(plane).copy()
    lib().orc_deblock_chroma(_p(p), p.shape[1], p.shape[0], bd, cu_step, ctb_h, qp, bs, beta_off,
                             tc_off, sub_w, sub_h)
    return p


def sao_region(src, dst, bd, bx, by, w, h, sao_type, band_or_class, offsets):
    src = _u16(src)
    dst = _u16(dst).copy()
    off = np.asarray(offsets, dtype=np.int32)
    rc = lib().orc_sao_region(_p(src), _p(dst), src.shape[1], src.shape[0], bd, bx, by, w, h,
                              sao_type, band_or_class, _p(off))
    return dst, rc


def alf_luma(plane, bd, aps=None):
    """Whole-plane luma ALF. aps: dict(coeff[n,12], clip_idx[n,12], delta_idx[25], luma_clip)."""
    p = _u16(plane).copy()
    if aps is None:
        rc = lib().orc_alf_luma(_p(p), p.shape[1], p.shape[0], bd, 0, 0, None, None, None)
    else:
        coeff = np.zeros((25, 12), dtype=np.int16)
        clip = np.zeros((25, 12), dtype=np.uint8)
        n = len(aps["coeff"])
        coeff[:n] = aps["coeff"]
        clip[:n] = aps.get("clip_idx", np.zeros((n, 12)))
        delta = np.ascontiguousarray(aps["delta_idx"], dtype=np.uint8)
        rc = lib().orc_alf_luma(_p(p), p.shape[1], p.shape[0], bd, n, int(aps.get("luma_clip", 0)),
                                _p(delta), _p(coeff), _p(clip))
    return p, rc


def alf_classify(plane, bd, bx, by):
    plane = _u16(plane)
    out = np.zeros(2, dtype=np.int32)
    lib().orc_alf_classify(_p(plane), plane.shape[1], plane.shape[0], bd, bx, by, _p(out))
    return int(out[0]), int(out[1])


# ----------------------------------------------------------------------- MC --

def mc_luma(ref, bd, bx, by, w, h, mvx, mvy, bi=False, affine=False, alt_hpel=False):
    ref = _u16(ref)
    out = np.zeros((h, w), dtype=np.int32)
    lib().orc_mc_luma(_p(ref), ref.shape[1], ref.shape[0], bd, bx, by, w, h, mvx, mvy, int(bi),
                      int(affine), int(alt_hpel), _p(out))
    return out


def mc_chroma(ref, bd, bxc, byc, cw, ch, mvx, mvy, bi=False, cf=CHROMA_420):
    ref = _u16(ref)
    out = np.zeros((ch, cw), dtype=np.int32)
    lib().orc_mc_chroma(_p(ref), ref.shape[1], ref.shape[0], bd, bxc, byc, cw, ch, mvx, mvy,
                        int(bi), cf, _p(out))
    return out


def bi_average(p0, p1, bcw, bd):
    p0, p1 = _i32(p0), _i32(p1)
    out = np.zeros(p0.shape, dtype=np.uint16)
    lib().orc_bi_average(_p(p0), _p(p1), p0.size, bcw, bd, _p(out))
    return out


def mc_luma_8(ref, bx, by, w, h, mvx, mvy, bi=False, affine=False, alt_hpel=False):
    """inter.rs:896-1051 interpolate_luma_block on an 8-bit plane."""
    ref = np.ascontiguousarray(ref, dtype=np.uint8)
    out = np.zeros((h, w), dtype=np.int32)
    lib().orc_mc_luma_8(_p(ref), ref.shape[1], ref.shape[0], ref.shape[1], bx, by, w, h, mvx, mvy, int(bi),
                        int(alt_hpel), int(affine), _p(out))
    return out


def mc_chroma_420_8(ref, cx, cy, cw, ch, mvx, mvy, bi=False):
    """inter.rs:1056-1182 interpolate_chroma_block_420 on an 8-bit plane."""
    ref = np.ascontiguousarray(ref, dtype=np.uint8)
    out = np.zeros((ch, cw), dtype=np.int32)
    lib().orc_mc_chroma_420_8(_p(ref), ref.shape[1], ref.shape[0], ref.shape[1], cx, cy, cw, ch, mvx, mvy,
                              int(bi), _p(out))
    return out


def bi_average_8(p0, p1, bcw):
    """inter.rs:1189-1201 weighted_average_bi."""
    p0, p1 = _i32(p0), _i32(p1)
    out = np.zeros(p0.shape, dtype=np.int32)
    lib().orc_bi_average_8(_p(p0), _p(p1), p0.size, bcw, _p(out))
    return out


# ------------------------------------------------------------ frame path --

# Record layouts of include/vvcg.h, as numpy structured dtypes.
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
TOOL_DEP_QUANT, TOOL_DEBLOCK, TOOL_SAO, TOOL_ALF = 1, 2, 4, 8
assert CU_DTYPE.itemsize == 16 and CTU_DTYPE.itemsize == 20 and PIC_DTYPE.itemsize == 32


def chroma_dims(w, h, cf):
    if cf == CHROMA_400:
        return 0, 0
    sw = 2 if cf in (CHROMA_420, CHROMA_422) else 1
    sh = 2 if cf == CHROMA_420 else 1
    return (w + sw - 1) // sw, (h + sh - 1) // sh


def encode_frame(y, u, v, bd, qp, ctu_log2=5, opts=OPT_FULL_INTRA | OPT_DEBLOCK, cf=CHROMA_420):
    """Restated slice::encode_vvc_frame_picture on coded-size planes.

    Returns (cus, levels, (rec_y, rec_u, rec_v)): cus is a CU_DTYPE array in
    tb-grid raster order, levels the int16 pool the records index.
    """
    y = _u16(y)
    h, w = y.shape
    cw, ch = chroma_dims(w, h, cf)
    u = _u16(u) if cf else np.zeros((1, 1), np.uint16)
    v = _u16(v) if cf else np.zeros((1, 1), np.uint16)
    tb = min(1 << ctu_log2, 32)
    cus = np.zeros((h // tb) * (w // tb), dtype=CU_DTYPE)
    cap = w * h * 3 + 64
    levels = np.zeros(cap, dtype=np.int16)
    used = C.c_uint64(0)
    ry = np.zeros((h, w), np.uint16)
    ru = np.zeros((max(ch, 1), max(cw, 1)), np.uint16)
    rv = np.zeros((max(ch, 1), max(cw, 1)), np.uint16)
    rc = lib().orc_encode_frame(_p(y), _p(u), _p(v), w, h, bd, cf, qp, ctu_log2, opts, _p(cus),
                                _p(levels), cap, C.byref(used), _p(ry), _p(ru), _p(rv))
    if rc:
        raise ValueError(f"encode_frame rejected ({rc})")
    return cus, levels[: used.value].copy(), (ry, ru, rv)


def strict_encode(y, u, v, qp, ctu_log2=5):
    """slice::encode_picture's decisions and reconstruction (slice.rs:325-455,
    without the CABAC writes) on an 8-bit 4:2:0 picture of coded size.

    Returns (cus, levels, (rec_y, rec_u, rec_v)): CU_DTYPE records in
    tb-grid raster order with the syntax decode_picture parses (modes, cbf,
    tu_tools: transform skip per coded TB, mts_idx, lfnst_idx), dense levels.
    """
    y, u, v = (np.ascontiguousarray(a, dtype=np.uint8) for a in (y, u, v))
    h, w = y.shape
    cus = np.zeros((h // 32) * (w // 32), dtype=CU_DTYPE)
    levels = np.zeros(w * h * 3 // 2 + 64, np.int16)
    used = C.c_uint64(0)
    ry, ru, rv = np.zeros_like(y), np.zeros_like(u), np.zeros_like(v)
    rc = lib().orc_strict_encode(_p(y), _p(u), _p(v), w, h, qp, ctu_log2, _p(cus), _p(levels), C.byref(used),
                                 _p(ry), _p(ru), _p(rv))
    if rc:
        raise ValueError(f"strict_encode rejected ({rc})")
    return cus, levels[:used.value].copy(), (ry, ru, rv)


def strict_decode(cus, levels, w, h, qp, ctu_log2=5):
    """slice::decode_picture's reconstruction (slice.rs:458-627) from parsed
    records (as strict_encode returns them); returns (y, u, v) uint8."""
    cus = np.ascontiguousarray(cus, dtype=CU_DTYPE)
    levels = np.ascontiguousarray(levels, dtype=np.int16)
    ry = np.zeros((h, w), np.uint8)
    ru = np.zeros((h // 2, w // 2), np.uint8)
    rv = np.zeros((h // 2, w // 2), np.uint8)
    rc = lib().orc_strict_decode(_p(cus), _p(levels), levels.size, w, h, qp, ctu_log2, _p(ry), _p(ru), _p(rv))
    if rc:
        raise ValueError(f"strict_decode rejected ({rc})")
    return ry, ru, rv


def strict_write(cus, levels, w, h, qp):
    """The slice data encode_picture writes (slice.rs:407-455, with
    cabac.rs BinEncoder and residual.rs / slice.rs residual coding) for
    records as strict_encode returns them; bytes."""
    cus = np.ascontiguousarray(cus, dtype=CU_DTYPE)
    levels = np.ascontiguousarray(levels, dtype=np.int16)
    cap = 64 + 4 * levels.size + 16 * len(cus)
    out = np.zeros(cap, np.uint8)
    n = C.c_uint64(0)
    rc = lib().orc_strict_write(_p(cus), _p(levels), levels.size, w, h, qp, _p(out), cap, C.byref(n))
    if rc:
        raise ValueError(f"strict_write rejected the records ({rc})")
    return out[:n.value].tobytes()


def block_write(levels, luma=True, dep_quant=False, sign_hiding=False, ts=False, qp=26):
    """One block's residual_coding (residual.rs encode_residual_with_options)
    or residual_ts_coding (slice.rs encode_ts_block) on fresh I-slice
    contexts, then the terminating bin and byte alignment; bytes."""
    lv = np.ascontiguousarray(levels, dtype=np.int32)
    h, w = lv.shape
    cap = 64 + 8 * lv.size
    out = np.zeros(cap, np.uint8)
    n = C.c_uint64(0)
    rc = lib().orc_block_write(_p(lv), w, h, int(luma), int(dep_quant), int(sign_hiding), int(ts), qp, _p(out), cap,
                               C.byref(n))
    if rc:
        raise ValueError(f"block_write rejected the block ({rc})")
    return out[:n.value].tobytes()


def recon_frame(pic, cus, levels, ctus, aps=None):
    """Restated decode_vvc_frame_picture_with_chroma_qp reconstruction + filters.

    pic: one PIC_DTYPE record; cus/ctus: the picture's own records. Returns
    (status, (y, u, v)) with coded-size planes; status -3 marks the input on
    which the reference aborts (fixed-filter ALF reaching class >= 16).
    """
    pic = np.asarray(pic, dtype=PIC_DTYPE).reshape(1).copy()
    w, h = int(pic[0]["width"]), int(pic[0]["height"])
    cf = int(pic[0]["chroma_format"])
    cw, ch = chroma_dims(w, h, cf)
    cus = np.ascontiguousarray(cus, dtype=CU_DTYPE)
    levels = np.ascontiguousarray(levels, dtype=np.int16)
    if levels.size == 0:
        levels = np.zeros(1, np.int16)
    ctus = np.ascontiguousarray(ctus, dtype=CTU_DTYPE)
    aps_arr = None if aps is None else np.asarray(aps, dtype=APS_DTYPE).reshape(1).copy()
    y = np.zeros((h, w), np.uint16)
    u = np.zeros((max(ch, 1), max(cw, 1)), np.uint16)
    v = np.zeros((max(ch, 1), max(cw, 1)), np.uint16)
    rc = lib().orc_recon_frame(_p(pic), _p(cus), _p(levels), _p(ctus),
                               None if aps_arr is None else _p(aps_arr), _p(y), _p(u), _p(v))
    return rc, (y, u, v)


# ------------------------------------------------------------ transform units --

TU_DTYPE = np.dtype([("log2_w", "u1"), ("log2_h", "u1"), ("bit_depth", "u1"), ("qp", "u1"),
                     ("flags", "u1"), ("mts_idx", "u1"), ("lfnst_idx", "u1"),
                     ("lfnst_mode", "u1"), ("in_off", "<u4"), ("out_off", "<u4")])
TU_DEP_QUANT, TU_TRANSFORM_SKIP, TU_BDPCM_HOR, TU_BDPCM_VER, TU_IMPLICIT_MTS, TU_INTER = 1, 2, 4, 8, 16, 32


def tu_batch(recs, data, out_count, forward=False):
    """Run a transform-unit batch (TU_DTYPE records) over int16 `data`.

    Returns (rc, out): rc is 0, or -(i + 1) for the first record the
    reference rejects (later records are not run).
    """
    recs = np.ascontiguousarray(recs, dtype=TU_DTYPE)
    data = np.ascontiguousarray(data, dtype=np.int16)
    out = np.zeros(out_count, np.int16)
    rc = lib().orc_tu_batch(1 if forward else 0, _p(recs), len(recs), _p(data), _p(out))
    return rc, out


def plane_metrics(a, b):
    """(sse, sad, samples) of two equally sized 2-D uint8 / uint16 arrays
    (accelerator.rs:258-292 CpuFrameMetrics::plane_metrics)."""
    assert a.shape == b.shape and a.dtype == b.dtype
    elem = a.dtype.itemsize
    h, w = a.shape
    out = np.zeros(3, np.uint64)
    rc = lib().orc_plane_metrics(a.ctypes.data_as(C.c_void_p), a.strides[0] // elem,
                                 b.ctypes.data_as(C.c_void_p), b.strides[0] // elem, w, h, elem, _p(out))
    assert rc == 0
    return int(out[0]), int(out[1]), int(out[2])


def luma_tx_search(pred, src, qp, mode, use_ts=False, lfnst=False):
    """slice.rs:810-874 encode_luma's transform choice for one square block.

    Returns (mts_idx, lfnst_idx, ts, cbf, sse, levels, samples)."""
    pred = np.ascontiguousarray(pred, dtype=np.int32)
    src = np.ascontiguousarray(src, dtype=np.int32)
    n = pred.shape[0]
    lv = np.zeros(n * n, np.int16)
    sm = np.zeros(n * n, np.int16)
    sse = C.c_uint64(0)
    r = lib().orc_luma_tx_search(n, _p(pred), _p(src), qp, mode, int(use_ts), int(lfnst), _p(lv), _p(sm),
                                 C.byref(sse))
    return (r >> 8) & 0xF, (r >> 4) & 0xF, (r >> 1) & 1, r & 1, sse.value, lv, sm


# ------------------------------------------------------- LMCS / joint chroma --

LMCS_APS_DTYPE = np.dtype([("bin_cw_delta", "<i2", (16,)), ("min_bin_idx", "u1"), ("max_bin_idx", "u1"),
                           ("chroma_res_scaling_offset", "i1"), ("reserved", "u1")])
LMCS_TABLES_DTYPE = np.dtype([("bit_depth", "u1"), ("min_bin_idx", "u1"), ("max_bin_idx", "u1"),
                              ("reserved", "u1"), ("reshape_pivot", "<i4", (17,)), ("chroma_adj_lut", "<i4", (16,)),
                              ("fwd_lut", "<u2", (4096,)), ("inv_lut", "<u2", (4096,))])
CRES_DTYPE = np.dtype([("log2_w", "u1"), ("log2_h", "u1"), ("bit_depth", "u1"), ("joint", "i1"),
                       ("flags", "<u4"), ("scale", "<i4"), ("cb_off", "<u4"), ("cr_off", "<u4")])


def lmcs_build(aps, bd):
    """LmcsReshaper16::from_aps (filter.rs:2628-2705) -> LMCS_TABLES_DTYPE record."""
    a = np.asarray(aps, dtype=LMCS_APS_DTYPE).reshape(1).copy()
    t = np.zeros(1, LMCS_TABLES_DTYPE)
    lib().orc_lmcs_build(_p(a), bd, _p(t))
    return t[0]


def lmcs_map_plane(tables, plane, inverse=True):
    t = np.asarray(tables, dtype=LMCS_TABLES_DTYPE).reshape(1).copy()
    out = np.ascontiguousarray(plane, dtype=np.uint16).copy()
    lib().orc_lmcs_map_plane(_p(t), int(inverse), _p(out), out.size)
    return out


def lmcs_chroma_scale(tables, luma, ctu, x, y):
    t = np.asarray(tables, dtype=LMCS_TABLES_DTYPE).reshape(1).copy()
    luma = np.ascontiguousarray(luma, dtype=np.uint16)
    h, w = luma.shape
    return lib().orc_lmcs_chroma_scale(_p(t), _p(luma), w, w, h, ctu, x, y)


def chroma_residuals(recs, res):
    recs = np.ascontiguousarray(recs, dtype=CRES_DTYPE)
    out = np.ascontiguousarray(res, dtype=np.int16).copy()
    for i in range(len(recs)):
        lib().orc_chroma_residuals(_p(recs[i:i + 1].copy()), _p(out))
    return out


def sao_bounded(plane, vis_w, vis_h, bd, ctu, ctu_cols, params):
    """The general decoder's SAO of one plane (filter.rs:1954-2033 per CTU,
    decode_general.rs:5189-5223); params: SAO_DTYPE-layout records per CTU."""
    src = _u16(plane)
    dst = np.zeros_like(src)
    prm = np.ascontiguousarray(params).view(np.uint8)
    lib().orc_sao_bounded(_p(src), _p(dst), src.shape[1], src.shape[0], vis_w, vis_h, bd, ctu, ctu_cols, _p(prm),
                          prm.size // 6)
    return dst


def mip_predict(above, left, w, h, mode, transposed, bd):
    """predict_mip_16 (predict.rs:4109 / predict_mip_bd :2461) of one block."""
    a, l = _i32(above), _i32(left)
    out = np.zeros(w * h, np.int32)
    lib().orc_mip_predict(_p(a), _p(l), w, h, mode, int(transposed), bd, _p(out))
    return out


def mip_search(above, left, src, w, h, bd):
    """choose_best_mip_mode_16 (predict.rs:4166): (mode, transposed, sad, pred)."""
    a, l, s = _i32(above), _i32(left), _i32(src)
    out = np.zeros(w * h, np.int32)
    sad = C.c_uint64(0)
    r = lib().orc_mip_search(_p(a), _p(l), _p(s), w, h, bd, _p(out), C.byref(sad))
    return r & 0xFF, r >> 8, sad.value, out


def deblock_general(planes, vis_w, vis_h, bd, ctu, cells, ccells, params):
    """apply_deblock of the general decoder (decode_general.rs:4977) on a
    4:2:0 picture; returns filtered copies of the (Y, Cb, Cr) planes. cells /
    ccells / params in the vvcg_dbk_cell / vvcg_dbk_ccell / vvcg_dbk_params
    layouts (2-D record arrays, rows x cols)."""
    y, u, v = (_u16(p).copy() for p in planes)
    c = np.ascontiguousarray(cells)
    cc = np.ascontiguousarray(ccells)
    prm = np.ascontiguousarray(params).reshape(1)
    lib().orc_deblock_general(_p(y), _p(u), _p(v), y.shape[1], u.shape[1], vis_w, vis_h, bd, ctu, _p(c),
                              c.shape[1], c.shape[0], _p(cc), cc.shape[1], cc.shape[0], _p(prm))
    return y, u, v


CTU_MOTION_DTYPE = np.dtype([("mv", "<i4", (3, 2)), ("ref", "<i4", (3,)), ("cbf", "u1"), ("reserved", "u1", (3,))])
assert CTU_MOTION_DTYPE.itemsize == 40


def inter_ctu_deblock(planes, ctu, qp, cells):
    """The deblocking part of apply_inter_loop_filters (slice.rs:2291-2554)
    on an 8-bit 4:2:0 picture: returns filtered copies of the (Y, Cb, Cr)
    planes. cells: (height/ctu, width/ctu) CTU_MOTION_DTYPE records."""
    y, u, v = (_u16(p).copy() for p in planes)
    c = np.ascontiguousarray(cells, dtype=CTU_MOTION_DTYPE)
    h, w = y.shape
    assert c.shape == (h // ctu, w // ctu)
    lib().orc_inter_ctu_deblock(_p(y), _p(u), _p(v), y.shape[1], u.shape[1], w, h, ctu, qp, _p(c))
    return y, u, v


def _i32c(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def bdof(pred0, pred1, w, h):
    """apply_bdof_luma (inter.rs:1218-1339): w x h 14-bit predictions -> 8-bit samples."""
    a, b = _i32c(pred0), _i32c(pred1)
    out = np.zeros(w * h, np.int32)
    lib().orc_bdof(_p(a), _p(b), w, h, _p(out))
    return out


def dmvr(ref0, ref1, bx, by, dx, dy, mv):
    """refine_dmvr_subblock (inter.rs:1371-1471) on 8-bit planes; mv =
    (mv0 hor, mv0 ver, mv1 hor, mv1 ver); returns the refined four."""
    r0, r1 = np.ascontiguousarray(ref0, dtype=np.uint8), np.ascontiguousarray(ref1, dtype=np.uint8)
    m = _i32c(mv).copy()
    lib().orc_dmvr(_p(r0), _p(r1), r0.shape[1], r0.shape[0], r0.shape[1], bx, by, dx, dy, _p(m))
    return m


def affine_mvs(cp, six_param, w, h, inter_dir):
    """derive_affine_subblock_mvs (inter.rs:1502-1579): (subblock MVs
    (n, 2), PROF horizontal deltas (16,), vertical (16,), PROF enabled)."""
    c = _i32c(cp).reshape(6)
    sub = np.zeros(2 * (w // 4) * (h // 4), np.int32)
    ph, pv = np.zeros(16, np.int32), np.zeros(16, np.int32)
    en = lib().orc_affine_mvs(_p(c), int(six_param), w, h, inter_dir, _p(sub), _p(ph), _p(pv))
    return sub.reshape(-1, 2), ph, pv, bool(en)


def prof(src6x6, dmv_x, dmv_y, bi):
    """apply_prof_4x4 (inter.rs:1581-1609)."""
    s, x, y = _i32c(src6x6), _i32c(dmv_x), _i32c(dmv_y)
    out = np.zeros(16, np.int32)
    lib().orc_prof(_p(s), _p(x), _p(y), int(bi), _p(out))
    return out


def ciip(inter, intra, left_intra, above_intra):
    """apply_ciip_blend (inter.rs:1615-1630)."""
    a, b = _i32c(inter), _i32c(intra)
    out = np.zeros(a.size, np.int32)
    lib().orc_ciip(_p(a), _p(b), a.size, int(left_intra), int(above_intra), _p(out))
    return out


def gpm(pred0, pred1, w, h, split_dir, scale_x=0, scale_y=0):
    """predict_gpm_block (inter.rs:1673-1731)."""
    a, b = _i32c(pred0), _i32c(pred1)
    out = np.zeros(w * h, np.int32)
    lib().orc_gpm(_p(a), _p(b), w, h, split_dir, scale_x, scale_y, _p(out))
    return out


def dbk_lens(luma, size_p, size_q, ctb_boundary=False):
    """luma_lens / chroma_lens (decode_general.rs:4916 / :4929)."""
    out = np.zeros(2, np.int32)
    lib().orc_dbk_lens(int(luma), size_p, size_q, int(ctb_boundary), _p(out))
    return int(out[0]), int(out[1])


def dbk_bs(p_intra, q_intra, p_cbf, q_cbf, tu_edge, pmv, qmv, pref, qref):
    """derive_boundary_strength (filter.rs:202-226)."""
    return lib().orc_dbk_bs(int(p_intra), int(q_intra), int(p_cbf), int(q_cbf), int(tu_edge), pmv[0], pmv[1],
                            qmv[0], qmv[1], pref, qref)


def alf_general(y, u, v, vis_w, vis_h, bd, ctu, ctu_cols, ctus, params):
    """apply_alf of the general decoder (decode_general.rs:5225) on a 4:2:0
    picture; ctus / params in the vvcg_alf_ctu / vvcg_alf_params layouts."""
    y, u, v = _u16(y), _u16(u), _u16(v)
    dy, du, dv = np.zeros_like(y), np.zeros_like(u), np.zeros_like(v)
    c = np.ascontiguousarray(ctus).view(np.uint8)
    p = np.ascontiguousarray(params).view(np.uint8)
    lib().orc_alf_general(_p(y), _p(u), _p(v), _p(dy), _p(du), _p(dv), y.shape[1], y.shape[0], vis_w, vis_h, bd,
                          ctu, ctu_cols, _p(c), _p(p))
    return dy, du, dv


# ------------------------------------------------- general-decoder pictures --

DBK_CELL_DTYPE = np.dtype([("tu_id", "<u4"), ("tu_w", "<u2"), ("tu_h", "<u2"), ("mv", "<i4", (2, 2)),
                           ("ref_idx", "i1", (2,)), ("flags", "u1"), ("reserved", "u1")])
DBK_CCELL_DTYPE = np.dtype([("tu_cb", "<u4"), ("tu_cr", "<u4"), ("tu_w", "<u2"), ("tu_h", "<u2")])
_DBK_CODED, _DBK_INTRA, _DBK_CBF, _DBK_NO_TU = 1, 2, 4, 0xFFFFFFFF


def mark_tu_maps(width, height, tbs):
    """The deblocking maps mark_tu (decode_general.rs:4837-4907) leaves after
    the picture's transform blocks, visited in decode order (tbs: records
    with a "pred" block (x, y, w, h in component samples, cu_*, comp) and a
    "coded" flag): per 4x4 luma cell the last luma block's id (its index),
    size and cbf, and the coded / intra flags of its coding unit; per 2x2
    chroma cell the last Cb / Cr block ids and size."""
    cols, rows = width // 4, height // 4
    cells = np.zeros((rows, cols), DBK_CELL_DTYPE)
    cells["tu_id"] = _DBK_NO_TU
    cells["ref_idx"] = -1
    cc = np.zeros((rows, cols), DBK_CCELL_DTYPE)
    cc["tu_cb"] = _DBK_NO_TU
    cc["tu_cr"] = _DBK_NO_TU
    for i, t in enumerate(tbs):
        r = t["pred"]
        x, y, w, h = int(r["x"]), int(r["y"]), int(r["w"]), int(r["h"])
        if int(r["comp"]) == 0:
            x1, y1 = min(x + w, cols * 4), min(y + h, rows * 4)
            sub = cells[y // 4:(y1 + 3) // 4, x // 4:(x1 + 3) // 4]
            sub["tu_id"], sub["tu_w"], sub["tu_h"] = i, w, h
            sub["flags"] = (sub["flags"] & (0xFF ^ _DBK_CBF)) | (_DBK_CBF if int(t["coded"]) else 0)
            cx, cy, cw_, ch_ = int(r["cu_x"]), int(r["cu_y"]), int(r["cu_w"]), int(r["cu_h"])
            cx1, cy1 = min(cx + cw_, cols * 4), min(cy + ch_, rows * 4)
            cu = cells[cy // 4:(cy1 + 3) // 4, cx // 4:(cx1 + 3) // 4]
            cu["flags"] |= _DBK_CODED | _DBK_INTRA
        else:
            x1, y1 = min(x + w, cols * 2), min(y + h, rows * 2)
            sub = cc[y // 2:(y1 + 1) // 2, x // 2:(x1 + 1) // 2]
            sub["tu_cb" if int(r["comp"]) == 1 else "tu_cr"] = i
            sub["tu_w"], sub["tu_h"] = w, h
    return cells, cc


def general_picture(pic, tbs, group_sizes, levels, slot_count, sao, alf_ctus, alf_params):
    """decode_general_picture's reconstruction and loop filters for one intra
    picture, composed from the restatements above in the reference's order
    (decode_general.rs:1134-1150): residuals of the coded blocks (tu_batch),
    reconstruction of every block in decode order (gen_intra_recon, one group
    after another), deblocking over mark_tu's maps (deblock_general), SAO per
    component (sao_bounded; chroma CTUs of half size) and ALF (alf_general),
    as the picture's tools select. Records as the GEN_* layouts of the
    package; offsets local to the picture. Returns the visible (Y, Cb, Cr)."""
    w, h = int(pic["width"]), int(pic["height"])
    vw, vh = int(pic["vis_width"]), int(pic["vis_height"])
    cvw, cvh = (vw + 1) // 2, (vh + 1) // 2
    bd, ctu, tools = int(pic["bit_depth"]), 1 << int(pic["ctu_log2"]), int(pic["tools"])
    coded = tbs[tbs["coded"] != 0]["tu"]
    rc, res = tu_batch(coded.view(TU_DTYPE) if coded.dtype != TU_DTYPE else coded, levels, slot_count)
    if rc:
        raise ValueError(f"tu_batch rejected record {-rc - 1}")
    Y = np.zeros((h, w), np.uint16)
    U = np.zeros((h // 2, w // 2), np.uint16)
    V = np.zeros((h // 2, w // 2), np.uint16)
    dy = np.zeros((h // 4, w // 4), np.uint8)
    dc = np.zeros((h // 2, w // 2), np.uint8)
    starts = np.concatenate([[0], np.cumsum(group_sizes)]).astype(np.uint32)
    Y, U, V, _, _, _ = gen_intra_recon(Y, U, V, dy, dc, bd, ctu, np.ascontiguousarray(tbs["pred"]), starts, res,
                                       slot_count, bool(int(pic["vert_collocated"])))
    cols, rows = -(-vw // ctu), -(-vh // ctu)
    nctu = cols * rows
    if tools & 2:  # deblocking
        cells, cc = mark_tu_maps(w, h, tbs)
        Y, U, V = deblock_general((Y, U, V), vw, vh, bd, ctu, cells, cc, pic["dbk"])
    if tools & 4:  # SAO
        Y = sao_bounded(Y, vw, vh, bd, ctu, cols, sao[:nctu])
        U = sao_bounded(U, cvw, cvh, bd, ctu // 2, cols, sao[nctu:2 * nctu])
        V = sao_bounded(V, cvw, cvh, bd, ctu // 2, cols, sao[2 * nctu:3 * nctu])
    if tools & 8:  # ALF
        Y, U, V = alf_general(Y, U, V, vw, vh, bd, ctu, cols, alf_ctus, alf_params)
    return Y[:vh, :vw], U[:cvh, :cvw], V[:cvh, :cvw]


# ---- the multi-tool stream (VvcMultiToolEncoder: IDR + P pictures) ----------
SLICE_DEP_QUANT, SLICE_SIGN_HIDING, SLICE_DEBLOCK, SLICE_FULL_INTRA_MODES = 1, 2, 4, 8
INTER_CU_MERGE, INTER_CU_SKIP, INTER_CU_ALT_HPEL = 1, 2, 4
INTER_CU_DTYPE = np.dtype([("mv", "<i4", (2, 2)), ("mvd", "<i4", (2,)), ("ref_idx", "i1", (2,)), ("inter_dir", "u1"),
                           ("bcw_idx", "u1"), ("flags", "u1"), ("mvp_idx", "u1"), ("cbf", "u1"), ("tu_tools", "u1"),
                           ("level_off", "<i4", (3,)), ("reserved", "<u4")])
assert INTER_CU_DTYPE.itemsize == 48


def derive_intra_mpms(left=None, above=None):
    """predict.rs:1455-1506: the 6 MPM candidates from the left / above modes."""
    out = np.zeros(6, np.uint8)
    lib().orc_derive_intra_mpms(-1 if left is None else int(left), -1 if above is None else int(above), _p(out))
    return out


def _planes8(y, u, v):
    return tuple(np.ascontiguousarray(a, dtype=np.uint8) for a in (y, u, v))


def _ref_ptrs(refs):
    refs = [_planes8(*r) for r in refs]
    arr = (C.c_void_p * (3 * len(refs)))(*[a.ctypes.data for r in refs for a in r])
    return refs, arr


def mt_encode(y, u, v, qp, opts=0, ctu_log2=5):
    """encode_picture_multitool's decisions and reconstruction (slice.rs:2575-2970)
    of one 8-bit 4:2:0 IDR picture; returns (cus, levels, (y, u, v))."""
    y, u, v = _planes8(y, u, v)
    h, w = y.shape
    tb = min(1 << ctu_log2, 32)
    cus = np.zeros((h // tb) * (w // tb), dtype=CU_DTYPE)
    levels = np.zeros(w * h * 3 // 2 + 64, np.int16)
    used = C.c_uint64(0)
    ry, ru, rv = np.zeros_like(y), np.zeros_like(u), np.zeros_like(v)
    rc = lib().orc_mt_encode(_p(y), _p(u), _p(v), w, h, qp, ctu_log2, opts, _p(cus), _p(levels), C.byref(used),
                             _p(ry), _p(ru), _p(rv))
    if rc:
        raise ValueError(f"mt_encode rejected ({rc})")
    return cus, levels[:used.value].copy(), (ry, ru, rv)


def mt_decode(cus, levels, w, h, qp, opts=0, ctu_log2=5):
    """decode_picture_multitool's reconstruction (slice.rs:3012-3300)."""
    cus = np.ascontiguousarray(cus, dtype=CU_DTYPE)
    levels = np.ascontiguousarray(levels, dtype=np.int16)
    ry = np.zeros((h, w), np.uint8)
    ru, rv = np.zeros((h // 2, w // 2), np.uint8), np.zeros((h // 2, w // 2), np.uint8)
    rc = lib().orc_mt_decode(_p(cus), _p(levels), levels.size, w, h, qp, ctu_log2, opts, _p(ry), _p(ru), _p(rv))
    if rc:
        raise ValueError(f"mt_decode rejected ({rc})")
    return ry, ru, rv


def _write(fn, cus, dtype, levels, w, h, qp, opts):
    cus = np.ascontiguousarray(cus, dtype=dtype)
    levels = np.ascontiguousarray(levels, dtype=np.int16)
    cap = 64 + 4 * levels.size + 32 * len(cus)
    out = np.zeros(cap, np.uint8)
    n = C.c_uint64(0)
    rc = fn(_p(cus), _p(levels), levels.size, w, h, qp, opts, _p(out), cap, C.byref(n))
    if rc:
        raise ValueError(f"the writer rejected the records ({rc})")
    return out[:n.value].tobytes()


def mt_write(cus, levels, w, h, qp, opts=0):
    """The slice data encode_picture_multitool writes (slice.rs:2867-2960); bytes."""
    return _write(lib().orc_mt_write, cus, CU_DTYPE, levels, w, h, qp, opts)


def p_write(cus, levels, w, h, qp, opts=0):
    """The slice data encode_inter_picture writes (slice.rs:3451-3536); bytes."""
    return _write(lib().orc_p_write, cus, INTER_CU_DTYPE, levels, w, h, qp, opts)


def inter_encode(y, u, v, qp, refs, opts=0):
    """encode_inter_picture (slice.rs:3307-3549) of one P picture against the
    L0 reference pictures `refs` ((y, u, v) each); returns (cus, levels, (y, u, v))."""
    y, u, v = _planes8(y, u, v)
    h, w = y.shape
    keep, arr = _ref_ptrs(refs)
    cus = np.zeros((h // 32) * (w // 32), dtype=INTER_CU_DTYPE)
    levels = np.zeros(w * h * 3 // 2 + 64, np.int16)
    used = C.c_uint64(0)
    ry, ru, rv = np.zeros_like(y), np.zeros_like(u), np.zeros_like(v)
    rc = lib().orc_inter_encode(_p(y), _p(u), _p(v), w, h, qp, 5, opts, arr, len(keep), _p(cus), _p(levels),
                                C.byref(used), _p(ry), _p(ru), _p(rv))
    if rc:
        raise ValueError(f"inter_encode rejected ({rc})")
    return cus, levels[:used.value].copy(), (ry, ru, rv)


def inter_resolve_motion(cus, w, h):
    """decode_inter_picture's motion derivation (slice.rs:3617-3677): fills
    the motion of merge / skip records (candidate 0) and AMVP records
    (predictor mvp_idx + mvd) in place order; returns a new array."""
    cus = np.array(cus, dtype=INTER_CU_DTYPE, copy=True)
    rc = lib().orc_inter_resolve_motion(_p(cus), w, h, 5)
    if rc:
        raise ValueError(f"inter_resolve_motion rejected ({rc})")
    return cus


def inter_decode(cus, levels, w, h, qp, refs, opts=0):
    """decode_inter_picture's reconstruction (slice.rs:3677-3834) from records with motion."""
    cus = np.ascontiguousarray(cus, dtype=INTER_CU_DTYPE)
    levels = np.ascontiguousarray(levels, dtype=np.int16)
    keep, arr = _ref_ptrs(refs)
    ry = np.zeros((h, w), np.uint8)
    ru, rv = np.zeros((h // 2, w // 2), np.uint8), np.zeros((h // 2, w // 2), np.uint8)
    rc = lib().orc_inter_decode(_p(cus), _p(levels), levels.size, w, h, qp, 5, opts, arr, len(keep), _p(ry), _p(ru),
                                _p(rv))
    if rc:
        raise ValueError(f"inter_decode rejected ({rc})")
    return ry, ru, rv


def multitool_stream(frames, qp, keyint=3, opts=0):
    """VvcMultiToolEncoder::encode_i420 (mod.rs:1512-1720) over 8-bit 4:2:0
    frames of coded size: an IDR picture whenever poc = index % keyint is 0,
    else a P picture predicting from the most recent picture (the DPB's
    build_ref_lists, inter.rs:481). Returns one dict per picture: kind ("I" /
    "P"), data (slice data), cus, levels, recon (y, u, v)."""
    out, last = [], None
    for i, (y, u, v) in enumerate(frames):
        h, w = np.asarray(y).shape
        if i % max(keyint, 1) == 0 or last is None:
            cus, levels, rec = mt_encode(y, u, v, qp, opts)
            data = mt_write(cus, levels, w, h, qp, opts)
            out.append(dict(kind="I", data=data, cus=cus, levels=levels, recon=rec))
        else:
            cus, levels, rec = inter_encode(y, u, v, qp, [last], opts)
            data = p_write(cus, levels, w, h, qp, opts)
            out.append(dict(kind="P", data=data, cus=cus, levels=levels, recon=rec))
        last = rec
    return out
