"""CPU: the reference's own loop-filter and LMCS tests (crates/rustmpeg-video/
src/vvc/filter.rs:2855-3023) ported to the oracle's 16-bit functions at bit
depth 8, where the reference requires them to equal its 8-bit path: an
identity LMCS keeps all 256 levels and scales chroma by 1 << 11, deblocking
smooths a step edge below beta, a band offset moves the matching band, and
ALF with fixed filter 4 of the normative table keeps a constant plane."""
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_identity_lmcs_preserves_all_256_levels(orc):
    aps = np.zeros(1, orc.LMCS_APS_DTYPE)
    aps["min_bin_idx"], aps["max_bin_idx"] = 0, 15
    t = orc.lmcs_build(aps, 8)
    levels = np.arange(256)
    assert np.array_equal(t["fwd_lut"][:256], levels)
    assert np.array_equal(t["inv_lut"][:256], levels)
    luma = np.full((64, 64), 128, np.uint16)
    assert orc.lmcs_chroma_scale(t, luma, 64, 0, 0) == 1 << 11


def test_deblocking_smooths_step_edge_when_below_beta(orc):
    # an 8-sample edge at x = 8: p side 100, q side 108, QP 30, bS 2
    plane = np.full((8, 16), 100, np.uint16)
    plane[:, 8:] = 108
    out = orc.deblock_luma(plane, 8, 8, 16, 30, bs=2)
    assert (out[:, 7] > 100).all()
    assert (out[:, 8] < 108).all()


def test_sao_band_offset_modifies_matching_samples(orc):
    src = np.full((8, 8), 64, np.uint16)  # 64 >> 3 == band 8
    dst, rc = orc.sao_region(src, src, 8, 0, 0, 8, 8, 1, 8, [5, -2, 0, 0])
    assert rc == 0
    assert (dst == 69).all()


def _fixed_filter(k):
    text = open(os.path.join(ROOT, "rustmpeg-next_b200", "csrc", "vvc_tables.h")).read()
    body = re.search(r"kAlfFixedCoeff\[832\]\s*=\s*\{(.*?)\};", text, re.S).group(1)
    vals = [int(v) for v in re.findall(r"-?\d+", body)]
    assert len(vals) == 832
    return vals[13 * k:13 * k + 12]


def test_alf_preserves_constant_plane(orc):
    plane = np.full((16, 16), 140, np.uint16)
    aps = dict(coeff=np.array([_fixed_filter(4)], np.int16), clip_idx=np.zeros((1, 12), np.uint8),
               delta_idx=np.zeros(25, np.uint8), luma_clip=1)
    out, rc = orc.alf_luma(plane, 8, aps)
    assert rc == 0
    assert (out == 140).all()
