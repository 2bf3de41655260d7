"""The normative tables of csrc/vvc_tables.h against the reference's own literals.

The kernels and the oracle compile the same header, so a transcription error
there would pass every GPU parity test. tests/golden/tables.json holds the
values of the reference's table constants (extracted from its Rust sources by
tests/golden/make_tables.py, each with the file:line it came from); every
header table is compared with it entry by entry.
"""
from __future__ import annotations

import json
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "rustmpeg-next_b200", "csrc", "vvc_tables.h")
GOLD = os.path.join(ROOT, "tests", "golden", "tables.json")

# header table -> the reference constants it holds, concatenated in order
PAIRS = {
    "kInvQuantScale": ["INV_QUANT_SCALES", "INV_QUANT_SCALES_SQRT2"],
    "kQuantScale": ["QUANT_SCALES", "QUANT_SCALES_SQRT2"],
    "kDct2N2": ["DCT2_2"], "kDct2N4": ["DCT2_4"], "kDct2N8": ["DCT2_8"], "kDct2N16": ["DCT2_16"],
    "kDct2N32": ["DCT2_32"], "kDct2N64": ["DCT2_64"],
    "kDst7N4": ["DST7_4"], "kDst7N8": ["DST7_8"], "kDst7N16": ["DST7_16"], "kDst7N32": ["DST7_32"],
    "kDct8N4": ["DCT8_4"], "kDct8N8": ["DCT8_8"], "kDct8N16": ["DCT8_16"], "kDct8N32": ["DCT8_32"],
    "kLfnst8x8": ["LFNST_8X8"], "kLfnst4x4": ["LFNST_4X4"], "kLfnstLut": ["LFNST_LUT"],
    "kDbfTc": ["DBF_TC_TABLE"], "kDbfBeta": ["DBF_BETA_TABLE"],
    "kAlfFixedCoeff": ["ALF_FIXED_FILTER_COEFF"], "kAlfClassToFilter": ["ALF_CLASS_TO_FILTER_MAPPING"],
    "kAlfClip": ["ALF_CLIP_VALS_8BIT", "ALF_CLIP_VALS_10BIT", "ALF_CLIP_VALS_12BIT"],
    "kAlfTransposePerm": ["ALF_TRANSPOSE_PERM"],
    "kLumaTaps8": ["LUMA_FILTER_8TAP"], "kLumaAltHpel": ["LUMA_ALT_HPEL_FILTER_8TAP"],
    "kAffineTaps8": ["AFFINE_LUMA_FILTER_8TAP"], "kBcwWeights": ["BCW_WEIGHTS"],
    "kGeoDis": ["GEO_DIS"], "kGeoAngleToMask": ["GEO_ANGLE_TO_MASK"], "kBilinear4": ["BILINEAR_FILTER_PREC4"],
    "kAngTable": ["ANG_TABLE"], "kInvAngTable": ["INV_ANG_TABLE"],
    "kIntraFilterThreshold": ["INTRA_FILTER_THRESHOLD"], "kChromaTaps4": ["CHROMA_FILTER_4TAP"],
    "kCclmDivSig": ["CCLM_DIV_SIG_TABLE"],
    "kMip4x4": ["MIP_MATRIX_4X4"], "kMip8x8": ["MIP_MATRIX_8X8"], "kMip16x16": ["MIP_MATRIX_16X16"],
    # vvc_cabac.h
    "kCtxInitI": ["CTX_INIT_I"], "kCtxInitP": ["CTX_INIT_P"], "kCtxInitB": ["CTX_INIT_B"],
    "kRenormLps": ["RENORM_LPS"], "kPrefixCtx": ["PREFIX_CTX"],
    "kMinInGroup": ["MIN_IN_GROUP"], "kGroupIdx": ["GROUP_IDX"], "kGoRicePars": ["GO_RICE_PARS_COEFF"],
}
CABAC_HDR = os.path.join(ROOT, "rustmpeg-next_b200", "csrc", "vvc_cabac.h")


def header_tables():
    """Every `static const <type> kName[..]...[..] = { ... };` (or constexpr)
    of the two headers, flattened row-major, keyed by name."""
    src = re.sub(r"//[^\n]*", "", open(HDR).read() + open(CABAC_HDR).read())
    src = src.replace("[kNumContexts]", "[379]")
    out = {}
    for m in re.finditer(r"(?:static\s+const|constexpr)\s+\w+\s+(k\w+)\s*((?:\[\s*\d+\s*\])+)\s*=\s*\{", src):
        depth, i = 0, m.end() - 1
        while True:
            if src[i] == "{":
                depth += 1
            elif src[i] == "}":
                depth -= 1
                if depth == 0:
                    break
            i += 1
        vals = [int(v) for v in re.findall(r"-?\d+", src[m.end():i])]
        dims = [int(d) for d in re.findall(r"\d+", m.group(2))]
        assert int(np.prod(dims)) == len(vals), (m.group(1), dims, len(vals))
        out[m.group(1)] = np.array(vals, dtype=np.int64)
    return out


@pytest.fixture(scope="module")
def gold():
    return json.load(open(GOLD))


@pytest.fixture(scope="module")
def hdr():
    return header_tables()


@pytest.mark.parametrize("name", sorted(PAIRS))
def test_header_table_equals_reference_literal(name, gold, hdr):
    assert name in hdr, f"{name} missing from vvc_tables.h"
    ref = np.concatenate([np.array(gold[r]["values"], dtype=np.int64) for r in PAIRS[name]])
    got = hdr[name]
    assert got.size == ref.size, f"{name}: {got.size} entries, reference {ref.size}"
    bad = np.flatnonzero(got != ref)
    where = ", ".join(gold[r]["at"] for r in PAIRS[name])
    assert bad.size == 0, (f"{name} differs from {where} at {bad.size} entries, first index {bad[0]}: "
                           f"header {got[bad[0]]}, reference {ref[bad[0]]}")


def test_every_golden_table_is_checked(gold):
    used = {r for refs in PAIRS.values() for r in refs}
    assert used == {k for k in gold if not k.startswith("_")}


def test_context_offsets_equal_the_reference(gold):
    """The first context of each syntax element's set (vvc_cabac.h kCtx*)
    against cabac.rs's ctx module, every constant."""
    src = open(CABAC_HDR).read()
    got = {m.group(1): int(m.group(2)) for m in re.finditer(r"constexpr\s+int\s+kCtx(\w+)\s*=\s*(\d+)\s*;", src)}
    ref = gold["_ctx_offsets"]["values"]
    camel = {"".join(w.capitalize() for w in k.lower().split("_")): v for k, v in ref.items()}
    assert got == camel, sorted(set(got.items()) ^ set(camel.items()))[:5]


def test_dct2_matrices_nest(hdr):
    """Property of the reference's DCT-II family: the N-point matrix is the
    even rows' left halves of the 2N-point one (dct.rs builds every size from
    the same basis), checked on the header independently of the golden file."""
    for n in (2, 4, 8, 16, 32):
        big = hdr[f"kDct2N{2 * n}"].reshape(2 * n, 2 * n)
        small = hdr[f"kDct2N{n}"].reshape(n, n)
        assert np.array_equal(big[::2, :n], small), n
