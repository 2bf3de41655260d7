"""CPU: the sparse level form the decoder accepts (TOOL_SPARSE_LEVELS).

synth.sparsify writes, per coded TB, the count of its nonzero levels at an
even offset, one unused word and (raster index, level) pairs with strictly
rising indices; densify inverts it. Checked here: the layout, the round trip
to the same raster levels, the flag's value against include/vvcg.h, and the
oracle's reconstruction of the round-tripped records.
"""
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SPECS = [
    dict(width=128, height=64, bit_depth=10, chroma_format=1, ctu_log2=5, qp=22),
    dict(width=128, height=128, bit_depth=8, chroma_format=2, ctu_log2=6, qp=30),
    dict(width=256, height=128, bit_depth=12, chroma_format=3, ctu_log2=7, qp=37),
    dict(width=64, height=64, bit_depth=10, chroma_format=0, ctu_log2=5, qp=27),
]


def _coded_tbs(synth, pics, cus):
    for p in pics:
        tb, sizes = synth._tb_sizes(p)
        c0 = int(p["cu_offset"])
        n = (int(p["width"]) // tb) * (int(p["height"]) // tb)
        for k in range(c0, c0 + n):
            for c in range(3 if int(p["chroma_format"]) else 1):
                o = int(cus["level_off"][k, c])
                if o >= 0 and (int(cus["cbf"][k]) >> c) & 1:
                    yield k, c, o, sizes[c]


def test_tool_flag_matches_the_header(pkg):
    hdr = open(os.path.join(ROOT, "include", "vvcg.h")).read()
    m = re.search(r"VVCG_TOOL_SPARSE_LEVELS\s*=\s*1u\s*<<\s*(\d+)", hdr)
    assert m and pkg.TOOL_SPARSE_LEVELS == 1 << int(m.group(1))


def test_sparse_layout_and_round_trip(pkg):
    from rustmpeg_next_b200 import synth

    pics, cus, levels, _, _ = synth.random_records(SPECS, seed=21, tools=pkg.TOOL_DEP_QUANT)
    sp, sc, sl = synth.sparsify(pics, cus, levels)
    assert (sp["tools"] & pkg.TOOL_SPARSE_LEVELS).all()
    assert (pics["tools"] & pkg.TOOL_SPARSE_LEVELS == 0).all()  # inputs untouched
    dense = {(k, c): levels[o:o + n] for k, c, o, n in _coded_tbs(synth, pics, cus)}
    seen = 0
    for k, c, o, n in _coded_tbs(synth, sp, sc):
        assert o % 2 == 0
        cnt = int(sl[o])
        pairs = sl[o + 2:o + 2 + 2 * cnt].reshape(-1, 2).astype(np.int64)
        assert (np.diff(pairs[:, 0]) > 0).all() and (pairs[:, 0] < n).all() and (pairs[:, 1] != 0).all()
        want = dense[(k, c)]
        assert cnt == np.count_nonzero(want)
        assert (want[pairs[:, 0]] == pairs[:, 1]).all()
        seen += 1
    assert seen == len(dense)
    assert len(sl) < len(levels)
    bp, bc, bl = synth.densify(sp, sc, sl)
    assert (bp["tools"] == pics["tools"]).all()
    for k, c, o, n in _coded_tbs(synth, bp, bc):
        assert (bl[o:o + n] == dense[(k, c)]).all()


def test_round_tripped_records_reconstruct_identically(pkg, orc):
    from rustmpeg_next_b200 import synth

    pics, cus, levels, ctus, _ = synth.random_records(SPECS[:2], seed=22, tools=pkg.TOOL_DEP_QUANT | pkg.TOOL_DEBLOCK)
    bp, bc, bl = synth.densify(*synth.sparsify(pics, cus, levels))
    for p, q in zip(pics, bp):
        tb = min(1 << int(p["ctu_log2"]), 32)
        n = (int(p["width"]) // tb) * (int(p["height"]) // tb)
        nc = (int(p["width"]) >> int(p["ctu_log2"])) * (int(p["height"]) >> int(p["ctu_log2"]))
        c0, t0 = int(p["cu_offset"]), int(p["ctu_offset"])
        ra, pa = orc.recon_frame(p, cus[c0:c0 + n], levels, ctus[t0:t0 + nc])
        rb, pb = orc.recon_frame(q, bc[c0:c0 + n], bl, ctus[t0:t0 + nc])
        assert ra == rb == 0
        for a, b in zip(pa, pb):
            assert a is None and b is None or (a == b).all()


def test_empty_and_all_zero_tbs(pkg):
    """A coded TB whose levels are all zero becomes a count of 0 (two words);
    a batch without coded TBs gives an empty pool."""
    from rustmpeg_next_b200 import synth

    pics, cus, levels, _, _ = synth.random_records(SPECS[:1], seed=23, tools=0)
    k = int(np.argmax(cus["cbf"] & 1))
    o = int(cus["level_off"][k, 0])
    levels = levels.copy()
    levels[o:o + 1024] = 0
    sp, sc, sl = synth.sparsify(pics, cus, levels)
    so = int(sc["level_off"][k, 0])
    assert sl[so] == 0 and sl[so + 1] == 0
    none = cus.copy()
    none["cbf"] = 0
    none["level_off"] = -1
    _, nc, nl = synth.sparsify(pics, none, levels)
    assert len(nl) == 0 and (nc["level_off"] == -1).all()
