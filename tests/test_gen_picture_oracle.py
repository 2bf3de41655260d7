"""CPU: the inputs and the oracle composition of the general decoder's picture
pass: the synthetic coding trees (blocks inside the picture, decode-order
groups, slots and level ranges), mark_tu's deblocking maps, and
oracle.general_picture (each loop filter changes the picture; the decode
order matters)."""
import numpy as np


def test_synthetic_general_pictures_are_well_formed(pkg):
    from rustmpeg_next_b200 import synth

    for seed, (w, h, ctu, bd) in enumerate([(200, 120, 64, 10), (128, 128, 32, 8), (256, 136, 128, 12),
                                             (96, 64, 16, 10)]):
        p, tbs, sizes, lv, slots, sao, alf, prm = synth.random_general_picture(w, h, ctu=ctu, bd=bd, seed=seed)
        assert int(sizes.sum()) == len(tbs) and (sizes > 0).all()
        r = tbs["pred"]
        luma, chroma = r["comp"] == 0, r["comp"] != 0
        pw, ph = int(p["width"]), int(p["height"])
        assert pw % ctu == 0 and ph % ctu == 0
        assert ((r["x"] + r["w"])[luma] <= pw).all() and ((r["y"] + r["h"])[luma] <= ph).all()
        assert ((r["x"] + r["w"])[chroma] <= pw // 2).all() and ((r["y"] + r["h"])[chroma] <= ph // 2).all()
        assert (r["w"][chroma] >= 2).all() and (r["w"][chroma] <= 32).all() and (r["h"][chroma] <= 32).all()
        assert (r["w"][luma] <= 64).all() and (r["h"][luma] <= 64).all()
        n = (r["w"].astype(np.int64) * r["h"])
        assert (r["out_off"][1:] == np.cumsum(n)[:-1]).all() and int(n.sum()) == slots
        c = tbs["coded"] != 0
        assert ((tbs["tu"]["in_off"][c].astype(np.int64) + n[c]) <= lv.size).all()
        assert (tbs["tu"]["out_off"] == r["out_off"]).all()
        # every visible luma sample is covered by exactly one luma block
        cover = np.zeros((ph, pw), np.int32)
        for t in r[luma]:
            cover[t["y"]:t["y"] + t["h"], t["x"]:t["x"] + t["w"]] += 1
        assert (cover[:h, :w] == 1).all()
        assert len(sao) == 3 * len(alf)


def test_mark_tu_maps_keep_the_last_block_of_a_cell(orc):
    from rustmpeg_next_b200 import GEN_TB_DTYPE

    tbs = np.zeros(5, GEN_TB_DTYPE)
    # a 4x16 CU split vertically into four 1x16 sub-partitions, then its chroma
    for i in range(4):
        tbs[i]["pred"]["x"], tbs[i]["pred"]["y"], tbs[i]["pred"]["w"], tbs[i]["pred"]["h"] = 8 + i, 0, 1, 16
        tbs[i]["pred"]["cu_x"], tbs[i]["pred"]["cu_w"], tbs[i]["pred"]["cu_h"] = 8, 4, 16
        tbs[i]["coded"] = i == 3
    tbs[4]["pred"]["comp"], tbs[4]["pred"]["x"], tbs[4]["pred"]["w"], tbs[4]["pred"]["h"] = 1, 4, 2, 8
    cells, cc = orc.mark_tu_maps(32, 32, tbs)
    assert (cells["tu_id"][0:4, 2] == 3).all() and (cells["tu_w"][0:4, 2] == 1).all()
    assert (cells["flags"][0:4, 2] == 1 | 2 | 4).all()
    assert (cells["tu_id"][0:4, 0] == 0xFFFFFFFF).all()
    assert (cc["tu_cb"][0:4, 2] == 4).all() and (cc["tu_cr"][0:4, 2] == 0xFFFFFFFF).all()


def test_general_picture_filters_and_decode_order(pkg, orc):
    from rustmpeg_next_b200 import synth

    p, tbs, sizes, lv, slots, sao, alf, prm = synth.random_general_picture(160, 96, ctu=32, bd=10, seed=7)
    outs = {}
    for tools in (0, 2, 2 | 4, 2 | 4 | 8):
        q = p.copy()
        q["tools"] = tools
        outs[tools] = orc.general_picture(q, tbs, sizes, lv, slots, sao, alf, prm)
    for a, b in ((0, 2), (2, 6), (6, 14)):
        assert any((x != y).any() for x, y in zip(outs[a], outs[b])), (a, b)
    again = orc.general_picture(p, tbs, sizes, lv, slots, sao, alf, prm)
    assert all((x == y).all() for x, y in zip(again, outs[14]))
    # the same blocks as one group each in reverse decode order reconstruct differently
    q = p.copy()
    q["tools"] = 0
    rev = tbs[::-1].copy()
    other = orc.general_picture(q, rev, np.ones(len(rev), np.uint32), lv, slots, sao, alf, prm)
    assert any((x != y).any() for x, y in zip(other, outs[0]))
