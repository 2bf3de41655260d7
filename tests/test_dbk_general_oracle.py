"""CPU: the oracle's restatement of the general decoder's deblocking
(apply_deblock, decode_general.rs:4977-5187).

Pins: the reference's known answers for luma_lens / chroma_lens
(decode_general.rs:5717-5736), the boundary-strength rule
(filter.rs:202-226) case by case, and a cross-check of the whole driver
against the frame path's plane drivers (deblock_luma_plane_16 /
deblock_chroma_plane_16, filter.rs:2344 / :2433) on a uniform grid of intra
transform blocks, where both must filter the same edges the same way.
"""
import numpy as np
import pytest


def test_luma_lens_known_answers(orc):
    # decode_general.rs:5719-5724
    assert orc.dbk_lens(True, 4, 32) == (1, 1)
    assert orc.dbk_lens(True, 32, 4) == (1, 1)
    assert orc.dbk_lens(True, 8, 8) == (3, 3)
    assert orc.dbk_lens(True, 32, 8) == (7, 3)
    assert orc.dbk_lens(True, 8, 64) == (3, 7)
    assert orc.dbk_lens(True, 16, 16) == (3, 3)


def test_chroma_lens_known_answers(orc):
    # decode_general.rs:5731-5735
    assert orc.dbk_lens(False, 8, 8, False) == (3, 3)
    assert orc.dbk_lens(False, 16, 8, False) == (3, 3)
    assert orc.dbk_lens(False, 8, 8, True) == (1, 3)
    assert orc.dbk_lens(False, 4, 16, False) == (1, 1)
    assert orc.dbk_lens(False, 16, 4, True) == (1, 1)


def test_boundary_strength_rules(orc):
    z = (0, 0)
    assert orc.dbk_bs(True, False, False, False, True, z, z, 0, 0) == 2
    assert orc.dbk_bs(False, True, True, True, True, z, z, 0, 0) == 2
    assert orc.dbk_bs(False, False, True, False, True, z, z, 0, 0) == 1
    assert orc.dbk_bs(False, False, True, False, False, z, z, 0, 0) == 0  # cbf counts on TU edges only
    assert orc.dbk_bs(False, False, False, False, True, z, z, 3, 4) == 1  # different reference pictures
    assert orc.dbk_bs(False, False, False, False, True, (8, 0), z, 2, 2) == 1  # half a sample apart
    assert orc.dbk_bs(False, False, False, False, True, (7, -7), z, 2, 2) == 0
    assert orc.dbk_bs(False, False, False, False, True, (0, -8), z, 2, 2) == 1


def _uniform_maps(pkg, pic_w, pic_h, tb, ctu):
    cols, rows = pic_w // 4, pic_h // 4
    cells = np.zeros((rows, cols), pkg.DBK_CELL_DTYPE)
    cells["ref_idx"] = -1
    yy, xx = np.mgrid[0:rows, 0:cols]
    cells["tu_id"] = (yy * 4 // tb) * 1000 + xx * 4 // tb
    cells["tu_w"] = tb
    cells["tu_h"] = tb
    cells["flags"] = pkg.DBK_CODED | pkg.DBK_INTRA
    cc = np.zeros((-(-pic_h // 4), -(-pic_w // 4)), pkg.DBK_CCELL_DTYPE)
    cy, cx = np.mgrid[0:cc.shape[0], 0:cc.shape[1]]
    cc["tu_cb"] = (cy * 2 // (tb // 2)) * 1000 + cx * 2 // (tb // 2)
    cc["tu_cr"] = cc["tu_cb"] + 500000
    cc["tu_w"] = tb // 2
    cc["tu_h"] = tb // 2
    return cells, cc


@pytest.mark.parametrize("w,h,tb,ctu,bd,qp", [(128, 96, 32, 32, 10, 37), (192, 128, 16, 64, 8, 42),
                                              (128, 128, 8, 32, 12, 33)])
def test_general_driver_matches_frame_drivers_on_a_uniform_grid(pkg, orc, w, h, tb, ctu, bd, qp):
    from rustmpeg_next_b200 import synth

    planes, _, _, _ = synth.random_deblock_picture(w, h, ctu, bd, seed=w + tb)
    cells, cc = _uniform_maps(pkg, w, h, tb, ctu)
    prm = np.zeros((), pkg.DBK_PARAMS_DTYPE)
    prm["qp"] = qp
    prm["beta_offset_div2"] = [1, -1, 0]
    prm["tc_offset_div2"] = [2, 0, -2]
    got = orc.deblock_general(planes, w, h, bd, ctu, cells, cc, prm)
    y = orc.deblock_luma(planes[0], bd, tb, ctu, qp, bs=2, beta_off=1, tc_off=2)
    u = orc.deblock_chroma(planes[1], bd, tb // 2, ctu // 2, qp, bs=2, beta_off=-1, tc_off=0)
    v = orc.deblock_chroma(planes[2], bd, tb // 2, ctu // 2, qp, bs=2, beta_off=0, tc_off=-2)
    # chroma blocks of 4 samples (tb 8) take the weak filter in the general
    # driver, which the frame driver's 8-sample lattice does not model
    n = 3 if tb >= 16 else 1
    for c, (a, b) in enumerate(list(zip(got, (y, u, v)))[:n]):
        assert np.array_equal(a, b), f"plane {c}: {np.count_nonzero(a != b)} samples differ"
    assert np.count_nonzero(got[0] != planes[0]) > 0


def test_general_driver_only_touches_samples_near_transform_edges(pkg, orc):
    from rustmpeg_next_b200 import synth

    planes, cells, cc, prm = synth.random_deblock_picture(256, 128, 32, 10, seed=5)
    got = orc.deblock_general(planes, 256, 128, 10, 32, cells, cc, prm)
    changed = got[0] != planes[0]
    assert changed.any()
    ids = cells["tu_id"]
    edge_v = np.zeros_like(ids, bool)
    edge_v[:, 1:] = ids[:, 1:] != ids[:, :-1]
    edge_h = np.zeros_like(ids, bool)
    edge_h[1:, :] = ids[1:, :] != ids[:-1, :]
    near = np.zeros(changed.shape, bool)
    for cy, cx in zip(*np.nonzero(edge_v)):
        near[4 * cy:4 * cy + 4, max(4 * cx - 7, 0):4 * cx + 7] = True
    for cy, cx in zip(*np.nonzero(edge_h)):
        near[max(4 * cy - 7, 0):4 * cy + 7, 4 * cx:4 * cx + 4] = True
    assert not (changed & ~near).any()
    # a single transform block over the picture leaves luma as it is
    one = cells.copy()
    one["tu_id"] = 7
    got1 = orc.deblock_general(planes, 256, 128, 10, 32, one, cc, prm)
    assert np.array_equal(got1[0], planes[0])
