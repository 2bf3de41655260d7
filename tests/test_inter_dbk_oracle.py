"""CPU: the oracle's restatement of the CTU-boundary deblocking of inter
pictures (apply_inter_loop_filters, slice.rs:2291-2554) against the
plane drivers it shares its edge filters with (deblock_luma_plane /
deblock_chroma_plane at bit depth 8, pinned by the reference's filter
tests): with the same boundary strength on every CTU edge the two agree,
and without residual or motion difference nothing is filtered."""
import numpy as np
import pytest


def _planes(w, h, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    y = 70 + (xx * 90) // w + (yy * 40) // h + rng.integers(-2, 3, (h, w)) + 5 * ((xx // 32 + yy // 32) % 2)
    cyy, cxx = np.mgrid[0:h // 2, 0:w // 2]
    u = 120 + (cxx * 16) // (w // 2) + rng.integers(-1, 2, (h // 2, w // 2)) + 3 * ((cxx // 16) % 2)
    return [np.clip(p, 0, 255).astype(np.uint16) for p in (y, u, u[::-1].copy())]


@pytest.mark.parametrize("w,h,ctu,qp", [(192, 128, 32, 34), (256, 128, 64, 40)])
def test_uniform_strength_equals_the_plane_drivers(orc, w, h, ctu, qp):
    planes = _planes(w, h, ctu)
    cells = np.zeros((h // ctu, w // ctu), orc.CTU_MOTION_DTYPE)
    cells["cbf"] = 7  # residual everywhere: bS 1 on every CTU edge
    got = orc.inter_ctu_deblock(planes, ctu, qp, cells)
    want_y = orc.deblock_luma(planes[0], 8, ctu, ctu, qp, bs=1)
    cqp = qp if qp <= 26 else qp - 1
    want_c = [orc.deblock_chroma(p, 8, ctu // 2, ctu // 2, cqp, bs=1) for p in planes[1:]]
    assert np.array_equal(got[0], want_y)
    assert np.array_equal(got[1], want_c[0]) and np.array_equal(got[2], want_c[1])
    assert (got[0] != planes[0]).any()


def test_no_residual_and_same_motion_filters_nothing(orc):
    planes = _planes(128, 128, 3)
    cells = np.zeros((4, 4), orc.CTU_MOTION_DTYPE)
    cells["mv"] = 40  # the same motion everywhere
    got = orc.inter_ctu_deblock(planes, 32, 37, cells)
    assert all(np.array_equal(a, b) for a, b in zip(got, planes))
    cells["mv"][1, 2, 0, 0] += 8  # half a sample apart on the edges of one CTU
    got = orc.inter_ctu_deblock(planes, 32, 37, cells)
    changed = np.argwhere(got[0] != planes[0])
    assert changed.size and changed[:, 0].min() >= 32 - 7 and changed[:, 0].max() < 64 + 7
