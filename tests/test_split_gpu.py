"""GPU parity: the quadrant-mean partition hook (vvcg_qt_mtt_split_dev,
choose_qt_mtt_partition_rdo_16 of slice.rs:4111-4167) equals the oracle on
every region, bit depths 8..12, regions inside, across and past the plane
edge and at the minimum sizes; malformed requests are rejected."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _regions(pkg, rng, w, h, n):
    r = np.zeros(n, pkg.SPLIT_REQ_DTYPE)
    r["w"] = rng.choice([4, 8, 9, 16, 24, 32, 64, 128], n)
    r["h"] = rng.choice([4, 8, 9, 16, 24, 32, 64, 128], n)
    r["x"] = rng.integers(0, w + 64, n)
    r["y"] = rng.integers(0, h + 64, n)
    r["qp"] = rng.integers(0, 64, n)
    r["min_cb"] = rng.choice([4, 8, 16, 32], n)
    return r


@pytest.mark.parametrize("bd", [8, 10, 12])
def test_split_matches_oracle(ctx, pkg, orc, bd):
    import torch

    rng = np.random.default_rng(100 + bd)
    h, w = 270, 480
    coarse = rng.integers(0, 1 << bd, (h // 8 + 1, w // 8 + 1))
    noise = rng.integers(-(1 << (bd - 6)), 1 << (bd - 6), (h, w))
    plane = np.clip(np.kron(coarse, np.ones((8, 8), np.int64))[:h, :w] + noise, 0, (1 << bd) - 1).astype(np.uint16)
    reqs = _regions(pkg, rng, w, h, 3000)
    got = ctx.qt_mtt_split(torch.from_numpy(plane.view(np.int16)).cuda(), bd, reqs)
    regions = np.stack([reqs["x"], reqs["y"], reqs["w"], reqs["h"], reqs["qp"], reqs["min_cb"]], 1).astype(np.int64)
    want = orc.qt_mtt_split(plane, bd, regions)
    assert np.array_equal(got, want)
    assert set(np.unique(want).tolist()) == {0, 1, 2, 3}


def test_split_rejects_malformed_requests(ctx, pkg):
    import torch

    plane = torch.zeros((64, 64), dtype=torch.int16, device="cuda")
    r = np.zeros(1, pkg.SPLIT_REQ_DTYPE)
    r["w"], r["h"], r["qp"] = 32, 32, 30
    bad = r.copy()
    bad["w"] = 0
    with pytest.raises(pkg.InvalidInput, match="region size"):
        ctx.qt_mtt_split(plane, 10, bad)
    bad = r.copy()
    bad["qp"] = 64
    with pytest.raises(pkg.InvalidInput, match="QP"):
        ctx.qt_mtt_split(plane, 10, bad)
    with pytest.raises(pkg.InvalidInput):
        ctx.qt_mtt_split(plane, 13, r)
    assert ctx.qt_mtt_split(plane, 10, r).tolist() == [pkg.SPLIT_NONE]
