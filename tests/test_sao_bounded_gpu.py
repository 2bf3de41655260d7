"""GPU parity: the general decoder's SAO of one plane (vvcg_sao_bounded_16_dev)
against the oracle's restatement of apply_sao_region_bounded_16 and its
per-CTU driver: band and all four edge classes, visible sizes that crop CTUs,
8..12-bit planes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pw,ph,vis_w,vis_h,bd,ctu", [
    (256, 128, 250, 120, 10, 64), (128, 64, 128, 64, 8, 32), (192, 96, 181, 77, 12, 32), (64, 64, 60, 33, 10, 16),
])
def test_sao_bounded_matches_oracle(ctx, pkg, orc, pw, ph, vis_w, vis_h, bd, ctu):
    import torch

    rng = np.random.default_rng(pw + ph + bd)
    plane = rng.integers(0, 1 << bd, (ph, pw)).astype(np.uint16)
    plane[:, : pw // 2] = (plane[:, : pw // 2] // 64) * 64 + 32  # flat regions for edge ties
    cols = -(-pw // ctu)
    rows = -(-ph // ctu)
    prm = np.zeros(rows * cols, pkg.SAO_DTYPE)
    kind = rng.integers(0, 3, rows * cols)
    prm["type"] = kind
    omax = (1 << (min(bd, 10) - 5)) - 1
    prm["band_or_class"] = np.where(kind == 1, rng.integers(0, 32, rows * cols), rng.integers(0, 4, rows * cols))
    prm["offsets"] = np.where((kind == 2)[:, None], rng.integers(0, omax + 1, (rows * cols, 4)) * np.array([1, 1, -1, -1]),
                              rng.integers(-omax, omax + 1, (rows * cols, 4)))
    want = orc.sao_bounded(plane, vis_w, vis_h, bd, ctu, cols, prm)
    src = torch.from_numpy(plane.view(np.int16)).cuda()
    dst = torch.zeros_like(src)
    ctx.sao_bounded(src, dst, vis_w, vis_h, bd, ctu, cols, torch.from_numpy(prm.view(np.uint8)).cuda())
    torch.cuda.synchronize()
    got = dst.cpu().numpy().view(np.uint16)
    assert (got == want).all()
    assert (got != plane).any()
