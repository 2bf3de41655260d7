"""GPU parity: CTU-boundary deblocking of inter pictures
(vvcg_deblock_ctu_edges_dev) against the oracle's restatement of the
deblocking part of apply_inter_loop_filters (slice.rs:2291-2554), bit-exact:
8-bit 4:2:0 pictures with per-CTU cbf flags and motion that give every
boundary strength (0: same motion, no residual; 1: residual, a different
reference or a motion difference of half a sample or more)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _picture(w, h, seed):
    """Smooth 8-bit content (ramps plus small noise, so the luma decisions
    filter) with blocky steps at CTU boundaries."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    y = 60 + (xx * 100) // w + (yy * 50) // h + rng.integers(-2, 3, (h, w)) + 6 * ((xx // 32 + yy // 32) % 2)
    ch, cw = h // 2, w // 2
    cyy, cxx = np.mgrid[0:ch, 0:cw]
    u = 128 + (cxx * 20) // cw + rng.integers(-1, 2, (ch, cw)) + 4 * ((cxx // 16) % 2)
    v = 120 - (cyy * 20) // ch + rng.integers(-1, 2, (ch, cw)) + 4 * ((cyy // 16) % 2)
    return [np.clip(p, 0, 255).astype(np.uint16) for p in (y, u, v)]


def _cells(pkg, rows, cols, seed):
    rng = np.random.default_rng(seed)
    c = np.zeros((rows, cols), pkg.CTU_MOTION_DTYPE)
    c["cbf"] = rng.integers(0, 8, (rows, cols)) * (rng.random((rows, cols)) < 0.5)
    base = rng.integers(-64, 64, (rows, cols, 1, 2))
    jitter = rng.integers(-9, 10, (rows, cols, 3, 2)) * (rng.random((rows, cols, 3, 1)) < 0.5)
    c["mv"] = base + jitter
    c["ref"] = rng.integers(0, 2, (rows, cols, 1)) * (rng.random((rows, cols, 1)) < 0.3)
    return c


@pytest.mark.parametrize("w,h,ctu,qp,seed", [(256, 192, 32, 32, 1), (192, 128, 64, 40, 2), (256, 256, 128, 45, 3),
                                             (64, 64, 32, 26, 4), (128, 96, 32, 51, 5)])
def test_ctu_edge_deblocking_matches_oracle(ctx, pkg, orc, w, h, ctu, qp, seed):
    import torch

    planes = _picture(w, h, seed)
    cells = _cells(pkg, h // ctu, w // ctu, seed)
    want = orc.inter_ctu_deblock(planes, ctu, qp, cells)
    dev = [torch.from_numpy(p.view(np.int16).copy()).cuda() for p in planes]
    ctx.deblock_ctu_edges(dev, ctu, qp, cells)
    torch.cuda.synchronize()
    changed = 0
    for k in range(3):
        got = dev[k].cpu().numpy().view(np.uint16)
        diff = np.argwhere(got != want[k])
        assert diff.size == 0, f"plane {k}: {len(diff)} samples differ, first {diff[:3].tolist()}"
        changed += int((want[k] != planes[k]).sum())
    assert changed > 0  # the case filters something


def test_ctu_edge_deblocking_rejects_bad_geometry(ctx, pkg):
    import torch

    planes = [torch.zeros((96, 100), dtype=torch.int16, device="cuda"),
              torch.zeros((48, 50), dtype=torch.int16, device="cuda"),
              torch.zeros((48, 50), dtype=torch.int16, device="cuda")]
    with pytest.raises(pkg.InvalidInput):
        ctx.deblock_ctu_edges(planes, 32, 30, np.zeros((3, 3), pkg.CTU_MOTION_DTYPE))
