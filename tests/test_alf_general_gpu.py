"""GPU parity: the general decoder's ALF (vvcg_alf_general_dev) against the
oracle's restatement of apply_alf: luma 7x7 with virtual boundaries (fixed
sets and APS filters, clipping), chroma 5x5 alternatives with virtual
boundaries, CCALF from the unfiltered luma, cropped visible sizes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(pkg, rng):
    a = np.zeros((), pkg.ALF_PARAMS_DTYPE)
    a["num_luma_filters"] = int(rng.integers(1, 26))
    a["luma_clip"] = int(rng.integers(0, 2))
    a["coeff_delta_idx"] = rng.integers(0, int(a["num_luma_filters"]), 25)
    a["luma_coeff"] = rng.integers(-40, 41, (25, 12))
    a["luma_clip_idx"] = rng.integers(0, 4, (25, 12))
    a["num_chroma_filters"] = int(rng.integers(1, 9))
    a["chroma_clip"] = int(rng.integers(0, 2))
    a["chroma_coeff"] = rng.integers(-40, 41, (8, 6))
    a["chroma_clip_idx"] = rng.integers(0, 4, (8, 6))
    a["num_cc_cb"], a["num_cc_cr"] = int(rng.integers(1, 5)), int(rng.integers(0, 5))
    a["cc_cb"] = rng.integers(-64, 65, (4, 7))
    a["cc_cr"] = rng.integers(-64, 65, (4, 7))
    return a


@pytest.mark.parametrize("pw,ph,vis_w,vis_h,bd,ctu", [
    (256, 192, 250, 181, 10, 64), (128, 128, 128, 128, 8, 32), (256, 256, 233, 256, 12, 128), (96, 64, 90, 60, 10, 32),
])
def test_alf_general_matches_oracle(ctx, pkg, orc, pw, ph, vis_w, vis_h, bd, ctu):
    import torch

    rng = np.random.default_rng(pw * 3 + ph + bd + ctu)
    maxv = (1 << bd) - 1
    yy, xx = np.mgrid[0:ph, 0:pw]
    y = np.clip((1 << (bd - 1)) + (maxv // 4) * np.sin(xx / 7.0) * np.cos(yy / 5.0) + rng.integers(-30, 31, (ph, pw)),
                0, maxv).astype(np.uint16)
    ch, cw = (ph + 1) // 2, (pw + 1) // 2
    u = np.clip(rng.integers(0, maxv + 1) + rng.integers(-60, 61, (ch, cw)), 0, maxv).astype(np.uint16)
    v = np.clip(rng.integers(0, maxv + 1) + rng.integers(-60, 61, (ch, cw)), 0, maxv).astype(np.uint16)
    cols, rows = -(-vis_w // ctu), -(-vis_h // ctu)
    ctus = np.zeros(rows * cols, pkg.ALF_CTU_DTYPE)
    ctus["luma_mode"] = rng.integers(0, 3, rows * cols)
    ctus["luma_set"] = rng.integers(0, 16, rows * cols)
    ctus["cb_alt"] = np.where(rng.random(rows * cols) < 0.7, rng.integers(0, 8, rows * cols), 0xFF)
    ctus["cr_alt"] = np.where(rng.random(rows * cols) < 0.7, rng.integers(0, 8, rows * cols), 0xFF)
    ctus["cc_cb"] = rng.integers(0, 5, rows * cols)
    ctus["cc_cr"] = rng.integers(0, 5, rows * cols)
    prm = _params(pkg, rng)
    want = orc.alf_general(y, u, v, vis_w, vis_h, bd, ctu, cols, ctus, prm)
    src = [torch.from_numpy(p.view(np.int16).copy()).cuda() for p in (y, u, v)]
    dst = [torch.zeros_like(t) for t in src]
    ctx.alf_general(src, dst, vis_w, vis_h, bd, ctu, cols, ctus, prm)
    torch.cuda.synchronize()
    for c in range(3):
        got = dst[c].cpu().numpy().view(np.uint16)
        bad = np.argwhere(got != want[c])
        assert bad.size == 0, f"plane {c}: {len(bad)} samples differ, first {bad[:4].tolist()}"
    assert (want[0] != y).any() and (want[1] != u).any()
