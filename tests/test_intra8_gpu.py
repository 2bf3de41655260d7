"""GPU parity: the 8-bit luma intra mode search (vvcg_luma_intra_search_8_dev)
against the oracle's choose_luma_intra_pred_mode and the multi-tool encoder's
MRL candidates: every block size 4..64, blocks on the picture's top row and
left column and at its right and bottom edges, all 67 modes or the MPMs, MRL
on and off, blocks on and below a CTU's first row."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _planes(w, h, seed):
    from rustmpeg_next_b200 import synth

    y, _, _ = synth.value_noise_frame(w, h, 10, frame=seed)
    recon = (y >> 2).astype(np.uint8)
    rng = np.random.default_rng(seed)
    src = np.clip(recon.astype(np.int32) + rng.integers(-12, 13, recon.shape), 0, 255).astype(np.uint8)
    # a few hard edges and flat areas so that the angular modes differ
    recon[h // 3:h // 3 + 20, :] = 30
    src[:, w // 2:w // 2 + 9] = 220
    return recon, src


def _reqs(pkg, w, h, n, seed, flags=None):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, pkg.ISR_REQ_DTYPE)
    for i in range(n):
        lw, lh = int(rng.integers(2, 7)), int(rng.integers(2, 7))
        bw, bh = 1 << lw, 1 << lh
        gx = int(rng.integers(0, (w - bw) // 4 + 1)) * 4
        gy = int(rng.integers(0, (h - bh) // 4 + 1)) * 4
        if i % 7 == 0:
            gx = 0
        if i % 11 == 0:
            gy = 0
        if i % 13 == 0:
            gx, gy = w - bw, h - bh
        r[i]["x"], r[i]["y"], r[i]["log2_w"], r[i]["log2_h"] = gx, gy, lw, lh
        r[i]["flags"] = int(rng.integers(0, 4)) if flags is None else flags
        r[i]["log2_ctu"] = int(rng.integers(4, 8))
        r[i]["mpm"] = rng.choice(67, 6, replace=False)
    return r


@pytest.mark.parametrize("w,h,n,seed,flags", [(256, 192, 300, 1, None), (128, 128, 200, 2, 2), (96, 80, 120, 3, 0),
                                             (64, 64, 60, 4, 3)])
def test_intra_search_matches_oracle(ctx, pkg, orc, w, h, n, seed, flags):
    import torch

    recon, src = _planes(w, h, seed)
    reqs = _reqs(pkg, w, h, n, seed, flags)
    got = ctx.luma_intra_search_8(torch.from_numpy(recon).cuda(), torch.from_numpy(src).cuda(), reqs)
    for i, q in enumerate(reqs):
        want = orc.luma_intra_search_8(recon, src, int(q["x"]), int(q["y"]), 1 << int(q["log2_w"]),
                                       1 << int(q["log2_h"]), q["mpm"], bool(q["flags"] & 1), bool(q["flags"] & 2),
                                       1 << int(q["log2_ctu"]))
        assert (int(got[i]["mode"]), int(got[i]["mrl_idx"]), int(got[i]["sad"])) == want, (i, q)


def test_intra_search_full_hd_ctus(ctx, pkg, orc):
    """The multi-tool encoder's call: one 32x32 CTU at a time, all 67 modes."""
    import torch

    w, h = 1920, 1080
    recon, src = _planes(w, h, 9)
    xs, ys = np.meshgrid(np.arange(0, w - 31, 32), np.arange(0, h - 31, 32))
    reqs = np.zeros(xs.size, pkg.ISR_REQ_DTYPE)
    reqs["x"], reqs["y"] = xs.ravel(), ys.ravel()
    reqs["log2_w"] = reqs["log2_h"] = 5
    reqs["log2_ctu"] = 5
    reqs["mpm"] = [0, 1, 50, 18, 46, 54]
    got = ctx.luma_intra_search_8(torch.from_numpy(recon).cuda(), torch.from_numpy(src).cuda(), reqs)
    rng = np.random.default_rng(0)
    for i in rng.choice(len(reqs), 60, replace=False):
        q = reqs[i]
        want = orc.luma_intra_search_8(recon, src, int(q["x"]), int(q["y"]), 32, 32, q["mpm"])
        assert (int(got[i]["mode"]), int(got[i]["mrl_idx"]), int(got[i]["sad"])) == want, i
    assert len(set(got["mode"].tolist())) > 10


def test_intra_search_rejects_bad_requests(ctx, pkg):
    import torch

    recon = torch.zeros((64, 64), dtype=torch.uint8, device="cuda")
    r = np.zeros(1, pkg.ISR_REQ_DTYPE)
    r["log2_w"], r["log2_h"], r["x"] = 5, 5, 40
    with pytest.raises(pkg.InvalidInput, match="outside the plane"):
        ctx.luma_intra_search_8(recon, recon, r)
    r["x"], r["mpm"] = 0, [0, 1, 2, 3, 4, 67]
    with pytest.raises(pkg.InvalidInput, match="MPM"):
        ctx.luma_intra_search_8(recon, recon, r)
    r["mpm"], r["log2_w"] = [0, 1, 2, 3, 4, 5], 7
    with pytest.raises(pkg.InvalidInput, match="block size"):
        ctx.luma_intra_search_8(recon, recon, r)
