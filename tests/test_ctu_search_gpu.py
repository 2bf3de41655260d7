"""GPU parity: the CTU full search of the GPU encoder (vvcg_ctu_search_dev)
against the oracle's restatement: all six split types, every block over the
67 modes or a candidate list, 8x8 Hadamard SATD + lambda * bits, bit depths
8, 10 and 12, CTUs on the picture's edges."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _src(w, h, bd, seed):
    from rustmpeg_next_b200 import synth

    y, _, _ = synth.value_noise_frame(w, h, 10, frame=seed)
    y = y.astype(np.int32)
    y = y << (bd - 10) if bd >= 10 else y >> (10 - bd)
    rng = np.random.default_rng(seed)
    y[h // 2:h // 2 + 5, :] = (1 << bd) - 1  # a hard edge
    return np.clip(y + rng.integers(-3, 4, y.shape), 0, (1 << bd) - 1).astype(np.uint16)


def _check(ctx, pkg, orc, src, bd, qp, reqs):
    import torch

    lam = orc.search_lambda_q8(qp)
    got = ctx.ctu_search(torch.from_numpy(src.view(np.int16)).cuda(), bd, lam, reqs)
    for i, q in enumerate(reqs):
        want = orc.ctu_search(src, bd, int(q["x"]), int(q["y"]), lam, int(q["split_mask"]),
                              tuple(int(c) for c in q["cand"][:int(q["n_cand"])]))
        g = got[i]
        assert int(g["cost"]) == want["cost"], (i, q, g, want)
        assert [int(v) for v in g["split_cost"]] == want["split_cost"], (i, g, want)
        assert (int(g["split"]), int(g["cu_mode"]), [int(v) for v in g["modes"]]) == \
            (want["split"], want["cu_mode"], want["modes"]), (i, g, want)
    return got


@pytest.mark.parametrize("bd,qp", [(10, 32), (8, 22), (12, 37)])
def test_ctu_search_full_matches_oracle(ctx, pkg, orc, bd, qp):
    w, h = 160, 96
    src = _src(w, h, bd, bd)
    xs, ys = np.meshgrid(np.arange(0, w, 32), np.arange(0, h, 32))
    reqs = np.zeros(xs.size, pkg.CTU_SEARCH_REQ_DTYPE)
    reqs["x"], reqs["y"], reqs["split_mask"] = xs.ravel(), ys.ravel(), 0x3F
    got = _check(ctx, pkg, orc, src, bd, qp, reqs)
    assert len(set(got["split"].tolist())) > 1


def test_ctu_search_pruned_matches_oracle(ctx, pkg, orc):
    w, h = 128, 128
    src = _src(w, h, 10, 5)
    rng = np.random.default_rng(5)
    xs, ys = np.meshgrid(np.arange(0, w, 32), np.arange(0, h, 32))
    reqs = np.zeros(xs.size, pkg.CTU_SEARCH_REQ_DTYPE)
    reqs["x"], reqs["y"] = xs.ravel(), ys.ravel()
    for q in reqs:
        q["split_mask"] = int(rng.integers(1, 64))
        q["n_cand"] = int(rng.integers(0, 7))
        q["cand"] = rng.choice(67, 6, replace=False)
    _check(ctx, pkg, orc, src, 10, 27, reqs)


def test_ctu_search_rejects_bad_requests(ctx, pkg):
    import torch

    src = torch.zeros((64, 64), dtype=torch.int16, device="cuda")
    r = np.zeros(1, pkg.CTU_SEARCH_REQ_DTYPE)
    r["x"], r["split_mask"] = 40, 1
    with pytest.raises(pkg.InvalidInput, match="outside the plane"):
        ctx.ctu_search(src, 10, 100, r)
    r["x"], r["split_mask"] = 0, 0
    with pytest.raises(pkg.InvalidInput, match="split mask"):
        ctx.ctu_search(src, 10, 100, r)
