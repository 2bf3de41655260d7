"""GPU parity: the motion-estimation hook (vvcg_inter_search_8_dev,
estimate_inter_block of inter.rs:1866-2003) equals the oracle on random merge
lists (uni / bi, BCW, alternative half-sample filter, unusable lists), AMVP
starts and block sizes, finds a shifted reference with SAD 0, and rejects
malformed requests."""
import numpy as np
import pytest

from test_inter_search_oracle import random_case, _smooth, _one

pytestmark = pytest.mark.gpu


def _cuda(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_inter_search_matches_oracle(ctx, pkg, orc, seed):
    src, refs0, refs1, cands, reqs = random_case(pkg, seed, n_req=150)
    got = ctx.inter_search_8(_cuda(src), [_cuda(r) for r in refs0], [_cuda(r) for r in refs1], cands, reqs)
    want = orc.inter_search_8(src, refs0, refs1, cands, reqs, pkg.ME_RES_DTYPE)
    bad = [i for i in range(len(reqs)) if got[i].tobytes() != want[i].tobytes()]
    assert not bad, (bad[:5], got[bad[0]], want[bad[0]])
    assert set(want["is_merge"].tolist()) == {0, 1}


def test_inter_search_without_references(ctx, pkg, orc):
    src, _, _, cands, reqs = random_case(pkg, 14, n_req=40)
    got = ctx.inter_search_8(_cuda(src), [], [], cands, reqs)
    want = orc.inter_search_8(src, [], [], cands, reqs, pkg.ME_RES_DTYPE)
    assert got.tobytes() == want.tobytes()


def test_inter_search_finds_a_shifted_reference(ctx, pkg):
    rng = np.random.default_rng(5)
    src = _smooth(rng, 64, 64, scale=16)
    ref = np.roll(src, (1, 2), (0, 1))
    got = ctx.inter_search_8(_cuda(src), [_cuda(ref)], [], np.zeros(0, pkg.MV_CAND_DTYPE),
                             _one(pkg, 24, 24, 16, 16))[0]
    assert int(got["sad"]) == 0 and not got["is_merge"]
    assert (int(got["cand"]["mv"][0][0]), int(got["cand"]["mv"][0][1])) == (32, 16)


def test_inter_search_rejects_malformed_requests(ctx, pkg):
    src = _cuda(np.zeros((32, 32), np.uint8))
    none = np.zeros(0, pkg.MV_CAND_DTYPE)
    with pytest.raises(pkg.InvalidInput, match="outside the plane"):
        ctx.inter_search_8(src, [], [], none, _one(pkg, 28, 0, 8, 8))
    with pytest.raises(pkg.InvalidInput, match="block size"):
        ctx.inter_search_8(src, [], [], none, _one(pkg, 0, 0, 0, 8))
    with pytest.raises(pkg.InvalidInput, match="candidates past"):
        ctx.inter_search_8(src, [], [], none, _one(pkg, 0, 0, 8, 8, n=1))
    with pytest.raises(pkg.LimitExceeded):
        ctx.inter_search_8(src, [src] * 17, [], none, _one(pkg, 0, 0, 8, 8))
