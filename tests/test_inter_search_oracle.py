"""CPU: the oracle of the encoders' motion-estimation hook
(estimate_inter_block, crates/rustmpeg-video/src/vvc/inter.rs:1866-2003)
against a Python restatement of its search that predicts through the oracle's
8-bit interpolation and BCW average (checked against the GPU elsewhere), on
random merge lists (uni / bi, BCW weights, alternative half-sample filter,
unusable lists) and AMVP starts; and known answers: a shifted reference is
found by the diamond search with SAD 0, an exact merge candidate wins ties,
and without references or candidates the default candidate comes back."""
import numpy as np
import pytest

U64_MAX = (1 << 64) - 1
BCW = (-2, 3, 4, 5, 10)


def _pred(orc, refs0, refs1, c, x, y, w, h):
    has0 = (c["inter_dir"] & 1) and c["ref_idx"][0] >= 0 and len(refs0) > 0
    has1 = (c["inter_dir"] & 2) and c["ref_idx"][1] >= 0 and len(refs1) > 0
    alt = bool(c["alt_hpel"])
    if has0 and has1:
        r0 = refs0[min(int(c["ref_idx"][0]), len(refs0) - 1)]
        r1 = refs1[min(int(c["ref_idx"][1]), len(refs1) - 1)]
        p0 = orc.mc_luma_8(r0, x, y, w, h, int(c["mv"][0][0]), int(c["mv"][0][1]), bi=True, alt_hpel=alt)
        p1 = orc.mc_luma_8(r1, x, y, w, h, int(c["mv"][1][0]), int(c["mv"][1][1]), bi=True, alt_hpel=alt)
        w1 = BCW[min(int(c["bcw_idx"]), 4)]
        return np.clip((p0.astype(np.int64) * (8 - w1) + p1 * w1 + 256 + (8192 << 3)) >> 9, 0, 255)
    if has0 or has1:
        l = 0 if has0 else 1
        r = (refs0 if has0 else refs1)[min(int(c["ref_idx"][l]), len(refs0 if has0 else refs1) - 1)]
        return orc.mc_luma_8(r, x, y, w, h, int(c["mv"][l][0]), int(c["mv"][l][1]), alt_hpel=alt)
    return np.full((h, w), 128)


def _py_search(orc, src, refs0, refs1, cands, q):
    x, y, w, h = int(q["x"]), int(q["y"]), int(q["w"]), int(q["h"])
    blk = src[y:y + h, x:x + w].astype(np.int64)
    sad = lambda p: int(np.abs(blk - p).sum())  # noqa: E731
    best, best_i = U64_MAX, 0
    for i in range(int(q["num_cands"])):
        s = sad(_pred(orc, refs0, refs1, cands[int(q["cand_off"]) + i], x, y, w, h))
        if s < best:
            best, best_i = s, i
    if not refs0:
        return True, best_i, best, None
    at = lambda mx, my: sad(orc.mc_luma_8(refs0[0], x, y, w, h, mx, my))  # noqa: E731
    mv = ((int(q["amvp"][0]) >> 4) << 4, (int(q["amvp"][1]) >> 4) << 4)
    s_best = at(*mv)
    for _ in range(max(int(q["search_range"]), 1)):
        cx, cy = mv[0] >> 4, mv[1] >> 4
        improved = False
        for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
            t = ((cx + dx) << 4, (cy + dy) << 4)
            s = at(*t)
            if s < s_best:
                s_best, mv, improved = s, t, True
        if not improved:
            break
    ic = mv
    for dx, dy in ((4, 0), (-4, 0), (0, 4), (0, -4)):
        t = (ic[0] + dx, ic[1] + dy)
        s = at(*t)
        if s < s_best:
            s_best, mv = s, t
    if best <= s_best:
        return True, best_i, best, None
    return False, 0, s_best, mv


def _smooth(rng, h, w, scale=12):
    coarse = rng.integers(0, 256, (h // scale + 3, w // scale + 3)).astype(np.float64)
    yy, xx = np.mgrid[0:h, 0:w] / scale
    y0, x0 = yy.astype(int), xx.astype(int)
    fy, fx = yy - y0, xx - x0
    v = (coarse[y0, x0] * (1 - fx) * (1 - fy) + coarse[y0, x0 + 1] * fx * (1 - fy)
         + coarse[y0 + 1, x0] * (1 - fx) * fy + coarse[y0 + 1, x0 + 1] * fx * fy)
    return np.clip(v, 0, 255).astype(np.uint8)


def random_case(pkg, seed, n_req=60, h=72, w=96):
    rng = np.random.default_rng(seed)
    src = _smooth(rng, h, w)
    refs0 = [np.roll(src, (int(rng.integers(-3, 4)), int(rng.integers(-3, 4))), (0, 1)) for _ in range(2)]
    refs1 = [np.clip(src.astype(int) + rng.integers(-6, 7, src.shape), 0, 255).astype(np.uint8)]
    cands = np.zeros(n_req * 3, pkg.MV_CAND_DTYPE)
    cands["mv"] = rng.integers(-48, 49, (len(cands), 2, 2))
    cands["ref_idx"] = rng.integers(-1, 3, (len(cands), 2))
    cands["inter_dir"] = rng.integers(0, 4, len(cands))
    cands["bcw_idx"] = rng.integers(0, 6, len(cands))
    cands["alt_hpel"] = rng.integers(0, 2, len(cands))
    reqs = np.zeros(n_req, pkg.ME_REQ_DTYPE)
    reqs["w"] = rng.choice([4, 8, 12, 16, 32], n_req)
    reqs["h"] = rng.choice([4, 8, 16, 24], n_req)
    reqs["x"] = [int(rng.integers(0, w - bw + 1)) for bw in reqs["w"]]
    reqs["y"] = [int(rng.integers(0, h - bh + 1)) for bh in reqs["h"]]
    reqs["cand_off"] = np.arange(n_req) * 3
    reqs["num_cands"] = rng.integers(0, 4, n_req)
    reqs["search_range"] = rng.integers(0, 6, n_req)
    reqs["amvp"] = rng.integers(-40, 41, (n_req, 2))
    return src, refs0, refs1, cands, reqs


@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_matches_restated_search(orc, pkg, seed):
    src, refs0, refs1, cands, reqs = random_case(pkg, seed)
    got = orc.inter_search_8(src, refs0, refs1, cands, reqs, pkg.ME_RES_DTYPE)
    kinds = set()
    for i, q in enumerate(reqs):
        is_merge, idx, sad, mv = _py_search(orc, src, refs0, refs1, cands, q)
        g = got[i]
        assert int(g["sad"]) == sad and bool(g["is_merge"]) == is_merge, i
        if is_merge:
            assert int(g["merge_idx"]) == idx
            if int(q["num_cands"]):
                assert g["cand"].tobytes() == cands[int(q["cand_off"]) + idx].tobytes()
        else:
            assert (int(g["cand"]["mv"][0][0]), int(g["cand"]["mv"][0][1])) == mv
            assert int(g["cand"]["inter_dir"]) == 1 and list(g["cand"]["ref_idx"]) == [0, -1]
        kinds.add(is_merge)
    assert kinds == {True, False}


def _one(pkg, x, y, w, h, amvp=(0, 0), rng_=4, off=0, n=0):
    q = np.zeros(1, pkg.ME_REQ_DTYPE)
    q["x"], q["y"], q["w"], q["h"], q["amvp"], q["search_range"] = x, y, w, h, amvp, rng_
    q["cand_off"], q["num_cands"] = off, n
    return q


def test_diamond_search_finds_a_shifted_reference(orc, pkg):
    rng = np.random.default_rng(5)
    src = _smooth(rng, 64, 64, scale=16)
    ref = np.roll(src, (1, 2), (0, 1))  # ref[y][x] = src[y - 1][x - 2]: the block moved by (+2, +1)
    got = orc.inter_search_8(src, [ref], [], np.zeros(0, pkg.MV_CAND_DTYPE), _one(pkg, 24, 24, 16, 16),
                             pkg.ME_RES_DTYPE)[0]
    assert int(got["sad"]) == 0 and not got["is_merge"]
    assert (int(got["cand"]["mv"][0][0]), int(got["cand"]["mv"][0][1])) == (32, 16)


def test_exact_merge_candidate_wins_the_tie(orc, pkg):
    rng = np.random.default_rng(6)
    src = _smooth(rng, 64, 64, scale=16)
    ref = np.roll(src, (1, 2), (0, 1))
    c = np.zeros(2, pkg.MV_CAND_DTYPE)
    c["inter_dir"], c["ref_idx"], c["bcw_idx"] = 1, [[0, -1], [0, -1]], 2
    c["mv"][0, 0] = (16, 0)     # not the shift
    c["mv"][1, 0] = (32, 16)    # the shift: SAD 0, like the search
    got = orc.inter_search_8(src, [ref], [], c, _one(pkg, 24, 24, 16, 16, n=2), pkg.ME_RES_DTYPE)[0]
    assert int(got["sad"]) == 0 and got["is_merge"] and int(got["merge_idx"]) == 1


def test_without_references_or_candidates_the_default_comes_back(orc, pkg):
    src = np.full((32, 32), 100, np.uint8)
    got = orc.inter_search_8(src, [], [], np.zeros(0, pkg.MV_CAND_DTYPE), _one(pkg, 0, 0, 8, 8), pkg.ME_RES_DTYPE)[0]
    assert int(got["sad"]) == U64_MAX and got["is_merge"] and int(got["merge_idx"]) == 0
    assert int(got["cand"]["inter_dir"]) == 1 and list(got["cand"]["ref_idx"]) == [0, -1]
    assert int(got["cand"]["bcw_idx"]) == 2
    # a candidate with no usable list predicts 128 everywhere: SAD 28 per sample
    c = np.zeros(1, pkg.MV_CAND_DTYPE)
    c["inter_dir"], c["ref_idx"] = 3, [-1, -1]
    got = orc.inter_search_8(src, [], [], c, _one(pkg, 0, 0, 8, 8, n=1), pkg.ME_RES_DTYPE)[0]
    assert int(got["sad"]) == 28 * 64 and got["is_merge"]
