"""GPU: the CNN-pruned CTU search (vvcg_ctu_search_pruned_dev): without
logits it equals the full search with host requests; with logits its
candidate and split choice (top-k of the softmax, full set when their
probability mass is below the threshold) equals the oracle's search on the
same candidates; and a pruner trained on full-search labels keeps the cost
close to the full search."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plane(w, h, seed):
    import torch
    from rustmpeg_next_b200 import synth

    y, _, _ = synth.value_noise_frame(w, h, 10, frame=seed)
    y = np.ascontiguousarray(y.astype(np.uint16))
    return y, torch.from_numpy(y.view(np.int16)).cuda()


def _xy(w, h):
    import torch

    xs, ys = np.meshgrid(np.arange(0, w - 31, 32), np.arange(0, h - 31, 32))
    a = np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32)
    return a, torch.from_numpy(a).cuda()


def test_unpruned_device_search_equals_host_requests(ctx, pkg):
    y, plane = _plane(256, 128, 1)
    a, xy = _xy(256, 128)
    reqs = np.zeros(len(a), pkg.CTU_SEARCH_REQ_DTYPE)
    reqs["x"], reqs["y"], reqs["split_mask"] = a[:, 0], a[:, 1], 0x3F
    want = ctx.ctu_search(plane, 10, 300, reqs)
    got = ctx.ctu_search_xy(plane, 10, 300, xy)
    assert np.array_equal(got.view(np.uint8), want.view(np.uint8))


def test_pruned_search_matches_oracle_on_its_candidates(ctx, pkg, orc):
    import torch

    y, plane = _plane(192, 128, 2)
    a, xy = _xy(192, 128)
    rng = np.random.default_rng(2)
    logits = rng.normal(0, 1.0, (len(a), 73)).astype(np.float32)
    # a clear winner per head (probability far above the threshold) ...
    logits[np.arange(len(a)), rng.integers(0, 67, len(a))] += 8.0
    logits[np.arange(len(a)), 67 + rng.integers(0, 6, len(a))] += 8.0
    # ... except flat heads (far below it): all modes / all splits
    logits[::3, :67] *= 0.01
    logits[1::4, 67:] *= 0.01
    got = ctx.ctu_search_xy(plane, 10, 250, xy, torch.from_numpy(logits).cuda(), 3, 2, 0.4)

    def top(v, k):  # ties: lower index first
        return [int(i) for i in sorted(range(len(v)), key=lambda j: (-v[j], j))[:k]]

    def mass(v, idx):
        e = np.exp(v.astype(np.float64) - v.max())
        return e[idx].sum() / e.sum()

    for i, (x, yy) in enumerate(a):
        li, ls = logits[i, :67], logits[i, 67:]
        cand = tuple(top(li, 3)) if mass(li, top(li, 3)) >= 0.4 else ()
        mask = sum(1 << s for s in top(ls, 2)) if mass(ls, top(ls, 2)) >= 0.4 else 0x3F
        want = orc.ctu_search(y, 10, int(x), int(yy), 250, mask, cand)
        g = got[i]
        assert (int(g["cost"]), int(g["split"]), [int(v) for v in g["modes"]]) == \
            (want["cost"], want["split"], want["modes"]), i


def test_trained_pruner_stays_close_to_full_search(ctx, pkg):
    import torch
    from rustmpeg_next_b200 import cnn

    data = cnn.training_set(ctx, n_frames=2, width=1024, height=512, qps=(27, 37), seed=3)
    params, losses = cnn.train(ctx, data, steps=300, batch=256, lr=2e-3, seed=3)
    assert losses[-1] < losses[0]
    y, plane = _plane(1024, 512, 77)
    a, xy = _xy(1024, 512)
    lam = cnn.search_lambda_q8(32)
    full = ctx.ctu_search_xy(plane, 10, lam, xy)
    logits, _, _ = ctx.cnn_forward(plane, 10, xy, params, 32)
    pruned = ctx.ctu_search_xy(plane, 10, lam, xy, logits, 6, 2, 0.7)
    total = full["cost"].astype(np.float64).sum()
    inc = pruned["cost"].astype(np.float64).sum() / total - 1.0
    assert 0.0 <= inc < 0.08, inc
    # what training buys: with the same pruning and no fallback, the trained
    # network's candidates cost less than an untrained network's
    untrained = torch.from_numpy(cnn.init_params(99)).cuda()
    lg_u, _, _ = ctx.cnn_forward(plane, 10, xy, untrained, 32)
    forced_t = ctx.ctu_search_xy(plane, 10, lam, xy, logits, 3, 2, 0.0)
    forced_u = ctx.ctu_search_xy(plane, 10, lam, xy, lg_u, 3, 2, 0.0)
    inc_t = forced_t["cost"].astype(np.float64).sum() / total - 1.0
    inc_u = forced_u["cost"].astype(np.float64).sum() / total - 1.0
    assert inc_t < 0.8 * inc_u, (inc_t, inc_u)


def test_mode_costs_of_the_unsplit_cu(ctx, pkg, orc):
    """vvcg_ctu_search_costs_dev: the same results as the full search, every
    mode's cost of the unsplit CU equal to the oracle's search restricted to
    that one mode, and the minimum over the 67 costs is the unsplit cost."""
    y, plane = _plane(192, 128, 5)
    a, xy = _xy(192, 128)
    want = ctx.ctu_search_xy(plane, 10, 280, xy)
    got, costs = ctx.ctu_search_costs(plane, 10, 280, xy)
    assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
    c = costs.cpu().numpy()
    assert c.shape == (len(a), 67)
    # the unsplit cost adds the split flag's one bit at lambda to the best mode's
    assert np.array_equal(c.min(1) + (280 * 1 >> 8), got["split_cost"][:, 0].astype(np.int64))
    assert np.array_equal(c.argmin(1), got["cu_mode"])
    rng = np.random.default_rng(5)
    for k in rng.choice(len(a), 4, replace=False):
        for m in (0, 1, int(rng.integers(2, 67)), int(c[k].argmin())):
            r = orc.ctu_search(y, 10, int(a[k, 0]), int(a[k, 1]), 280, split_mask=1, cand=(m,))
            assert r["split_cost"][0] == c[k, m] + (280 >> 8), (k, m)


def test_max_probability_rule_matches_oracle(ctx, pkg, orc):
    """The encoder configuration's own policy: top-3 modes, top-2 splits and
    the full set for a head whose most probable entry is below 0.4
    (PRUNE_MAX_PROB), against the oracle's search on those candidates."""
    import torch

    y, plane = _plane(160, 96, 9)
    a, xy = _xy(160, 96)
    rng = np.random.default_rng(9)
    logits = rng.normal(0, 1.0, (len(a), 73)).astype(np.float32)
    logits[np.arange(len(a)), rng.integers(0, 67, len(a))] += rng.uniform(0.0, 9.0, len(a)).astype(np.float32)
    logits[np.arange(len(a)), 67 + rng.integers(0, 6, len(a))] += rng.uniform(0.0, 3.0, len(a)).astype(np.float32)
    got = ctx.ctu_search_xy(plane, 10, 250, xy, torch.from_numpy(logits).cuda(), 3, 2, 0.4, rule=pkg.PRUNE_MAX_PROB)

    def top(v, k):
        return [int(i) for i in sorted(range(len(v)), key=lambda j: (-v[j], j))[:k]]

    def pmax(v):
        e = np.exp(v.astype(np.float64) - v.max())
        return 1.0 / e.sum()

    kept = 0
    for i, (x, yy) in enumerate(a):
        li, ls = logits[i, :67], logits[i, 67:]
        cand = tuple(top(li, 3)) if pmax(li) >= 0.4 else ()
        mask = sum(1 << s for s in top(ls, 2)) if pmax(ls) >= 0.4 else 0x3F
        kept += bool(cand) + (mask != 0x3F)
        want = orc.ctu_search(y, 10, int(x), int(yy), 250, mask, cand)
        g = got[i]
        assert (int(g["cost"]), int(g["split"]), [int(v) for v in g["modes"]]) == \
            (want["cost"], want["split"], want["modes"]), i
    assert 0 < kept < 2 * len(a)  # both pruned and fallback heads occur
