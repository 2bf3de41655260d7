"""GPU parity: the 8-bit strict encoder's luma transform search
(vvcg_luma_tx_search_dev) against the oracle's restatement of
slice::encode_luma: the same winner (mts_idx / lfnst_idx / transform skip),
cbf, SSE, levels and reconstructed samples for every block."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _blocks(n_blocks, seed):
    rng = np.random.default_rng(seed)
    recs, preds, srcs = [], [], []
    at = 0
    for i in range(n_blocks):
        lg = int(rng.integers(2, 6))
        n = 1 << lg
        yy, xx = np.mgrid[0:n, 0:n]
        base = 128 + 60 * np.sin(xx * rng.random() * 0.7 + yy * rng.random() * 0.7 + rng.random() * 6)
        src = np.clip(base + rng.normal(0, rng.choice([2, 8, 25]), (n, n)), 0, 255).astype(np.int16)
        if i % 2:
            pred = np.clip(base + rng.normal(0, 6, (n, n)) + rng.integers(-20, 21), 0, 255).astype(np.int16)
        else:  # oriented low-frequency residuals, where LFNST candidates win
            ang, f = rng.random() * np.pi, rng.random() * 0.5
            res = rng.normal(0, 12) * np.cos(f * (np.cos(ang) * xx + np.sin(ang) * yy)) + rng.normal(0, 1, (n, n))
            pred = np.clip(src - np.round(res), 0, 255).astype(np.int16)
        qp = int(rng.choice([4, 12, 22, 27, 32, 37, 45, 51]))
        flags = (1 if qp == 4 and rng.random() < 0.7 else 0) | (2 if rng.random() < 0.6 else 0)
        recs.append((lg, qp, int(rng.integers(0, 67)), flags, at, at, 0))
        preds.append(pred.reshape(-1))
        srcs.append(src.reshape(-1))
        at += n * n
    return recs, np.concatenate(preds), np.concatenate(srcs), at


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_luma_tx_search_matches_oracle(ctx, pkg, orc, seed):
    import torch

    recs, pred, src, total = _blocks(600, seed)
    reqs = np.array(recs, dtype=pkg.TXS_REQ_DTYPE)
    d_pred, d_src = torch.from_numpy(pred).cuda(), torch.from_numpy(src).cuda()
    d_lv = torch.zeros(total, dtype=torch.int16, device="cuda")
    d_sm = torch.zeros(total, dtype=torch.int16, device="cuda")
    res = ctx.luma_tx_search(reqs, d_pred, d_src, d_lv, d_sm)
    lv, sm = d_lv.cpu().numpy(), d_sm.cpu().numpy()
    chosen = set()
    for i, r in enumerate(reqs):
        n = 1 << int(r["log2_size"])
        o = int(r["in_off"])
        m, l, ts, cbf, sse, wl, ws = orc.luma_tx_search(pred[o:o + n * n].reshape(n, n), src[o:o + n * n].reshape(n, n),
                                                         int(r["qp"]), int(r["mode"]), bool(r["flags"] & 1),
                                                         bool(r["flags"] & 2))
        g = res[i]
        assert (int(g["mts_idx"]), int(g["lfnst_idx"]), int(g["transform_skip"]), int(g["cbf"]), int(g["sse"])) == \
            (m, l, ts, cbf, sse), f"block {i} {r}"
        assert (lv[o:o + n * n] == wl).all() and (sm[o:o + n * n] == ws).all(), f"block {i} data"
        chosen.add((m, l, ts))
    # the search picks among several candidate kinds, LFNST among them
    assert len(chosen) >= 5 and any(c[1] for c in chosen)
