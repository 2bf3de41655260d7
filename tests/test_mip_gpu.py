"""GPU parity: matrix-based intra prediction (vvcg_mip_predict_dev) against
the oracle's restatement of predict_mip_bd and choose_best_mip_mode_16, over
every block size 4x4..64x64 (all three size classes, every upsampling case),
every mode in both orientations, and the SAD search."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(rng, search_frac):
    recs, refs, srcs = [], [], []
    ref_at = out_at = 0
    for lw in range(2, 7):
        for lh in range(2, 7):
            for _ in range(6):
                w, h = 1 << lw, 1 << lh
                bd = int(rng.choice([8, 10, 12]))
                a = rng.integers(0, 1 << bd, w + h)
                if rng.random() < 0.5:  # smooth references
                    a = np.clip(np.cumsum(rng.integers(-9, 10, w + h)) + (1 << (bd - 1)), 0, (1 << bd) - 1)
                search = rng.random() < search_frac
                nm = 16 if (w == 4 and h == 4) else (8 if (w == 4 or h == 4 or (w == 8 and h == 8)) else 6)
                mode = 0xFF if search else int(rng.integers(0, nm + 3))
                recs.append((lw, lh, bd, mode, int(rng.integers(0, 2)), (0, 0, 0), ref_at, out_at))
                refs.append(a.astype(np.int16))
                src = np.clip(rng.integers(0, 1 << bd) + rng.integers(-40, 41, w * h), 0, (1 << bd) - 1)
                srcs.append(src.astype(np.int16))
                ref_at += w + h
                out_at += w * h
    return recs, np.concatenate(refs), np.concatenate(srcs), out_at


@pytest.mark.parametrize("seed,search_frac", [(1, 0.0), (2, 0.5)])
def test_mip_matches_oracle(ctx, pkg, orc, seed, search_frac):
    import torch

    rng = np.random.default_rng(seed)
    recs, refs, srcs, total = _case(rng, search_frac)
    reqs = np.array(recs, dtype=pkg.MIP_REQ_DTYPE)
    d_refs, d_src = torch.from_numpy(refs).cuda(), torch.from_numpy(srcs).cuda()
    d_pred = torch.zeros(total, dtype=torch.int16, device="cuda")
    res = ctx.mip_predict(reqs, d_refs, d_pred, d_src)
    pred = d_pred.cpu().numpy()
    for i, r in enumerate(reqs):
        w, h = 1 << int(r["log2_w"]), 1 << int(r["log2_h"])
        ro, oo, bd = int(r["ref_off"]), int(r["out_off"]), int(r["bit_depth"])
        above, left = refs[ro:ro + w], refs[ro + w:ro + w + h]
        if int(r["mode"]) == 0xFF:
            m, t, sad, want = orc.mip_search(above, left, srcs[oo:oo + w * h], w, h, bd)
            assert (int(res[i]["mode"]), int(res[i]["transposed"]), int(res[i]["sad"])) == (m, t, sad), f"request {i}"
        else:
            want = orc.mip_predict(above, left, w, h, int(r["mode"]), int(r["transposed"]), bd)
        assert (pred[oo:oo + w * h].astype(np.int32) == want).all(), f"request {i} {r}"
