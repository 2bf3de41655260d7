"""CPU: the oracle's CTU full search (the GPU encoder's candidate-cost stage;
no reference counterpart): a flat picture keeps the unsplit CU with Planar,
split costs add up from their blocks, and the SATD is the 8x8 Hadamard sum
(scipy's Sylvester Hadamard matrix) of the block residual."""
import numpy as np


def test_flat_picture_keeps_one_planar_cu(orc):
    src = np.full((64, 64), 300, np.uint16)
    lam = orc.search_lambda_q8(32)
    r = orc.ctu_search(src, 10, 32, 32, lam)
    assert (r["split"], r["cu_mode"], r["modes"][0]) == (0, 0, 0)
    # SATD 0 everywhere: each cost is lambda * (split bits + 8 + 2 per Planar block)
    counts, sbits = [1, 4, 2, 2, 3, 3], [1, 2, 3, 3, 4, 4]
    want = [(lam * sbits[s]) // 256 + counts[s] * ((lam * 10) // 256) for s in range(6)]
    assert r["split_cost"] == want


def test_satd_of_a_single_mode_equals_hadamard_sum(orc):
    from scipy.linalg import hadamard

    rng = np.random.default_rng(1)
    src = rng.integers(0, 1024, (64, 64)).astype(np.uint16)
    lam = 0
    r = orc.ctu_search(src, 10, 32, 32, lam, split_mask=1, cand=(18,))
    pred = orc.predict_block(src, 10, 32, 32, 32, 32, 18).astype(np.int64)
    d = src[32:64, 32:64].astype(np.int64) - pred
    H = hadamard(8)
    satd = 0
    for ty in range(0, 32, 8):
        for tx in range(0, 32, 8):
            satd += (int(np.abs(H @ d[ty:ty + 8, tx:tx + 8] @ H.T).sum()) + 2) >> 2
    assert r["split_cost"][0] == satd and r["cu_mode"] == 18
