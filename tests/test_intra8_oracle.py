"""CPU: the oracle's 8-bit luma predictors and mode search
(predict.rs:1058-1958, :2619-2801; slice.rs:2698-2731).

Pins: the reference's own predictor tests (predict.rs:4247-4325: flat planes
stay flat under Planar, DC and all 65 angular modes; the top-left block
predicts the neutral 128; Planar wins a tie) and its cross-path test
planar_16_matches_the_8bit_reference_path (predict.rs:4565-4612), extended
here to all 67 modes: the 8-bit restatement equals the 16-bit one
(predict_block_16) on the same 8-bit samples.
"""
import numpy as np
import pytest


def _ramp(size=64):
    i = np.arange(size * size)
    return ((37 * (i % size) + 91 * (i // size) + 7 * (i % 13)) % 256).astype(np.uint8).reshape(size, size)


def test_flat_planes_stay_flat(orc):
    p77 = np.full((64, 64), 77, np.uint8)
    assert np.all(orc.predict_luma_8(p77, 32, 32, 32, 32, 0) == 77)
    p42 = np.full((64, 64), 42, np.uint8)
    assert np.all(orc.predict_luma_8(p42, 32, 32, 32, 32, 1) == 42)
    p93 = np.full((64, 64), 93, np.uint8)
    for d in range(2, 67):
        assert np.all(orc.predict_luma_8(p93, 16, 16, 16, 16, d) == 93), d


def test_top_left_block_is_neutral_and_planar_wins_ties(orc):
    z = np.zeros((32, 32), np.uint8)
    assert np.all(orc.predict_luma_8(z, 0, 0, 32, 32, 0) == 128)
    src = np.full((32, 32), 128, np.uint8)
    assert orc.luma_intra_search_8(z, src, 0, 0, 32, 32, [0, 1, 50, 18, 46, 54]) == (0, 0, 0)


@pytest.mark.parametrize("w,h", [(4, 4), (4, 8), (8, 4), (8, 8), (16, 16), (32, 32), (32, 16), (16, 32), (64, 64),
                                 (4, 64), (64, 4)])
def test_8bit_predictors_equal_the_16bit_ones(orc, w, h):
    p8 = _ramp()
    for bx, by in [(0, 0), (32, 0), (0, 32), (16, 16), (32, 32)]:
        if bx + w > 64 or by + h > 64:
            continue
        for mode in range(67):
            a = orc.predict_luma_8(p8, bx, by, w, h, mode)
            b = orc.predict_block(p8.astype(np.uint16), 8, bx, by, w, h, mode)
            assert np.array_equal(a, b.astype(np.int32)), (w, h, bx, by, mode)


def test_search_returns_the_best_of_the_predictions(orc):
    rng = np.random.default_rng(4)
    recon = _ramp()
    src = rng.integers(0, 256, (64, 64)).astype(np.uint8)
    mode, mrl, sad = orc.luma_intra_search_8(recon, src, 32, 32, 32, 32, [0, 1, 50, 18, 46, 54])
    sads = [int(np.abs(src[32:, 32:].astype(np.int64) - orc.predict_luma_8(recon, 32, 32, 32, 32, m)).sum())
            for m in range(67)]
    assert sad == min(sads) and mode == sads.index(min(sads)) and mrl == 0
    # MRL lines: a block below the CTU's first row; line 0 stays when no line is strictly better
    mode2, mrl2, sad2 = orc.luma_intra_search_8(recon, src, 16, 16, 16, 16, [0, 1, 50, 18, 46, 54], mrl=True, ctu=32)
    base = orc.luma_intra_search_8(recon, src, 16, 16, 16, 16, [0, 1, 50, 18, 46, 54])
    assert sad2 <= base[2]
    if mrl2:
        p = orc.predict_luma_8(recon, 16, 16, 16, 16, mode2, mrl=mrl2, ctu=32)
        assert int(np.abs(src[16:32, 16:32].astype(np.int64) - p).sum()) == sad2
