"""CPU: the oracle's general-decoder intra prediction (decode_general.rs
Gen::gather_len / gather_mrl / cclm_predict, predict_luma, predict_chroma).

Pin: with the neighbourhood a raster decode leaves (the rows above and the
columns to the left down to the block's bottom decoded, nothing below-left),
the general path's Planar / DC / angular predictions equal the 16-bit frame
path's predict_block_16 (predict.rs:3079-3410, pinned by the reference's
own tests) for luma and chroma, every mode and block size."""
import numpy as np
import pytest


def _state(w, h, bd, seed):
    rng = np.random.default_rng(seed)
    maxv = (1 << bd) - 1
    yy, xx = np.mgrid[0:h, 0:w]
    Y = np.clip((maxv // 2) + (maxv // 5) * np.sin(xx / 5.0 + yy / 9.0) + rng.integers(-20, 21, (h, w)), 0,
                maxv).astype(np.uint16)
    U = np.clip(rng.integers(maxv // 3, 2 * maxv // 3, (h // 2, w // 2)), 0, maxv).astype(np.uint16)
    V = np.clip(rng.integers(maxv // 3, 2 * maxv // 3, (h // 2, w // 2)), 0, maxv).astype(np.uint16)
    return Y, U, V


@pytest.mark.parametrize("bw,bh", [(4, 4), (8, 8), (16, 16), (32, 32), (64, 64), (8, 32), (32, 8), (4, 16), (16, 4)])
def test_general_luma_equals_frame_path_on_raster_neighbourhoods(pkg, orc, bw, bh):
    Y, U, V = _state(192, 192, 10, bw * 7 + bh)
    x, y = 64, 64
    dy = np.zeros((48, 48), np.uint8)
    cy, cx = np.mgrid[0:48, 0:48]
    dy[(cy * 4 < y) | ((cx * 4 < x) & (cy * 4 < y + bh))] = 1
    dc = np.zeros((96, 96), np.uint8)
    reqs = np.zeros(67, pkg.GEN_INTRA_REQ_DTYPE)
    for m in range(67):
        reqs[m] = (x, y, bw, bh, x, y, bw, bh, 0, m, 0, 0, 0, (0, 0, 0), m * bw * bh)
    got = orc.gen_intra_predict(Y, U, V, dy, dc, 10, 64, reqs, 67 * bw * bh)
    for m in range(67):
        want = orc.predict_block(Y, 10, x, y, bw, bh, m).astype(np.int16).ravel()
        assert np.array_equal(got[m * bw * bh:(m + 1) * bw * bh], want), m


@pytest.mark.parametrize("bw,bh", [(4, 4), (8, 8), (16, 16), (32, 32), (4, 16), (16, 4), (2, 8), (8, 2)])
def test_general_chroma_equals_frame_path_on_raster_neighbourhoods(pkg, orc, bw, bh):
    Y, U, V = _state(192, 192, 10, bw * 5 + bh)
    x, y = 32, 32  # chroma samples
    dy = np.ones((48, 48), np.uint8)
    cy, cx = np.mgrid[0:96, 0:96]
    dc = ((cy < y) | ((cx < x) & (cy < y + bh))).astype(np.uint8)
    reqs = np.zeros(67, pkg.GEN_INTRA_REQ_DTYPE)
    for m in range(67):
        reqs[m] = (x, y, bw, bh, 0, 0, 0, 0, 1, m, 0, 0, 0, (0, 0, 0), m * bw * bh)
    got = orc.gen_intra_predict(Y, U, V, dy, dc, 10, 64, reqs, 67 * bw * bh)
    # below 4 samples the general path leaves PDPC out of Planar / DC
    # (decode_general.rs:4767 / :4781) where predict_block_16 applies it
    for m in range(0 if min(bw, bh) >= 4 else 2, 67):
        want = orc.predict_block(U, 10, x, y, bw, bh, m, is_luma=False).astype(np.int16).ravel()
        assert np.array_equal(got[m * bw * bh:(m + 1) * bw * bh], want), m


@pytest.mark.parametrize("bw,bh", [(4, 4), (8, 8), (16, 16), (8, 4), (4, 8), (16, 8)])
def test_general_cclm_lm_and_lm_l_equal_frame_path(pkg, orc, bw, bh):
    """LM and LM-L with nothing decoded below-left equal
    predict_cclm_with_format_16 (predict.rs:3996-4066). LM-T differs by
    design: the general path extends the top template over the decoded
    above-right samples (numTopRight, decode_general.rs:4404-4412), the
    frame path stops at the block width."""
    for x, y in ((32, 32), (32, 16), (16, 32)):
        Y, U, V = _state(192, 192, 10, bw + bh + x)
        dy = np.ones((48, 48), np.uint8)
        cy, cx = np.mgrid[0:96, 0:96]
        dc = ((cy < y) | ((cx < x) & (cy < y + bh))).astype(np.uint8)
        for mode in (0, 1):
            r = np.zeros(1, pkg.GEN_INTRA_REQ_DTYPE)
            r[0] = (x, y, bw, bh, 0, 0, 0, 0, 1, 81 + mode, 0, 0, 0, (0, 0, 0), 0)
            got = orc.gen_intra_predict(Y, U, V, dy, dc, 10, 64, r, bw * bh)
            want = orc.predict_cclm(Y, U, 10, x, y, bw, bh, mode, 1, 64).astype(np.int16).ravel()
            assert np.array_equal(got, want), (x, y, mode)
