"""CPU: the oracle's transform-unit composites (oracle/orc_tu.cpp) against the
component functions they chain, and the reference's round-trip properties."""
import numpy as np

import oracle as orc_mod


def _rec(lw, lh, bd=10, qp=32, flags=0, mts=0, lfnst=0, mode=0):
    r = np.zeros(1, orc_mod.TU_DTYPE)
    r["log2_w"], r["log2_h"], r["bit_depth"], r["qp"] = lw, lh, bd, qp
    r["flags"], r["mts_idx"], r["lfnst_idx"], r["lfnst_mode"] = flags, mts, lfnst, mode
    return r


def test_inverse_composite_equals_dequant_then_inverse_transform(orc):
    rng = np.random.default_rng(0)
    for lw, lh in [(2, 2), (3, 4), (5, 5), (6, 6), (4, 2)]:
        w, h = 1 << lw, 1 << lh
        lv = np.zeros(w * h, np.int16)
        lv[rng.integers(0, min(w * h, 64), 5)] = rng.integers(-20, 21, 5)
        rc, got = orc.tu_batch(_rec(lw, lh), lv, w * h)
        assert rc == 0
        deq = orc.dequantize(lv.reshape(h, w), 32, bd=10)
        want = orc.inverse_transform(deq, skip_w=max(0, w - 32), skip_h=max(0, h - 32), bd=10)
        assert (got.reshape(h, w) == want).all()


def test_forward_then_inverse_reconstructs_at_low_qp(orc):
    rng = np.random.default_rng(1)
    # white-noise residuals: units without zero-out (a 32-point MTS keeps only 16)
    for lw, lh, mts in [(3, 3, 0), (4, 4, 1), (5, 5, 0), (2, 4, 2), (4, 3, 3)]:
        w, h = 1 << lw, 1 << lh
        res = rng.integers(-200, 201, w * h).astype(np.int16)
        r = _rec(lw, lh, bd=10, qp=16, mts=mts)
        rc, lv = orc.tu_batch(r, res, w * h, forward=True)
        assert rc == 0
        rc, back = orc.tu_batch(r, lv, w * h)
        assert rc == 0
        assert np.abs(back.astype(int) - res).mean() < 4


def test_transform_skip_is_lossless_at_qp4(orc):
    # transform.rs:796-801: quantize_ts / dequantize_ts round trip exactly at QP 4
    res = np.arange(-128, 128, dtype=np.int16)
    r = _rec(4, 4, qp=4, flags=orc_mod.TU_TRANSFORM_SKIP)
    rc, lv = orc.tu_batch(r, res, 256, forward=True)
    rc2, back = orc.tu_batch(r, lv, 256)
    assert rc == rc2 == 0 and (back == res).all()


def test_bdpcm_accumulates_with_saturation(orc):
    lv = np.zeros(16, np.int16)
    lv[:4] = [100, 100, 100, 100]
    r = _rec(2, 2, qp=4, flags=orc_mod.TU_TRANSFORM_SKIP | orc_mod.TU_BDPCM_HOR)
    rc, out = orc.tu_batch(r, lv, 16)
    assert rc == 0 and out[:4].tolist() == [100, 200, 300, 400]
    lv[:] = 32767
    rc, out = orc.tu_batch(_rec(2, 2, qp=4, flags=orc_mod.TU_TRANSFORM_SKIP | orc_mod.TU_BDPCM_VER), lv, 16)
    assert rc == 0 and (out == 32767).all()


def test_lfnst_units_round_trip_and_reject_mts(orc):
    rng = np.random.default_rng(2)
    res = rng.integers(-100, 101, 64).astype(np.int16)
    r = _rec(3, 3, qp=20, lfnst=1, mode=18)
    rc, lv = orc.tu_batch(r, res, 64, forward=True)
    # lfnst.rs:196-203: the 48 LFNST positions past the 8 outputs of an 8x8
    # unit are cleared; the bottom-right 4x4 keeps its primary coefficients
    scan8 = orc.coeff_scan(8, 8)
    assert rc == 0 and (lv[scan8[8:48]] == 0).all()
    rc, back = orc.tu_batch(r, lv, 64)
    assert rc == 0 and np.abs(back.astype(int) - res).mean() < 60
    assert orc.tu_batch(_rec(3, 3, lfnst=1, mts=1), res, 64, forward=True)[0] == -1
