"""CPU: the oracle's restatement of the strict 8-bit intra profile
(slice.rs:325-455 encode_picture, :458-627 decode_picture), pinned by the
reference's own tests of that profile:

- picture_round_trip_is_exact_at_qp4 (slice.rs:5155-5182) and
  flat_and_gradient_picture_round_trips_at_qp4 (:5222-5254): at QP 4 the
  transform-skip path is lossless, so the decoded picture equals the source;
- qp50_selection_uses_mts_and_lfnst (:5287-5321): on a smooth ramp with flat
  chroma at QP 50 the luma transform search selects both MTS and LFNST;
- closed loop (what every round-trip test of the reference asserts): the
  decoder's reconstruction of the encoder's records equals the encoder's own
  reconstruction, here on the small-picture configuration's content.
"""
import numpy as np
import pytest


def _mts_lfnst_counts(pkg, cus):
    t = cus["tu_tools"].astype(int)
    return int(((t >> pkg.CU_MTS_SHIFT) & 7).astype(bool).sum()), int((t >> pkg.CU_LFNST_SHIFT).astype(bool).sum())


def test_qp4_round_trip_is_exact(orc):
    w = h = 64
    j, i = np.mgrid[0:h, 0:w]
    y = ((i * 3 + j * 5) % 251).astype(np.uint8)
    u = np.full((h // 2, w // 2), 90, np.uint8)
    v = np.full((h // 2, w // 2), 160, np.uint8)
    cus, levels, rec = orc.strict_encode(y, u, v, 4)
    assert all((r == s).all() for r, s in zip(rec, (y, u, v)))
    dec = orc.strict_decode(cus, levels, w, h, 4)
    assert all((d == s).all() for d, s in zip(dec, (y, u, v)))
    assert (cus["tu_tools"] & 1).any()  # luma transform skip at QP 4


def test_flat_and_gradient_round_trip_at_qp4(orc):
    w, h = 96, 64
    j, i = np.mgrid[0:h, 0:w]
    y = np.where(i < 48, 100, (i * 3 + j * 5) % 251).astype(np.uint8)
    u = np.full((h // 2, w // 2), 96, np.uint8)
    v = np.full((h // 2, w // 2), 148, np.uint8)
    cus, levels, rec = orc.strict_encode(y, u, v, 4)
    dec = orc.strict_decode(cus, levels, w, h, 4)
    for d, r, s in zip(dec, rec, (y, u, v)):
        assert (d == s).all() and (r == s).all()


def test_qp50_selects_mts_and_lfnst(pkg, orc):
    from rustmpeg_next_b200 import synth

    w, h = 200, 120
    j, i = np.mgrid[0:h, 0:w]
    y = synth.pad_to((16 + (i + j) % 40).astype(np.uint8), 224, 128)
    u = synth.pad_to(np.full((60, 100), 128, np.uint8), 112, 64)
    v = u.copy()
    cus, levels, rec = orc.strict_encode(y, u, v, 50)
    mts, lfnst = _mts_lfnst_counts(pkg, cus)
    assert mts > 0 and lfnst > 0, (mts, lfnst)
    dec = orc.strict_decode(cus, levels, 224, 128, 50)
    assert all((d == r).all() for d, r in zip(dec, rec))


@pytest.mark.parametrize("qp", [22, 26, 37, 50])
def test_closed_loop_on_the_small_picture_content(pkg, orc, qp):
    from rustmpeg_next_b200 import synth

    for f in range(3):
        y, u, v = synth.config1_frame(f)
        cus, levels, rec = orc.strict_encode(y, u, v, qp)
        dec = orc.strict_decode(cus, levels, 64, 64, qp)
        assert all((d == r).all() for d, r in zip(dec, rec)), (qp, f)
        # the records only carry what decode_picture parses
        t = cus["tu_tools"].astype(int)
        assert ((t & 7) & ~cus["cbf"].astype(int) == 0).all()
        assert not (((t >> pkg.CU_MTS_SHIFT) & 7).astype(bool) & (t >> pkg.CU_LFNST_SHIFT).astype(bool)).any()


def test_small_picture_content_matches_its_description(pkg):
    from rustmpeg_next_b200 import synth

    y0, u0, _ = synth.config1_frame(0)
    y1, _, _ = synth.config1_frame(1)
    assert y0.shape == (64, 64) and u0.shape == (32, 32)
    assert (y0[24:40, 8:24] == 200).all() and (y1[24:40, 10:26] == 200).all()
    assert abs(int(u0.astype(int).mean()) - 128) <= 1 and u0.min() >= 124 and u0.max() <= 132
    ramp = np.rint(16 + 219 * np.arange(64) / 63)
    assert np.abs(y0[:8].astype(int) - ramp[None, :]).max() <= 8


def test_strict_decode_rejects_bad_tools(pkg, orc):
    from rustmpeg_next_b200 import synth

    y, u, v = synth.config1_frame(0)
    cus, levels, _ = orc.strict_encode(y, u, v, 30)
    bad = cus.copy()
    bad["tu_tools"][0] = (1 << pkg.CU_MTS_SHIFT) | (1 << pkg.CU_LFNST_SHIFT)
    with pytest.raises(ValueError):
        orc.strict_decode(bad, levels, 64, 64, 30)
