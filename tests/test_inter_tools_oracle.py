"""CPU: properties of the oracle's inter-tool restatements that follow from
the reference's definitions (inter.rs): BDOF of two equal predictions is
their rounded average; DMVR keeps motion whose two predictions already
match; GPM
split directions cover 64 (angle, distance) pairs and weight one side 8/8
far from the edge; CIIP with no intra neighbour weights intra 1/4; the
4-parameter affine model at zero spread gives one MV everywhere."""
import numpy as np


def test_bdof_of_equal_predictions_is_the_average(orc):
    rng = np.random.default_rng(0)
    p = rng.integers(-2000, 18000, 64)
    got = orc.bdof(p, p, 8, 8)
    want = np.clip((2 * p + (1 << 6) + 2 * 8192) >> 7, 0, 255)
    assert np.array_equal(got, want)


def test_dmvr_keeps_motion_that_already_matches(orc):
    """Identical references under equal motion: the zero offset's cost is
    0, below the early-termination bound, so the pair stays."""
    rng = np.random.default_rng(1)
    r = rng.integers(0, 256, (48, 48))
    assert np.array_equal(orc.dmvr(r, r, 16, 16, 16, 16, (32, -16, 32, -16)), [32, -16, 32, -16])


def test_gpm_weights(orc):
    p0, p1 = np.full(64 * 64, 200), np.full(64 * 64, 0)
    seen = set()
    for split in range(64):
        out = orc.gpm(p0, p1, 64, 64, split).reshape(64, 64)
        assert out.min() == 0 and out.max() == 200  # both partitions present
        seen.add(tuple(out[::8, ::8].ravel()))
    assert len(seen) == 64


def test_ciip_weights(orc):
    inter, intra = np.full(16, 100), np.full(16, 200)
    assert (orc.ciip(inter, intra, False, False) == 125).all()
    assert (orc.ciip(inter, intra, True, True) == 175).all()


def test_affine_translation(orc):
    sub, ph, pv, en = orc.affine_mvs([[20, -12], [20, -12], [20, -12]], False, 16, 16, 1)
    assert (sub == [20, -12]).all() and not en and not ph.any() and not pv.any()
