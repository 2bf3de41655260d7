"""CPU: two more of the reference's intra tests (crates/rustmpeg-video/src/
vvc/predict.rs:4247-4704) ported to the oracle: MIP predictions of every 8x8
mode, transposed or not, stay within 8 bits on a flat 110 boundary; and
gather_references_16 substitutes the below-left references of a block
instead of reading them (shown by prediction: changing those samples leaves
a below-left mode's prediction unchanged, changing the left column does not),
on the reference test's ramp plane."""
import numpy as np
import pytest


def _ramp(w, h, bd):
    mx = (1 << bd) - 1
    y, x = np.mgrid[0:h, 0:w].astype(np.int64)
    return np.minimum((37 * x + 91 * y + 11 * ((x * y) % 17)) % mx, mx).astype(np.uint16)


@pytest.mark.parametrize("transposed", [False, True])
def test_mip_prediction_on_flat_boundary_stays_within_8bit_range(orc, transposed):
    above = np.full(8, 110, np.int32)
    left = np.full(8, 110, np.int32)
    for mode in range(8):  # get_num_modes_mip(8, 8)
        pred = orc.mip_predict(above, left, 8, 8, mode, transposed, 8)
        assert pred.size == 64 and pred.min() >= 0 and pred.max() <= 255


@pytest.mark.parametrize("x,y,size", [(32, 0, 32), (32, 32, 16)])
def test_gather_references_16_substitutes_below_left_instead_of_reading_it(orc, x, y, size):
    plane = _ramp(64, 64, 10)
    mode = 2  # bottom-left diagonal: reads left[size..2 size)
    base = orc.predict_block(plane, 10, x, y, size, size, mode)
    below = plane.copy()
    below[y + size:y + 2 * size, x - 1] ^= 0x155  # the below-left samples
    assert np.array_equal(orc.predict_block(below, 10, x, y, size, size, mode), base)
    left = plane.copy()
    left[y:y + size, x - 1] ^= 0x155  # the left column proper
    assert not np.array_equal(orc.predict_block(left, 10, x, y, size, size, mode), base)
