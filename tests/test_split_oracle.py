"""CPU: the oracle of the encoders' quadrant-mean partition hook
(choose_qt_mtt_partition_rdo_16 / choose_qt_mtt_partition_rdo,
crates/rustmpeg-video/src/vvc/slice.rs:4111-4167) against a line-by-line
Python restatement on random planes and regions (inside, across and past the
plane edge), and on designed content whose split is known: flat (none),
left/right halves (binary vertical), top/bottom halves (binary horizontal),
quadrant pattern (quad; binary on a non-square region), regions at or below
the minimum size (none), and 10-bit samples whose 8-bit rounding saturates."""
import numpy as np
import pytest

NONE, QT, BT_H, BT_V = 0, 1, 2, 3


def _py_split(plane, bd, x, y, w, h, qp, min_cb):
    if w <= max(min_cb, 8) or h <= max(min_cb, 8):
        return NONE
    shift = max(bd - 8, 0)
    add = (1 << (shift - 1)) if shift > 0 else 0
    p8 = np.minimum(np.minimum(plane.astype(np.int64) + add, 65535) >> shift, 255)
    ph, pw = plane.shape
    hw, hh = w // 2, h // 2

    def mean(qx, qy, qw, qh):
        s = int(p8[qy:min(qy + qh, ph), qx:min(qx + qw, pw)].sum()) if qx < pw and qy < ph else 0
        return s // max(qw * qh, 1)

    m00, m10 = mean(x, y, hw, hh), mean(x + hw, y, hw, hh)
    m01, m11 = mean(x, y + hh, hw, hh), mean(x + hw, y + hh, hw, hh)
    hor = abs(m00 - m01) + abs(m10 - m11)
    ver = abs(m00 - m10) + abs(m01 - m11)
    thr = max(qp, 4) // 2 + 8
    if w == h and hor > thr and ver > thr:
        return QT
    if hor > ver and hor > thr:
        return BT_H
    if ver > thr:
        return BT_V
    return NONE


@pytest.mark.parametrize("bd", [8, 10, 12])
def test_oracle_matches_restatement_on_random_regions(orc, bd):
    rng = np.random.default_rng(bd)
    h, w = 96, 160
    # blocky content so that every outcome occurs
    coarse = rng.integers(0, 1 << bd, (h // 8 + 1, w // 8 + 1))
    plane = np.kron(coarse, np.ones((8, 8), np.int64))[:h, :w].astype(np.uint16)
    regions = []
    for _ in range(400):
        rw, rh = (int(v) for v in rng.choice([4, 8, 12, 16, 24, 32, 48, 64], 2))
        x, y = int(rng.integers(0, w + 16)), int(rng.integers(0, h + 16))
        regions.append((x, y, rw, rh, int(rng.integers(0, 64)), int(rng.choice([4, 8, 16]))))
    got = orc.qt_mtt_split(plane, bd, regions)
    want = [_py_split(plane, bd, *r) for r in regions]
    assert got.tolist() == want
    assert set(want) == {NONE, QT, BT_H, BT_V}


def _plane(f, h=64, w=64):
    yy, xx = np.mgrid[0:h, 0:w]
    return f(xx, yy).astype(np.uint16)


def test_designed_content(orc):
    flat = _plane(lambda x, y: 100 + 0 * x)
    lr = _plane(lambda x, y: np.where(x < 16, 20, 200))
    tb = _plane(lambda x, y: np.where(y < 16, 20, 200))
    quad = _plane(lambda x, y: np.where((x < 16) ^ (y < 16), 20, 200))
    region = (0, 0, 32, 32, 32, 4)
    assert orc.qt_mtt_split(flat, 8, [region]).tolist() == [NONE]
    assert orc.qt_mtt_split(lr, 8, [region]).tolist() == [BT_V]
    assert orc.qt_mtt_split(tb, 8, [region]).tolist() == [BT_H]
    assert orc.qt_mtt_split(quad, 8, [region]).tolist() == [QT]
    # no quad split for a non-square region: the larger difference decides
    assert orc.qt_mtt_split(quad, 8, [(0, 0, 32, 16, 32, 4)]).tolist() == [BT_V]
    # at or below max(min_cb, 8) in either dimension: no split
    assert orc.qt_mtt_split(quad, 8, [(0, 0, 8, 32, 32, 4), (0, 0, 32, 32, 32, 32)]).tolist() == [NONE, NONE]
    # a weak edge stays below max(qp, 4) / 2 + 8
    weak = _plane(lambda x, y: np.where(x < 16, 100, 110))
    assert orc.qt_mtt_split(weak, 8, [(0, 0, 32, 32, 0, 4)]).tolist() == [BT_V]   # 2 * 10 > 10
    assert orc.qt_mtt_split(weak, 8, [(0, 0, 32, 32, 30, 4)]).tolist() == [NONE]  # 20 <= 23


def test_high_bit_depth_rounds_and_saturates_at_255(orc):
    # 10-bit 1023 rounds to (1023 + 2) >> 2 = 256 -> 255; 1020 -> 255; 900 -> 225
    left_right = _plane(lambda x, y: np.where(x < 16, 900, 1023))
    r = (0, 0, 32, 32, 4, 4)
    assert orc.qt_mtt_split(left_right, 10, [r]).tolist() == [BT_V]  # |225 - 255| * 2 = 60 > 10
    assert _py_split(left_right, 10, *r) == BT_V


def test_region_past_the_plane_divides_by_the_full_area(orc):
    # only the top-left quadrant lies inside: its mean is 200, the others 0
    plane = np.full((16, 16), 200, np.uint16)
    got = orc.qt_mtt_split(plane, 8, [(0, 0, 32, 32, 32, 4), (8, 0, 32, 32, 32, 4)])
    want = [_py_split(plane, 8, 0, 0, 32, 32, 32, 4), _py_split(plane, 8, 8, 0, 32, 32, 32, 4)]
    assert got.tolist() == want and want[0] == QT
