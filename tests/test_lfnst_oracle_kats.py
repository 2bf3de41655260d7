"""CPU: the reference's own LFNST tests (crates/rustmpeg-video/src/vvc/
lfnst.rs:319-388) ported to the oracle's forward_lfnst_rect /
inverse_lfnst_rect: Planar and DC share the untransposed set 0, invalid
indexes are rejected, the forward transform leaves nothing past the zero-out
length of the top-left diagonal scan, forward then inverse keeps the
low-frequency block within the reference's error bound, and transposed
directional modes round trip within int16. Blocks come from the reference
test's generator (LCG 1664525 / 1013904223, (seed >> 20) % 81 - 40)."""
import numpy as np
import pytest


def _block(size, seed):
    out = np.zeros(size * size, np.int32)
    for i in range(size * size):
        seed = (seed * 1664525 + 1013904223) & 0xFFFFFFFF
        out[i] = ((seed >> 20) % 81) - 40
    return out


def _top_left_diag_scan():
    """Up-right diagonal order of 4x4 sub-blocks, and of positions inside
    each, over the top-left 8x8 (the LFNST coefficient order)."""
    def diag(n):
        return [(x, d - x) for d in range(2 * n - 1) for x in range(n) if 0 <= d - x < n]
    return [(4 * sx + x, 4 * sy + y) for sx, sy in diag(2) for x, y in diag(4)]


def test_scan_generator_starts_like_the_lfnst_scan():
    assert _top_left_diag_scan()[:10] == [(0, 0), (0, 1), (1, 0), (0, 2), (1, 1), (2, 0), (0, 3), (1, 2), (2, 1),
                                          (3, 0)]


def test_planar_and_dc_use_the_same_untransposed_set(orc):
    for size in (4, 8, 16):
        c = _block(size, 0x2468 + size)
        _, a = orc.lfnst(c, size, size, 1, 0, True)
        _, b = orc.lfnst(c, size, size, 1, 1, True)
        assert np.array_equal(a, b)


def test_rejects_invalid_indexes(orc):
    c = np.zeros(16, np.int32)
    assert orc.lfnst(c, 4, 4, 0, 0, True)[0] != 0
    assert orc.lfnst(c, 4, 4, 3, 0, True)[0] != 0
    assert orc.lfnst(c, 4, 4, 0, 0, False)[0] != 0


@pytest.mark.parametrize("size", [4, 8, 16, 32])
@pytest.mark.parametrize("index", [1, 2])
def test_forward_zeroes_everything_outside_the_low_frequency_region(orc, size, index):
    rc, c = orc.lfnst(_block(size, 0x12345678), size, size, index, 0, True)
    assert rc == 0
    zero_out = 8 if size in (4, 8) else 16
    scan_len = 48 if size >= 8 else 16
    nonzero = 0
    for k, (x, y) in enumerate(_top_left_diag_scan()[:scan_len]):
        if c[y * size + x] != 0:
            assert k < zero_out, (size, index, k)
            nonzero += 1
    assert nonzero <= zero_out


@pytest.mark.parametrize("size", [8, 16, 32])
@pytest.mark.parametrize("index", [1, 2])
def test_inverse_of_forward_preserves_low_frequencies_approximately(orc, size, index):
    original = _block(size, 0x9ABCDEF0 ^ size ^ index)
    rc, c = orc.lfnst(original, size, size, index, 0, True)
    assert rc == 0
    rc, back = orc.lfnst(c, size, size, index, 0, False)
    assert rc == 0
    sse = int(((original.astype(np.int64) - back) ** 2).sum())
    assert sse < 200_000_000, sse


@pytest.mark.parametrize("mode", [35, 50, 66, 81, 94])
def test_transposed_directional_modes_round_trip(orc, mode):
    for size in (4, 8, 16):
        rc, c = orc.lfnst(_block(size, 0x55AA0000 ^ mode), size, size, 1, mode, True)
        assert rc == 0
        rc, back = orc.lfnst(c, size, size, 1, mode, False)
        assert rc == 0
        assert back.min() >= -32768 and back.max() <= 32767
