"""CPU: the library's host-side CABAC parser (vvcg_parse_residual_block,
vvcg_parse_strict) against the oracle's restatement of the reference's
encoder side (cabac.rs BinEncoder, residual.rs encode_residual_with_options,
slice.rs encode_ts_block and encode_picture's syntax writes), on the
reference's own round-trip cases:

- residual.rs tests regular_residual_round_trips_sparse_blocks (sizes 4..32,
  QP 4..63), regular_residual_round_trips_chroma_blocks,
  dep_quant_and_sign_hiding_round_trip, inferred_last_group_flags_round_trip;
- slice.rs tests ts_block_round_trips_coefficients (16 / 32 at QP 4 / 26 /
  40) and ts_block_inferred_significance_positions_round_trip;
- slice.rs picture_round_trip_is_exact_at_qp4: the strict encoder's records
  through slice data and back, and the decoded picture equal to the source.

The parser and the writer are independent restatements of inverse
functions, so every case decodes exactly what was coded only when both
follow the reference.
"""
import numpy as np
import pytest


def _lcg(seed):
    seed = (seed * 1664525 + 1013904223) & 0xFFFFFFFF
    return seed, ((seed >> 8) % 121) - 60


def _sparse_block(size, seed):
    """residual.rs sparse_block: every fifth coefficient an LCG value in
    -60..60 (0 replaced by 1), the last one forced positive."""
    c = np.zeros(size * size, np.int32)
    for i in range(size * size):
        if i % 5 == 0:
            seed, v = _lcg(seed)
            c[i] = 1 if v == 0 else v
    seed, v = _lcg(seed)
    c[-1] = max(v, 1)
    return c.reshape(size, size)


def _dense_ts_block(size, seed):
    """slice.rs ts_block_round_trips_coefficients: LCG values, |v| < 6 -> 0."""
    c = np.zeros(size * size, np.int32)
    for i in range(size * size):
        seed, v = _lcg(seed)
        c[i] = 0 if abs(v) < 6 else v
    return c.reshape(size, size)


@pytest.mark.parametrize("size", [4, 8, 16, 32])
@pytest.mark.parametrize("qp", [4, 10, 26, 40, 63])
def test_regular_residual_round_trips(pkg, orc, size, qp):
    block = _sparse_block(size, 0x12345678 ^ size ^ qp)
    data = orc.block_write(block, luma=True, qp=qp)
    assert (pkg.parse_residual_block(data, size, size, pkg.PARSE_LUMA, qp) == block).all()


@pytest.mark.parametrize("size", [4, 8, 16])
def test_chroma_residual_round_trips(pkg, orc, size):
    block = _sparse_block(size, 0x9ABCDEF0 ^ size)
    data = orc.block_write(block, luma=False, qp=26)
    assert (pkg.parse_residual_block(data, size, size, 0, 26) == block).all()


@pytest.mark.parametrize("size", [4, 8, 16])
@pytest.mark.parametrize("dq,sdh", [(True, False), (False, True), (True, True)])
def test_dependent_quantisation_and_sign_hiding_round_trip(pkg, orc, size, dq, sdh):
    block = _sparse_block(size, 0xCAFEBABE ^ size)
    data = orc.block_write(block, luma=True, dep_quant=dq, sign_hiding=sdh, qp=26)
    flags = pkg.PARSE_LUMA | (pkg.PARSE_DEP_QUANT if dq else 0) | (pkg.PARSE_SIGN_HIDING if sdh else 0)
    got = pkg.parse_residual_block(data, size, size, flags, 26)
    if sdh and not dq:
        assert (np.abs(got) == np.abs(block)).all()  # hidden signs follow the parity, not the input
    else:
        assert (got == block).all()


def test_inferred_last_group_flags_round_trip(pkg, orc):
    block = np.zeros((32, 32), np.int32)
    block[0, 0], block[0, 31], block[31, 31] = 9, -5, 7
    data = orc.block_write(block, luma=True, qp=26)
    assert (pkg.parse_residual_block(data, 32, 32, pkg.PARSE_LUMA, 26) == block).all()


@pytest.mark.parametrize("size,shape", [(4, (4, 4)), (8, (8, 8)), (16, (4, 16)), (32, (32, 8))])
def test_rectangular_and_small_blocks_round_trip(pkg, orc, size, shape):
    h, w = shape
    rng = np.random.default_rng(size)
    block = np.where(rng.random((h, w)) < 0.3, rng.integers(-300, 301, (h, w)), 0).astype(np.int32)
    block[0, 0] = 17
    for luma in (True, False):
        data = orc.block_write(block, luma=luma, qp=30)
        assert (pkg.parse_residual_block(data, w, h, pkg.PARSE_LUMA if luma else 0, 30) == block).all()


@pytest.mark.parametrize("size", [16, 32])
@pytest.mark.parametrize("qp", [4, 26, 40])
def test_transform_skip_residual_round_trips(pkg, orc, size, qp):
    block = _dense_ts_block(size, 0x12345678 ^ size)
    data = orc.block_write(block, ts=True, qp=qp)
    assert (pkg.parse_residual_block(data, size, size, pkg.PARSE_TRANSFORM_SKIP, qp) == block).all()


@pytest.mark.parametrize("size", [16, 32])
def test_transform_skip_inferred_significance_round_trips(pkg, orc, size):
    for case in ([(31, 31)], [(0, 0)], [(3, 3)], [(30, 31), (31, 30), (31, 31)]):
        block = np.zeros((size, size), np.int32)
        for x, y in case:
            x, y = min(x, size - 1), min(y, size - 1)
            block[y, x] = 7 if (x + y) % 2 == 0 else -3
        data = orc.block_write(block, ts=True, qp=26)
        assert (pkg.parse_residual_block(data, size, size, pkg.PARSE_TRANSFORM_SKIP, 26) == block).all(), case


def test_malformed_substream_is_rejected(pkg, orc):
    block = _sparse_block(16, 77)
    data = bytearray(orc.block_write(block, luma=True, qp=26))
    with pytest.raises(pkg.InvalidInput):
        pkg.parse_residual_block(bytes(data[: len(data) // 3]), 16, 16, pkg.PARSE_LUMA, 26)


def _strict_records(orc, synth, frames, qp):
    out = []
    for f in frames:
        y, u, v = f
        cus, levels, rec = orc.strict_encode(y, u, v, qp)
        out.append((cus, levels, rec, orc.strict_write(cus, levels, y.shape[1], y.shape[0], qp)))
    return out


@pytest.mark.parametrize("qp", [4, 26, 37, 50])
def test_strict_slice_data_parses_back_to_the_records(pkg, orc, qp):
    from rustmpeg_next_b200 import synth

    frames = [synth.config1_frame(f) for f in range(3)]
    coded = _strict_records(orc, synth, frames, qp)
    pics, cus, levels, used = pkg.parse_strict([(b, 64, 64, qp) for _, _, _, b in coded], threads=3)
    at = 0
    for i, (c0, l0, rec, _) in enumerate(coded):
        c1 = cus[at:at + len(c0)]
        at += len(c0)
        for f in ("luma_mode", "chroma_mode", "cbf", "tu_tools"):
            assert (c1[f] == c0[f]).all(), (i, f)
        for k in range(len(c0)):
            for c, n in ((0, 1024), (1, 256), (2, 256)):
                if c0["level_off"][k, c] >= 0:
                    a = l0[c0["level_off"][k, c]:][:n]
                    b = levels[c1["level_off"][k, c]:][:n]
                    assert (a == b).all(), (i, k, c)
        # decoding the parsed records gives the encoder's reconstruction
        rel = c1.copy()
        dec = orc.strict_decode(rel, levels, 64, 64, qp)
        assert all((d == r).all() for d, r in zip(dec, rec))
    if qp == 4:
        for (_, _, rec, _), f in zip(coded, frames):
            assert all((r == s).all() for r, s in zip(rec, f))  # lossless at QP 4


def test_sparse_parse_matches_dense(pkg, orc):
    from rustmpeg_next_b200 import synth

    frames = [synth.config1_frame(f) for f in range(3)]
    coded = _strict_records(orc, synth, frames, 30)
    streams = [(b, 64, 64, 30) for _, _, _, b in coded]
    pd, cd, ld, _ = pkg.parse_strict(streams)
    ps, cs, ls, _ = pkg.parse_strict(streams, sparse=True)
    assert (ps["tools"] & pkg.TOOL_SPARSE_LEVELS).all()
    back_p, back_c, back_l = synth.densify(ps, cs, ls)
    for k in range(len(cd)):
        for c, n in ((0, 1024), (1, 256), (2, 256)):
            if cd["level_off"][k, c] >= 0:
                assert (ld[cd["level_off"][k, c]:][:n] == back_l[back_c["level_off"][k, c]:][:n]).all()


def test_strict_slice_data_with_every_luma_mode_and_chroma_candidate(pkg, orc):
    """Records with MPM and non-MPM luma modes (truncated binary remainder)
    and non-DM chroma modes through the writer and the parser."""
    from rustmpeg_next_b200 import synth

    y, u, v = synth.config1_frame(0)
    cus, levels, _ = orc.strict_encode(y, u, v, 32)
    rng = np.random.default_rng(5)
    streams, want = [], []
    for rep in range(17):
        c = cus.copy()
        c["luma_mode"] = [(rep * 4 + k) % 67 for k in range(len(c))]
        cand = np.array([0, 50, 18, 1])
        ch = cand[rng.integers(0, 4, len(c))]
        c["chroma_mode"] = np.where(ch == c["luma_mode"], 66, ch)
        c["tu_tools"] &= ~np.uint8(0xF8)  # the transform indices depend on the levels' syntax; keep skip flags
        streams.append((orc.strict_write(c, levels, 64, 64, 32), 64, 64, 32))
        want.append(c)
    _, got, _, _ = pkg.parse_strict(streams)
    want = np.concatenate(want)
    for f in ("luma_mode", "chroma_mode", "cbf"):
        assert (got[f] == want[f]).all(), f
