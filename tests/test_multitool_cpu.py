"""CPU: the multi-tool stream (VvcMultiToolEncoder, mod.rs:1512-1720): the
oracle's restatement of its IDR encoder / decoder (slice.rs:2575 / :3012)
and P-picture encoder / decoder (slice.rs:3307 / :3552) in closed loop, and
the library's host parser (vvcg_parse_multitool_idr / _p) against the
oracle's restatement of the encoder side's CABAC writes, on:

- the small-picture configuration's sequence (64x64 8-bit, QP 26, an IDR
  picture and two P pictures; ramp + noise + a moving square);
- the reference's inter_p_slice_conformance_cases_qp4_qp10_qp40_round_trip
  cases (mod.rs:4150-4197: 64x64 at QP 4 / 10, 200x120 at QP 40, with and
  without dependent quantisation, sign hiding where DQ is off) and its
  multi_tool_encoder_and_decoder_round_trip_gop_sequence (mod.rs:4103-4146)
  with the options this library supports (CCLM, MIP, joint Cb-Cr, SAO and
  ALF are not);
- AMVP coding units with coded motion vector differences (which the
  reference's encoder never writes, but its decoder reads), whose motion the
  parser must derive as the oracle's restatement of decode_inter_picture does.
"""
import numpy as np
import pytest


def _gradient(w, h, shift=0):
    """mod.rs:3219-3235 gradient, luma shifted as the conformance test does."""
    j, i = np.mgrid[0:h, 0:w]
    y = (((i * 3 + j * 5) % 251) + shift) % 256
    return y.astype(np.uint8), np.full((h // 2, w // 2), 90, np.uint8), np.full((h // 2, w // 2), 160, np.uint8)


def _coded(frame, w, h):
    from rustmpeg_next_b200 import synth

    cw, ch = (w + 31) // 32 * 32, (h + 31) // 32 * 32
    y, u, v = frame
    return synth.pad_to(y, cw, ch), synth.pad_to(u, cw // 2, ch // 2), synth.pad_to(v, cw // 2, ch // 2)


def _as_streams(st, w, h, qp, opts):
    return [(p["kind"], p["data"], w, h, qp, opts) for p in st]


def _hides_signs(opts):
    """Sign hiding without dependent quantisation: the reference's encoder
    writes its levels unchanged and skips the hidden signs, so the decoder
    infers those signs from the parity of the sums (residual.rs decode side)
    and its reconstruction can differ from the encoder's."""
    return bool(opts & 2) and not (opts & 1)


def _check_parse(pkg, orc, st, w, h, qp, opts, sparse=False):
    """Every picture's parsed records equal the encoder's, levels included
    (their magnitudes where signs are hidden)."""
    streams = _as_streams(st, w, h, qp, opts)
    for kind in ("I", "P"):
        idx = [k for k, p in enumerate(st) if p["kind"] == kind]
        if not idx:
            continue
        pics, cus, levels, _ = pkg.parse_multitool([streams[k] for k in idx], kind, sparse=sparse, threads=2)
        ncu = (w // 32) * (h // 32)
        for j, k in enumerate(idx):
            want, got = st[k]["cus"], cus[j * ncu:(j + 1) * ncu]
            fields = ("luma_mode", "chroma_mode", "cbf", "tu_tools") if kind == "I" else (
                "mv", "ref_idx", "inter_dir", "bcw_idx", "flags", "cbf", "tu_tools", "mvd", "mvp_idx")
            for f in fields:
                assert (got[f] == want[f]).all(), (k, f)
            if sparse:
                continue
            for r0, r1 in zip(want, got):
                for c, n in ((0, 1024), (1, 256), (2, 256)):
                    if r0["level_off"][c] >= 0:
                        a = st[k]["levels"][r0["level_off"][c]:][:n]
                        b = levels[r1["level_off"][c]:][:n]
                        if _hides_signs(opts):
                            a, b = np.abs(a), np.abs(b)
                        assert (a == b).all(), (k, c)


def _closed_loop(orc, st, w, h, qp, opts):
    """The oracle's decoders reproduce each picture's encoder reconstruction
    (not with hidden signs, see _hides_signs)."""
    if _hides_signs(opts):
        return
    prev = None
    for p in st:
        if p["kind"] == "I":
            dec = orc.mt_decode(p["cus"], p["levels"], w, h, qp, opts)
        else:
            moved = orc.inter_resolve_motion(p["cus"], w, h)
            assert (moved["mv"] == p["cus"]["mv"]).all() and (moved["ref_idx"] == p["cus"]["ref_idx"]).all()
            dec = orc.inter_decode(p["cus"], p["levels"], w, h, qp, [prev], opts)
        assert all((a == b).all() for a, b in zip(dec, p["recon"]))
        prev = p["recon"]


def test_mpm_list_matches_the_reference_cases(orc):
    """predict.rs:4327-4367 MPM cases (VTM PU::getIntraMPMs)."""
    assert list(orc.derive_intra_mpms()) == [0, 1, 50, 18, 46, 54]
    assert list(orc.derive_intra_mpms(30)) == [0, 30, 29, 31, 28, 32]
    assert list(orc.derive_intra_mpms(30, 30)) == [0, 30, 29, 31, 28, 32]
    assert list(orc.derive_intra_mpms(30, 31)) == [0, 30, 31, 29, 32, 28]
    assert list(orc.derive_intra_mpms(2, 66)) == [0, 2, 66, 3, 65, 4]
    assert list(orc.derive_intra_mpms(20, 40)) == [0, 20, 40, 19, 21, 39]


@pytest.mark.parametrize("opts", [0, 1, 2, 4 | 1])
def test_small_picture_sequence_ip_p(pkg, orc, opts):
    from rustmpeg_next_b200 import synth

    frames = [synth.config1_frame(f) for f in range(3)]
    st = orc.multitool_stream(frames, 26, keyint=3, opts=opts)
    assert [p["kind"] for p in st] == ["I", "P", "P"]
    _closed_loop(orc, st, 64, 64, 26, opts)
    _check_parse(pkg, orc, st, 64, 64, 26, opts)
    _check_parse(pkg, orc, st, 64, 64, 26, opts, sparse=True)


@pytest.mark.parametrize("w,h,qp,dq", [(64, 64, 4, False), (64, 64, 4, True), (64, 64, 10, False),
                                       (64, 64, 10, True), (200, 120, 40, False), (200, 120, 40, True)])
def test_inter_p_slice_conformance_cases(pkg, orc, w, h, qp, dq):
    opts = (1 if dq else 2) | 4 | 8  # DQ or sign hiding, deblocking, full intra modes
    frames = [_coded(_gradient(w, h, idx * 11), w, h) for idx in range(3)]
    cw, ch = frames[0][0].shape[1], frames[0][0].shape[0]
    st = orc.multitool_stream(frames, qp, keyint=4, opts=opts)
    _closed_loop(orc, st, cw, ch, qp, opts)
    _check_parse(pkg, orc, st, cw, ch, qp, opts)
    if qp == 4 and not dq:  # transform skip on the IDR picture: lossless luma there
        assert (st[0]["recon"][0] == frames[0][0]).all()


def test_gop_sequence_with_a_brighter_p_picture(pkg, orc):
    """mod.rs:4103-4146: an IDR picture and a P picture whose luma is 2 brighter, QP 24."""
    f0 = _gradient(64, 64)
    f1 = (np.minimum(f0[0].astype(int) + 2, 255).astype(np.uint8), f0[1], f0[2])
    opts = 1 | 4 | 8
    st = orc.multitool_stream([f0, f1], 24, keyint=4, opts=opts)
    assert [p["kind"] for p in st] == ["I", "P"]
    _closed_loop(orc, st, 64, 64, 24, opts)
    _check_parse(pkg, orc, st, 64, 64, 24, opts)


def _amvp_records(orc, rng, w, h, base, n_levels):
    """P records mixing skip, merge and AMVP coding units (mvp_idx, mvd) on
    top of an encoder picture's residuals; motion derived by the oracle."""
    cus = base.copy()
    for k in range(len(cus)):
        r = rng.random()
        if r < 0.45:
            cus[k]["flags"] = 0  # AMVP
            cus[k]["mvp_idx"] = rng.integers(0, 2)
            cus[k]["mvd"] = rng.integers(-300, 301, 2) * (rng.random() < 0.8)
        else:
            cus[k]["flags"] = orc.INTER_CU_MERGE
            cus[k]["mvp_idx"] = 0
            cus[k]["mvd"] = 0
            if cus[k]["cbf"] == 0:
                cus[k]["flags"] |= orc.INTER_CU_SKIP
    return orc.inter_resolve_motion(cus, w, h)


def test_amvp_coding_units_parse_to_the_derived_motion(pkg, orc):
    from rustmpeg_next_b200 import synth

    rng = np.random.default_rng(11)
    w, h = 160, 96
    src = [synth.pad_to(a, s[0], s[1]) for a, s in zip(synth.config1_frame(1), ((w, h), (w // 2, h // 2), (w // 2, h // 2)))]
    ref = [synth.pad_to(a, s[0], s[1]) for a, s in zip(synth.config1_frame(0), ((w, h), (w // 2, h // 2), (w // 2, h // 2)))]
    base, levels, _ = orc.inter_encode(*src, 30, [ref])
    for rep in range(4):
        cus = _amvp_records(orc, rng, w, h, base, len(levels))
        assert (cus["flags"] & orc.INTER_CU_MERGE == 0).any()
        data = orc.p_write(cus, levels, w, h, 30)
        _, got, glv, _ = pkg.parse_multitool([("P", data, w, h, 30, 0)], "P")
        for f in ("mv", "ref_idx", "inter_dir", "flags", "mvd", "mvp_idx", "cbf", "tu_tools"):
            assert (got[f] == cus[f]).all(), (rep, f)
        # and the oracle reconstructs the same picture from either record set
        a = orc.inter_decode(cus, levels, w, h, 30, [ref])
        b = orc.inter_decode(got, glv, w, h, 30, [ref])
        assert all((x == y).all() for x, y in zip(a, b))


def test_transform_skip_residuals_in_p_pictures_parse(pkg, orc):
    """decode_inter_picture reads transform_skip_flag per coded TB
    (slice.rs:3727-3775) though the reference's encoder writes 0."""
    from rustmpeg_next_b200 import synth

    y, u, v = synth.config1_frame(2)
    ref = synth.config1_frame(1)
    cus, levels, _ = orc.inter_encode(y, u, v, 30, [ref])
    rng = np.random.default_rng(3)
    lv = levels.copy()
    for k in range(len(cus)):
        for c, n in ((0, 1024), (1, 256), (2, 256)):
            o = cus[k]["level_off"][c]
            if o >= 0 and rng.random() < 0.5:
                cus[k]["tu_tools"] |= 1 << c
                lv[o:o + n] = np.clip(lv[o:o + n], -200, 200)
    data = orc.p_write(cus, lv, 64, 64, 30)
    _, got, glv, _ = pkg.parse_multitool([("P", data, 64, 64, 30, 0)], "P")
    assert (got["tu_tools"] == cus["tu_tools"]).all()
    a = orc.inter_decode(cus, lv, 64, 64, 30, [ref])
    b = orc.inter_decode(got, glv, 64, 64, 30, [ref])
    assert all((x == y).all() for x, y in zip(a, b))


def test_intra_coding_unit_in_a_p_picture_is_rejected(pkg, orc):
    """decode_inter_picture returns Unsupported("intra CU inside inter fast
    slice") for pred_mode_flag 1 (slice.rs:3640-3642): a substream whose first
    coding unit is not skipped and carries pred_mode_flag 1 fails the parse."""
    from rustmpeg_next_b200 import synth

    y, u, v = synth.config1_frame(1)
    cus, levels, _ = orc.inter_encode(y, u, v, 30, [synth.config1_frame(0)])
    pkg.parse_multitool([("P", orc.p_write(cus, levels, 64, 64, 30), 64, 64, 30, 0)], "P")
    for k in (0, 2):
        bad = cus.copy()
        bad[k]["flags"] |= 0x80  # the oracle writer's intra coding unit
        with pytest.raises(pkg.InvalidInput, match="intra coding unit"):
            pkg.parse_multitool([("P", orc.p_write(bad, levels, 64, 64, 30), 64, 64, 30, 0)], "P")


def test_unsupported_options_and_ctu_sizes_are_rejected(pkg, orc):
    from rustmpeg_next_b200 import synth

    st = orc.multitool_stream([synth.config1_frame(0)], 26)
    with pytest.raises(pkg.InvalidInput):
        pkg.parse_multitool([("I", st[0]["data"], 64, 64, 26, 16)], "I")  # an option outside VVCG_SLICE_*
    with pytest.raises(pkg.InvalidInput):
        pkg.parse_multitool([("I", st[0]["data"], 64, 48, 26, 0)], "I")  # not a multiple of 32


def _fixture_pictures(name):
    import os

    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "multitool_streams.npz"))
    data, offs = z[f"{name}_data"], z[f"{name}_offsets"]
    w, h = (int(x) for x in z[f"{name}_size"])
    pics = [(str(z[f"{name}_kind"][i]), data[offs[i]:offs[i + 1]].tobytes(), w, h, int(z[f"{name}_qp"][i]), 0)
            for i in range(len(offs) - 1)]
    return pics, [int(x) for x in z[f"{name}_stream"]], [str(x) for x in z[f"{name}_sha256"]]


def _sha(planes):
    import hashlib

    hh = hashlib.sha256()
    for p in planes:
        hh.update(np.ascontiguousarray(p, dtype=np.uint8).tobytes())
    return hh.hexdigest()


@pytest.mark.parametrize("name", ["small", "hd"])
def test_committed_streams_parse_and_decode_to_their_hashes(pkg, orc, name):
    """tests/golden/multitool_streams.npz: the parser's records, decoded by
    the oracle picture after picture (each P picture from the previous
    picture of its stream), give the committed reconstruction hashes."""
    pics, sid, hashes = _fixture_pictures(name)
    prev = {}
    for i, (kind, data, w, h, qp, opts) in enumerate(pics):
        _, cus, levels, _ = pkg.parse_multitool([(kind, data, w, h, qp, opts)], kind, threads=1)
        if kind == "I":
            dec = orc.mt_decode(cus, levels, w, h, qp, opts)
        else:
            dec = orc.inter_decode(cus, levels, w, h, qp, [prev[sid[i]]], opts)
        assert _sha(dec) == hashes[i], i
        prev[sid[i]] = dec
