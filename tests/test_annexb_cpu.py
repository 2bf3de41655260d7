"""CPU: Annex-B access units of the default stream (vvcg_hls_rbsp,
vvcg_annexb_idr, vvcg_annexb_read_idr).

Pinned on the reference's own byte vectors: the profile_tier_level of level
16 with 64x64 CTUs (hls.rs:5482-5489 ptl_matches_the_vtm_validated_reference,
here the bytes after the VPS's first three), the AUD, picture header and
slice header bytes (hls.rs:5492-5496), the VPS and SPS prefixes of the
128x128 test configuration (hls.rs:5499-5510, configuration at :5435-5447)
and the emulation-prevention round trip (bits.rs:334-338). Then the round
trip of strict-profile slice data written by the oracle's encoder side
through an access unit and back, at picture sizes that need a conformance
window, and the rejections.
"""
import numpy as np
import pytest

# hls.rs:5484-5486
PTL_LEVEL16_CTU64 = bytes([0x02, 0x10, 0xBA, 0x2F, 0xB6, 0x9B, 0xFF, 0xFF, 0xFF, 0x4F, 0xFF, 0xC0, 0x00, 0x00])
REF_CFG = dict(width=128, height=128, qp=26, level_idc=16, ctu_log2=6, min_cb_log2=3, ts_log2=3)


def test_parameter_sets_match_the_reference_vectors(pkg):
    vps = pkg.hls_rbsp(pkg.HLS_VPS, **REF_CFG)
    assert vps[:3] == bytes([0x10, 0x00, 0x00])
    assert vps[3:17] == PTL_LEVEL16_CTU64
    sps = pkg.hls_rbsp(pkg.HLS_SPS, **REF_CFG)
    assert sps[:3] == bytes([0x01, 0x0B, 0x02])
    assert sps[2:16] == PTL_LEVEL16_CTU64  # after the SPS's first 16 bits (ids, chroma format, CTU size, ...)
    assert pkg.hls_rbsp(pkg.HLS_AUD, **REF_CFG) == bytes([0x88])
    assert pkg.hls_rbsp(pkg.HLS_PH, **REF_CFG, arg=0) == bytes([0x88, 0x04])
    assert pkg.hls_rbsp(pkg.HLS_SLICE_HEADER, **REF_CFG, arg=0) == bytes([0x28])


def _ue(bits, pos):
    z = 0
    while bits[pos + z] == "0":
        z += 1
    return int(bits[pos + z:pos + 2 * z + 1], 2) - 1, pos + 2 * z + 1


def test_sps_parses_as_the_reference_reads_it(pkg):
    """What the reference's own test reads back from its SPS
    (hls.rs:5504-5508: 128x128, level 16, profile 1): profile and level in
    the PTL, then after sps_gdr_enabled_flag and
    sps_ref_pic_resampling_enabled_flag the two sizes as ue(v)."""
    sps = pkg.hls_rbsp(pkg.HLS_SPS, **REF_CFG)
    bits = "".join(f"{b:08b}" for b in sps)
    assert int(bits[16:23], 2) == 1 and int(bits[24:32], 2) == 16  # general_profile_idc, general_level_idc
    w, pos = _ue(bits, 16 + 14 * 8 + 2)
    h, pos = _ue(bits, pos)
    assert (w, h) == (128, 128)
    assert bits[pos] == "0"  # no conformance window


def test_sps_carries_the_size_and_the_conformance_window(pkg):
    a = pkg.hls_rbsp(pkg.HLS_SPS, **REF_CFG)
    b = pkg.hls_rbsp(pkg.HLS_SPS, **dict(REF_CFG, crop_right=8, crop_bottom=4))
    assert len(b) > len(a) and a[:17] == b[:17]
    c = pkg.hls_rbsp(pkg.HLS_SPS, **dict(REF_CFG, ctu_log2=5))
    assert c != a  # sps_log2_ctu_size_minus5 and the PTL's CTU constraint
    with pytest.raises(pkg.InvalidInput):
        pkg.hls_rbsp(pkg.HLS_SPS, **dict(REF_CFG, ctu_log2=4))
    with pytest.raises(pkg.InvalidInput):
        pkg.hls_rbsp(pkg.HLS_SPS, **dict(REF_CFG, crop_right=3))
    with pytest.raises(pkg.InvalidInput):
        pkg.hls_rbsp(9, **REF_CFG)


def _nals(au):
    """Split at 4-byte start codes; (type, payload)."""
    parts = au.split(b"\x00\x00\x00\x01")
    assert parts[0] == b""
    return [((p[1] >> 3), p[2:]) for p in parts[1:]]


def test_access_unit_layout_and_emulation_prevention(pkg):
    # slice data full of start-code emulations (bits.rs:335 and more)
    data = bytes([0, 0, 0, 1, 0, 0, 2, 0, 0, 3, 9, 0, 0, 0, 0, 0, 1, 0xFF, 0, 0])
    au = pkg.annexb_idr(data + b"\x80", 64, 64, 26)
    nals = _nals(au)
    assert [t for t, _ in nals] == [20, 14, 15, 16, 19, 8]  # AUD VPS SPS PPS PH IDR_N_LP
    for _, payload in nals:  # no 00 00 0x (x <= 3) left unescaped inside a NAL unit
        for i in range(len(payload) - 2):
            if payload[i] == 0 and payload[i + 1] == 0:
                assert payload[i + 2] == 3 or payload[i + 2] > 3
    got, w, h, qp = pkg.annexb_read_idr(au)
    assert got == data + b"\x80" and (w, h, qp) == (64, 64, 26)
    # two access units back to back, 3-byte start code and leading zeros: the first IDR slice
    au2 = b"\x00\x00" + au + pkg.annexb_idr(b"\x12\x34", 64, 64, 30).replace(b"\x00\x00\x00\x01", b"\x00\x00\x01", 1)
    assert pkg.annexb_read_idr(au2)[0] == data + b"\x80"


def test_encoder_slice_data_round_trips(pkg, orc):
    from rustmpeg_next_b200 import synth

    for k, (w, h, qp) in enumerate([(64, 64, 26), (120, 60, 32), (1920, 1080, 22)]):
        cw, ch = (w + 31) // 32 * 32, (h + 31) // 32 * 32
        if w == 1920:  # a smaller picture's slice data: only the headers depend on the size here
            y, u, v = synth.config1_frame(k % 3)
            cw, ch = 64, 64
        else:
            y, u, v = (synth.config1_frame(k % 3) if (cw, ch) == (64, 64) else
                       (np.random.default_rng(k).integers(0, 256, (ch, cw), dtype=np.uint8),
                        np.random.default_rng(k + 1).integers(0, 256, (ch // 2, cw // 2), dtype=np.uint8),
                        np.random.default_rng(k + 2).integers(0, 256, (ch // 2, cw // 2), dtype=np.uint8)))
        cus, levels, _ = orc.strict_encode(y, u, v, qp)
        data = orc.strict_write(cus, levels, cw, ch, qp)
        au = pkg.annexb_idr(data, w, h, qp)
        got, gw, gh, gqp = pkg.annexb_read_idr(au)
        assert got == data
        assert (gw, gh, gqp) == ((w + 31) // 32 * 32, (h + 31) // 32 * 32, qp)
        sps = dict(_nals(au))[15]
        level = sps[3]  # general_level_idc: the byte after profile_idc and tier (no emulation this early)
        assert level == (64 if w == 1920 else 16)


def test_read_rejects_streams_outside_the_layout(pkg):
    au = pkg.annexb_idr(b"\x55\xAA", 64, 64, 26)
    nals = au.split(b"\x00\x00\x00\x01")[1:]
    no_pps = b"".join(b"\x00\x00\x00\x01" + n for n in nals if (n[1] >> 3) != 16)
    with pytest.raises(pkg.InvalidInput):
        pkg.annexb_read_idr(no_pps)
    no_slice = b"".join(b"\x00\x00\x00\x01" + n for n in nals if (n[1] >> 3) != 8)
    with pytest.raises(pkg.InvalidInput):
        pkg.annexb_read_idr(no_slice)
    with pytest.raises(pkg.InvalidInput):
        pkg.annexb_read_idr(b"")
    # a slice header whose byte_alignment() is broken: the stop bit cleared
    bad = au[:-3] + bytes([au[-3] & 0xF7]) + au[-2:]
    with pytest.raises(pkg.InvalidInput):
        pkg.annexb_read_idr(bad)
