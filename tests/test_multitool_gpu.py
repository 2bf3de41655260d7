"""GPU parity: the multi-tool stream (VvcMultiToolEncoder: IDR + P pictures)
from slice data to pixels on the GPU, bit-exact against the oracle's
restatement of the reference decoder (decode_picture_multitool,
slice.rs:3012; decode_inter_picture, slice.rs:3552) fed the same parsed
records, and against the encoder's reconstruction where the two agree:

- the small-picture configuration's sequence: 64x64 8-bit, an IDR picture
  and two P pictures at QP 26 (ramp + noise + a moving square), default
  options and with dependent quantisation, sign hiding, deblocking and the
  67-mode intra search;
- the reference's conformance cases (mod.rs:4150-4197) and GOP sequence
  (mod.rs:4103-4146) with this library's options;
- P records with AMVP motion (fractional, far outside the picture), sparse
  levels, transform-skip residuals and several references, through
  vvcg_decode_p_batch directly, one and many pictures per call;
- malformed records rejected without disturbing the context.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle_decode(orc, pkg, streams, sparse=False):
    """The oracle's decoder over the library's parsed records (the reference
    decoder's view of the slice data), picture by picture."""
    from rustmpeg_next_b200 import synth

    out, prev = [], None
    for kind, data, w, h, qp, opts in streams:
        _, cus, levels, _ = pkg.parse_multitool([(kind, data, w, h, qp, opts)], kind)
        if kind == "I":
            dec = orc.mt_decode(cus, levels, w, h, qp, opts)
        else:
            dec = orc.inter_decode(cus, levels, w, h, qp, [prev], opts)
        out.append(dec)
        prev = dec
    return out


def _assert_same(got, want, what):
    for c in range(3):
        d = np.argwhere(got[c].astype(np.int32) != want[c].astype(np.int32))
        assert d.size == 0, f"{what} plane {c}: {len(d)} samples differ, first {d[:3].tolist()}"


def _run_stream(ctx, pkg, orc, frames, qp, opts, keyint=3, sparse=False):
    st = orc.multitool_stream(frames, qp, keyint=keyint, opts=opts)
    h, w = frames[0][0].shape
    streams = [(p["kind"], p["data"], w, h, qp, opts) for p in st]
    got = ctx.decode_multitool_stream(streams, sparse=sparse, threads=2)
    want = _oracle_decode(orc, pkg, streams)
    for k, (g, o) in enumerate(zip(got, want)):
        _assert_same(g, o, f"picture {k} ({st[k]['kind']})")
    hides = (opts & 2) and not (opts & 1)
    if not hides:  # the decoder reproduces the encoder's reconstruction
        for k, (g, p) in enumerate(zip(got, st)):
            _assert_same(g, p["recon"], f"picture {k} against the encoder")
    return st, got


@pytest.mark.parametrize("opts", [0, 1, 2, 1 | 4, 4 | 8])
@pytest.mark.parametrize("sparse", [False, True])
def test_small_picture_sequence_i_p_p(ctx, pkg, orc, opts, sparse):
    from rustmpeg_next_b200 import synth

    frames = [synth.config1_frame(f) for f in range(3)]
    st, _ = _run_stream(ctx, pkg, orc, frames, 26, opts, sparse=sparse)
    assert [p["kind"] for p in st] == ["I", "P", "P"]


def _gradient(w, h, shift=0):
    j, i = np.mgrid[0:h, 0:w]
    y = ((((i * 3 + j * 5) % 251) + shift) % 256).astype(np.uint8)
    return y, np.full((h // 2, w // 2), 90, np.uint8), np.full((h // 2, w // 2), 160, np.uint8)


@pytest.mark.parametrize("w,h,qp,dq", [(64, 64, 4, False), (64, 64, 4, True), (64, 64, 10, False),
                                       (64, 64, 10, True), (224, 128, 40, False), (224, 128, 40, True)])
def test_conformance_cases(ctx, pkg, orc, w, h, qp, dq):
    opts = (1 if dq else 2) | 4 | 8
    frames = [_gradient(w, h, idx * 11) for idx in range(3)]
    _run_stream(ctx, pkg, orc, frames, qp, opts, keyint=4)


def test_gop_with_two_idr_pictures(ctx, pkg, orc):
    """keyint 2: I P I P, each P predicting from the picture before it."""
    from rustmpeg_next_b200 import synth

    frames = [synth.config1_frame(f % 3) for f in range(4)]
    st, _ = _run_stream(ctx, pkg, orc, frames, 30, 1 | 4, keyint=2)
    assert [p["kind"] for p in st] == ["I", "P", "I", "P"]


def _planes(frame, w, h):
    from rustmpeg_next_b200 import synth

    return tuple(synth.pad_to(a, s[0], s[1]) for a, s in zip(frame, ((w, h), (w // 2, h // 2), (w // 2, h // 2))))


def _random_motion(orc, rng, base, w, h, far=False):
    """AMVP / merge / skip records on an encoded picture's residuals, with
    fractional motion vector differences (far ones reach outside the picture)."""
    cus = base.copy()
    for k in range(len(cus)):
        if rng.random() < 0.6:
            cus[k]["flags"] = 0
            cus[k]["mvp_idx"] = rng.integers(0, 2)
            span = 6000 if far else 200
            cus[k]["mvd"] = rng.integers(-span, span + 1, 2)
        else:
            cus[k]["flags"] = orc.INTER_CU_MERGE | (orc.INTER_CU_SKIP if cus[k]["cbf"] == 0 else 0)
            cus[k]["mvd"] = 0
            cus[k]["mvp_idx"] = 0
    return orc.inter_resolve_motion(cus, w, h)


@pytest.mark.parametrize("far", [False, True])
def test_p_pictures_with_amvp_motion(ctx, pkg, orc, far):
    from rustmpeg_next_b200 import synth

    rng = np.random.default_rng(5 + far)
    w, h = 192, 128
    refs = [_planes(synth.config1_frame(f), w, h) for f in range(3)]
    src = _planes(synth.config1_frame(2), w, h)
    base, levels, _ = orc.inter_encode(*src, 28, refs[:1])
    ctx.dpb_reserve(4, w, h)
    for s, r in enumerate(refs):
        ctx.dpb_upload(s, r)
    for rep in range(3):
        cus = _random_motion(orc, rng, base, w, h, far)
        cus["ref_idx"][:, 0] = np.where(cus["ref_idx"][:, 0] >= 0, rng.integers(0, 3, len(cus)), -1)
        assert (np.abs(cus["mv"][:, 0]) % 16 != 0).any()
        pic = np.zeros(1, pkg.P_PIC_DTYPE)
        pic["width"], pic["height"], pic["qp"], pic["num_refs"], pic["out_slot"] = w, h, 28, 3, 3
        pic[0]["ref_slot"][:3] = [0, 1, 2]
        ctx.decode_p_batch(pic, cus, levels)
        want = orc.inter_decode(cus, levels, w, h, 28, refs)
        _assert_same(ctx.dpb_download(3), want, f"repetition {rep}")


def test_p_pictures_sparse_levels_and_transform_skip(ctx, pkg, orc):
    from rustmpeg_next_b200 import synth

    w, h = 128, 96
    ref = _planes(synth.config1_frame(0), w, h)
    cus, levels, _ = orc.inter_encode(*_planes(synth.config1_frame(1), w, h), 24, [ref])
    rng = np.random.default_rng(9)
    lv = levels.copy()
    for k in range(len(cus)):
        for c, n in ((0, 1024), (1, 256), (2, 256)):
            o = cus[k]["level_off"][c]
            if o >= 0 and rng.random() < 0.4:
                cus[k]["tu_tools"] |= 1 << c
                lv[o:o + n] = np.clip(lv[o:o + n], -300, 300)
    streams = [("P", orc.p_write(cus, lv, w, h, 24), w, h, 24, 0)]
    want = orc.inter_decode(cus, lv, w, h, 24, [ref])
    for sparse in (False, True):
        pics, pc, pl, _ = pkg.parse_multitool(streams, "P", sparse=sparse)
        ctx.dpb_reserve(2, w, h)
        ctx.dpb_upload(0, ref)
        pics[0]["ref_slot"][0], pics[0]["out_slot"] = 0, 1
        ctx.decode_p_batch(pics, pc, pl)
        _assert_same(ctx.dpb_download(1), want, f"sparse={sparse}")


def test_many_streams_in_one_call(ctx, pkg, orc):
    """Six independent 2-picture P chains in one vvcg_decode_p_batch call:
    the first pictures of every chain run in one launch, the second ones in
    the next."""
    from rustmpeg_next_b200 import synth

    w, h = 96, 64
    n = 6
    ctx.dpb_reserve(3 * n, w, h)
    pics, all_cus, all_lv, wants = [], [], [], []
    for s in range(n):
        frames = [_planes(synth.config1_frame((s + f) % 3), w, h) for f in range(3)]
        st = orc.multitool_stream(frames, 22 + 3 * s, keyint=3, opts=(s % 2))
        ctx.dpb_upload(3 * s, st[0]["recon"])
        for k in (1, 2):
            p = np.zeros((), pkg.P_PIC_DTYPE)
            p["width"], p["height"], p["qp"], p["num_refs"] = w, h, 22 + 3 * s, 1
            p["options"] = s % 2
            p["ref_slot"][0], p["out_slot"] = 3 * s + k - 1, 3 * s + k
            p["cu_offset"] = sum(len(c) for c in all_cus)
            cus = st[k]["cus"].copy()
            lo = cus["level_off"]
            cus["level_off"] = np.where(lo >= 0, lo + sum(len(x) for x in all_lv), -1)
            pics.append(p)
            all_cus.append(cus)
            all_lv.append(st[k]["levels"])
            wants.append((3 * s + k, st[k]["recon"]))
    order = [i for k in (0, 1) for i in range(k, len(pics), 2)]  # the first P of every chain first
    ctx.decode_p_batch(np.array([pics[i] for i in order]), np.concatenate(all_cus), np.concatenate(all_lv))
    for slot, want in wants:
        _assert_same(ctx.dpb_download(slot), want, f"slot {slot}")


def test_bad_p_records_are_rejected(ctx, pkg, orc):
    from rustmpeg_next_b200 import synth

    ref = synth.config1_frame(0)
    cus, levels, rec = orc.inter_encode(*synth.config1_frame(1), 26, [ref])
    ctx.dpb_reserve(2, 64, 64)
    ctx.dpb_upload(0, ref)
    pic = np.zeros(1, pkg.P_PIC_DTYPE)
    pic["width"], pic["height"], pic["qp"], pic["num_refs"], pic["out_slot"] = 64, 64, 26, 1, 1
    coded = np.flatnonzero(cus["cbf"] & 1)
    assert coded.size
    for mutate in ("off", "tools", "slot"):
        bad, p = cus.copy(), pic.copy()
        if mutate == "off":
            bad[coded[0]]["level_off"][0] = len(levels) - 10
        elif mutate == "tools":
            bad[0]["tu_tools"] = 8
        else:
            p[0]["out_slot"] = 0  # its own reference
        with pytest.raises(pkg.InvalidInput):
            ctx.decode_p_batch(p, bad, levels)
    ctx.decode_p_batch(pic, cus, levels)  # the context still works
    _assert_same(ctx.dpb_download(1), rec, "after rejections")


def test_picture_buffer_round_trip_and_store(ctx, pkg, orc):
    from rustmpeg_next_b200 import synth

    y, u, v = synth.config1_frame(1)
    ctx.dpb_reserve(2, 64, 64)
    ctx.dpb_upload(1, (y, u, v))
    _assert_same(ctx.dpb_download(1), (y, u, v), "upload / download")
    cus, levels, rec = orc.strict_encode(y, u, v, 30)
    batch = pkg.Batch(np.array([synth.strict_picture(64, 64, 30)]), cus, levels, np.zeros(4, pkg.CTU_DTYPE))
    ctx.decode_batch(batch)
    ctx.dpb_store(0, 0)
    _assert_same(ctx.dpb_download(0), rec, "frame-path picture stored")


@pytest.mark.parametrize("name", ["small", "hd"])
@pytest.mark.parametrize("sparse", [False, True])
def test_committed_streams_decode_to_their_hashes(ctx, pkg, name, sparse):
    """tests/golden/multitool_streams.npz (the small-picture I P P sequence;
    four 1920x1088 I P P P streams at QP 22..37) from slice data to pixels in
    one call: every picture's SHA-256 equals the committed reconstruction's."""
    from test_multitool_cpu import _fixture_pictures, _sha

    pics, sid, hashes = _fixture_pictures(name)
    got = ctx.decode_multitool_stream(pics, sparse=sparse, threads=4, stream_ids=sid)
    for i, g in enumerate(got):
        assert _sha(g) == hashes[i], i
