"""GPU parity: libvvcg's reconstruction and loop filters against the oracle.

Every comparison is bit-exact (integer sample work). Inputs are (a) records
produced by the oracle's restatement of the reference encoder
(slice::encode_vvc_frame_picture), the closed loop the reference's own
round-trip tests use, and (b) seeded synthetic records with random modes,
sparse levels, SAO parameters and ALF switches, in batches of pictures with
different sizes, bit depths, chroma formats and CTU sizes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def oracle_outputs(orc, pics, cus, levels, ctus, aps):
    outs = []
    for p in pics:
        tb = min(1 << int(p["ctu_log2"]), 32)
        n = (int(p["width"]) // tb) * (int(p["height"]) // tb)
        nc = (int(p["width"]) >> int(p["ctu_log2"])) * (int(p["height"]) >> int(p["ctu_log2"]))
        a = None if aps is None or int(p["alf_aps"]) < 0 else aps[int(p["alf_aps"])]
        rc, planes = orc.recon_frame(p, cus[int(p["cu_offset"]):][:n], levels,
                                     ctus[int(p["ctu_offset"]):][:nc], a)
        vw, vh, cf = int(p["visible_width"]), int(p["visible_height"]), int(p["chroma_format"])
        cw, ch = orc.chroma_dims(vw, vh, cf)
        outs.append((rc, planes[0][:vh, :vw], planes[1][:ch, :cw] if cf else None,
                     planes[2][:ch, :cw] if cf else None))
    return outs


def assert_same(gpu_outs, orc_outs):
    for i, (g, o) in enumerate(zip(gpu_outs, orc_outs)):
        assert o[0] == 0
        for c in range(3):
            if o[c + 1] is None:
                continue
            diff = np.argwhere(g[c] != o[c + 1])
            assert diff.size == 0, f"picture {i} plane {c}: {len(diff)} samples differ, first {diff[:3].tolist()}"


def encoded_picture(orc, pkg, w, h, bd, qp, ctu_log2, opts, cf=1, seed=0, vis=None):
    from rustmpeg_next_b200 import synth

    vw, vh = vis or (w, h)
    y, u, v = synth.value_noise_frame(vw, vh, 10, frame=seed)
    if bd != 10:
        y = (y.astype(np.int32) << bd >> 10).astype(np.uint16) if bd > 10 else (y >> (10 - bd)).astype(np.uint16)
        u = (u.astype(np.int32) << bd >> 10).astype(np.uint16) if bd > 10 else (u >> (10 - bd)).astype(np.uint16)
        v = (v.astype(np.int32) << bd >> 10).astype(np.uint16) if bd > 10 else (v >> (10 - bd)).astype(np.uint16)
    cw, ch = orc.chroma_dims(w, h, cf)
    if cf == 3:
        u = np.kron(u, np.ones((2, 2), np.uint16))[:vh, :vw]
        v = np.kron(v, np.ones((2, 2), np.uint16))[:vh, :vw]
    elif cf == 2:
        u = np.repeat(u, 2, axis=0)[:vh]
        v = np.repeat(v, 2, axis=0)[:vh]
    y = synth.pad_to(y, w, h)
    u = synth.pad_to(u, cw, ch)
    v = synth.pad_to(v, cw, ch)
    cus, levels, _ = orc.encode_frame(y, u, v, bd, qp, ctu_log2, opts, cf=cf)
    p = np.zeros((), pkg.PIC_DTYPE)
    p["width"], p["height"] = w, h
    p["visible_width"], p["visible_height"] = vw, vh
    p["bit_depth"], p["chroma_format"], p["ctu_log2"] = bd, cf, ctu_log2
    p["slice_qp"], p["chroma_qp_scaled"] = qp, orc.chroma_qp(qp, bd)
    p["tools"] = (pkg.TOOL_DEP_QUANT if opts & orc.OPT_DEP_QUANT else 0) | \
                 (pkg.TOOL_DEBLOCK if opts & orc.OPT_DEBLOCK else 0)
    p["alf_aps"] = -1
    return p, cus, levels


@pytest.mark.parametrize("bd,qp,ctu_log2,opts,cf", [
    (10, 22, 5, 1 | 2 | 8, 1),
    (10, 37, 5, 1 | 2 | 8, 1),
    (10, 27, 5, 1 | 2 | 4 | 8, 1),
    (8, 32, 6, 1 | 2 | 8, 1),
    (12, 30, 7, 1 | 8, 1),
    (10, 27, 5, 1 | 8, 2),
    (10, 27, 6, 1 | 2 | 8, 3),
    (10, 45, 5, 0, 1),
])
def test_recon_matches_oracle_on_encoder_records(ctx, pkg, orc, bd, qp, ctu_log2, opts, cf):
    ctu = 1 << ctu_log2
    vis = (200, 120)
    w = -(-vis[0] // ctu) * ctu
    h = -(-vis[1] // ctu) * ctu
    p, cus, levels = encoded_picture(orc, pkg, w, h, bd, qp, ctu_log2, opts, cf=cf, seed=qp, vis=vis)
    ctus = np.zeros((h // ctu) * (w // ctu), pkg.CTU_DTYPE)
    batch = pkg.Batch(np.array([p]), cus, levels, ctus)
    gpu = ctx.decode_batch(batch)
    assert_same(gpu, oracle_outputs(orc, batch.pics, cus, levels, ctus, None))


def test_mixed_batch_of_encoded_pictures(ctx, pkg, orc):
    parts = [encoded_picture(orc, pkg, 128, 64, 10, 27, 5, 1 | 2 | 8, seed=1),
             encoded_picture(orc, pkg, 64, 128, 8, 33, 6, 1 | 4 | 8, seed=2),
             encoded_picture(orc, pkg, 96, 64, 10, 22, 5, 1 | 2, seed=3)]
    pics, cus, levels = [], [], []
    ncu = nlev = 0
    for p, c, l in parts:
        p = p.copy()
        p["cu_offset"] = ncu
        c = c.copy()
        c["level_off"] = np.where(c["level_off"] >= 0, c["level_off"] + nlev, -1)
        pics.append(p)
        cus.append(c)
        levels.append(l)
        ncu += len(c)
        nlev += len(l)
    pics = np.array(pics)
    cus = np.concatenate(cus)
    levels = np.concatenate(levels)
    ctus = np.zeros(64, pkg.CTU_DTYPE)
    batch = pkg.Batch(pics, cus, levels, ctus)
    gpu = ctx.decode_batch(batch)
    assert_same(gpu, oracle_outputs(orc, pics, cus, levels, ctus, None))


SPECS = [
    dict(width=256, height=128, visible_width=250, visible_height=120, bit_depth=10, chroma_format=1, ctu_log2=5, qp=22),
    dict(width=128, height=128, bit_depth=8, chroma_format=1, ctu_log2=6, qp=30),
    dict(width=256, height=256, bit_depth=12, chroma_format=1, ctu_log2=7, qp=37),
    dict(width=96, height=64, bit_depth=10, chroma_format=2, ctu_log2=5, qp=27),
    dict(width=64, height=96, bit_depth=10, chroma_format=3, ctu_log2=5, qp=32),
    dict(width=64, height=64, bit_depth=10, chroma_format=0, ctu_log2=5, qp=25),
]


@pytest.mark.parametrize("tools_name", ["recon", "deblock", "deblock_sao", "dq_deblock_sao_alf"])
def test_synthetic_batch_matches_oracle(ctx, pkg, orc, tools_name):
    from rustmpeg_next_b200 import synth

    tools = {"recon": 0, "deblock": pkg.TOOL_DEBLOCK, "deblock_sao": pkg.TOOL_DEBLOCK | pkg.TOOL_SAO,
             "dq_deblock_sao_alf": pkg.TOOL_DEP_QUANT | pkg.TOOL_DEBLOCK | pkg.TOOL_SAO | pkg.TOOL_ALF}[tools_name]
    pics, cus, levels, ctus, aps = synth.random_records(SPECS, seed=11, tools=tools,
                                                        alf_aps=bool(tools & pkg.TOOL_ALF))
    batch = pkg.Batch(pics, cus, levels, ctus, aps)
    gpu = ctx.decode_batch(batch)
    assert_same(gpu, oracle_outputs(orc, pics, cus, levels, ctus, aps))


def test_staged_run_equals_whole_call_and_reruns_are_identical(ctx, pkg, orc):
    from rustmpeg_next_b200 import synth

    pics, cus, levels, ctus, aps = synth.random_records(SPECS[:3], seed=5,
                                                        tools=pkg.TOOL_DEBLOCK | pkg.TOOL_SAO)
    batch = pkg.Batch(pics, cus, levels, ctus, aps)
    first = ctx.decode_batch(batch)
    ctx.prepare(batch)
    ctx.upload(batch)
    for _ in range(3):
        ctx.run(pkg.STAGE_ALL)
    ctx.sync()
    again = ctx.download(batch.output_planes())
    for a, b in zip(first, again):
        for c in range(3):
            if a[c] is not None:
                assert (a[c] == b[c]).all()


def test_timeout_is_reported_and_context_stays_usable(pkg, orc):
    """A one-poll wait limit makes the wavefront waits give up (no fault, no
    hang); the host reads the status word and the context keeps working."""
    from rustmpeg_next_b200 import synth

    spec = [dict(width=1024, height=512, bit_depth=10, chroma_format=1, ctu_log2=5, qp=27)] * 4
    pics, cus, levels, ctus, _ = synth.random_records(spec, seed=9, tools=0)
    batch = pkg.Batch(pics, cus, levels, ctus)
    with pkg.Context(0, spin_limit=1) as c:
        with pytest.raises(pkg.Timeout):
            c.decode_batch(batch)
    with pkg.Context(0) as c:
        out = c.decode_batch(batch)
        ref = oracle_outputs(orc, pics[:1], cus, levels, ctus, None)
        assert (out[0][0] == ref[0][1]).all()


def test_invalid_inputs_are_rejected(ctx, pkg):
    from rustmpeg_next_b200 import synth

    spec = [dict(width=128, height=64, bit_depth=10, chroma_format=1, ctu_log2=5, qp=27)]
    pics, cus, levels, ctus, _ = synth.random_records(spec, seed=1, tools=0)
    bad = cus.copy()
    k = int(np.argmax(bad["cbf"] & 1))
    bad["level_off"][k, 0] = len(levels)  # past the end of the pool
    with pytest.raises(pkg.InvalidInput):
        ctx.decode_batch(pkg.Batch(pics, bad, levels, ctus))
    p2 = pics.copy()
    p2["ctu_log2"] = 4
    with pytest.raises(pkg.InvalidInput):
        ctx.decode_batch(pkg.Batch(p2, cus, levels, ctus))
    p3 = pics.copy()
    p3["width"], p3["height"] = 8192, 8192
    with pytest.raises((pkg.LimitExceeded, pkg.InvalidInput)):
        ctx.decode_batch(pkg.Batch(p3, cus, levels, ctus))
    out = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus))  # still usable
    assert out[0][0].shape == (64, 128)


def test_sao_edge_class3_on_picture_edge_aborts_like_the_reference(ctx, pkg, orc):
    """apply_sao_region_16 indexes row -1 for edge class 3 on the first picture
    row (a panic in the reference); the GPU rejects the same input."""
    from rustmpeg_next_b200 import synth

    spec = [dict(width=128, height=64, bit_depth=10, chroma_format=1, ctu_log2=5, qp=27)]
    pics, cus, levels, ctus, _ = synth.random_records(spec, seed=4, tools=pkg.TOOL_SAO)
    ctus["sao"]["type"] = 0
    ctus["sao"][1, 0]["type"] = 2
    ctus["sao"][1, 0]["band_or_class"] = 3
    ref = oracle_outputs(orc, pics, cus, levels, ctus, None)
    assert ref[0][0] == -3
    with pytest.raises(pkg.InvalidInput):
        ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus))
    # class 3 inside the picture is fine
    ctus["sao"][1, 0]["band_or_class"] = 2
    out = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus))
    assert_same(out, oracle_outputs(orc, pics, cus, levels, ctus, None))


def test_fixed_filter_alf_abort_matches_the_reference(ctx, pkg, orc):
    """The reference's whole-plane fixed-filter ALF aborts when a 4x4 block's
    class is 16 or more; the GPU reports that input as invalid too."""
    from rustmpeg_next_b200 import synth

    spec = [dict(width=128, height=128, bit_depth=10, chroma_format=1, ctu_log2=5, qp=22)]
    pics, cus, levels, ctus, _ = synth.random_records(spec, seed=2, tools=pkg.TOOL_ALF)
    ctus["alf_luma"] = 1
    ref = oracle_outputs(orc, pics, cus, levels, ctus, None)
    if ref[0][0] == 0:
        pytest.skip("content produced no class >= 16")
    assert ref[0][0] == -3
    with pytest.raises(pkg.InvalidInput):
        ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus))


def test_graph_replay_equals_direct_runs(ctx, pkg, orc):
    """vvcg_batch_run_graph: captured once, replayed; interleaved with direct
    runs, every run reconstructs and filters the same pictures."""
    from rustmpeg_next_b200 import synth

    pics, cus, levels, ctus, aps = synth.random_records(SPECS[:4], seed=21,
                                                        tools=pkg.TOOL_DEBLOCK | pkg.TOOL_SAO | pkg.TOOL_ALF,
                                                        alf_aps=True)
    batch = pkg.Batch(pics, cus, levels, ctus, aps)
    want = ctx.decode_batch(batch)
    ctx.prepare(batch)
    ctx.upload(batch)
    for graph in (True, True, False, True, False):
        n0 = ctx.kernel_launches
        ctx.run(pkg.STAGE_ALL, graph=graph)
        ctx.sync()
        assert ctx.kernel_launches > n0
        got = ctx.download(batch.output_planes())
        for a, b in zip(want, got):
            for c in range(3):
                if a[c] is not None:
                    assert (a[c] == b[c]).all(), f"graph={graph}"


@pytest.mark.parametrize("chunk,lanes", [(1, 2), (2, 3), (3, 1)])
def test_pipelined_decode_equals_whole_batch(ctx, pkg, orc, chunk, lanes):
    """vvcg_decode_batch_pipelined: chunks of pictures on internal lanes give
    the pictures vvcg_decode_batch gives, whatever the chunking, also when a
    picture's levels are not in picture order in the pool."""
    from rustmpeg_next_b200 import synth

    pics, cus, levels, ctus, aps = synth.random_records(SPECS + SPECS[:2], seed=33,
                                                        tools=pkg.TOOL_DEBLOCK | pkg.TOOL_SAO | pkg.TOOL_ALF,
                                                        alf_aps=True)
    # move picture 1's levels to the end of the pool
    p1 = pics[1]
    tb = min(1 << int(p1["ctu_log2"]), 32)
    n1 = (int(p1["width"]) // tb) * (int(p1["height"]) // tb)
    sel = cus[int(p1["cu_offset"]):int(p1["cu_offset"]) + n1].copy()
    extra, at = [], len(levels)
    for k in range(n1):
        for c in range(3):
            if sel["cbf"][k] >> c & 1 and sel["level_off"][k, c] >= 0:
                o = int(sel["level_off"][k, c])
                n = tb * tb if c == 0 else max(tb // 2, 2) ** 2
                sel["level_off"][k, c] = at
                extra.append(levels[o:o + n].copy())
                at += n
    cus[int(p1["cu_offset"]):int(p1["cu_offset"]) + n1] = sel
    levels = np.concatenate([levels] + extra)
    batch = pkg.Batch(pics, cus, levels, ctus, aps)
    want = ctx.decode_batch(batch)
    got = ctx.decode_batch_pipelined(batch, chunk_pictures=chunk, lanes=lanes)
    for i, (a, b) in enumerate(zip(want, got)):
        for c in range(3):
            if a[c] is not None:
                assert (a[c] == b[c]).all(), f"picture {i} plane {c}"


def test_async_decode_on_two_contexts_equals_decode_batch(ctx, pkg, orc):
    """vvcg_decode_batch_async + vvcg_batch_sync, alternating two contexts as a
    streaming caller does, gives vvcg_decode_batch's pictures for every batch."""
    import torch
    from rustmpeg_next_b200 import synth

    batches = []
    for seed in (41, 42, 43):
        pics, cus, levels, ctus, aps = synth.random_records(SPECS[:4], seed=seed,
                                                            tools=pkg.TOOL_DEBLOCK | pkg.TOOL_SAO | pkg.TOOL_ALF,
                                                            alf_aps=True)
        pin = lambda a: torch.from_numpy(a.view(np.uint8)).pin_memory().numpy().view(a.dtype)  # noqa: E731
        batches.append(pkg.Batch(pics, pin(cus), pin(levels), pin(ctus), pin(aps)))
    want = [ctx.decode_batch(b) for b in batches]
    with pkg.Context(0) as c1, pkg.Context(0) as c2:
        lanes = [c1, c2]
        outs = [b.output_planes() for b in batches]
        for i, b in enumerate(batches):
            if i >= 2:
                lanes[i % 2].sync()
            lanes[i % 2].decode_batch_async(b, outs[i])
        c1.sync()
        c2.sync()
    for i in range(len(batches)):
        for a, g in zip(want[i], outs[i]):
            for c in range(3):
                if a[c] is not None:
                    assert (a[c] == g[c]).all(), f"batch {i}"
