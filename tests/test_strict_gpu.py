"""GPU parity: the strict 8-bit intra profile (slice.rs:458-627 decode_picture)
on the frame path with per-TB transform tools (VVCG_TOOL_TU_TOOLS: transform
skip per component, luma MTS and LFNST), bit-exact against the oracle's
restatement of decode_picture and the encoder's own reconstruction: the
small-picture configuration's three 64x64 frames at QP 26 (and other QPs),
the reference's QP 4 lossless pictures and its QP 50 MTS / LFNST picture,
batched with each other and with a 10-bit frame-path picture, and through
the allocation-free entry point.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _strict_case(orc, synth, y, u, v, qp):
    cus, levels, rec = orc.strict_encode(y, u, v, qp)
    h, w = y.shape
    dec = orc.strict_decode(cus, levels, w, h, qp)
    assert all((d == r).all() for d, r in zip(dec, rec))
    return synth.strict_picture(w, h, qp), cus, levels, rec


def _batch(pkg, cases):
    pics, cus, levels, ncu, nlv = [], [], [], 0, 0
    for p, c, lv, _ in cases:
        p = p.copy()
        p["cu_offset"] = ncu
        c = c.copy()
        c["level_off"] = np.where(c["level_off"] >= 0, c["level_off"] + nlv, -1)
        pics.append(p)
        cus.append(c)
        levels.append(lv)
        ncu += len(c)
        nlv += len(lv)
    ctus = np.zeros(sum((int(p["width"]) // 32) * (int(p["height"]) // 32) for p in pics), pkg.CTU_DTYPE)
    return pkg.Batch(np.array(pics), np.concatenate(cus), np.concatenate(levels), ctus)


def _assert_planes(got, rec, what):
    for c in range(3):
        diff = np.argwhere(got[c] != rec[c])
        assert diff.size == 0, f"{what} plane {c}: {len(diff)} samples differ, first {diff[:3].tolist()}"


def _small_picture_cases(orc, synth, qps):
    out = []
    for qp in qps:
        for f in range(3):
            out.append(_strict_case(orc, synth, *synth.config1_frame(f), qp))
    return out


def test_small_picture_sequence_at_qp26_matches_oracle(ctx, pkg, orc):
    from rustmpeg_next_b200 import synth

    cases = _small_picture_cases(orc, synth, [26])
    got = ctx.decode_batch(_batch(pkg, cases))
    for i, (g, case) in enumerate(zip(got, cases)):
        _assert_planes(g, case[3], f"frame {i}")


def test_mts_lfnst_and_transform_skip_pictures_match_oracle(ctx, pkg, orc):
    from rustmpeg_next_b200 import synth

    cases = _small_picture_cases(orc, synth, [4, 22, 37, 50])
    j, i = np.mgrid[0:120, 0:200]
    y = synth.pad_to((16 + (i + j) % 40).astype(np.uint8), 224, 128)
    u = synth.pad_to(np.full((60, 100), 128, np.uint8), 112, 64)
    cases.append(_strict_case(orc, synth, y, u, u.copy(), 50))
    j, i = np.mgrid[0:64, 0:96]
    y = np.where(i < 48, 100, (i * 3 + j * 5) % 251).astype(np.uint8)
    cases.append(_strict_case(orc, synth, y, np.full((32, 48), 96, np.uint8), np.full((32, 48), 148, np.uint8), 4))
    tools = np.concatenate([c[1]["tu_tools"] for c in cases]).astype(int)
    assert (tools & 7).any() and ((tools >> pkg.CU_MTS_SHIFT) & 7).any() and (tools >> pkg.CU_LFNST_SHIFT).any()
    got = ctx.decode_batch(_batch(pkg, cases))
    for k, (g, case) in enumerate(zip(got, cases)):
        _assert_planes(g, case[3], f"picture {k} (QP {int(case[0]['slice_qp'])})")


def test_strict_pictures_batch_with_a_frame_path_picture(ctx, pkg, orc):
    """TU-tool pictures and a 10-bit DQ picture without them in one batch."""
    from rustmpeg_next_b200 import synth
    from test_recon_gpu import oracle_outputs

    cases = _small_picture_cases(orc, synth, [30])
    spec = [dict(width=128, height=64, bit_depth=10, chroma_format=1, ctu_log2=5, qp=27)]
    pics, cus, levels, ctus, _ = synth.random_records(spec, seed=81, tools=pkg.TOOL_DEP_QUANT)
    b = _batch(pkg, cases)
    p = pics[0].copy()
    p["cu_offset"] = len(b.cus)
    p["ctu_offset"] = len(b.ctus)
    c = cus.copy()
    c["level_off"] = np.where(c["level_off"] >= 0, c["level_off"] + len(b.levels), -1)
    batch = pkg.Batch(np.concatenate([b.pics, np.array([p])]), np.concatenate([b.cus, c]),
                      np.concatenate([b.levels, levels]), np.concatenate([b.ctus, ctus]))
    got = ctx.decode_batch(batch)
    for k, case in enumerate(cases):
        _assert_planes(got[k], case[3], f"strict picture {k}")
    want = oracle_outputs(orc, pics, cus, levels, ctus, None)[0]
    for c_ in range(3):
        assert (got[-1][c_] == want[c_ + 1]).all()


def test_strict_picture_through_the_static_entry(ctx, pkg, orc):
    import torch
    from rustmpeg_next_b200 import synth

    p, cus, levels, rec = _strict_case(orc, synth, *synth.config1_frame(2), 26)
    planes = [torch.zeros((64, 64), dtype=torch.int16, device="cuda"),
              torch.zeros((32, 32), dtype=torch.int16, device="cuda"),
              torch.zeros((32, 32), dtype=torch.int16, device="cuda")]
    d_cus = torch.from_numpy(cus.view(np.uint8).copy()).cuda()
    d_lev = torch.from_numpy(levels.copy()).cuda()
    torch.cuda.synchronize()
    pkg.recon_picture_static(p, d_cus, d_lev, planes)
    _assert_planes([t.cpu().numpy().view(np.uint16) for t in planes], rec, "static")


def test_bad_transform_tools_are_rejected(ctx, pkg, orc):
    from rustmpeg_next_b200 import synth

    p, cus, levels, rec = _strict_case(orc, synth, *synth.config1_frame(0), 37)
    for t in ((5 << pkg.CU_MTS_SHIFT), (3 << pkg.CU_LFNST_SHIFT),
              (1 << pkg.CU_MTS_SHIFT) | (1 << pkg.CU_LFNST_SHIFT), pkg.CU_TS_Y | (2 << pkg.CU_MTS_SHIFT)):
        bad = cus.copy()
        bad["tu_tools"][1] = t
        with pytest.raises(pkg.InvalidInput):
            ctx.decode_batch(_batch(pkg, [(p, bad, levels, rec)]))
    got = ctx.decode_batch(_batch(pkg, [(p, cus, levels, rec)]))  # the context still works
    _assert_planes(got[0], rec, "after rejections")


@pytest.mark.parametrize("sparse", [False, True])
def test_strict_bitstreams_decode_on_the_gpu(ctx, pkg, orc, sparse):
    """From slice data to pixels: the small-picture sequence at QP 26 (and
    the QP 4 / 50 pictures) written as CABAC slice data by the oracle's
    encoder side, parsed by the library's host parser (dense or sparse
    levels) and decoded on the GPU, equal to the encoder's reconstruction."""
    from rustmpeg_next_b200 import synth

    streams, recs = [], []
    for qp in (26, 26, 26, 4, 50):
        y, u, v = synth.config1_frame(len(streams) % 3)
        cus, levels, rec = orc.strict_encode(y, u, v, qp)
        streams.append((orc.strict_write(cus, levels, 64, 64, qp), 64, 64, qp))
        recs.append(rec)
    pics, cus, levels, _ = pkg.parse_strict(streams, sparse=sparse, threads=4)
    ctus = np.zeros(4 * len(pics), pkg.CTU_DTYPE)
    for i in range(len(pics)):
        pics["ctu_offset"][i] = 4 * i
    got = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus))
    for k, (g, rec) in enumerate(zip(got, recs)):
        _assert_planes(g, rec, f"stream {k}")


def test_annexb_access_units_decode_on_the_gpu(ctx, pkg, orc):
    """From Annex-B access units to pixels: the oracle encoder's slice data
    wrapped as the reference encoder's IDR access units (vvcg_annexb_idr),
    read back (vvcg_annexb_read_idr: size and QP from the PPS and slice
    header), parsed and decoded on the GPU, equal to the encoder's
    reconstruction."""
    from rustmpeg_next_b200 import synth

    aus, recs = [], []
    rng = np.random.default_rng(8)
    for k, qp in enumerate((26, 37, 22)):
        if k < 2:
            y, u, v = synth.config1_frame(k)
        else:  # 96x64 noise: a second coded size in the batch
            y = rng.integers(0, 256, (64, 96), dtype=np.uint8)
            u, v = (rng.integers(0, 256, (32, 48), dtype=np.uint8) for _ in range(2))
        cus, levels, rec = orc.strict_encode(y, u, v, qp)
        h, w = y.shape
        aus.append(pkg.annexb_idr(orc.strict_write(cus, levels, w, h, qp), w, h, qp))
        recs.append(rec)
    streams = [pkg.annexb_read_idr(au) for au in aus]
    assert [(w, h, qp) for _, w, h, qp in streams] == [(64, 64, 26), (64, 64, 37), (96, 64, 22)]
    pics, cus, levels, _ = pkg.parse_strict(streams, threads=2)
    n_ctu = [(int(p["width"]) // 32) * (int(p["height"]) // 32) for p in pics]
    pics["ctu_offset"] = np.concatenate([[0], np.cumsum(n_ctu)[:-1]])
    got = ctx.decode_batch(pkg.Batch(pics, cus, levels, np.zeros(sum(n_ctu), pkg.CTU_DTYPE)))
    for k, (g, rec) in enumerate(zip(got, recs)):
        _assert_planes(g, rec, f"access unit {k}")
