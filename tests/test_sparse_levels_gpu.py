"""GPU parity: the sparse level form (TOOL_SPARSE_LEVELS, per coded TB a count
and (raster index, level) pairs) gives the pictures the dense raster form
gives, and both equal the oracle's, bit-exact: synthetic and encoder
records, whole-batch, pipelined and allocation-free calls, batches that mix
both forms, and malformed sparse records rejected without harm to the
context.
"""
import numpy as np
import pytest

from test_recon_gpu import SPECS, assert_same, encoded_picture, oracle_outputs

pytestmark = pytest.mark.gpu

ALL_TOOLS = 1 | 2 | 4 | 8  # DEP_QUANT | DEBLOCK | SAO | ALF


def _same_planes(a_list, b_list):
    for i, (a, b) in enumerate(zip(a_list, b_list)):
        for c in range(3):
            if a[c] is not None:
                assert (a[c] == b[c]).all(), f"picture {i} plane {c}"


def test_sparse_synthetic_batch_matches_dense_and_oracle(ctx, pkg, orc):
    from rustmpeg_next_b200 import synth

    pics, cus, levels, ctus, aps = synth.random_records(SPECS, seed=71, tools=ALL_TOOLS, alf_aps=True)
    sp, sc, sl = synth.sparsify(pics, cus, levels)
    assert len(sl) < len(levels)
    dense = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus, aps))
    sparse = ctx.decode_batch(pkg.Batch(sp, sc, sl, ctus, aps))
    _same_planes(dense, sparse)
    assert_same(sparse, oracle_outputs(orc, pics, cus, levels, ctus, aps))


@pytest.mark.parametrize("bd,qp,ctu_log2,opts,cf", [
    (10, 22, 5, 1 | 2 | 8, 1),
    (8, 37, 6, 1 | 2 | 8, 1),
    (12, 27, 7, 1 | 8, 2),
    (10, 32, 5, 1 | 2 | 8, 3),
])
def test_sparse_encoder_records_match_oracle(ctx, pkg, orc, bd, qp, ctu_log2, opts, cf):
    from rustmpeg_next_b200 import synth

    ctu = 1 << ctu_log2
    vis = (200, 120)
    w, h = -(-vis[0] // ctu) * ctu, -(-vis[1] // ctu) * ctu
    p, cus, levels = encoded_picture(orc, pkg, w, h, bd, qp, ctu_log2, opts, cf=cf, seed=qp + 1, vis=vis)
    ctus = np.zeros((h // ctu) * (w // ctu), pkg.CTU_DTYPE)
    sp, sc, sl = synth.sparsify(np.array([p]), cus, levels)
    got = ctx.decode_batch(pkg.Batch(sp, sc, sl, ctus))
    assert_same(got, oracle_outputs(orc, np.array([p]), cus, levels, ctus, None))


def test_mixed_dense_and_sparse_pictures_in_one_batch(ctx, pkg):
    """Dense pictures leave odd offsets in the shared pool; the sparse ones
    after them start on even offsets (one pad word), whole-batch and
    pipelined in chunks whose level windows start on odd offsets."""
    from rustmpeg_next_b200 import synth

    pics, cus, levels, ctus, aps = synth.random_records(SPECS + SPECS[:2], seed=72, tools=ALL_TOOLS, alf_aps=True)
    want = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus, aps))
    sp, sc, sl = synth.sparsify(pics, cus, levels)
    pool = [np.zeros(1, np.int16)]  # one word first: every dense offset becomes odd
    at = 1
    mix_p, mix_c = pics.copy(), cus.copy()
    for i in range(len(pics)):
        p = pics[i]
        tb, sizes = synth._tb_sizes(p)
        c0 = int(p["cu_offset"])
        n = (int(p["width"]) // tb) * (int(p["height"]) // tb)
        src_c, src_l = (sc, sl) if i % 2 else (cus, levels)
        if i % 2:
            mix_p["tools"][i] = sp["tools"][i]
            if at & 1:
                pool.append(np.zeros(1, np.int16))
                at += 1
        rec = src_c[c0:c0 + n].copy()
        offs = rec["level_off"].astype(np.int64)
        used = offs >= 0
        lo_, hi_ = int(offs[used].min()), 0
        for k in range(n):
            for c in range(3):
                o = int(offs[k, c])
                if o < 0:
                    continue
                hi_ = max(hi_, o + (2 + 2 * int(src_l[o]) if i % 2 else sizes[c]))
        pool.append(np.asarray(src_l[lo_:hi_], np.int16))
        rec["level_off"] = np.where(used, offs - lo_ + at, -1).astype(np.int32)
        mix_c[c0:c0 + n] = rec
        at += hi_ - lo_
    mix_l = np.concatenate(pool)
    batch = pkg.Batch(mix_p, mix_c, mix_l, ctus, aps)
    _same_planes(want, ctx.decode_batch(batch))
    for chunk, lanes in ((1, 2), (3, 2)):
        _same_planes(want, ctx.decode_batch_pipelined(batch, chunk_pictures=chunk, lanes=lanes))


def test_sparse_levels_through_the_static_entry(ctx, pkg):
    import torch
    from rustmpeg_next_b200 import synth

    spec = [dict(width=256, height=128, bit_depth=10, chroma_format=1, ctu_log2=5, qp=27)]
    pics, cus, levels, ctus, _ = synth.random_records(spec, seed=73, tools=1 | 2)
    want = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus))[0]
    sp, sc, sl = synth.sparsify(pics, cus, levels)
    planes = [torch.zeros((128, 256), dtype=torch.int16, device="cuda"),
              torch.zeros((64, 128), dtype=torch.int16, device="cuda"),
              torch.zeros((64, 128), dtype=torch.int16, device="cuda")]
    d_cus = torch.from_numpy(sc.view(np.uint8).copy()).cuda()
    d_lev = torch.from_numpy(sl.copy()).cuda()
    torch.cuda.synchronize()
    pkg.recon_picture_static(sp[0], d_cus, d_lev, planes)
    for c in range(3):
        assert (planes[c].cpu().numpy().view(np.uint16) == want[c]).all(), c


def _first_tb_with(sc, sl, at_least):
    for k in range(len(sc)):
        o = int(sc["level_off"][k, 0])
        if sc["cbf"][k] & 1 and o >= 0 and int(sl[o]) >= at_least:
            return k, o
    raise AssertionError("no TB with enough levels")


def test_malformed_sparse_records_are_rejected(ctx, pkg):
    from rustmpeg_next_b200 import synth

    spec = [dict(width=128, height=64, bit_depth=10, chroma_format=1, ctu_log2=5, qp=22)]
    pics, cus, levels, ctus, _ = synth.random_records(spec, seed=74, tools=1 | 2)
    sp, sc, sl = synth.sparsify(pics, cus, levels)
    k, o = _first_tb_with(sc, sl, 2)
    cases = []
    bad = sl.copy()
    bad[o + 2] = 1024  # index past a 32x32 TB (checked on the device)
    cases.append((sc, bad))
    bad = sl.copy()
    bad[o + 4] = bad[o + 2]  # second index not above the first (device)
    cases.append((sc, bad))
    bad = sl.copy()
    bad[o] = 1025  # count above the TB's size (host)
    cases.append((sc, bad))
    odd = sc.copy()
    odd["level_off"][k, 0] = o + 1  # odd offset (host)
    cases.append((odd, sl))
    for c_, l_ in cases:
        with pytest.raises(pkg.InvalidInput):
            ctx.decode_batch(pkg.Batch(sp, c_, l_, ctus))
    want = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus))
    _same_planes(want, ctx.decode_batch(pkg.Batch(sp, sc, sl, ctus)))  # the context still works
