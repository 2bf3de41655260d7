"""GPU parity: transform-unit batches (vvcg_tu_inverse_batch / vvcg_tu_forward_batch)
against the oracle, bit-exact, over every TU shape 1x2..64x64 and the tools of
the residual path (DQ, transform skip, BDPCM, implicit / explicit MTS, LFNST),
bit depths 8..12 and the full Qp' range."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(ctx, pkg, recs, data, total, forward):
    import torch

    d_in = torch.from_numpy(data).cuda()
    d_out = torch.full((total,), -7, dtype=torch.int16, device="cuda")
    (ctx.tu_forward if forward else ctx.tu_inverse)(recs, d_in, d_out)
    torch.cuda.synchronize()
    return d_out.cpu().numpy()


def _compare(orc, got, recs, data, total, forward):
    rc, want = orc.tu_batch(recs, data, total, forward=forward)
    assert rc == 0
    bad = np.nonzero(got != want)[0]
    if bad.size:
        starts = recs["out_off"].astype(np.int64)
        i = int(np.searchsorted(starts, bad[0], side="right") - 1)
        raise AssertionError(f"{bad.size} values differ; first in unit {i}: {recs[i]}")


@pytest.mark.parametrize("forward", [False, True])
@pytest.mark.parametrize("seed,bds,odd", [(1, (8, 10), 0.05), (2, (8, 9, 10, 11, 12), 0.3), (3, (12,), 0.1)])
def test_tu_batch_matches_oracle(ctx, pkg, orc, forward, seed, bds, odd):
    from rustmpeg_next_b200 import synth

    recs, data, total = synth.random_tu_records(3000, seed=seed, forward=forward, bit_depths=bds,
                                                odd_frac=odd)
    got = _run(ctx, pkg, recs, data, total, forward)
    _compare(orc, got, recs, data, total, forward)


@pytest.mark.parametrize("forward", [False, True])
def test_tu_batch_full_qp_range_and_every_lfnst_mode(ctx, pkg, orc, forward):
    from rustmpeg_next_b200 import synth

    recs, data, total = synth.random_tu_records(4000, seed=17, forward=forward, bit_depths=(8, 10, 12),
                                                qp_range=(-12, 63))
    recs["lfnst_mode"] = np.arange(len(recs)) % 95
    got = _run(ctx, pkg, recs, data, total, forward)
    _compare(orc, got, recs, data, total, forward)


def test_tu_batch_rejects_what_the_reference_rejects(ctx, pkg, orc):
    import torch

    r = np.zeros(1, pkg.TU_DTYPE)
    r["log2_w"], r["log2_h"], r["bit_depth"], r["qp"] = 6, 6, 10, 30
    data = torch.zeros(4096, dtype=torch.int16, device="cuda")
    out = torch.zeros(4096, dtype=torch.int16, device="cuda")
    bad = r.copy()
    bad["mts_idx"] = 1  # DST-7 has no 64-point matrix
    assert orc.tu_batch(bad, np.zeros(4096, np.int16), 4096)[0] < 0
    with pytest.raises(pkg.InvalidInput, match="transform"):
        ctx.tu_inverse(bad, data, out)
    bad = r.copy()
    bad["lfnst_idx"], bad["mts_idx"], bad["log2_w"], bad["log2_h"] = 1, 1, 4, 4
    assert orc.tu_batch(bad, np.zeros(4096, np.int16), 4096, forward=True)[0] < 0
    with pytest.raises(pkg.InvalidInput, match="MTS combined with LFNST"):
        ctx.tu_forward(bad, data, out)
    bad = r.copy()
    bad["out_off"] = 1  # past the end of the output
    with pytest.raises(pkg.InvalidInput, match="output range"):
        ctx.tu_inverse(bad, data, out)
    ctx.tu_inverse(r, data, out)  # still usable
    torch.cuda.synchronize()
    assert int(out.abs().max()) == 0
