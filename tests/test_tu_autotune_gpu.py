"""GPU: the block-size-binning autotuner of the transform-unit batches
(vvcg_tu_autotune). It times each CTA width of every size group on the
caller's batch and keeps the fastest; the outputs of the tuning call and of
later batches equal the untuned batch and the oracle bit for bit, the chosen
widths are ones the library has, and a group without units reports 0."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WIDTHS = ({2, 4, 8}, {2, 4, 8}, {1, 2, 4})


def _groups(recs):
    el = 1 << (recs["log2_w"].astype(np.int64) + recs["log2_h"])
    return [bool(np.any(el <= 256)), bool(np.any((el > 256) & (el <= 1024))), bool(np.any(el > 1024))]


@pytest.mark.parametrize("forward", [False, True])
def test_tuned_batches_equal_untuned_and_oracle(ctx, pkg, orc, forward):
    import torch
    from rustmpeg_next_b200 import synth

    recs, data, total = synth.random_tu_records(3000, seed=41, forward=forward, bit_depths=(8, 10, 12))
    d_in = torch.from_numpy(data).cuda()
    run = ctx.tu_forward if forward else ctx.tu_inverse
    before = torch.full((total,), -7, dtype=torch.int16, device="cuda")
    run(recs, d_in, before)
    tuned_out = torch.full((total,), -7, dtype=torch.int16, device="cuda")
    warps = ctx.tu_autotune(recs, d_in, tuned_out, forward)
    after = torch.full((total,), -7, dtype=torch.int16, device="cuda")
    run(recs, d_in, after)
    torch.cuda.synchronize()
    want = before.cpu().numpy()
    assert np.array_equal(tuned_out.cpu().numpy(), want)
    assert np.array_equal(after.cpu().numpy(), want)
    rc, oracle_out = orc.tu_batch(recs, data, total, forward=forward)
    assert rc == 0 and np.array_equal(want, oracle_out)
    for g, present in enumerate(_groups(recs)):
        assert (warps[g] in WIDTHS[g]) if present else warps[g] == 0, (g, warps)


def test_group_without_units_reports_zero(ctx, pkg):
    import torch

    r = np.zeros(64, pkg.TU_DTYPE)
    r["log2_w"], r["log2_h"], r["bit_depth"], r["qp"] = 3, 3, 10, 32
    r["in_off"] = r["out_off"] = np.arange(64, dtype=np.uint32) * 64
    data = torch.ones(64 * 64, dtype=torch.int16, device="cuda")
    out = torch.zeros(64 * 64, dtype=torch.int16, device="cuda")
    warps = ctx.tu_autotune(r, data, out, False)
    assert warps[0] in WIDTHS[0] and warps[1] == 0 and warps[2] == 0


def test_autotune_rejects_what_the_batch_rejects(ctx, pkg):
    import torch

    r = np.zeros(1, pkg.TU_DTYPE)
    r["log2_w"], r["log2_h"], r["bit_depth"], r["qp"] = 6, 6, 10, 30
    data = torch.zeros(4096, dtype=torch.int16, device="cuda")
    out = torch.zeros(4096, dtype=torch.int16, device="cuda")
    r["qp"] = 88
    with pytest.raises(pkg.InvalidInput):
        ctx.tu_autotune(r, data, out, False)
