"""GPU parity: the general decoder's deblocking (vvcg_deblock_general_dev)
against the oracle's restatement of apply_deblock on random coding trees:
QT / BT / TT partitions with ISP sub-partitions of 1..64 samples, intra and
inter blocks with motion, shared and separate chroma trees, bit depths 8, 10
and 12, CTU sizes 32..128, visible sizes that are not multiples of 8."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(ctx, planes, vis_w, vis_h, bd, ctu, cells, cc, prm, device_maps=False):
    import torch

    t = [torch.from_numpy(p.astype(np.int16)).cuda() for p in planes]
    if device_maps:
        cells = torch.from_numpy(cells.view(np.uint8).reshape(cells.shape[0], -1).copy()).cuda()
        cc = torch.from_numpy(cc.view(np.uint8).reshape(cc.shape[0], -1).copy()).cuda()
    ctx.deblock_general(t, vis_w, vis_h, bd, ctu, cells, cc, prm)
    torch.cuda.synchronize()
    return [x.cpu().numpy().view(np.uint16) for x in t]


@pytest.mark.parametrize("vis_w,vis_h,ctu,bd,dual,seed", [
    (256, 128, 32, 10, False, 1), (200, 136, 64, 8, True, 2), (122, 70, 32, 12, False, 3),
    (384, 256, 128, 10, True, 4), (64, 64, 16, 10, False, 5), (1920, 1080, 128, 10, False, 6),
])
def test_deblock_general_matches_oracle(ctx, pkg, orc, vis_w, vis_h, ctu, bd, dual, seed):
    from rustmpeg_next_b200 import synth

    planes, cells, cc, prm = synth.random_deblock_picture(vis_w, vis_h, ctu, bd, seed=seed, dual_tree=dual)
    want = orc.deblock_general(planes, vis_w, vis_h, bd, ctu, cells, cc, prm)
    got = _run(ctx, planes, vis_w, vis_h, bd, ctu, cells, cc, prm, device_maps=seed % 2 == 0)
    for c in range(3):
        diff = np.argwhere(got[c] != want[c])
        assert diff.size == 0, f"plane {c}: {len(diff)} samples differ, first {diff[:4].tolist()}"
        assert np.count_nonzero(want[c] != planes[c]) > 0, f"plane {c}: nothing filtered"


def test_deblock_general_all_inter_without_residual(ctx, pkg, orc):
    """bS from motion alone: every block inter, no cbf, motion fields that
    differ by less and by more than half a sample."""
    from rustmpeg_next_b200 import synth

    planes, cells, cc, prm = synth.random_deblock_picture(256, 192, 64, 10, seed=11, intra_prob=0.0, isp_prob=0.0)
    cells["flags"] &= 0xFF ^ pkg.DBK_CBF
    want = orc.deblock_general(planes, 256, 192, 10, 64, cells, cc, prm)
    got = _run(ctx, planes, 256, 192, 10, 64, cells, cc, prm)
    for c in range(3):
        assert np.array_equal(got[c], want[c]), c


def test_deblock_general_rejects_bad_arguments(ctx, pkg):
    import torch
    from rustmpeg_next_b200 import synth

    planes, cells, cc, prm = synth.random_deblock_picture(64, 64, 32, 10, seed=1)
    t = [torch.from_numpy(p.astype(np.int16)).cuda() for p in planes]
    with pytest.raises(pkg.InvalidInput, match="luma cell map"):
        ctx.deblock_general(t, 64, 64, 10, 32, cells[:, :8], cc, prm)
    with pytest.raises(pkg.InvalidInput, match="CTU size"):
        ctx.deblock_general(t, 64, 64, 10, 24, cells, cc, prm)
    bad = prm.copy()
    bad["num_ref"] = [17, 0]
    with pytest.raises(pkg.InvalidInput, match="reference list"):
        ctx.deblock_general(t, 64, 64, 10, 32, cells, cc, bad)
