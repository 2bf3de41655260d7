"""GPU parity: sequential reconstruction of the general decoder's transform
blocks (vvcg_gen_intra_recon_dev) against the oracle's restatement of
reconstruct_tu in decode order: ISP coding units (horizontal and vertical
sub-partitions of 1..32 samples, including the shared 4-wide region of
narrow vertical ones), each sub-partition predicted from the ones
reconstructed before it, followed by the CU's chroma blocks (CCLM reads the
CU's reconstructed luma); planes and decoded maps compared bit-exactly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (cu_w, cu_h) of ISP coding units and their sub-partition counts (H.266
# 7.4.9.5: 2 for 4x8 / 8x4, else 4)
SHAPES = [(4, 8), (8, 4), (8, 8), (4, 16), (16, 4), (8, 16), (16, 8), (16, 16), (32, 16), (16, 32), (32, 32),
          (4, 32), (32, 4), (8, 32)]


def _case(pkg, w, h, bd, seed):
    from rustmpeg_next_b200 import synth

    rng = np.random.default_rng(seed)
    (Y, U, V), dy, dc = synth.random_gen_intra_state(w, h, bd, seed=seed, hole_prob=0.05)
    dy[:] = 1
    dc[:] = 1
    reqs, groups, off = [], [0], 0
    for gy in range(0, h - 31, 64):
        for gx in range(0, w - 31, 64):
            cw, ch = SHAPES[rng.integers(len(SHAPES))]
            isp = int(rng.integers(1, 3))
            if (cw, ch) in ((4, 8), (4, 16), (4, 32)):
                isp = 2 if rng.random() < 0.7 else 1
            n = 2 if (cw, ch) in ((4, 8), (8, 4)) else 4
            sw, sh = (cw, ch // n) if isp == 1 else (cw // n, ch)
            mode = int(rng.integers(0, 67))
            dy[gy // 4:(gy + ch + 3) // 4, gx // 4:(gx + cw + 3) // 4] = 0
            dc[gy // 2:(gy + ch) // 2, gx // 2:(gx + cw) // 2] = 0
            for k in range(n):
                x, y = (gx, gy + k * sh) if isp == 1 else (gx + k * sw, gy)
                reqs.append((x, y, sw, sh, gx, gy, cw, ch, 0, mode, 0, isp, 0, (0, 0, 0), off))
                off += sw * sh
            if cw >= 8 and ch >= 8:  # the CU's chroma blocks after its luma
                cm = int(rng.choice([0, 1, 18, 50, 66, 81, 82, 83]))
                for comp in (1, 2):
                    reqs.append((gx // 2, gy // 2, cw // 2, ch // 2, gx, gy, cw, ch, comp, cm, 0, 0, 0, (0, 0, 0),
                                 off))
                    off += (cw // 2) * (ch // 2)
            groups.append(len(reqs))
    reqs = np.array(reqs, pkg.GEN_INTRA_REQ_DTYPE)
    res = rng.integers(-24, 25, off).astype(np.int16)
    return (Y, U, V), dy, dc, reqs, np.array(groups, np.uint32), res, off


@pytest.mark.parametrize("w,h,bd,ctu,seed", [(256, 192, 10, 64, 1), (192, 128, 8, 32, 2), (320, 256, 12, 128, 3)])
def test_sequential_reconstruction_matches_oracle(ctx, pkg, orc, w, h, bd, ctu, seed):
    import torch

    (Y, U, V), dy, dc, reqs, groups, res, n = _case(pkg, w, h, bd, seed)
    want = orc.gen_intra_recon(Y, U, V, dy, dc, bd, ctu, reqs, groups, res, n)
    planes = [torch.from_numpy(p.view(np.int16).copy()).cuda() for p in (Y, U, V)]
    dyt, dct = torch.from_numpy(dy.copy()).cuda(), torch.from_numpy(dc.copy()).cuda()
    pred = ctx.gen_intra_recon(planes, dyt, dct, bd, ctu, reqs, groups, torch.from_numpy(res).cuda(), n)
    assert np.array_equal(pred.cpu().numpy()[:n], want[5][:n])
    for k in range(3):
        got = planes[k].cpu().numpy().view(np.uint16)
        diff = np.argwhere(got != want[k])
        assert diff.size == 0, f"plane {k}: {len(diff)} samples differ, first {diff[:3].tolist()}"
    assert np.array_equal(dyt.cpu().numpy(), want[3]) and np.array_equal(dct.cpu().numpy(), want[4])
    # the sub-partitions depend on each other: predicting them all from the
    # starting state (one call of independent blocks) gives other samples
    indep = orc.gen_intra_predict(Y, U, V, dy, dc, bd, ctu, reqs, n)
    assert not np.array_equal(indep[:n], want[5][:n])


def test_sequential_reconstruction_rejects_bad_groups(ctx, pkg):
    import torch

    (Y, U, V), dy, dc, reqs, groups, res, n = _case(pkg, 128, 128, 10, 5)
    planes = [torch.from_numpy(p.view(np.int16).copy()).cuda() for p in (Y, U, V)]
    dyt, dct = torch.from_numpy(dy).cuda(), torch.from_numpy(dc).cuda()
    bad = groups.copy()
    bad[-1] -= 1
    with pytest.raises(pkg.InvalidInput, match="groups"):
        ctx.gen_intra_recon(planes, dyt, dct, 10, 64, reqs, bad, None, n)
