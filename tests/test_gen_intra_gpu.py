"""GPU parity: the general decoder's intra prediction
(vvcg_gen_intra_predict_dev) against the oracle's restatement: luma
Planar / DC / angular with MRL lines 0..2, BDPCM, ISP sub-partitions of
1..64 samples (with the shared 4-wide region of narrow vertical ones),
chroma Planar / DC / angular and CCLM LM / LM-L / LM-T, on random decoded
maps with holes, bit depths 8, 10, 12, both chroma sample positions."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h,bd,ctu,vc,seed", [(256, 192, 10, 64, False, 1), (192, 128, 8, 32, True, 2),
                                                (320, 256, 12, 128, False, 3), (128, 128, 10, 16, True, 4)])
def test_gen_intra_matches_oracle(ctx, pkg, orc, w, h, bd, ctu, vc, seed):
    import torch
    from rustmpeg_next_b200 import synth

    (Y, U, V), dy, dc = synth.random_gen_intra_state(w, h, bd, seed=seed)
    reqs, n = synth.random_gen_intra_reqs(w, h, 600, seed=seed)
    want = orc.gen_intra_predict(Y, U, V, dy, dc, bd, ctu, reqs, n, vert_collocated=vc)
    planes = [torch.from_numpy(p.view(np.int16)).cuda() for p in (Y, U, V)]
    got = ctx.gen_intra_predict(planes, torch.from_numpy(dy).cuda(), torch.from_numpy(dc).cuda(), bd, ctu, reqs, n,
                                vert_collocated=vc).cpu().numpy()[:n]
    bad = [i for i, q in enumerate(reqs)
           if not np.array_equal(got[q["out_off"]:q["out_off"] + q["w"] * q["h"]],
                                 want[q["out_off"]:q["out_off"] + q["w"] * q["h"]])]
    assert not bad, [(i, reqs[i]) for i in bad[:3]]


def test_gen_intra_rejects_bad_requests(ctx, pkg):
    import torch
    from rustmpeg_next_b200 import synth

    (Y, U, V), dy, dc = synth.random_gen_intra_state(64, 64, 10, seed=9)
    planes = [torch.from_numpy(p.view(np.int16)).cuda() for p in (Y, U, V)]
    dyt, dct = torch.from_numpy(dy).cuda(), torch.from_numpy(dc).cuda()
    r = np.zeros(1, pkg.GEN_INTRA_REQ_DTYPE)
    r[0] = (60, 0, 8, 8, 60, 0, 8, 8, 0, 0, 0, 0, 0, (0, 0, 0), 0)
    with pytest.raises(pkg.InvalidInput, match="luma block"):
        ctx.gen_intra_predict(planes, dyt, dct, 10, 64, r, 64)
    r[0] = (0, 0, 4, 4, 0, 0, 4, 4, 1, 81, 0, 0, 0, (0, 0, 0), 0)
    r["x"] = 1
    with pytest.raises(pkg.InvalidInput, match="CCLM position"):
        ctx.gen_intra_predict(planes, dyt, dct, 10, 64, r, 64)
    r[0] = (0, 0, 4, 4, 0, 0, 4, 4, 0, 0, 0, 0, 0, (0, 0, 0), 60)
    with pytest.raises(pkg.InvalidInput, match="output"):
        ctx.gen_intra_predict(planes, dyt, dct, 10, 64, r, 64)
