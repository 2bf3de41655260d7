"""LMCS and joint Cb-Cr residuals: the library's host-side table build
against the oracle (CPU), and the GPU mapping, chroma scale derivation and
residual combination against the oracle (bit-exact)."""
import numpy as np
import pytest


@pytest.mark.parametrize("bd", [8, 10, 12])
def test_lmcs_tables_match_oracle(pkg, orc, bd):
    from rustmpeg_next_b200 import synth

    rng = np.random.default_rng(bd)
    for _ in range(20):
        a = synth.random_lmcs_aps(rng)
        got = pkg.lmcs_build(a, bd)
        want = orc.lmcs_build(np.frombuffer(a.tobytes(), orc.LMCS_APS_DTYPE)[0], bd)
        assert got.tobytes() == want.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("bd", [8, 10, 12])
def test_lmcs_gpu_matches_oracle(ctx, pkg, orc, bd):
    import torch
    from rustmpeg_next_b200 import synth

    rng = np.random.default_rng(100 + bd)
    tables = pkg.lmcs_build(synth.random_lmcs_aps(rng), bd)
    otab = np.frombuffer(tables.tobytes(), orc.LMCS_TABLES_DTYPE)[0]
    h, w = 136, 250
    plane = rng.integers(0, 1 << bd, (h, w)).astype(np.uint16)
    plane[0, :8] = (1 << bd) - 1
    for inverse in (True, False):
        t = torch.from_numpy(plane.view(np.int16).copy()).cuda()
        ctx.lmcs_map_plane(tables, t, inverse)
        torch.cuda.synchronize()
        assert (t.cpu().numpy().view(np.uint16) == orc.lmcs_map_plane(otab, plane, inverse)).all()
    for ctu in (32, 64, 128):
        pos = np.stack([rng.integers(0, w, 200), rng.integers(0, h, 200)], 1).astype(np.uint32)
        pos[:3] = [[0, 0], [5, 0], [0, 70]]
        d_pos = torch.from_numpy(pos.view(np.int32)).cuda()
        out = torch.zeros(len(pos), dtype=torch.int32, device="cuda")
        ctx.lmcs_chroma_scales(tables, torch.from_numpy(plane.view(np.int16)).cuda(), ctu, d_pos, out)
        torch.cuda.synchronize()
        want = [orc.lmcs_chroma_scale(otab, plane, ctu, int(x), int(y)) for x, y in pos]
        assert out.cpu().numpy().tolist() == want


@pytest.mark.gpu
def test_chroma_residuals_gpu_match_oracle(ctx, pkg, orc):
    import torch

    rng = np.random.default_rng(7)
    recs, at = [], 0
    for i in range(500):
        lw, lh = int(rng.integers(1, 6)), int(rng.integers(1, 6))
        n = (1 << lw) * (1 << lh)
        single = rng.random() < 0.2
        flags = (pkg.CRES_SCALE if rng.random() < 0.7 else 0) | (pkg.CRES_SINGLE if single else 0)
        recs.append((lw, lh, int(rng.choice([8, 10, 12])), int(rng.integers(-3, 4)), flags,
                     int(rng.choice([512, 1024, 1800, 2048, 2600, 4096, 30000])), at, at + n))
        at += 2 * n
    recs = np.array(recs, dtype=pkg.CRES_DTYPE)
    res = rng.integers(-600, 601, at).astype(np.int16)
    res[:64] = rng.choice([-32768, 32767, -5000, 5000], 64)
    d = torch.from_numpy(res.copy()).cuda()
    ctx.chroma_residuals(recs, d)
    torch.cuda.synchronize()
    want = orc.chroma_residuals(np.frombuffer(recs.tobytes(), orc.CRES_DTYPE), res)
    assert (d.cpu().numpy() == want).all()
