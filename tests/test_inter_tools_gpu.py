"""GPU parity: the inter-prediction tools beyond plain motion compensation
(BDOF, DMVR, affine subblock motion with PROF deltas, PROF, CIIP, GPM)
against the oracle's restatements of inter.rs, bit-exact, on seeded
batches of blocks of every size the tools take."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cuda(a, dtype=np.int32):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _smooth(rng, n, lo, hi):
    """Correlated 14-bit-like intermediates: a ramp plus noise."""
    base = rng.integers(lo, hi)
    return (base + np.cumsum(rng.integers(-40, 41, n))).clip(-8192, 24575)


def test_bdof_matches_oracle(ctx, pkg, orc):
    rng = np.random.default_rng(1)
    sizes = [(8, 8), (16, 16), (8, 16), (16, 8), (4, 4), (32, 16), (12, 8), (128, 4)] * 6
    reqs, p0, p1, off = [], [], [], 0
    for w, h in sizes:
        a = _smooth(rng, w * h, -4000, 20000)
        b = a + rng.integers(-300, 301, w * h) + rng.integers(-200, 200)
        reqs.append((w, h, off))
        p0.append(a)
        p1.append(b)
        off += w * h
    p0, p1 = np.concatenate(p0), np.concatenate(p1)
    out = _cuda(np.zeros(off))
    ctx.bdof(np.array(reqs, pkg.BDOF_REQ_DTYPE), _cuda(p0), _cuda(p1), out)
    got = out.cpu().numpy()
    for w, h, o in reqs:
        want = orc.bdof(p0[o:o + w * h], p1[o:o + w * h], w, h)
        assert np.array_equal(got[o:o + w * h], want), (w, h)


def test_dmvr_matches_oracle(ctx, pkg, orc):
    import torch

    rng = np.random.default_rng(2)
    h, w = 96, 128
    yy, xx = np.mgrid[0:h, 0:w]
    r0 = (128 + 60 * np.sin(xx / 7.0) * np.cos(yy / 9.0) + rng.integers(-6, 7, (h, w))).clip(0, 255).astype(np.uint8)
    r1 = np.roll(np.roll(r0, 1, axis=1), -1, axis=0)
    r1 = (r1.astype(int) + rng.integers(-3, 4, (h, w))).clip(0, 255).astype(np.uint8)
    reqs = []
    for k in range(120):
        dx, dy = [(8, 8), (16, 16), (16, 8), (8, 16)][k % 4]
        reqs.append((int(rng.integers(-8, w)), int(rng.integers(-8, h)), dx, dy,
                     ((int(rng.integers(-64, 65)), int(rng.integers(-64, 65))),
                      (int(rng.integers(-64, 65)), int(rng.integers(-64, 65))))))
    reqs = np.array(reqs, pkg.DMVR_REQ_DTYPE)
    out = torch.zeros(4 * len(reqs), dtype=torch.int32, device="cuda")
    ctx.dmvr(_cuda(r0, np.uint8), _cuda(r1, np.uint8), reqs, out)
    got = out.cpu().numpy().reshape(-1, 4)
    refined = 0
    for i, r in enumerate(reqs):
        want = orc.dmvr(r0, r1, int(r["bx"]), int(r["by"]), int(r["dx"]), int(r["dy"]), r["mv"].reshape(4))
        assert np.array_equal(got[i], want), (i, got[i], want)
        refined += int((want != r["mv"].reshape(4)).any())
    assert refined > 10


def test_affine_mvs_and_prof_match_oracle(ctx, pkg, orc):
    import torch

    rng = np.random.default_rng(3)
    reqs, off = [], 0
    for k in range(200):
        w, h = int(2 ** rng.integers(3, 8)), int(2 ** rng.integers(3, 8))
        spread = [4, 40, 400, 4000][k % 4]
        cp = rng.integers(-spread, spread + 1, (3, 2))
        reqs.append((cp, w, h, int(k % 2), int(1 + k % 3), (0, 0), off))
        off += (w // 4) * (h // 4)
    reqs = np.array(reqs, pkg.AFFINE_REQ_DTYPE)
    sub = torch.zeros(2 * off, dtype=torch.int32, device="cuda")
    prof = torch.zeros(33 * len(reqs), dtype=torch.int32, device="cuda")
    ctx.affine_mvs(reqs, sub, prof)
    gs, gp = sub.cpu().numpy().reshape(-1, 2), prof.cpu().numpy().reshape(-1, 33)
    kinds = set()
    for i, r in enumerate(reqs):
        w, h = int(r["w"]), int(r["h"])
        s, ph, pv, en = orc.affine_mvs(r["cp"], int(r["six_param"]), w, h, int(r["inter_dir"]))
        o = int(r["sub_off"])
        assert np.array_equal(gs[o:o + len(s)], s), i
        assert np.array_equal(gp[i, :16], ph) and np.array_equal(gp[i, 16:32], pv) and gp[i, 32] == int(en), i
        kinds.add(en)
    assert kinds == {True, False}
    # PROF on 4x4 subblocks with those deltas
    preqs, src, dmv, outn = [], [], [], 0
    for i in range(len(reqs)):
        preqs.append((36 * i, 32 * i, 16 * i, i % 2, (0, 0, 0)))
        src.append(_smooth(rng, 36, -2000, 15000))
        dmv.append(gp[i, :32])
    preqs = np.array(preqs, pkg.PROF_REQ_DTYPE)
    src, dmv = np.concatenate(src), np.concatenate(dmv)
    out = torch.zeros(16 * len(preqs), dtype=torch.int32, device="cuda")
    ctx.prof(preqs, _cuda(src), _cuda(dmv), out)
    got = out.cpu().numpy()
    for i, r in enumerate(preqs):
        want = orc.prof(src[36 * i:36 * i + 36], dmv[32 * i:32 * i + 16], dmv[32 * i + 16:32 * i + 32], int(r["bi"]))
        assert np.array_equal(got[16 * i:16 * i + 16], want), i


def test_ciip_and_gpm_match_oracle(ctx, pkg, orc):
    import torch

    rng = np.random.default_rng(4)
    creqs, inter, intra, off = [], [], [], 0
    for k in range(40):
        n = int(rng.choice([16, 64, 256, 1024]))
        creqs.append((n, off, k % 2, (k // 2) % 2, (0, 0)))
        inter.append(rng.integers(0, 256, n))
        intra.append(rng.integers(0, 256, n))
        off += n
    creqs = np.array(creqs, pkg.CIIP_REQ_DTYPE)
    inter, intra = np.concatenate(inter), np.concatenate(intra)
    out = torch.zeros(off, dtype=torch.int32, device="cuda")
    ctx.ciip_blend(creqs, _cuda(inter), _cuda(intra), out)
    got = out.cpu().numpy()
    for r in creqs:
        o, n = int(r["off"]), int(r["n"])
        assert np.array_equal(got[o:o + n], orc.ciip(inter[o:o + n], intra[o:o + n], r["left_intra"], r["above_intra"]))
    greqs, p0, p1, off = [], [], [], 0
    for split in range(64):
        for w, h, sx in ((16, 8, 0), (8, 32, 0), (4, 4, 1), (32, 32, 0)):
            greqs.append((w, h, split, sx, sx, 0, off))
            p0.append(rng.integers(0, 256, w * h))
            p1.append(rng.integers(0, 256, w * h))
            off += w * h
    greqs = np.array(greqs, pkg.GPM_REQ_DTYPE)
    p0, p1 = np.concatenate(p0), np.concatenate(p1)
    out = torch.zeros(off, dtype=torch.int32, device="cuda")
    ctx.gpm_blend(greqs, _cuda(p0), _cuda(p1), out)
    got = out.cpu().numpy()
    for r in greqs:
        o, w, h = int(r["off"]), int(r["w"]), int(r["h"])
        want = orc.gpm(p0[o:o + w * h], p1[o:o + w * h], w, h, int(r["split_dir"]), int(r["scale_x"]), int(r["scale_y"]))
        assert np.array_equal(got[o:o + w * h], want), (int(r["split_dir"]), w, h)


def test_inter_tools_reject_bad_requests(ctx, pkg):
    import torch

    z = torch.zeros(64, dtype=torch.int32, device="cuda")
    with pytest.raises(pkg.InvalidInput):
        ctx.bdof(np.array([(6, 8, 0)], pkg.BDOF_REQ_DTYPE), z, z, z)
    with pytest.raises(pkg.InvalidInput):
        ctx.gpm_blend(np.array([(8, 8, 64, 0, 0, 0, 0)], pkg.GPM_REQ_DTYPE), z, z, z)
    with pytest.raises(pkg.InvalidInput):
        ctx.ciip_blend(np.array([(65, 0, 0, 0, (0, 0))], pkg.CIIP_REQ_DTYPE), z, z, z)
