"""GPU parity: batched motion-compensation interpolation against the oracle's
restatement of inter.rs (interpolate_luma_block_16,
interpolate_chroma_block_format_16, weighted_average_bi_16), bit-exact, over
all 16 (luma) / 32 (chroma) fractional phases, bi and uni outputs, affine and
alternative half-pel taps, blocks reaching outside the picture, bit depths
8/10/12."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run_blocks(ctx, pkg, ref, bd, blocks, chroma=0):
    import torch

    dev = torch.device("cuda:0")
    t_ref = torch.from_numpy(ref.astype(np.int16)).to(dev)
    arr = np.zeros(len(blocks), pkg.MC_BLOCK_DTYPE)
    off = 0
    for i, b in enumerate(blocks):
        for k in ("x", "y", "w", "h", "mv_x", "mv_y", "flags"):
            arr[i][k] = b[k]
        arr[i]["out_offset"] = off
        off += b["w"] * b["h"]
    t_blk = torch.from_numpy(arr.view(np.uint8)).to(dev)
    out = torch.zeros(off, dtype=torch.int32, device=dev)
    if chroma:
        ctx.mc_chroma(t_ref, bd, chroma, t_blk, out)
    else:
        ctx.mc_luma(t_ref, bd, t_blk, out)
    torch.cuda.synchronize()
    return out.cpu().numpy(), arr


@pytest.mark.parametrize("bd", [8, 10, 12])
def test_luma_mc_matches_oracle(ctx, pkg, orc, bd):
    rng = np.random.default_rng(bd)
    H, W = 96, 160
    ref = rng.integers(0, 1 << bd, (H, W)).astype(np.uint16)
    blocks = []
    for fy in range(16):
        for fx in range(16):
            flags = int(rng.integers(0, 8))
            w, h = [(4, 4), (8, 8), (16, 8), (8, 32), (32, 32), (64, 16)][(fx + fy) % 6]
            x = int(rng.integers(-20, W))
            y = int(rng.integers(-20, H))
            mvx = int(rng.integers(-40, 40)) * 16 + fx
            mvy = int(rng.integers(-40, 40)) * 16 + fy
            blocks.append(dict(x=x, y=y, w=w, h=h, mv_x=mvx, mv_y=mvy, flags=flags))
    blocks.append(dict(x=10, y=5, w=128, h=72, mv_x=-37, mv_y=91, flags=0))
    blocks.append(dict(x=10, y=5, w=128, h=72, mv_x=-37, mv_y=91, flags=1))
    got, arr = run_blocks(ctx, pkg, ref, bd, blocks)
    for b, a in zip(blocks, arr):
        exp = orc.mc_luma(ref, bd, b["x"], b["y"], b["w"], b["h"], b["mv_x"], b["mv_y"],
                          bi=bool(b["flags"] & 1), affine=bool(b["flags"] & 2),
                          alt_hpel=bool(b["flags"] & 4))
        o = int(a["out_offset"])
        g = got[o:o + b["w"] * b["h"]].reshape(b["h"], b["w"])
        assert (g == exp).all(), b


@pytest.mark.parametrize("bd,cf", [(10, 1), (8, 2), (12, 3)])
def test_chroma_mc_matches_oracle(ctx, pkg, orc, bd, cf):
    rng = np.random.default_rng(100 + bd)
    H, W = 48, 80
    ref = rng.integers(0, 1 << bd, (H, W)).astype(np.uint16)
    blocks = []
    for ph in range(32):
        w, h = [(2, 2), (4, 4), (8, 4), (16, 16), (32, 8)][ph % 5]
        blocks.append(dict(x=int(rng.integers(-10, W)), y=int(rng.integers(-10, H)), w=w, h=h,
                           mv_x=int(rng.integers(-400, 400)) + ph, mv_y=int(rng.integers(-400, 400)) - ph,
                           flags=int(rng.integers(0, 2))))
    got, arr = run_blocks(ctx, pkg, ref, bd, blocks, chroma=cf)
    for b, a in zip(blocks, arr):
        exp = orc.mc_chroma(ref, bd, b["x"], b["y"], b["w"], b["h"], b["mv_x"], b["mv_y"],
                            bi=bool(b["flags"] & 1), cf=cf)
        o = int(a["out_offset"])
        g = got[o:o + b["w"] * b["h"]].reshape(b["h"], b["w"])
        assert (g == exp).all(), b


def test_bi_average_matches_oracle(ctx, pkg, orc):
    import torch

    rng = np.random.default_rng(7)
    for bd in (8, 10, 12):
        p0 = rng.integers(-9000, 9000, 4096).astype(np.int32)
        p1 = rng.integers(-9000, 9000, 4096).astype(np.int32)
        for bcw in range(5):
            t0 = torch.from_numpy(p0).cuda()
            t1 = torch.from_numpy(p1).cuda()
            out = torch.zeros(4096, dtype=torch.int16, device="cuda")
            ctx.mc_bi_average(t0, t1, bcw, bd, out)
            torch.cuda.synchronize()
            got = out.cpu().numpy().view(np.uint16)
            assert (got == orc.bi_average(p0, p1, bcw, bd)).all(), (bd, bcw)


def _blocks_8(rng, W, H, luma):
    blocks = []
    nph = 16 if luma else 32
    for fy in range(nph):
        for fx in range(0, nph, 3 if luma else 5):
            w, h = [(4, 4), (8, 8), (16, 8), (8, 32), (32, 32), (64, 16)][(fx + fy) % 6]
            scale = 16 if luma else 32
            blocks.append(dict(x=int(rng.integers(-20, W)), y=int(rng.integers(-20, H)), w=w, h=h,
                               mv_x=int(rng.integers(-40, 40)) * scale + fx, mv_y=int(rng.integers(-40, 40)) * scale + fy,
                               flags=int(rng.integers(0, 8)) if luma else int(rng.integers(0, 2))))
    return blocks


def test_luma_mc_8bit_matches_oracle(ctx, pkg, orc):
    """interpolate_luma_block (inter.rs:896-1051) on 8-bit planes, including its
    2-D uni-prediction rounding, which differs from the 16-bit function's."""
    import torch

    rng = np.random.default_rng(81)
    H, W = 96, 160
    ref = rng.integers(0, 256, (H, W)).astype(np.uint8)
    blocks = _blocks_8(rng, W, H, True)
    arr = np.zeros(len(blocks), pkg.MC_BLOCK_DTYPE)
    off = 0
    for i, b in enumerate(blocks):
        for k in ("x", "y", "w", "h", "mv_x", "mv_y", "flags"):
            arr[i][k] = b[k]
        arr[i]["out_offset"] = off
        off += b["w"] * b["h"]
    out = torch.zeros(off, dtype=torch.int32, device="cuda")
    ctx.mc_luma_8(torch.from_numpy(ref).cuda(), torch.from_numpy(arr.view(np.uint8)).cuda(), out)
    got = out.cpu().numpy()
    for b, a in zip(blocks, arr):
        exp = orc.mc_luma_8(ref, b["x"], b["y"], b["w"], b["h"], b["mv_x"], b["mv_y"], bi=bool(b["flags"] & 1),
                            affine=bool(b["flags"] & 2), alt_hpel=bool(b["flags"] & 4))
        o = int(a["out_offset"])
        assert (got[o:o + b["w"] * b["h"]].reshape(b["h"], b["w"]) == exp).all(), b


def test_chroma_mc_420_8bit_and_bi_average_match_oracle(ctx, pkg, orc):
    import torch

    rng = np.random.default_rng(82)
    H, W = 48, 80
    ref = rng.integers(0, 256, (H, W)).astype(np.uint8)
    blocks = _blocks_8(rng, W, H, False)
    arr = np.zeros(len(blocks), pkg.MC_BLOCK_DTYPE)
    off = 0
    for i, b in enumerate(blocks):
        for k in ("x", "y", "w", "h", "mv_x", "mv_y", "flags"):
            arr[i][k] = b[k]
        arr[i]["out_offset"] = off
        off += b["w"] * b["h"]
    out = torch.zeros(off, dtype=torch.int32, device="cuda")
    ctx.mc_chroma_420_8(torch.from_numpy(ref).cuda(), torch.from_numpy(arr.view(np.uint8)).cuda(), out)
    got = out.cpu().numpy()
    for b, a in zip(blocks, arr):
        exp = orc.mc_chroma_420_8(ref, b["x"], b["y"], b["w"], b["h"], b["mv_x"], b["mv_y"], bi=bool(b["flags"] & 1))
        o = int(a["out_offset"])
        assert (got[o:o + b["w"] * b["h"]].reshape(b["h"], b["w"]) == exp).all(), b
    # weighted_average_bi (inter.rs:1189) is the 16-bit average at bit depth 8
    p0 = rng.integers(-8192, 8192, 4096).astype(np.int32)
    p1 = rng.integers(-8192, 8192, 4096).astype(np.int32)
    for bcw in range(5):
        o16 = torch.zeros(4096, dtype=torch.int16, device="cuda")
        ctx.mc_bi_average(torch.from_numpy(p0).cuda(), torch.from_numpy(p1).cuda(), bcw, 8, o16)
        torch.cuda.synchronize()
        assert (o16.cpu().numpy().astype(np.int32) == orc.bi_average_8(p0, p1, bcw)).all()
