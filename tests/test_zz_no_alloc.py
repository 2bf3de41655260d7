"""GPU: the allocation-free entry point vvcg_recon_picture_static.

Its output on device-resident records must equal vvcg_decode_batch's on the
same records, call after call: the calls share one fixed device array that
keeps the previous call's contents, so consecutive calls on different
pictures (size, bit depth, chroma format, CTU size, tools, plane strides)
are compared, and the device's free memory must not move across any call
after the first.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPECS = [
    dict(width=512, height=256, bit_depth=10, chroma_format=1, ctu_log2=5, qp=27),
    dict(width=256, height=256, bit_depth=12, chroma_format=2, ctu_log2=6, qp=33),
    dict(width=192, height=128, bit_depth=8, chroma_format=3, ctu_log2=5, qp=22),
    # chroma 80 samples wide: a stride that is a multiple of 8 but not of 64
    dict(width=160, height=96, bit_depth=10, chroma_format=1, ctu_log2=5, qp=30),
    dict(width=224, height=160, bit_depth=10, chroma_format=0, ctu_log2=5, qp=25),  # 4:0:0
]
TOOLS = [1 | 2, 2, 0, 2, 1 | 2]  # DEP_QUANT | DEBLOCK, DEBLOCK, none, DEBLOCK, DEP_QUANT | DEBLOCK
PAD = [0, 0, 0, 0, 24]  # extra samples per row beyond the plane width (stride > width)


def _inputs(pkg, k, seed):
    from rustmpeg_next_b200 import synth

    pics, cus, levels, ctus, _ = synth.random_records([SPECS[k]], seed=seed, tools=TOOLS[k])
    return pics, cus, levels, ctus


def _device_inputs(pkg, k, pics, cus, levels, seed):
    """Records, levels and planes on the device; the planes start with junk
    (they are the work space too) and, with PAD[k], have a stride larger
    than their width."""
    import torch

    p = pics[0]
    w, h, cf = int(p["width"]), int(p["height"]), int(p["chroma_format"])
    cw, ch = pkg.chroma_dims(w, h, cf)
    g = torch.Generator(device="cuda").manual_seed(seed)

    def plane(ph, pw):
        full = torch.randint(-32768, 32767, (ph, pw + PAD[k]), dtype=torch.int16, device="cuda", generator=g)
        return full[:, :pw]

    planes = [plane(h, w)] + ([plane(ch, cw), plane(ch, cw)] if cf else [None, None])
    d_cus = torch.from_numpy(cus.view(np.uint8).copy()).cuda()
    d_lev = torch.from_numpy(levels.astype(np.int16)).cuda()
    return d_cus, d_lev, planes


def test_static_entry_matches_decode_batch_on_consecutive_calls(ctx, pkg):
    import torch

    order = [(0, 101), (1, 202), (3, 505), (0, 303), (4, 606), (2, 404)]
    cases = []
    # every input and every expected output exists before the first static call
    for k, seed in order:
        pics, cus, levels, ctus = _inputs(pkg, k, seed)
        want = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus))[0]
        cases.append((k, pics, want, _device_inputs(pkg, k, pics, cus, levels, seed)))
    torch.cuda.synchronize()
    moved = []
    for i, (k, pics, want, (d_cus, d_lev, planes)) in enumerate(cases):
        torch.cuda.synchronize()
        free0, reserved0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
        pkg.recon_picture_static(pics[0], d_cus, d_lev, planes)
        torch.cuda.synchronize()
        free1, reserved1 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
        if i >= 1:  # the first call on the device may load the module
            moved.append((i, free0 - free1, reserved1 - reserved0))
        got = [None if t is None else t.cpu().numpy().view(np.uint16) for t in planes]
        for c in range(3):
            if want[c] is None:
                assert got[c] is None
                continue
            diff = np.argwhere(got[c] != want[c])
            assert diff.size == 0, f"call {i} (spec {k}) plane {c}: {len(diff)} samples differ, first {diff[:3].tolist()}"
    # calls after the first allocate nothing on the device
    assert all(f == 0 and r == 0 for _, f, r in moved), moved


def test_static_entry_rejects_what_it_cannot_hold(pkg):
    import torch

    pics, cus, levels, _ = _inputs(pkg, 0, 7)
    d_cus = torch.from_numpy(cus.view(np.uint8).copy()).cuda()
    d_lev = torch.from_numpy(levels.astype(np.int16)).cuda()
    p = pics[0]
    w, h = int(p["width"]), int(p["height"])
    planes = [torch.zeros((h, w), dtype=torch.int16, device="cuda"),
              torch.zeros((h // 2, w // 2), dtype=torch.int16, device="cuda"),
              torch.zeros((h // 2, w // 2), dtype=torch.int16, device="cuda")]
    tall = p.copy()
    tall["width"], tall["height"] = 32, 32 * 257  # one CTU row more than the array holds
    tall["visible_width"], tall["visible_height"] = 32, 32 * 257
    tall_planes = [torch.zeros((32 * 257, 32), dtype=torch.int16, device="cuda"),
                   torch.zeros((16 * 257, 16), dtype=torch.int16, device="cuda"),
                   torch.zeros((16 * 257, 16), dtype=torch.int16, device="cuda")]
    with pytest.raises(pkg.LimitExceeded, match="CTU rows"):
        pkg.recon_picture_static(tall, d_cus, d_lev, tall_planes)
    sao = p.copy()
    sao["tools"] = pkg.TOOL_SAO
    with pytest.raises(pkg.InvalidInput, match="SAO and ALF"):
        pkg.recon_picture_static(sao, d_cus, d_lev, planes)
    flat = torch.zeros(h * w + 1, dtype=torch.int16, device="cuda")
    odd = [flat[1:].view(h, w)] + planes[1:]  # 2-byte aligned luma plane
    with pytest.raises(pkg.InvalidInput, match="aligned"):
        pkg.recon_picture_static(p, d_cus, d_lev, odd)
    # checked in the binding, before the library sees the pointers
    with pytest.raises(pkg.InvalidInput, match="coded size"):
        pkg.recon_picture_static(p, d_cus, d_lev, [planes[0][: h - 8]] + planes[1:])
    with pytest.raises(pkg.InvalidInput, match="16-bit"):
        pkg.recon_picture_static(p, d_cus, d_lev, [planes[0].float()] + planes[1:])
    with pytest.raises(pkg.InvalidInput, match="unit column stride"):
        pkg.recon_picture_static(p, d_cus, d_lev, [planes[0].t().contiguous().t()] + planes[1:])
    with pytest.raises(pkg.InvalidInput, match="uint8"):
        pkg.recon_picture_static(p, d_cus.view(torch.int16), d_lev, planes)
    with pytest.raises(pkg.InvalidInput, match="int16"):
        pkg.recon_picture_static(p, d_cus, d_lev.int(), planes)
    with pytest.raises(pkg.InvalidInput, match="CUDA tensor"):
        pkg.recon_picture_static(p, d_cus.cpu(), d_lev, planes)
