"""GPU: the allocation-free entry point vvcg_recon_picture_static.

Its output on device-resident records must equal vvcg_decode_batch's on the
same records, call after call: the calls share one fixed device array that
keeps the previous call's contents, so consecutive calls on different
pictures (size, bit depth, chroma format, CTU size, tools) are compared, and
the device's free memory must not move across calls after the first.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPECS = [
    dict(width=512, height=256, bit_depth=10, chroma_format=1, ctu_log2=5, qp=27),
    dict(width=256, height=256, bit_depth=12, chroma_format=2, ctu_log2=6, qp=33),
    dict(width=192, height=128, bit_depth=8, chroma_format=3, ctu_log2=5, qp=22),
]
TOOLS = [1 | 2, 2, 0]  # DEP_QUANT | DEBLOCK, DEBLOCK, none


def _inputs(pkg, k, seed):
    from rustmpeg_next_b200 import synth

    pics, cus, levels, ctus, _ = synth.random_records([SPECS[k]], seed=seed, tools=TOOLS[k])
    return pics, cus, levels, ctus


def _static_call(pkg, pics, cus, levels, seed):
    import torch

    p = pics[0]
    w, h, cf = int(p["width"]), int(p["height"]), int(p["chroma_format"])
    cw, ch = pkg.chroma_dims(w, h, cf)
    g = torch.Generator(device="cuda").manual_seed(seed)
    # the planes are also the work space: start them with junk
    planes = [torch.randint(-32768, 32767, (h, w), dtype=torch.int16, device="cuda", generator=g)]
    if cf:
        planes += [torch.randint(-32768, 32767, (ch, cw), dtype=torch.int16, device="cuda", generator=g)
                   for _ in range(2)]
    else:
        planes += [None, None]
    d_cus = torch.from_numpy(cus.view(np.uint8).copy()).cuda()
    d_lev = torch.from_numpy(levels.astype(np.int16)).cuda()
    torch.cuda.synchronize()
    pkg.recon_picture_static(p, d_cus, d_lev, planes)
    return [None if t is None else t.cpu().numpy().view(np.uint16) for t in planes]


def test_static_entry_matches_decode_batch_on_consecutive_calls(ctx, pkg):
    import torch

    order = [(0, 101), (1, 202), (0, 303), (2, 404)]
    free = []
    for i, (k, seed) in enumerate(order):
        pics, cus, levels, ctus = _inputs(pkg, k, seed)
        want = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus))[0]
        if i >= 1:
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info()[0])
        got = _static_call(pkg, pics, cus, levels, seed)
        for c in range(3):
            if want[c] is None:
                continue
            diff = np.argwhere(got[c] != want[c])
            assert diff.size == 0, f"call {i} plane {c}: {len(diff)} samples differ, first {diff[:3].tolist()}"
    torch.cuda.synchronize()
    free.append(torch.cuda.mem_get_info()[0])
    # calls after the first allocate nothing on the device
    assert len(set(free)) == 1, free


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
    with pytest.raises(pkg.LimitExceeded, match="CTU rows"):
        pkg.recon_picture_static(tall, d_cus, d_lev, planes)
    sao = p.copy()
    sao["tools"] = pkg.TOOL_SAO
    with pytest.raises(pkg.InvalidInput, match="SAO and ALF"):
        pkg.recon_picture_static(sao, d_cus, d_lev, planes)
    flat = torch.zeros(h * w + 1, dtype=torch.int16, device="cuda")
    odd = [flat[1:].view(h, w)] + planes[1:]  # 2-byte aligned luma plane
    with pytest.raises(pkg.InvalidInput, match="aligned"):
        pkg.recon_picture_static(p, d_cus, d_lev, odd)
