"""GPU: destroying a context returns every device buffer it grew (CTU
search, CNN training and motion-estimation workspaces included): device
memory after several create / use / destroy cycles equals what it was after
the first."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cycle(pkg, plane, xy, labels, params):
    from test_inter_search_oracle import random_case
    import torch

    c = pkg.Context(0)
    try:
        c.ctu_search_xy(plane, 10, 300, xy)
        c.cnn_forward(plane, 10, xy, params, 32)
        c.cnn_train_step(plane, 10, 32, xy, labels, params)
        src, refs0, refs1, cands, reqs = random_case(pkg, 3, n_req=20)
        c.inter_search_8(torch.from_numpy(src).cuda(), [torch.from_numpy(r).cuda() for r in refs0], [], cands, reqs)
        torch.cuda.synchronize()
    finally:
        c.close()


def test_destroy_returns_device_memory(pkg):
    import torch
    from rustmpeg_next_b200 import cnn

    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    pkg.build()
    h, w = 512, 1024
    plane = torch.randint(0, 1024, (h, w), dtype=torch.int16, device="cuda")
    xs, ys = np.meshgrid(np.arange(0, w - 31, 32), np.arange(0, h - 31, 32))
    xy = torch.from_numpy(np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32)).cuda()
    labels = torch.zeros((xy.shape[0], 2), dtype=torch.uint8, device="cuda")
    params = torch.from_numpy(cnn.init_params(1)).cuda()
    _cycle(pkg, plane, xy, labels, params)  # first use: module, tables and torch's cache settle
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(4):
        _cycle(pkg, plane, xy, labels, params)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 - free1 < (16 << 20), (free0 - free1) / 2**20
