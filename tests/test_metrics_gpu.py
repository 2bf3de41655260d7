"""GPU parity: plane metrics (vvcg_plane_metrics_8_dev / _16_dev) against the
oracle's CpuFrameMetrics::plane_metrics restatement: exact SSE, SAD and sample
counts for 8- and 16-bit planes, padded strides, unaligned views, ragged
widths and empty planes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,w,h,pad,off", [
    (np.uint8, 1920, 1080, 0, 0), (np.uint8, 37, 19, 5, 1), (np.uint8, 64, 64, 64, 0),
    (np.uint16, 1920, 1088, 64, 0), (np.uint16, 333, 77, 3, 1), (np.uint16, 960, 540, 0, 0),
    (np.uint8, 0, 10, 0, 0),
])
def test_plane_metrics_match_oracle(ctx, pkg, orc, dtype, w, h, pad, off):
    import torch

    rng = np.random.default_rng(w * 7 + h)
    maxv = 255 if dtype == np.uint8 else 4095
    base_a = rng.integers(0, maxv + 1, (h, w + pad + off)).astype(dtype)
    base_b = np.clip(base_a.astype(np.int32) + rng.integers(-40, 41, base_a.shape), 0, maxv).astype(dtype)
    a, b = base_a[:, off:off + w], base_b[:, off:off + w]
    want = orc.plane_metrics(np.ascontiguousarray(a), np.ascontiguousarray(b))
    tdt = torch.uint8 if dtype == np.uint8 else torch.int16
    ta = torch.from_numpy(base_a.view(np.int16) if dtype == np.uint16 else base_a).cuda()[:, off:off + w]
    tb = torch.from_numpy(base_b.view(np.int16) if dtype == np.uint16 else base_b).cuda()[:, off:off + w]
    assert ta.dtype == tdt
    got = ctx.plane_metrics(ta, tb)
    assert got == want


def test_plane_metrics_reject_mismatched_views(ctx, pkg):
    import torch

    a = torch.zeros((4, 8), dtype=torch.uint8, device="cuda")
    b = torch.zeros((4, 9), dtype=torch.uint8, device="cuda")
    with pytest.raises(pkg.InvalidInput, match="differ"):
        ctx.plane_metrics(a, b)
