"""GPU: the tensor-core (tcgen05) path of the CNN pruner against a plain
PyTorch fp32 reference (floating point; bf16 operands, fp32 accumulation)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tensor_core_selftest_matches_fp32_matmul(ctx, pkg):
    import torch

    g = torch.Generator(device="cpu").manual_seed(0)
    a = torch.randn((128, 16), generator=g).to(torch.bfloat16)
    b = torch.randn((32, 16), generator=g).to(torch.bfloat16)
    d = ctx.tc_selftest(a.cuda().view(torch.int16), b.cuda().view(torch.int16)).cpu()
    want = a.float() @ b.float().T
    assert torch.allclose(d, want, rtol=1e-5, atol=1e-5), (d - want).abs().max()
