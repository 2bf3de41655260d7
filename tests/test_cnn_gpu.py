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


def _blocks(n, bd, seed):
    import torch
    from rustmpeg_next_b200 import synth

    y, _, _ = synth.value_noise_frame(32 * 8, max(64, 32 * ((n + 7) // 8)), 10, frame=seed)
    y = y.astype(np.int32)
    y = y << (bd - 10) if bd >= 10 else y >> (10 - bd)
    plane = np.ascontiguousarray(y.astype(np.uint16))
    xy = np.array([[32 * (i % 8), 32 * (i // 8)] for i in range(n)], np.int32)
    blocks = np.stack([plane[yy:yy + 32, xx:xx + 32] for xx, yy in xy]).astype(np.float32)
    return torch.from_numpy(plane.view(np.int16)).cuda(), torch.from_numpy(xy).cuda(), blocks


@pytest.mark.parametrize("n,bd,seed", [(1, 10, 1), (37, 10, 2), (300, 8, 3)])
def test_cnn_forward_matches_fp32_reference(ctx, pkg, n, bd, seed):
    import torch
    from rustmpeg_next_b200 import cnn

    plane, xy, blocks = _blocks(n, bd, seed)
    params = cnn.init_params(seed)
    qp = 22 + 5 * seed
    logits, gap, acts = ctx.cnn_forward(plane, bd, xy, torch.from_numpy(params).cuda(), qp, want_acts=True)
    ref_logits, ref_gap, ref_acts = cnn.reference_forward(blocks, bd, params, qp)
    # layer 1 is fp32 on both sides: equal up to summation order and bf16 ties
    a1 = acts[:, 0].float().cpu().reshape(n, 32, 32, 32).permute(0, 3, 1, 2)
    assert (a1 - ref_acts[0]).abs().max() <= 1e-2 * max(1.0, float(ref_acts[0].abs().max()))
    for l in (1, 2, 3):
        got = acts[:, l].float().cpu().reshape(n, 32, 32, 32).permute(0, 3, 1, 2)
        err = (got - ref_acts[l]).abs().max() / max(1e-6, float(ref_acts[l].abs().max()))
        assert err < 2e-2, (l, float(err))
    assert torch.allclose(gap.cpu(), ref_gap, rtol=2e-2, atol=2e-3), (gap.cpu() - ref_gap).abs().max()
    assert torch.allclose(logits.cpu(), ref_logits, rtol=2e-2, atol=2e-2), (logits.cpu() - ref_logits).abs().max()


@pytest.mark.parametrize("n,seed", [(3, 1), (150, 2)])
def test_cnn_gradients_match_autograd(ctx, pkg, n, seed):
    """Loss and the gradient of every parameter group against PyTorch
    autograd through the fp32 restatement."""
    import torch
    from rustmpeg_next_b200 import cnn

    plane, xy, blocks = _blocks(n, 10, seed)
    rng = np.random.default_rng(seed)
    labels = np.stack([rng.integers(0, 67, n), rng.integers(0, 6, n)], axis=1).astype(np.uint8)
    params = cnn.init_params(seed)
    p = torch.from_numpy(params).cuda()
    loss, grads = ctx.cnn_train_step(plane, 10, 27, xy, torch.from_numpy(labels).cuda(), p)
    ref_loss, ref = cnn.reference_loss_and_grads(blocks, labels, 10, params, 27)
    assert abs(float(loss.item()) - ref_loss) <= 1e-3 * max(1.0, abs(ref_loss))
    g = grads.cpu().numpy()
    groups = [("w1", cnn.OFF_W1, 576), ("b1", cnn.OFF_B1, 32)] + \
        [(f"w{l}", cnn.off_w(l), 9216) for l in (2, 3, 4)] + [(f"b{l}", cnn.off_b(l), 32) for l in (2, 3, 4)] + \
        [("wi", cnn.OFF_WI, 67 * 32), ("bi", cnn.OFF_BI, 67), ("ws", cnn.OFF_WS, 192), ("bs", cnn.OFF_BS, 6)]
    for name, off, cnt in groups:
        a, b = g[off:off + cnt], ref[off:off + cnt]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel < 3e-2, (name, rel)
    # params untouched without a learning rate
    assert torch.equal(p.cpu(), torch.from_numpy(params))


@pytest.mark.parametrize("n,seed", [(5, 3), (150, 4)])
def test_cnn_soft_target_gradients_match_autograd(ctx, pkg, n, seed):
    """The mode head trained against a distribution over the 67 modes (the
    softmax of negated search costs): loss and gradients against autograd."""
    import torch
    from rustmpeg_next_b200 import cnn

    plane, xy, blocks = _blocks(n, 10, seed)
    rng = np.random.default_rng(seed)
    labels = np.stack([rng.integers(0, 67, n), rng.integers(0, 6, n)], axis=1).astype(np.uint8)
    z = rng.normal(0.0, 2.0, (n, 67))
    soft = (np.exp(z - z.max(1, keepdims=True)) / np.exp(z - z.max(1, keepdims=True)).sum(1, keepdims=True))
    soft = soft.astype(np.float32)
    params = cnn.init_params(seed)
    p = torch.from_numpy(params).cuda()
    loss, grads = ctx.cnn_train_step(plane, 10, 27, xy, torch.from_numpy(labels).cuda(), p,
                                     soft=torch.from_numpy(soft).cuda())
    ref_loss, ref = cnn.reference_loss_and_grads(blocks, labels, 10, params, 27, soft=soft)
    assert abs(float(loss.item()) - ref_loss) <= 1e-3 * max(1.0, abs(ref_loss))
    g = grads.cpu().numpy()
    for name, off, cnt in [("w1", cnn.OFF_W1, 576), ("wi", cnn.OFF_WI, 67 * 32), ("bi", cnn.OFF_BI, 67),
                           ("ws", cnn.OFF_WS, 192), ("w4", cnn.off_w(4), 9216)]:
        a, b = g[off:off + cnt], ref[off:off + cnt]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel < 3e-2, (name, rel)
    # a one-hot soft target is the hard label
    onehot = np.zeros((n, 67), np.float32)
    onehot[np.arange(n), labels[:, 0]] = 1.0
    l1, g1 = ctx.cnn_train_step(plane, 10, 27, xy, torch.from_numpy(labels).cuda(), p,
                                soft=torch.from_numpy(onehot).cuda())
    l0, g0 = ctx.cnn_train_step(plane, 10, 27, xy, torch.from_numpy(labels).cuda(), p)
    assert abs(float(l1.item()) - float(l0.item())) <= 1e-5 * max(1.0, abs(float(l0.item())))
    assert torch.allclose(g1, g0, rtol=1e-4, atol=1e-7)


def test_cnn_adam_steps_reduce_the_loss(ctx, pkg):
    import torch
    from rustmpeg_next_b200 import cnn

    plane, xy, blocks = _blocks(256, 10, 7)
    # labels that the network can learn: classes of the block's brightness
    mean = blocks.mean(axis=(1, 2)) / 1023.0
    span = (mean - mean.min()) / max(1e-6, float(mean.max() - mean.min()))
    labels = torch.from_numpy(np.stack([np.minimum((span * 8).astype(int), 7) * 8,
                                        np.minimum((span * 6).astype(int), 5)], 1).astype(np.uint8))
    p = torch.from_numpy(cnn.init_params(7)).cuda()
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    losses = []
    for step in range(1, 41):
        loss, _ = ctx.cnn_train_step(plane, 10, 37, xy, labels.cuda(), p, m, v, step, 3e-3)
        losses.append(float(loss.item()))
    assert losses[-1] < 0.7 * losses[0], losses


def test_cnn_training_is_deterministic(ctx, pkg):
    """Two runs of the same training steps give bit-identical losses and
    parameters: every gradient and the loss are summed in a fixed order (no
    floating-point atomics)."""
    import torch
    from rustmpeg_next_b200 import cnn

    plane, xy, blocks = _blocks(512, 10, 9)
    mean = blocks.mean(axis=(1, 2)) / 1023.0
    labels = torch.from_numpy(np.stack([(mean * 60).astype(int) % 67, (mean * 50).astype(int) % 6],
                                       1).astype(np.uint8)).cuda()
    runs = []
    for _ in range(2):
        p = torch.from_numpy(cnn.init_params(9)).cuda()
        m, v = torch.zeros_like(p), torch.zeros_like(p)
        losses = []
        for step in range(1, 11):
            loss, _ = ctx.cnn_train_step(plane, 10, 32, xy, labels, p, m, v, step, 1e-3)
            losses.append(float(loss.item()))
        runs.append((losses, p.cpu().numpy()))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1])
