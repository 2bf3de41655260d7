"""Host side of the CNN pruner: parameter layout, initialisation, and a
plain PyTorch fp32 restatement of the network used by the tests to check
the tensor-core kernels (the library itself runs only its CUDA kernels).

Parameter vector (fp32, CNN_PARAMS entries): conv1 W [32][2][9] and b[32]
(input 0: the samples, input 1: a constant plane QP / 63);
conv2..4 W [32 out][32 in][9] and b[32]; intra head W [67][32], b[67];
split head W [6][32], b[6]. Taps are row-major over (dy, dx) in -1..1.
"""
from __future__ import annotations

import numpy as np

CH, MODES, SPLITS = 32, 67, 6
OFF_W1, OFF_B1 = 0, 576


def off_w(layer):
    return 608 + (layer - 2) * (CH * CH * 9 + CH)


def off_b(layer):
    return off_w(layer) + CH * CH * 9


OFF_WI = off_w(5)
OFF_BI = OFF_WI + MODES * CH
OFF_WS = OFF_BI + MODES
OFF_BS = OFF_WS + SPLITS * CH
N_PARAMS = OFF_BS + SPLITS


def init_params(seed=0):
    """He-initialised weights, zero biases (fp32 numpy vector)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[OFF_W1:OFF_W1 + 576] = rng.normal(0, np.sqrt(2 / 18), 576)
    for layer in (2, 3, 4):
        p[off_w(layer):off_w(layer) + CH * CH * 9] = rng.normal(0, np.sqrt(2 / (CH * 9)), CH * CH * 9)
    p[OFF_WI:OFF_WI + MODES * CH] = rng.normal(0, np.sqrt(1 / CH), MODES * CH)
    p[OFF_WS:OFF_WS + SPLITS * CH] = rng.normal(0, np.sqrt(1 / CH), SPLITS * CH)
    return p


def unpack(params):
    """torch tensors (conv weights as [out, in, 3, 3]) from the vector."""
    import torch

    p = params if isinstance(params, torch.Tensor) else torch.as_tensor(params, dtype=torch.float32)
    w1 = p[OFF_W1:OFF_W1 + 576].reshape(CH, 2, 3, 3)
    b1 = p[OFF_B1:OFF_B1 + CH]
    convs = [(p[off_w(layer):off_w(layer) + CH * CH * 9].reshape(CH, CH, 3, 3), p[off_b(layer):off_b(layer) + CH])
             for layer in (2, 3, 4)]
    wi, bi = p[OFF_WI:OFF_WI + MODES * CH].reshape(MODES, CH), p[OFF_BI:OFF_BI + MODES]
    ws, bs = p[OFF_WS:OFF_WS + SPLITS * CH].reshape(SPLITS, CH), p[OFF_BS:OFF_BS + SPLITS]
    return w1, b1, convs, wi, bi, ws, bs


def qp_input(qp):
    """The constant input plane's value: QP / 63 rounded to bf16."""
    import torch

    return float(torch.tensor(qp / 63.0, dtype=torch.float32).to(torch.bfloat16).float())


def reference_forward(blocks, bit_depth, params, qp):
    """fp32 restatement of the kernels' forward pass on (n, 32, 32) sample
    blocks with the same bf16 roundings (input, activations of layers 1-3,
    conv weights of layers 2-4); returns (logits (n, 73), gap (n, 32),
    activations [a1..a4] as (n, 32, 32, 32) fp32)."""
    import torch
    import torch.nn.functional as F

    bf = lambda t: t.to(torch.bfloat16).to(torch.float32)  # noqa: E731
    w1, b1, convs, wi, bi, ws, bs = unpack(params)
    x = bf(torch.as_tensor(blocks, dtype=torch.float32)[:, None] * (1.0 / ((1 << bit_depth) - 1)))
    x = torch.cat([x, torch.full_like(x, qp_input(qp))], dim=1)
    a = bf(F.relu(F.conv2d(x, w1, b1, padding=1)))
    acts = [a]
    for i, (w, b) in enumerate(convs):
        wq = w + (bf(w) - w).detach()  # bf16 values, fp32 weight gradients
        a = F.relu(F.conv2d(a, wq, b, padding=1))
        if i < 2:
            a = bf(a)
        acts.append(a)
    gap = a.mean(dim=(2, 3))
    logits = torch.cat([gap @ wi.T + bi, gap @ ws.T + bs], dim=1)
    return logits, gap, acts


def reference_loss_and_grads(blocks, labels, bit_depth, params, qp, soft=None):
    """Mean cross-entropy of both heads and its gradient w.r.t. the
    parameter vector, by autograd through reference_forward (fp32 with the
    kernels' bf16 roundings). `soft` (N x 67 rows summing to 1) replaces the
    mode head's one-hot target."""
    import torch

    p = torch.tensor(np.asarray(params, np.float32), requires_grad=True)
    logits, _, _ = reference_forward(blocks, bit_depth, p, qp)
    lab = torch.as_tensor(np.asarray(labels), dtype=torch.long)
    mode_target = lab[:, 0] if soft is None else torch.as_tensor(np.asarray(soft, np.float32))
    loss = torch.nn.functional.cross_entropy(logits[:, :MODES], mode_target) + \
        torch.nn.functional.cross_entropy(logits[:, MODES:], lab[:, 1])
    loss.backward()
    return float(loss.detach()), p.grad.numpy()


def search_lambda_q8(qp, bit_depth=10):
    """lambda of the CTU search (SATD domain) in 1/256 units:
    sqrt(0.57 * 2^((qp - 12) / 3)) * 2^(bit_depth - 8)."""
    return int(round(256.0 * np.sqrt(0.57 * 2.0 ** ((qp - 12) / 3.0)) * 2.0 ** (bit_depth - 8)))


def training_set(ctx, n_frames=8, width=1920, height=1080, qps=(22, 27, 32, 37), seed=0, soft_t=None):
    """Labelled 32x32 luma blocks for the pruner: value-noise 10-bit frames
    (the 1080p synthetic content), every CTU labelled by the full search at
    each QP (intra mode of the unsplit CU, best split type). Returns a list
    of (plane (H, W) int16 CUDA, xy (n, 2) int32 CUDA, labels (n, 2) uint8
    CUDA, qp, soft) per frame and QP. With soft_t, soft ((n, 67) fp32 CUDA)
    is each CTU's target over the 67 modes of the unsplit CU,
    softmax(-(cost - best cost) / (soft_t * lambda)): modes within a few
    lambda-weighted bits of the best share the probability; else None."""
    import torch

    from . import synth

    out = []
    with ctx.torch_stream_scope():
        xs, ys = np.meshgrid(np.arange(0, width - 31, 32), np.arange(0, height - 31, 32))
        xy = torch.from_numpy(np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32)).cuda()
        _label_frames(ctx, synth, xy, out, n_frames, width, height, qps, seed, soft_t)
    return out


def _label_frames(ctx, synth, xy, out, n_frames, width, height, qps, seed, soft_t):
    import torch

    for f in range(n_frames):
        y, _, _ = synth.value_noise_frame(width, height, 10, frame=seed * 1000 + f)
        plane = torch.from_numpy(np.ascontiguousarray(y.astype(np.uint16)).view(np.int16)).cuda()
        for qp in qps:
            lam = search_lambda_q8(qp)
            soft = None
            if soft_t is None:
                r = ctx.ctu_search_xy(plane, 10, lam, xy)
            else:
                r, costs = ctx.ctu_search_costs(plane, 10, lam, xy)
                rel = (costs - costs.min(dim=1, keepdim=True).values).to(torch.float32)
                soft = torch.softmax(-rel / (soft_t * lam / 256.0), dim=1).contiguous()
            lab = torch.from_numpy(np.stack([r["cu_mode"], r["split"]], 1).astype(np.uint8)).cuda()
            out.append((plane, xy, lab, qp, soft))


def train(ctx, data, steps=300, batch=1024, lr=1e-3, seed=0, params=None, schedule="constant", lr_min=0.0):
    """Adam on the labelled blocks of training_set (batches drawn from one
    frame at a time); returns (params CUDA tensor, losses). schedule
    "cosine" decays the step size from lr to lr_min over the steps."""
    import torch

    rng = np.random.default_rng(seed)
    with ctx.torch_stream_scope():
        p = torch.from_numpy(init_params(seed) if params is None else params).cuda()
        m, v = torch.zeros_like(p), torch.zeros_like(p)
        losses = []
        for step in range(1, steps + 1):
            plane, xy, lab, qp, soft = data[int(rng.integers(0, len(data)))]
            idx = torch.from_numpy(rng.choice(xy.shape[0], min(batch, xy.shape[0]), replace=False)).cuda()
            lr_t = lr if schedule == "constant" else \
                lr_min + (lr - lr_min) * 0.5 * (1.0 + np.cos(np.pi * (step - 1) / max(1, steps)))
            loss, _ = ctx.cnn_train_step(plane, 10, qp, xy[idx], lab[idx], p, m, v, step, float(lr_t), sync=False,
                                         soft=None if soft is None else soft[idx])
            losses.append(loss)
        torch.cuda.synchronize()
    return p, [float(x.item()) for x in losses]
