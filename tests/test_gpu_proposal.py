"""The proposal network's device steps against plain PyTorch fp32 references of
the same operations: the tcgen05 GEMM (every epilogue mode), the strided
convolution built from im2col + GEMM, the full forward and backward pass of
the network, the binning of light curves and the top-k selection.

Operands are bf16 (inputs rounded to bf16 for the fp32 reference too) and the
tensor cores accumulate in fp32, so a GEMM's fp32 output matches to ~1e-5
relative; bf16 outputs are compared at bf16 precision (2^-8 relative); the
backward pass, which rounds its intermediate gradients to bf16, is compared by
relative L2 error (<= 3e-2) per parameter.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    # the references in true fp32 (cuDNN convolutions default to TF32)
    torch.backends.cudnn.allow_tf32 = False
    torch.backends.cuda.matmul.allow_tf32 = False
    return torch


@pytest.fixture(scope="module")
def ops():
    from cuperiod_b200.proposal import Ops
    return Ops()


def _bf(torch, shape, seed, scale=1.0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    return (torch.randn(shape, generator=g) * scale).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (300, 64, 448), (256, 200, 104),
                                   (1000, 256, 512), (64, 1024, 256), (129, 512, 16)])
def test_gemm_matches_torch(torch, ops, M, N, K):
    A = _bf(torch, (M, K), 1)
    B = _bf(torch, (N, K), 2)
    ref = A.float() @ B.float().T
    out = torch.empty((M, N), dtype=torch.float32, device="cuda")
    ops.gemm(A, B, out, M=M, N=N, K=K, lda=K, ldb=K, ldo=N, mode=1)
    ops.check()
    torch.testing.assert_close(out, ref, rtol=1e-4, atol=1e-3 * float(ref.abs().max()))


def test_gemm_epilogues(torch, ops):
    M, N, K = 384, 128, 320
    A = _bf(torch, (M, K), 3)
    B = _bf(torch, (N, K), 4)
    bias = torch.randn(N, device="cuda")
    ref = A.float() @ B.float().T + bias
    # bias + ReLU, bf16 store
    out = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
    ops.gemm(A, B, out, M=M, N=N, K=K, lda=K, ldb=K, ldo=N, mode=0, bias=bias, relu=True)
    ops.check()
    torch.testing.assert_close(out.float(), ref.clamp_min(0.0), rtol=1e-2, atol=1e-2)
    # mask by a bf16 tensor's sign
    mask = _bf(torch, (M, N), 5)
    out2 = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
    ops.gemm(A, B, out2, M=M, N=N, K=K, lda=K, ldb=K, ldo=N, mode=0, bias=bias, mask=mask)
    ops.check()
    torch.testing.assert_close(out2.float(), torch.where(mask.float() > 0, ref, 0.0),
                               rtol=1e-2, atol=1e-2)
    # split-K atomic accumulation into a transposed fp32 output, twice
    acc = torch.zeros((N, M), dtype=torch.float32, device="cuda")
    for _ in range(2):
        ops.gemm(A, B, acc, M=M, N=N, K=K, lda=K, ldb=K, ldo=M, mode=2, transpose=True,
                 bias=bias, splits=3)
    ops.check()
    torch.testing.assert_close(acc, 2.0 * ref.T, rtol=1e-4, atol=1e-3 * float(ref.abs().max()))


@pytest.mark.parametrize("C,L", [(2, 4096), (64, 128)])
def test_strided_convolution_matches_torch(torch, ops, C, L):
    import torch.nn.functional as F

    from cuperiod_b200.proposal import WIDTH, kp
    B, O = 3, 64
    k = kp(0 if C == 2 else 1)
    x = _bf(torch, (B, L, C), 6)
    w = _bf(torch, (O, C, WIDTH), 7, 0.2)
    # the GEMM's weight layout: column k*C + c holds tap k of input channel c
    wk = torch.zeros((O, k), dtype=torch.bfloat16, device="cuda")
    wk[:, :WIDTH * C] = w.permute(0, 2, 1).reshape(O, WIDTH * C)
    col = torch.empty((B * L // 2, k), dtype=torch.bfloat16, device="cuda")
    ops.im2col(x, col, B, L, C, k)
    y = torch.empty((B * L // 2, O), dtype=torch.float32, device="cuda")
    ops.gemm(col, wk, y, M=B * L // 2, N=O, K=k, lda=k, ldb=k, ldo=O, mode=1)
    ops.check()
    ref = F.conv1d(x.float().permute(0, 2, 1), w.float(), stride=2, padding=3)   # (B, O, L/2)
    torch.testing.assert_close(y.view(B, L // 2, O), ref.permute(0, 2, 1), rtol=1e-4, atol=1e-3)


def _torch_net(torch, weights):
    import torch.nn.functional as F

    from cuperiod_b200.proposal import CHANNELS, IN_CHANNELS, N_CONV, WIDTH
    params = [torch.tensor(a, device="cuda").to(torch.bfloat16).float().requires_grad_(True)
              for a in weights.arrays()]

    def bf(t):
        # the device keeps activations (and so their gradients) in bf16
        return t.to(torch.bfloat16).float()

    def forward(x):
        act = x.float().permute(0, 2, 1)
        for layer in range(N_CONV):
            c = IN_CHANNELS if layer == 0 else CHANNELS
            w = params[layer][:, :WIDTH * c].reshape(CHANNELS, WIDTH, c).permute(0, 2, 1)
            act = bf(F.relu(F.conv1d(act, w, params[N_CONV + layer], stride=2, padding=3)))
        flat = act.permute(0, 2, 1).reshape(act.shape[0], -1)
        h = bf(F.relu(flat @ params[2 * N_CONV].T + params[2 * N_CONV + 1]))
        return h @ params[2 * N_CONV + 2].T + params[2 * N_CONV + 3]
    return params, forward


def test_network_forward_and_backward_match_torch(torch):
    from cuperiod_b200.proposal import (IN_CHANNELS, N_BINS, N_CLASSES, ProposalNet, Weights)
    w = Weights.init(seed=3)
    net = ProposalNet(w, train=True)
    B = 16
    x = _bf(torch, (B, N_BINS, IN_CHANNELS), 8)
    labels = torch.randint(0, N_CLASSES, (B,), dtype=torch.int32, device="cuda")
    logits = net.forward(x)
    d, loss = net.loss_and_grad(logits, labels, side=0.1)
    net.zero_grad()
    net.backward(d)
    net.ops.check()

    params, fwd = _torch_net(torch, w)
    ref = fwd(x)
    rel = float((logits - ref.detach()).norm() / ref.detach().norm())
    assert rel < 2e-2, rel
    tgt = torch.zeros_like(ref)
    lab = labels.long()
    tgt[torch.arange(B), lab] += 0.8
    tgt[torch.arange(B), (lab - 1).clamp_min(0)] += 0.1
    tgt[torch.arange(B), (lab + 1).clamp_max(N_CLASSES - 1)] += 0.1
    ref_loss = -(tgt * torch.log_softmax(ref, dim=1)).sum()
    assert abs(float(loss.item()) - float(ref_loss.detach())) <= 2e-2 * abs(float(ref_loss.detach()))
    (ref_loss / B).backward()
    errs = [float((g - p.grad).norm() / max(float(p.grad.norm()), 1e-12))
            for g, p in zip(net.g, params)]
    assert max(errs) < 3e-2, errs


def test_adam_step_moves_the_loss_down(torch):
    from cuperiod_b200.proposal import IN_CHANNELS, N_BINS, N_CLASSES, ProposalNet, Weights
    net = ProposalNet(Weights.init(seed=4), train=True)
    B = 32
    x = _bf(torch, (B, N_BINS, IN_CHANNELS), 9)
    labels = torch.randint(0, N_CLASSES, (B,), dtype=torch.int32, device="cuda")
    losses = []
    for _ in range(30):
        logits = net.forward(x)
        d, loss = net.loss_and_grad(logits, labels)
        losses.append(float(loss.item()) / B)
        net.zero_grad()
        net.backward(d)
        net.adam(1e-3)
    net.ops.check()
    assert losses[-1] < 0.5 * losses[0], losses


def test_binning_and_topk(torch, ops):
    from cuperiod_b200.proposal import N_BINS, ProposalNet, Weights
    rng = np.random.default_rng(0)
    curves = [np.sort(rng.uniform(0.0, 27.0, n)) for n in (500, 3000)]
    ys = [1.0 + rng.normal(0.0, 1e-3, t.size) for t in curves]
    t = torch.tensor(np.concatenate(curves), device="cuda")
    y = torch.tensor(np.concatenate(ys), device="cuda")
    off = torch.tensor([0, curves[0].size, curves[0].size + curves[1].size], dtype=torch.int64,
                       device="cuda")
    out = torch.empty((2, N_BINS, 2), dtype=torch.bfloat16, device="cuda")
    ops.bin_curves(t, y, off, 2, out)
    ops.check()
    got = out.float().cpu().numpy()
    for c, (tc, yc) in enumerate(zip(curves, ys)):
        k = np.clip(((tc - tc.min()) * (N_BINS / (tc.max() - tc.min()))).astype(int), 0,
                    N_BINS - 1)
        z = (yc - yc.mean()) / yc.std()
        s = np.bincount(k, z, N_BINS)
        n = np.bincount(k, None, N_BINS)
        mean = np.where(n > 0, s / np.maximum(n, 1), 0.0)
        np.testing.assert_array_equal(got[c, :, 1], (n > 0).astype(float))
        np.testing.assert_allclose(got[c, :, 0], mean, rtol=1e-2, atol=2e-2)
    net = ProposalNet(Weights.init(seed=1))
    logits = torch.randn((5, 1024), device="cuda")
    idx, mass = net.topk(logits, 16)
    ops.check()
    ref = torch.topk(logits, 16, dim=1)
    assert torch.equal(idx.long(), ref.indices)
    torch.testing.assert_close(mass, torch.softmax(logits, 1).gather(1, ref.indices).sum(1),
                               rtol=1e-4, atol=1e-5)
