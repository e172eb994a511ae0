"""The learned corrector's BF16 tensor-core convolutions against an FP32 reference, its
gradients against the FP32 autograd of the same network on the CPU, and its training."""

import numpy as np
import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


def _bf16(t):
    return t.to(torch.bfloat16).float()


def _reference_conv(x, w, b=None):
    """x (B, H, W, C) -> (B, H, W, O) by torch's FP32 convolution."""
    y = F.conv2d(x.permute(0, 3, 1, 2), w, b, padding=2)
    return y.permute(0, 2, 3, 1)


@pytest.mark.parametrize("cin,cout", [(4, 32), (32, 32), (32, 2), (2, 32)])
def test_conv_forward_matches_fp32(cin, cout):
    from cuwave_b200 import _native as nat
    from cuwave_b200.corrector import pack

    gen = torch.Generator().manual_seed(cin * 100 + cout)
    x = torch.randn((2, 37, 29, cin), generator=gen).to(torch.bfloat16).cuda()
    w = torch.randn((cout, cin, 5, 5), generator=gen).cuda() * 0.1
    b = torch.randn(cout, generator=gen).cuda()
    y = torch.empty((2, 37, 29, cout), device="cuda")
    nat.conv_fwd(x, pack(w), b, y32=y)
    ref = _reference_conv(x.float(), _bf16(w), b)
    assert float((y - ref).norm() / ref.norm()) < 1e-5
    y16 = torch.empty((2, 37, 29, cout), dtype=torch.bfloat16, device="cuda")
    nat.conv_fwd(x, pack(w), b, y16=y16, relu=True)
    assert torch.allclose(y16.float(), ref.clamp(min=0), rtol=1e-2, atol=1e-2)


@pytest.mark.parametrize("cin,cout", [(4, 32), (32, 32), (32, 2)])
def test_conv_gradients_match_fp32_autograd(cin, cout):
    from cuwave_b200 import _native as nat
    from cuwave_b200.corrector import pack, pack_transposed, unpack

    gen = torch.Generator().manual_seed(7 + cin + cout)
    x = torch.randn((2, 33, 41, cin), generator=gen).relu().to(torch.bfloat16).cuda()
    w = _bf16(torch.randn((cout, cin, 5, 5), generator=gen).cuda() * 0.1)
    dy = torch.randn((2, 33, 41, cout), generator=gen).to(torch.bfloat16).cuda()
    xr = x.float().requires_grad_(True)
    wr = w.clone().requires_grad_(True)
    br = torch.zeros(cout, device="cuda", requires_grad=True)
    _reference_conv(xr, wr, br).backward(dy.float())
    dw = torch.zeros((cout, (25 * cin + 15) // 16 * 16), device="cuda")
    db = torch.zeros(cout, device="cuda")
    nat.conv_bwd(dy, x, dw, db)
    assert float((unpack(dw, cin) - wr.grad).norm() / wr.grad.norm()) < 1e-5
    assert float((db - br.grad).norm() / br.grad.norm()) < 1e-5
    dx = torch.empty((2, 33, 41, cin), device="cuda")
    nat.conv_fwd(dy, pack_transposed(w), None, y32=dx, mask=x)
    want = xr.grad * (x.float() > 0)
    assert float((dx - want).norm() / want.norm()) < 1e-5


def test_network_gradient_matches_the_cpu_autograd():
    """The whole network's backward (BF16 activations and gradients, FP32 sums) against
    torch's FP32 autograd of the same network on the CPU."""
    from cuwave_b200.corrector import CHANNELS, Corrector

    net = Corrector(seed=3)
    gen = torch.Generator().manual_seed(11)
    x = torch.randn((2, 24, 20, 4), generator=gen)
    x[..., 3] = 0
    x = x.to(torch.bfloat16)
    target = torch.randn((2, 24, 20, 2), generator=gen)
    out = net.forward(x.cuda())
    err = out - target.cuda()
    grads = net.backward(2.0 * err / err.numel())
    # the CPU reference, weights rounded to BF16 as the kernels read them
    ws = [_bf16(w).cpu().requires_grad_(True) for w in net.w]
    bs = [b.cpu().requires_grad_(True) for b in net.b]
    h = x.float()
    for k in range(len(ws)):
        h = _reference_conv(h, ws[k], bs[k])
        if k < len(ws) - 1:
            h = h.relu()
    loss = (h - target).pow(2).mean()
    loss.backward()
    assert len(CHANNELS) == 4
    for got, ref in zip(grads, [w.grad for w in ws] + [b.grad for b in bs]):
        ref = ref.cuda()
        scale = float(ref.norm())
        if scale == 0.0:
            continue
        assert float((got - ref).norm()) / scale < 5e-2


def test_training_lowers_the_loss():
    from cuwave_b200.corrector import Corrector, grid_pair, train, training_pairs

    pair = grid_pair(40, 1.0, 2.0, 260)
    rng = np.random.default_rng(0)
    inputs, targets = training_pairs(pair, rng, shots=2, windows=6)
    net = Corrector(seed=1)
    losses = train(net, inputs, targets, steps=150, batch=4, lr=2e-3)
    assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:5])
