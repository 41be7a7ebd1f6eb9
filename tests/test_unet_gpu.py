"""The pressure-guess U-Net: forward and gradients of the tensor-core implementation
against the same network in torch float64 on the CPU (gradient check), and a short
training run that must reduce the loss.  BF16 activations bound the agreement: the
tolerances are 3e-2 (forward, norm-relative) and 8e-2 per layer for gradients."""
import numpy as np
import pytest

from coffee_sim_b200 import unet

torch = pytest.importorskip("torch")


def test_param_count_and_layout():
    n = unet.param_count()
    assert 240_000 < n < 260_000
    sl = unet.layer_slices()
    assert sl["head"][2] == n
    p = unet.init_params(0)
    assert p.shape == (n,) and np.isfinite(p).all()


def _inputs(dims, seed):
    g = torch.Generator().manual_seed(seed)
    nv = dims[0] * dims[1] * dims[2]
    feat = torch.randn(nv, unet.FEATURES, generator=g)
    feat[:, unet.REAL_INPUTS:] = 0.0
    feat = feat.to(torch.bfloat16)
    target = torch.randn(nv, generator=g)
    mask = (torch.rand(nv, generator=g) > 0.3).float()
    return feat, target, mask


@pytest.mark.gpu
def test_forward_and_gradients_match_float64_reference():
    from coffee_sim_b200.sim import engine_library

    dims = (8, 8, 8)
    params = unet.init_params(3)
    feat, target, mask = _inputs(dims, 5)
    net = unet.UNet(dims, engine_library(), params)
    net.pack()
    out = net.forward(feat.cuda())
    loss, dout = net.loss_and_grad(out, target.cuda(), mask.cuda())
    g = net.backward(dout).detach().cpu().double()
    torch.cuda.synchronize()
    net.check_errors()

    pt = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    ref = unet.reference_forward(pt, feat.double(), dims)
    out_c = out.detach().cpu().double()
    assert torch.linalg.norm(out_c - ref.detach()) <= 3e-2 * torch.linalg.norm(ref.detach())
    ref_loss = ((ref - target.double()) * mask.double()).pow(2).sum() / mask.sum()
    ref_loss.backward()
    assert abs(loss.item() - ref_loss.item()) <= 5e-2 * ref_loss.item()
    gr = pt.grad
    for name, (a, b, c) in unet.layer_slices().items():
        for lo, hi, what in ((a, b, "w"), (b, c, "b")):
            d = torch.linalg.norm(g[lo:hi] - gr[lo:hi])
            s = torch.linalg.norm(gr[lo:hi])
            assert d <= 8e-2 * s + 1e-6, (name, what, float(d / max(s, 1e-30)))


@pytest.mark.gpu
def test_training_reduces_the_loss():
    from coffee_sim_b200.sim import engine_library

    dims = (16, 16, 16)
    feat, _, mask = _inputs(dims, 7)
    # a target the network can learn: a function of the inputs
    target = feat[:, 0].float() * 0.5 + feat[:, 2].float() * 0.25
    net = unet.UNet(dims, engine_library(), seed=1)
    f, t, m = feat.cuda(), target.cuda(), mask.cuda()
    first = None
    for k in range(150):
        loss = net.train_step(f, t, m, lr=2e-3)
        if k == 0:
            first = loss.item()
    last = loss.item()
    net.check_errors()
    assert last < 0.2 * first, (first, last)
