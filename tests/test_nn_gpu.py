"""Tensor-core (tcgen05) BF16 3-D convolution layers against torch's float32 convolution
of the same bf16-rounded operands: forward (+bias, ReLU), input gradient (flipped
weights), weight gradient."""
import ctypes as C

import numpy as np
import pytest

from coffee_sim_b200.sim import engine_library

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
F = torch.nn.functional


def _lib():
    return engine_library()


def _p(t):
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _pack(w, cin_pad, cout_pad, flip=False):
    cout, _, cin = w.shape
    if flip:
        rows, kin = (cin + 15) // 16 * 16, cout_pad
    else:
        rows, kin = cout_pad, cin_pad
    kpad = (27 * kin + 63) // 64 * 64
    out = torch.zeros(rows, kpad, dtype=torch.bfloat16, device="cuda")
    _lib().call("cs_nn_pack_weights", _p(w), _p(out), cin, cin_pad if not flip else cin_pad, cout, cout_pad,
                1 if flip else 0, _stream())
    return out


def _to_ncdhw(x, dims, c):
    gx, gy, gz = dims
    return x[:, :c].float().reshape(gz, gy, gx, c).permute(3, 0, 1, 2).unsqueeze(0)


def _torch_w(w):
    cout, _, cin = w.shape
    # tap t = (dz+1)*9 + (dy+1)*3 + (dx+1)  ->  kernel index [kz][ky][kx]
    return w.reshape(cout, 3, 3, 3, cin).permute(0, 4, 1, 2, 3).contiguous()


@pytest.mark.parametrize("dims,cin,cout", [((12, 10, 9), 16, 16), ((8, 8, 8), 8, 32), ((16, 6, 5), 32, 64)])
def test_conv_forward_matches_torch(dims, cin, cout):
    torch.manual_seed(0)
    gx, gy, gz = dims
    nv = gx * gy * gz
    x = torch.randn(nv, cin, device="cuda").to(torch.bfloat16)
    w = (torch.randn(cout, 27, cin, device="cuda") * 0.1).contiguous()
    b = torch.randn(cout, device="cuda").contiguous()
    wp = _pack(w, cin, cout)
    y = torch.zeros(nv, cout, dtype=torch.bfloat16, device="cuda")
    y32 = torch.zeros(nv, cout, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib().call("cs_nn_conv3d", _p(x), _p(wp), _p(b), _p(y), _p(y32), gx, gy, gz, cin, cout, 1, _p(err), _stream())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    wb = w.to(torch.bfloat16).float()
    ref = F.relu(F.conv3d(_to_ncdhw(x, dims, cin), _torch_w(wb), b, padding=1))
    ref = ref.squeeze(0).permute(1, 2, 3, 0).reshape(nv, cout)
    scale = ref.abs().max().item()
    assert (y32 - ref).abs().max().item() <= 1e-4 * scale + 1e-5
    assert (y.float() - ref).abs().max().item() <= 1e-2 * scale


@pytest.mark.parametrize("dims,cin,cout", [((12, 10, 9), 16, 16), ((8, 8, 8), 32, 64)])
def test_conv_gradients_match_torch(dims, cin, cout):
    torch.manual_seed(1)
    gx, gy, gz = dims
    nv = gx * gy * gz
    x = torch.randn(nv, cin, device="cuda").to(torch.bfloat16)
    dy = torch.randn(nv, cout, device="cuda").to(torch.bfloat16)
    w = (torch.randn(cout, 27, cin, device="cuda") * 0.1).contiguous()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    # input gradient: the convolution with flipped, transposed weights
    wf = _pack(w, cin, cout, flip=True)
    cinp16 = (cin + 15) // 16 * 16
    dx32 = torch.zeros(nv, cinp16, dtype=torch.float32, device="cuda")
    _lib().call("cs_nn_conv3d", _p(dy), _p(wf), None, None, _p(dx32), gx, gy, gz, cout, cinp16, 0, _p(err),
                _stream())
    # weight gradient, split over CTAs
    dwt = torch.zeros(27 * cin, cout, dtype=torch.float32, device="cuda")
    _lib().call("cs_nn_conv3d_wgrad", _p(x), _p(dy), _p(dwt), gx, gy, gz, cin, cout, 7, _p(err), _stream())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    xt = _to_ncdhw(x, dims, cin).requires_grad_(True)
    wt = _torch_w(w.to(torch.bfloat16).float()).requires_grad_(True)
    out = F.conv3d(xt, wt, None, padding=1)
    out.backward(_to_ncdhw(dy, dims, cout))
    gx_ref = xt.grad.squeeze(0).permute(1, 2, 3, 0).reshape(nv, cin)
    s = gx_ref.abs().max().item()
    assert (dx32[:, :cin] - gx_ref).abs().max().item() <= 1e-4 * s + 1e-5
    if cinp16 > cin:
        assert dx32[:, cin:].abs().max().item() == 0.0
    # torch weight grad [cout][cin][kz][ky][kx] -> ours [t*cin + ci][co]
    gw_ref = wt.grad.permute(2, 3, 4, 1, 0).reshape(27 * cin, cout)
    s = gw_ref.abs().max().item()
    assert (dwt - gw_ref).abs().max().item() <= 1e-4 * s + 1e-5
