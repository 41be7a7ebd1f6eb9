"""Pressure-guess U-Net for the learned warm start (CS_WARM_LEARNED).

Three levels (16 / 32 / 64 channels), 3x3x3 convolutions with ReLU, 2x2x2 average
pooling, nearest upsampling with skip concatenation, and a 1x1x1 output layer:
about 246k parameters.  Activations are BF16 (channels-last), accumulation is FP32
in tensor memory; every convolution (forward, input gradient, weight gradient) runs on
the tcgen05 tensor cores through the engine library (`cs_nn_*`), and the glue
(pooling, concatenation, ReLU masks, loss, Adam) through its CUDA-core kernels.
torch only allocates the device memory and supplies the stream.

Inputs (8 channels per cell): r / s, fill fraction, fluid, bed and solid masks, three
zero channels, where r is the FP64 residual of the previous-substep pressure under the
pressure operator and s its RMS over the fluid cells.  The output times s is the
predicted pressure correction, so the network is a learned approximate inverse of the
operator; the guess is the previous pressure plus the correction (a zero output is the
plain warm start).  No counterpart in the reference.
"""
import ctypes as C
import math

import numpy as np

# name, level, input channels (padded to 8), output channels
LAYERS = [
    ("e1a", 0, 8, 16), ("e1b", 0, 16, 16),
    ("e2a", 1, 16, 32), ("e2b", 1, 32, 32),
    ("e3a", 2, 32, 64),
    ("d2a", 1, 96, 32), ("d2b", 1, 32, 32),
    ("d1a", 0, 48, 16), ("d1b", 0, 16, 16),
]
HEAD_C = 16
FEATURES = 8
REAL_INPUTS = 5


def param_count():
    return sum(cout * 27 * cin + cout for _, _, cin, cout in LAYERS) + HEAD_C + 1


def layer_slices():
    """Offsets of every layer's weights [cout][27][cin] and bias [cout] in the flat
    parameter vector (the head: HEAD_C weights then the bias)."""
    out, o = {}, 0
    for name, _, cin, cout in LAYERS:
        w = cout * 27 * cin
        out[name] = (o, o + w, o + w + cout)
        o += w + cout
    out["head"] = (o, o + HEAD_C, o + HEAD_C + 1)
    return out


def init_params(seed=0):
    """He-normal weights, zero biases (the first layer scaled to its real inputs)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(param_count(), dtype=np.float32)
    for name, (a, b, c) in layer_slices().items():
        if name == "head":
            p[a:b] = rng.normal(0.0, math.sqrt(1.0 / HEAD_C), HEAD_C)
            continue
        cin = next(l[2] for l in LAYERS if l[0] == name)
        fan = 27 * (REAL_INPUTS if name == "e1a" else cin)
        p[a:b] = rng.normal(0.0, math.sqrt(2.0 / fan), b - a)
    return p


def _r16(c):
    return (c + 15) // 16 * 16


class UNet:
    """The network on the GPU for training and inference (torch tensors as storage)."""

    def __init__(self, dims, lib, params=None, seed=0):
        import torch

        self.torch = torch
        self.lib = lib
        gx, gy, gz = dims
        if gx % 4 or gy % 4 or gz % 4:
            raise ValueError("grid dims must be multiples of 4")
        self.dims = [(gx, gy, gz), (gx // 2, gy // 2, gz // 2), (gx // 4, gy // 4, gz // 4)]
        self.nv = [a * b * c for a, b, c in self.dims]
        dev = "cuda"
        init = params if params is not None else init_params(seed)
        self.p = torch.tensor(np.asarray(init, dtype=np.float32), device=dev)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step_count = 0
        self.sl = layer_slices()
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.wf, self.wb = {}, {}
        for name, _, cin, cout in LAYERS:
            k = (27 * cin + 63) // 64 * 64
            self.wf[name] = torch.zeros(_r16(cout), k, dtype=torch.bfloat16, device=dev)
            kb = (27 * _r16(cout) + 63) // 64 * 64
            self.wb[name] = torch.zeros(_r16(cin), kb, dtype=torch.bfloat16, device=dev)
        self.act = {}

    # -- helpers --
    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _p(t):
        return None if t is None else C.c_void_p(t.data_ptr())

    def _w(self, name):
        a, b, _ = self.sl[name]
        return self.p[a:b]

    def _b(self, name):
        _, b, c = self.sl[name]
        return self.p[b:c]

    def pack(self):
        """bf16 GEMM operands of the current weights (forward and input gradient)."""
        for name, _, cin, cout in LAYERS:
            self.lib.call("cs_nn_pack_weights", self._p(self._w(name)), self._p(self.wf[name]), cin, cin, cout,
                          _r16(cout), 0, self._s())
            self.lib.call("cs_nn_pack_weights", self._p(self._w(name)), self._p(self.wb[name]), cin, cin, cout,
                          _r16(cout), 1, self._s())

    def _conv(self, name, x, lvl, relu=True):
        _, _, cin, cout = next(l for l in LAYERS if l[0] == name)
        gx, gy, gz = self.dims[lvl]
        y = self.torch.empty(self.nv[lvl], _r16(cout), dtype=self.torch.bfloat16, device="cuda")
        self.lib.call("cs_nn_conv3d", self._p(x), self._p(self.wf[name]), self._p(self._b(name)), self._p(y), None,
                      gx, gy, gz, cin, _r16(cout), 1 if relu else 0, self._p(self.err), self._s())
        return y

    # -- forward --
    def forward(self, feat):
        """feat: bf16 [voxels][8] -> f32 [voxels] (the guess in units of s)."""
        t = self.torch
        a = self.act
        d0, d1 = self.dims[0], self.dims[1]
        a["in"] = feat
        a["e1a"] = self._conv("e1a", feat, 0)
        a["e1b"] = self._conv("e1b", a["e1a"], 0)
        a["p1"] = t.empty(self.nv[1], 16, dtype=t.bfloat16, device="cuda")
        self.lib.call("cs_nn_pool", self._p(a["e1b"]), self._p(a["p1"]), None, None, *d0, 16, 0, self._s())
        a["e2a"] = self._conv("e2a", a["p1"], 1)
        a["e2b"] = self._conv("e2b", a["e2a"], 1)
        a["p2"] = t.empty(self.nv[2], 32, dtype=t.bfloat16, device="cuda")
        self.lib.call("cs_nn_pool", self._p(a["e2b"]), self._p(a["p2"]), None, None, *d1, 32, 0, self._s())
        a["e3a"] = self._conv("e3a", a["p2"], 2)
        a["u2"] = t.empty(self.nv[1], 96, dtype=t.bfloat16, device="cuda")
        self.lib.call("cs_nn_upcat", self._p(a["e3a"]), self._p(a["e2b"]), self._p(a["u2"]), None, None, None, *d1,
                      64, 32, 0, self._s())
        a["d2a"] = self._conv("d2a", a["u2"], 1)
        a["d2b"] = self._conv("d2b", a["d2a"], 1)
        a["u1"] = t.empty(self.nv[0], 48, dtype=t.bfloat16, device="cuda")
        self.lib.call("cs_nn_upcat", self._p(a["d2b"]), self._p(a["e1b"]), self._p(a["u1"]), None, None, None, *d0,
                      32, 16, 0, self._s())
        a["d1a"] = self._conv("d1a", a["u1"], 0)
        a["d1b"] = self._conv("d1b", a["d1a"], 0)
        out = t.empty(self.nv[0], dtype=t.float32, device="cuda")
        ha, _, hc = self.sl["head"]
        self.lib.call("cs_nn_head", self._p(a["d1b"]), self._p(self.p[ha:hc]), self._p(out), None, None, None,
                      self.nv[0], HEAD_C, 0, self._s())
        a["out"] = out
        return out

    # -- backward --
    def _layer_bwd(self, name, lvl, g32, x, need_input_grad=True):
        """g32: f32 gradient of the layer's (ReLU) output; returns f32 gradient of x."""
        t = self.torch
        _, _, cin, cout = next(l for l in LAYERS if l[0] == name)
        gx, gy, gz = self.dims[lvl]
        nv = self.nv[lvl]
        gb = t.empty(nv, _r16(cout), dtype=t.bfloat16, device="cuda")
        a0, b0, c0 = self.sl[name]
        self.lib.call("cs_nn_relu_grad", self._p(g32), self._p(self.act[name]), self._p(gb), self._p(self.g[b0:c0]),
                      nv * _r16(cout), _r16(cout), self._s())
        dwt = t.zeros(27 * cin, _r16(cout), dtype=t.float32, device="cuda")
        tiles = (27 * cin + 127) // 128
        splits = max(1, min(296 // tiles, nv // 64))
        self.lib.call("cs_nn_conv3d_wgrad", self._p(x), self._p(gb), self._p(dwt), gx, gy, gz, cin, _r16(cout),
                      splits, self._p(self.err), self._s())
        self.lib.call("cs_nn_wgrad_master", self._p(dwt), self._p(self.g[a0:b0]), cin, cout, _r16(cout), self._s())
        if not need_input_grad:
            return None
        dx = t.empty(nv, _r16(cin), dtype=t.float32, device="cuda")
        self.lib.call("cs_nn_conv3d", self._p(gb), self._p(self.wb[name]), None, None, self._p(dx), gx, gy, gz,
                      _r16(cout), _r16(cin), 0, self._p(self.err), self._s())
        return dx[:, :cin].contiguous() if _r16(cin) != cin else dx

    def backward(self, dout):
        """dout: f32 [voxels] gradient of the loss w.r.t. the output; fills self.g."""
        t = self.torch
        a = self.act
        d0, d1 = self.dims[0], self.dims[1]
        self.g.zero_()
        ha, _, hc = self.sl["head"]
        g_d1b = t.empty(self.nv[0], HEAD_C, dtype=t.float32, device="cuda")
        self.lib.call("cs_nn_head", self._p(a["d1b"]), self._p(self.p[ha:hc]), None, self._p(dout), self._p(g_d1b),
                      self._p(self.g[ha:hc]), self.nv[0], HEAD_C, 1, self._s())
        g_d1a = self._layer_bwd("d1b", 0, g_d1b, a["d1a"])
        g_u1 = self._layer_bwd("d1a", 0, g_d1a, a["u1"])
        g_d2b = t.zeros(self.nv[1], 32, dtype=t.float32, device="cuda")
        g_e1b = t.zeros(self.nv[0], 16, dtype=t.float32, device="cuda")
        self.lib.call("cs_nn_upcat", None, None, None, self._p(g_u1), self._p(g_d2b), self._p(g_e1b), *d0, 32, 16, 1,
                      self._s())
        g_d2a = self._layer_bwd("d2b", 1, g_d2b, a["d2a"])
        g_u2 = self._layer_bwd("d2a", 1, g_d2a, a["u2"])
        g_e3a = t.zeros(self.nv[2], 64, dtype=t.float32, device="cuda")
        g_e2b = t.zeros(self.nv[1], 32, dtype=t.float32, device="cuda")
        self.lib.call("cs_nn_upcat", None, None, None, self._p(g_u2), self._p(g_e3a), self._p(g_e2b), *d1, 64, 32, 1,
                      self._s())
        g_p2 = self._layer_bwd("e3a", 2, g_e3a, a["p2"])
        self.lib.call("cs_nn_pool", None, None, self._p(g_p2), self._p(g_e2b), *d1, 32, 1, self._s())
        g_e2a = self._layer_bwd("e2b", 1, g_e2b, a["e2a"])
        g_p1 = self._layer_bwd("e2a", 1, g_e2a, a["p1"])
        self.lib.call("cs_nn_pool", None, None, self._p(g_p1), self._p(g_e1b), *d0, 16, 1, self._s())
        g_e1a = self._layer_bwd("e1b", 0, g_e1b, a["e1a"])
        self._layer_bwd("e1a", 0, g_e1a, a["in"], need_input_grad=False)
        return self.g

    def loss_and_grad(self, out, target, mask):
        """Masked mean squared error over the fluid cells; returns (loss tensor, dout)."""
        n = float(mask.sum().item())
        dout = self.torch.empty_like(out)
        self.loss.zero_()
        self.lib.call("cs_nn_mse", self._p(out), self._p(target), self._p(mask), self._p(dout), self._p(self.loss),
                      out.numel(), 1.0 / max(n, 1.0), self._s())
        return self.loss, dout

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        self.lib.call("cs_nn_adam", self._p(self.p), self._p(self.g), self._p(self.m), self._p(self.v),
                      self.p.numel(), lr, b1, b2, eps, self.step_count, self._s())

    def train_step(self, feat, target, mask, lr=1e-3):
        self.pack()
        out = self.forward(feat)
        loss, dout = self.loss_and_grad(out, target, mask)
        self.backward(dout)
        self.adam(lr)
        return loss

    def check_errors(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("a tensor-core convolution timed out waiting for its MMAs")

    def params_numpy(self):
        return self.p.detach().cpu().numpy()


def reference_forward(params, feat, dims):
    """The same network in torch float64 on the CPU (the gradient-check oracle): feat is
    a float64 tensor [voxels][8]; returns the output [voxels]."""
    import torch
    import torch.nn.functional as F

    sl = layer_slices()
    p = params

    def conv(name, x, relu=True):
        _, _, cin, cout = next(l for l in LAYERS if l[0] == name)
        a, b, c = sl[name]
        # tap t = kz * 9 + ky * 3 + kx with offsets (kx - 1, ky - 1, kz - 1)
        w = p[a:b].reshape(cout, 3, 3, 3, cin).permute(0, 4, 1, 2, 3)
        y = F.conv3d(x, w, p[b:c], padding=1)
        return F.relu(y) if relu else y

    gx, gy, gz = dims
    x = feat.reshape(gz, gy, gx, FEATURES).permute(3, 0, 1, 2).unsqueeze(0)
    e1 = conv("e1b", conv("e1a", x))
    e2 = conv("e2b", conv("e2a", F.avg_pool3d(e1, 2)))
    e3 = conv("e3a", F.avg_pool3d(e2, 2))
    u2 = torch.cat([F.interpolate(e3, scale_factor=2, mode="nearest"), e2], dim=1)
    d2 = conv("d2b", conv("d2a", u2))
    u1 = torch.cat([F.interpolate(d2, scale_factor=2, mode="nearest"), e1], dim=1)
    d1 = conv("d1b", conv("d1a", u1))
    a, b, _ = sl["head"]
    out = torch.einsum("bczyx,c->bzyx", d1, p[a:b]) + p[b]
    return out.reshape(-1)


# ---- training on solver-generated pairs ----
def collect_samples(sim, sub_dt, substeps, torch_mod=None):
    """Step `sim` (an engine MpmSim3D) `substeps` times with sample capture on and return
    the (inputs, target, mask) pairs as CUDA tensors: network inputs before each solve,
    (solved - previous pressure) / s after it, and the fluid mask."""
    import torch

    n = sim.settings.cells
    out = []
    sim.learned_capture(True)
    try:
        for _ in range(substeps):
            sim.step_substep(sub_dt)
            feat = torch.empty(n, FEATURES, dtype=torch.bfloat16, device="cuda")
            target = torch.empty(n, dtype=torch.float32, device="cuda")
            mask = torch.empty(n, dtype=torch.float32, device="cuda")
            sim.learned_read_sample(feat, target, mask)
            out.append((feat, target, mask))
    finally:
        sim.learned_capture(False)
    return out


def train(samples, dims, lib, steps=1000, lr=1e-3, seed=0, params=None, log_every=0):
    """Adam on the masked MSE between the guess and the solved pressure (units of s),
    one pair per step in a seeded random order.  Returns (flat params, loss history)."""
    import torch

    net = UNet(dims, lib, params=params, seed=seed)
    rng = np.random.default_rng(seed)
    hist = []
    for k in range(steps):
        f, t, m = samples[int(rng.integers(len(samples)))]
        step_lr = lr * (0.1 ** (k / max(steps, 1)))  # exponential decay to lr / 10
        loss = net.train_step(f, t, m, lr=step_lr)
        if log_every and (k % log_every == 0 or k == steps - 1):
            hist.append((k, float(loss.item())))
    torch.cuda.synchronize()
    net.check_errors()
    return net.params_numpy(), hist
