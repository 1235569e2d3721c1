"""Learned warm start for the TV-regularised reconstruction: a 3-level 3D
U-Net whose 3x3x3 convolutions run on the sm_100a tensor cores.

The reference starts every VMLM-B reconstruction from zero
(``Tomography_3D/Ytrtt3D_optim.i:663``).  Here a small network maps the
normalised backprojection of the data to an estimate of the converged TV
reconstruction; VMLM-B then starts from that estimate and runs the
unchanged iteration to the same stopping rule, so the plain method stays
the arbiter of the result (a bad estimate only costs iterations).

Architecture (``UNet3D.LAYERS``): two convolutions per level at 16, 32 and
64 channels, leaky ReLU, 2x2x2 average pooling down, nearest-neighbour
upsampling up, skip connections by channel concatenation, and a residual
head ``out = x + conv(...)`` whose weights start at zero (the untrained
network is the identity).  Every convolution, its input gradient and its
weight gradient are the BF16 tcgen05 kernels of ``csrc/unet.cu`` (FP32
accumulation in tensor memory); the optimiser is Adam on FP32 master
weights.  Activations are kept in the padded channels-last layout of
``include/trtt_b200.h`` (``trtt_b200_conv3_forward``).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib

SLOPE = 0.1  # leaky ReLU slope


def _torch():
    import torch
    return torch


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream():
    torch = _torch()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _r16(c):
    return (c + 15) // 16 * 16


class UNet3D:
    """3-level 3D U-Net (16/32/64 channels) on the tcgen05 convolutions.

    ``forward(x)`` maps dense FP32 volumes (nb, d, h, w) (d, h, w multiples
    of 4) to dense FP32 volumes of the same shape; ``train_step(x, target)``
    runs forward, the mean-squared-error loss, backward and one Adam step and
    returns the loss.  Inputs and targets are multiplied by ``scale`` inside
    the network (and outputs divided by it) so that typical values are O(1).
    """

    # name, input channels (first tensor), input channels (skip tensor),
    # output channels, level (0: full resolution)
    LAYERS = [
        ("e1a", 16, 0, 16, 0), ("e1b", 16, 0, 16, 0),
        ("e2a", 16, 0, 32, 1), ("e2b", 32, 0, 32, 1),
        ("e3a", 32, 0, 64, 2), ("e3b", 64, 0, 64, 2),
        ("d2a", 64, 32, 32, 1), ("d2b", 32, 0, 32, 1),
        ("d1a", 32, 16, 16, 0), ("d1b", 16, 0, 16, 0),
        ("head", 16, 0, 16, 0),  # only output channel 0 is used
    ]

    def __init__(self, scale: float = 1.0, seed: int = 0, device=None, lr: float = 1e-3,
                 weight_decay: float = 0.0):
        torch = _torch()
        if not torch.cuda.is_available():
            raise _lib.TrttError("UNet3D needs a CUDA device (no CPU fallback)")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.scale = float(scale)
        self.lr, self.weight_decay = float(lr), float(weight_decay)
        self.step_count = 0
        g = torch.Generator().manual_seed(seed)
        self.params = {}
        for name, c1, c2, co, _ in self.LAYERS:
            cin = c1 + c2
            fan_in = 27 * (1 if name == "e1a" else cin)
            w = torch.randn(co, 27, cin, generator=g) * math.sqrt(2.0 / fan_in)
            if name == "e1a":
                w[:, :, 1:] = 0.0  # input channels 1..15 are padding
            if name == "head":
                w.zero_()
            b = torch.zeros(co)
            self.params[name] = {"w": w.to(self.device), "b": b.to(self.device)}
        self._adam = {k: {n: (torch.zeros_like(t), torch.zeros_like(t)) for n, t in v.items()}
                      for k, v in self.params.items()}
        self._grads = {k: {n: torch.zeros_like(t) for n, t in v.items()} for k, v in self.params.items()}
        self._packs = {}
        self._shape = None
        self._pack_all()

    # -- parameters ---------------------------------------------------------
    def _pack_all(self):
        torch = _torch()
        lib = _lib.load()
        st = _stream()
        for name, c1, c2, co, _ in self.LAYERS:
            cin = c1 + c2
            w = self.params[name]["w"]
            if name not in self._packs:
                self._packs[name] = (
                    torch.empty(27 * _r16(co) * cin, dtype=torch.bfloat16, device=self.device),
                    torch.empty(27 * cin * _r16(co), dtype=torch.bfloat16, device=self.device))
            fw, bw = self._packs[name]
            _lib.check(lib.trtt_b200_conv3_pack(_p(w), co, cin, 0, _p(fw), st), "conv3_pack")
            if name != "e1a":
                _lib.check(lib.trtt_b200_conv3_pack(_p(w), co, cin, 1, _p(bw), st), "conv3_pack")

    def state_dict(self):
        return {f"{k}.{n}": t.detach().cpu().numpy() for k, v in self.params.items() for n, t in v.items()} | \
            {"scale": np.array(self.scale)}

    def load_state_dict(self, sd):
        torch = _torch()
        for k, v in self.params.items():
            for n in v:
                v[n].copy_(torch.as_tensor(np.asarray(sd[f"{k}.{n}"]), device=self.device))
        if "scale" in sd:
            self.scale = float(np.asarray(sd["scale"]))
        self._pack_all()

    def save(self, path):
        np.savez(path, **self.state_dict())

    @classmethod
    def load(cls, path, **kw):
        sd = dict(np.load(path))
        net = cls(**kw)
        net.load_state_dict(sd)
        return net

    # -- buffers --------------------------------------------------------------
    def _ensure(self, nb, d, h, w):
        torch = _torch()
        if (d % 4) or (h % 4) or (w % 4):
            raise ValueError("volume dimensions must be multiples of 4")
        if self._shape == (nb, d, h, w):
            return
        self._shape = (nb, d, h, w)
        dims = [(d, h, w), (d // 2, h // 2, w // 2), (d // 4, h // 4, w // 4)]
        self._dims = dims
        rows = [nb * (a + 2) * (b + 2) * (c + 2) for a, b, c in dims]
        self._rows = rows

        def t(level, c, dtype=torch.bfloat16):
            return torch.zeros(rows[level], c, dtype=dtype, device=self.device)

        A = {}
        A["xin"] = t(0, 16)
        A["xf"] = torch.zeros(rows[0], dtype=torch.float32, device=self.device)
        A["out"] = torch.zeros(rows[0], dtype=torch.float32, device=self.device)
        for name, c1, c2, co, lv in self.LAYERS[:-1]:
            A[name] = t(lv, co)
        A["p1"], A["p2"] = t(1, 16), t(2, 32)
        A["u2"], A["u1"] = t(1, 64), t(0, 32)
        self.act = A
        G = {}
        G["dout"] = t(0, 16)
        for name, c1, c2, co, lv in self.LAYERS[:-1]:
            G[name] = t(lv, co)
        G["p1"], G["p2"] = t(1, 16), t(2, 32)
        G["u2"], G["u1"] = t(1, 64), t(0, 32)
        self.grad = G
        lib = _lib.load()
        need = 0
        for name, c1, c2, co, lv in self.LAYERS:
            a, b, c = dims[lv]
            need = max(need, lib.trtt_b200_conv3_wgrad_scratch(_r16(co), c1 + c2, nb, a, b, c))
        self._scratch = torch.empty(need // 4 + 1, dtype=torch.float32, device=self.device)
        self._loss = torch.zeros(1, dtype=torch.float64, device=self.device)

    # -- kernels ----------------------------------------------------------------
    def _conv(self, name, x1, x2, y, mode=0, resid=None):
        spec = {n: (c1, c2, co, lv) for n, c1, c2, co, lv in self.LAYERS}[name]
        c1, c2, co, lv = spec
        nb = self._shape[0]
        d, h, w = self._dims[lv]
        _lib.check(_lib.load().trtt_b200_conv3_forward(
            _p(x1), c1, _p(x2), c2, _p(self._packs[name][0]), _r16(co), _p(self.params[name]["b"]),
            mode, SLOPE, _p(y), None, 0, 0, _p(resid), nb, d, h, w, _stream()), f"conv3_forward {name}")

    def _conv_dx(self, name, gy, g1, g2, accumulate=0):
        c1, c2, co, lv = {n: (a, b, c, l) for n, a, b, c, l in self.LAYERS}[name]
        nb = self._shape[0]
        d, h, w = self._dims[lv]
        _lib.check(_lib.load().trtt_b200_conv3_forward(
            _p(gy), _r16(co), None, 0, _p(self._packs[name][1]), c1 + c2, None, 3, 1.0,
            _p(g1), _p(g2), c1, accumulate, None, nb, d, h, w, _stream()), f"conv3 input gradient {name}")

    def _conv_dw(self, name, gy, x1, x2):
        c1, c2, co, lv = {n: (a, b, c, l) for n, a, b, c, l in self.LAYERS}[name]
        nb = self._shape[0]
        d, h, w = self._dims[lv]
        gr = self._grads[name]
        _lib.check(_lib.load().trtt_b200_conv3_wgrad(
            _p(gy), _r16(co), _p(x1), c1, _p(x2), c2, _p(gr["w"]), _p(gr["b"]), _p(self._scratch),
            self._scratch.numel() * 4, nb, d, h, w, _stream()), f"conv3_wgrad {name}")

    def _resample(self, fine, coarse, c, level, mode, accumulate=0):
        nb = self._shape[0]
        d, h, w = self._dims[level]
        _lib.check(_lib.load().trtt_b200_unet_resample(_p(fine), _p(coarse), c, nb, d, h, w, mode,
                                                        accumulate, _stream()), "unet_resample")

    def _act_grad(self, g, y):
        _lib.check(_lib.load().trtt_b200_unet_act_grad(_p(g), _p(y), g.shape[0], g.shape[1], SLOPE,
                                                        _stream()), "unet_act_grad")

    # -- network ------------------------------------------------------------------
    def _forward_padded(self, x):
        lib = _lib.load()
        nb, d, h, w = x.shape
        self._ensure(nb, d, h, w)
        A = self.act
        _lib.check(lib.trtt_b200_unet_pad_input(_p(x), _p(A["xin"]), _p(A["xf"]), self.scale,
                                                nb, d, h, w, _stream()), "unet_pad_input")
        self._conv("e1a", A["xin"], None, A["e1a"])
        self._conv("e1b", A["e1a"], None, A["e1b"])
        self._resample(A["e1b"], A["p1"], 16, 0, 0)
        self._conv("e2a", A["p1"], None, A["e2a"])
        self._conv("e2b", A["e2a"], None, A["e2b"])
        self._resample(A["e2b"], A["p2"], 32, 1, 0)
        self._conv("e3a", A["p2"], None, A["e3a"])
        self._conv("e3b", A["e3a"], None, A["e3b"])
        self._resample(A["u2"], A["e3b"], 64, 1, 2)
        self._conv("d2a", A["u2"], A["e2b"], A["d2a"])
        self._conv("d2b", A["d2a"], None, A["d2b"])
        self._resample(A["u1"], A["d2b"], 32, 0, 2)
        self._conv("d1a", A["u1"], A["e1b"], A["d1a"])
        self._conv("d1b", A["d1a"], None, A["d1b"])
        self._conv("head", A["d1b"], None, A["out"], mode=2, resid=A["xf"])
        return A["out"]

    def forward(self, x, out=None):
        """Dense FP32 (nb, d, h, w) -> dense FP32 (nb, d, h, w)."""
        torch = _torch()
        x = x.contiguous()
        if x.dim() == 3:
            x = x.unsqueeze(0)
        nb, d, h, w = x.shape
        yp = self._forward_padded(x)
        if out is None:
            out = torch.empty_like(x)
        _lib.check(_lib.load().trtt_b200_unet_unpad(_p(yp), _p(out), 1.0 / self.scale, nb, d, h, w,
                                                    _stream()), "unet_unpad")
        return out

    __call__ = forward

    def backward(self, x, target, extra_grad=None):
        """Forward pass, loss mean((out - scale target)^2) and the gradients of
        every parameter (left in self._grads).  ``extra_grad`` (dense FP32
        like x): the gradient of an additional loss term with respect to the
        network output (in the units of x), added to the MSE gradient.
        Returns the MSE loss (device)."""
        lib = _lib.load()
        x = x.contiguous()
        target = target.contiguous()
        nb, d, h, w = x.shape
        out = self._forward_padded(x)
        A, G = self.act, self.grad
        self._loss.zero_()
        _lib.check(lib.trtt_b200_unet_mse(_p(out), _p(target), _p(G["dout"]), self.scale, _p(self._loss),
                                          nb, d, h, w, _stream()), "unet_mse")
        if extra_grad is not None:
            eg = extra_grad.contiguous()
            _lib.check(lib.trtt_b200_unet_add_output_grad(_p(G["dout"]), _p(eg), 1.0 / self.scale, nb, d, h, w,
                                                          _stream()), "unet_add_output_grad")
        self._conv_dw("head", G["dout"], A["d1b"], None)
        self._conv_dx("head", G["dout"], G["d1b"], None)
        self._act_grad(G["d1b"], A["d1b"])
        self._conv_dw("d1b", G["d1b"], A["d1a"], None)
        self._conv_dx("d1b", G["d1b"], G["d1a"], None)
        self._act_grad(G["d1a"], A["d1a"])
        self._conv_dw("d1a", G["d1a"], A["u1"], A["e1b"])
        self._conv_dx("d1a", G["d1a"], G["u1"], G["e1b"])
        self._resample(G["u1"], G["d2b"], 32, 0, 3)
        self._act_grad(G["d2b"], A["d2b"])
        self._conv_dw("d2b", G["d2b"], A["d2a"], None)
        self._conv_dx("d2b", G["d2b"], G["d2a"], None)
        self._act_grad(G["d2a"], A["d2a"])
        self._conv_dw("d2a", G["d2a"], A["u2"], A["e2b"])
        self._conv_dx("d2a", G["d2a"], G["u2"], G["e2b"])
        self._resample(G["u2"], G["e3b"], 64, 1, 3)
        self._act_grad(G["e3b"], A["e3b"])
        self._conv_dw("e3b", G["e3b"], A["e3a"], None)
        self._conv_dx("e3b", G["e3b"], G["e3a"], None)
        self._act_grad(G["e3a"], A["e3a"])
        self._conv_dw("e3a", G["e3a"], A["p2"], None)
        self._conv_dx("e3a", G["e3a"], G["p2"], None)
        self._resample(G["e2b"], G["p2"], 32, 1, 1, accumulate=1)
        self._act_grad(G["e2b"], A["e2b"])
        self._conv_dw("e2b", G["e2b"], A["e2a"], None)
        self._conv_dx("e2b", G["e2b"], G["e2a"], None)
        self._act_grad(G["e2a"], A["e2a"])
        self._conv_dw("e2a", G["e2a"], A["p1"], None)
        self._conv_dx("e2a", G["e2a"], G["p1"], None)
        self._resample(G["e1b"], G["p1"], 16, 0, 1, accumulate=1)
        self._act_grad(G["e1b"], A["e1b"])
        self._conv_dw("e1b", G["e1b"], A["e1a"], None)
        self._conv_dx("e1b", G["e1b"], G["e1a"], None)
        self._act_grad(G["e1a"], A["e1a"])
        self._conv_dw("e1a", G["e1a"], A["xin"], None)
        return self._loss

    def step(self):
        """One Adam step on every parameter from the gradients of backward()."""
        lib = _lib.load()
        self.step_count += 1
        for name in self.params:
            for n, w in self.params[name].items():
                g = self._grads[name][n]
                m, v = self._adam[name][n]
                _lib.check(lib.trtt_b200_adam(_p(w), _p(g), _p(m), _p(v), w.numel(), self.lr, 0.9, 0.999,
                                              1e-8, self.step_count, self.weight_decay, _stream()), "adam")
        self._pack_all()

    def train_step(self, x, target, extra_grad=None):
        loss = self.backward(x, target, extra_grad)
        self.step()
        return loss

    def status(self):
        _lib.check(_lib.load().trtt_b200_unet_status(_stream()), "unet")

    # -- CPU reference ----------------------------------------------------------------
    def torch_reference(self, x, dtype=None):
        """The same network in plain PyTorch on the CPU (test oracle of the
        kernels), with the current weights; x dense (nb, d, h, w)."""
        torch = _torch()
        import torch.nn.functional as F
        dtype = dtype or torch.float64

        def W(name):
            w = self.params[name]["w"].detach().cpu().to(dtype)
            co, _, cin = w.shape
            return w.permute(0, 2, 1).reshape(co, cin, 3, 3, 3), self.params[name]["b"].detach().cpu().to(dtype)

        def conv(name, t, act=True):
            w, b = W(name)
            y = F.conv3d(t, w, b, padding=1)
            return F.leaky_relu(y, SLOPE) if act else y

        x = x.detach().cpu().to(dtype) * self.scale
        if x.dim() == 3:
            x = x.unsqueeze(0)
        xin = torch.zeros((x.shape[0], 16) + tuple(x.shape[1:]), dtype=dtype)
        xin[:, 0] = x
        e1a = conv("e1a", xin)
        e1b = conv("e1b", e1a)
        e2a = conv("e2a", F.avg_pool3d(e1b, 2))
        e2b = conv("e2b", e2a)
        e3a = conv("e3a", F.avg_pool3d(e2b, 2))
        e3b = conv("e3b", e3a)
        d2a = conv("d2a", torch.cat([F.interpolate(e3b, scale_factor=2, mode="nearest"), e2b], 1))
        d2b = conv("d2b", d2a)
        d1a = conv("d1a", torch.cat([F.interpolate(d2b, scale_factor=2, mode="nearest"), e1b], 1))
        d1b = conv("d1b", d1a)
        out = x + conv("head", d1b, act=False)[:, 0]
        return out / self.scale
