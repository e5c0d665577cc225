"""Warm-start surrogate: a 3-level 3D U-Net over the voxel geometry,
trained and run by the library's own kernels (include/dsmc_surrogate.h).

Input per sample: the solid mask of an S^3 voxel box (S a power of two,
>= 16) and one scalar feature (log10 of the Knudsen number).  Output per
voxel: 4 fp32 channels, the steady gas density relative to the box's mean
and the three drift velocity components in units of `velocity_scale`.
Every 3x3x3 convolution is periodic, as the geometry is; the network is
fully convolutional, so one trained on 64^3 boxes runs on 256^3 ones.

Architecture (channels per level 16 / 32 / 64, BF16 weights and activations,
FP32 accumulation, ReLU after every 3x3x3 convolution):

    x(16) -c1a-> 16 -c1b-> 16 =skip1 -pool-> -c2a-> 32 -c2b-> 32 =skip2 -pool->
    -c3a-> 64 -c3b-> 64 -up-> [64 | skip2] -c2c-> 32 -c2d-> 32 -up->
    [32 | skip1] -c1c-> 16 -c1d-> 16 -head(1x1, fp32)-> 4

The reference has no counterpart: it always starts a run from a Maxwellian at
rest (System::setup_molecules, dsmc/system.cpp:398-430).  torch tensors are
used only as device memory; every operation is a call into libdsmc_b200.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import capi

# (name, cin, cout, level): level 0 = S, 1 = S/2, 2 = S/4
LAYERS = [
    ("c1a", 16, 16, 0), ("c1b", 16, 16, 0),
    ("c2a", 16, 32, 1), ("c2b", 32, 32, 1),
    ("c3a", 32, 64, 2), ("c3b", 64, 64, 2),
    ("c2c", 96, 32, 1), ("c2d", 32, 32, 1),
    ("c1c", 48, 16, 0), ("c1d", 16, 16, 0),
]
HEAD_IN, HEAD_OUT = 16, 4


def parameter_layout():
    """Offsets of every parameter in the flat fp32 vector: per layer its
    weights [cout][27][cin] then its bias [cout]; then the head weights
    [4][16] and bias [4]."""
    off, out = 0, {}
    for name, cin, cout, _ in LAYERS:
        out[name + ".w"] = (off, (cout, 27, cin))
        off += cout * 27 * cin
        out[name + ".b"] = (off, (cout,))
        off += cout
    out["head.w"] = (off, (HEAD_OUT, HEAD_IN))
    off += HEAD_OUT * HEAD_IN
    out["head.b"] = (off, (HEAD_OUT,))
    off += HEAD_OUT
    return out, off


def init_parameters(seed: int = 0) -> np.ndarray:
    """He-normal weights (std sqrt(2 / fan_in)), zero biases, a small head."""
    layout, n = parameter_layout()
    rng = np.random.default_rng(seed)
    p = np.zeros(n, np.float32)
    for name, cin, cout, _ in LAYERS:
        o, shape = layout[name + ".w"]
        p[o:o + int(np.prod(shape))] = rng.normal(0.0, math.sqrt(2.0 / (27 * cin)), int(np.prod(shape)))
    o, shape = layout["head.w"]
    p[o:o + 64] = rng.normal(0.0, math.sqrt(1.0 / HEAD_IN), 64)
    return p


@dataclass
class Buffers:
    batch: int
    S: int
    t: dict


class UNet:
    """The network on one CUDA device: fp32 master parameters, their bf16
    forward and input-gradient copies, Adam moments, and the activation
    buffers of the last batch shape."""

    def __init__(self, device: int = 0, params: np.ndarray | None = None, seed: int = 0):
        import torch
        self.torch = torch
        self.lib = capi.load()
        self.dev = torch.device("cuda", device)
        self.layout, self.nparams = parameter_layout()
        p = params if params is not None else init_parameters(seed)
        assert p.shape == (self.nparams,)
        self.p = torch.tensor(p, dtype=torch.float32, device=self.dev)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.adam_step = 0
        self.wf, self.wd = {}, {}
        for name, cin, cout, _ in LAYERS:
            self.wf[name] = torch.empty(cout * 27 * cin, dtype=torch.int16, device=self.dev)
            self.wd[name] = torch.empty(cout * 27 * cin, dtype=torch.int16, device=self.dev)
        self.buf: Buffers | None = None
        self.loss_acc = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.flux_work = None
        self.stream = None  # the current torch stream at each call
        self.pack_weights()

    # ---- helpers -----------------------------------------------------------
    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    @staticmethod
    def _ptr(t):
        return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)

    def _pp(self, key):
        off, shape = self.layout[key]
        return C.c_void_p(self.p.data_ptr() + 4 * off)

    def _gp(self, key):
        off, shape = self.layout[key]
        return C.c_void_p(self.g.data_ptr() + 4 * off)

    def _check(self, rc):
        capi.check(rc)

    def pack_weights(self):
        for name, cin, cout, _ in LAYERS:
            self._check(self.lib.dsmc_sg_pack_weights(self._s(), self._pp(name + ".w"), cout, cin,
                                                      self._ptr(self.wf[name]), self._ptr(self.wd[name])))

    def parameters_host(self) -> np.ndarray:
        return self.p.detach().cpu().numpy()

    def _buffers(self, batch: int, S: int) -> Buffers:
        if self.buf is not None and self.buf.batch == batch and self.buf.S == S:
            return self.buf
        torch = self.torch
        assert S >= 16 and S & (S - 1) == 0, "edge must be a power of two >= 16"
        H, Q = S // 2, S // 4

        def vol(edge, c):
            return torch.zeros((batch, edge, edge, edge, c), dtype=torch.int16, device=self.dev)
        t = {
            "x0": vol(S, 16), "a1": vol(S, 16), "cat1": vol(S, 48), "p1": vol(H, 16), "a2": vol(H, 32),
            "cat2": vol(H, 96), "p2": vol(Q, 32), "a3": vol(Q, 64), "b3": vol(Q, 64), "d2": vol(H, 32),
            "e2": vol(H, 32), "d1": vol(S, 16), "e1": vol(S, 16),
            "out": torch.zeros((batch, S, S, S, 4), dtype=torch.float32, device=self.dev),
            # gradients
            "de1": vol(S, 16), "dd1": vol(S, 16), "dcat1": vol(S, 48), "de2": vol(H, 32), "dd2": vol(H, 32),
            "dcat2": vol(H, 96), "db3": vol(Q, 64), "da3": vol(Q, 64), "dp2": vol(Q, 32), "dc2b": vol(H, 32),
            "da2": vol(H, 32), "dp1": vol(H, 16), "dc1b": vol(S, 16), "da1": vol(S, 16),
        }
        self.buf = Buffers(batch, S, t)
        return self.buf

    # ---- primitive calls -----------------------------------------------------
    def _conv(self, B, S, x, xcs, xoff, cin, name, cout, y, ycs, yoff, relu=True, mask=None, mcs=0, moff=0,
              dgrad=False):
        w = self.wd[name] if dgrad else self.wf[name]
        bias = C.c_void_p(0) if dgrad else self._pp(name + ".b")
        self._check(self.lib.dsmc_sg_conv3(self._s(), B, S, self._ptr(x), xcs, xoff, cin, self._ptr(w), bias, cout,
                                           self._ptr(y), ycs, yoff, 1 if relu else 0, self._ptr(mask), mcs, moff))

    def _wgrad(self, B, S, dy, dycs, dyoff, cout, x, xcs, xoff, cin, name):
        self._check(self.lib.dsmc_sg_conv3_wgrad(self._s(), B, S, self._ptr(dy), dycs, dyoff, cout, self._ptr(x),
                                                 xcs, xoff, cin, self._gp(name + ".w")))
        self._check(self.lib.dsmc_sg_bias_grad(self._s(), B, S, self._ptr(dy), dycs, dyoff, cout,
                                               self._gp(name + ".b")))

    # ---- forward / backward ------------------------------------------------
    def forward(self, solid, feature):
        """solid: uint8 tensor (B, S, S, S) on the device (1 = solid voxel),
        feature: float32 tensor (B,).  Returns the fp32 output (B, S, S, S, 4)
        (a buffer reused by the next call)."""
        B, S = int(solid.shape[0]), int(solid.shape[1])
        H, Q = S // 2, S // 4
        t = self._buffers(B, S).t
        L = self.lib
        s = self._s()
        self._check(L.dsmc_sg_pack_input(s, B, S, self._ptr(solid.contiguous()), self._ptr(feature.contiguous()),
                                          self._ptr(t["x0"])))
        self._conv(B, S, t["x0"], 16, 0, 16, "c1a", 16, t["a1"], 16, 0)
        self._conv(B, S, t["a1"], 16, 0, 16, "c1b", 16, t["cat1"], 48, 32)
        self._check(L.dsmc_sg_pool2(s, B, S, self._ptr(t["cat1"]), 48, 32, 16, self._ptr(t["p1"]), 16, 0))
        self._conv(B, H, t["p1"], 16, 0, 16, "c2a", 32, t["a2"], 32, 0)
        self._conv(B, H, t["a2"], 32, 0, 32, "c2b", 32, t["cat2"], 96, 64)
        self._check(L.dsmc_sg_pool2(s, B, H, self._ptr(t["cat2"]), 96, 64, 32, self._ptr(t["p2"]), 32, 0))
        self._conv(B, Q, t["p2"], 32, 0, 32, "c3a", 64, t["a3"], 64, 0)
        self._conv(B, Q, t["a3"], 64, 0, 64, "c3b", 64, t["b3"], 64, 0)
        self._check(L.dsmc_sg_up2(s, B, H, self._ptr(t["b3"]), 64, 0, 64, self._ptr(t["cat2"]), 96, 0))
        self._conv(B, H, t["cat2"], 96, 0, 96, "c2c", 32, t["d2"], 32, 0)
        self._conv(B, H, t["d2"], 32, 0, 32, "c2d", 32, t["e2"], 32, 0)
        self._check(L.dsmc_sg_up2(s, B, S, self._ptr(t["e2"]), 32, 0, 32, self._ptr(t["cat1"]), 48, 0))
        self._conv(B, S, t["cat1"], 48, 0, 48, "c1c", 16, t["d1"], 16, 0)
        self._conv(B, S, t["d1"], 16, 0, 16, "c1d", 16, t["e1"], 16, 0)
        self._check(L.dsmc_sg_head(s, B, S, self._ptr(t["e1"]), 16, 0, self._pp("head.w"), self._pp("head.b"),
                                   self._ptr(t["out"])))
        return t["out"]

    def backward(self, target, valid, channel_weight, flux_weight: float = 0.0) -> None:
        """Gradients of the weighted squared error of the last forward's
        output against target (B, S, S, S, 4) over the voxels with valid != 0
        (uint8 (B, S, S, S)), into self.g (zeroed first); with flux_weight,
        plus flux_weight times the squared error of each sample's mean x
        drift over its valid voxels (its flux), averaged over the batch.  The
        loss is added to self.loss_acc."""
        t = self.buf.t
        B, S = self.buf.batch, self.buf.S
        H, Q = S // 2, S // 4
        L = self.lib
        s = self._s()
        self.g.zero_()
        count = max(1, int(valid.sum().item()))
        cw = channel_weight if hasattr(channel_weight, "data_ptr") else self.torch.tensor(
            channel_weight, dtype=self.torch.float32, device=self.dev)
        target = target.contiguous()
        valid = valid.contiguous()
        coef = None
        if flux_weight > 0:
            if self.flux_work is None or self.flux_work.numel() < 3 * B:
                self.flux_work = self.torch.zeros(3 * B, dtype=self.torch.float64, device=self.dev)
            coef = self.flux_work[2 * B:3 * B]
            self._check(L.dsmc_sg_sample_flux_loss(s, B, S, self._ptr(t["out"]), self._ptr(target), self._ptr(valid),
                                                   1, C.c_float(flux_weight), self._ptr(self.flux_work),
                                                   self._ptr(coef), self._ptr(self.loss_acc)))
        self._check(L.dsmc_sg_loss_head_bwd(s, B, S, self._ptr(t["out"]), self._ptr(target),
                                            self._ptr(valid), self._ptr(cw), C.c_float(1.0 / count),
                                            self._ptr(t["e1"]), 16, 0, self._pp("head.w"), self._gp("head.w"),
                                            self._gp("head.b"), self._ptr(t["de1"]), 16, 0,
                                            self._ptr(self.loss_acc), self._ptr(coef), 1))
        # level 0 decoder
        self._wgrad(B, S, t["de1"], 16, 0, 16, t["d1"], 16, 0, 16, "c1d")
        self._conv(B, S, t["de1"], 16, 0, 16, "c1d", 16, t["dd1"], 16, 0, relu=False, mask=t["d1"], mcs=16,
                   dgrad=True)
        self._wgrad(B, S, t["dd1"], 16, 0, 16, t["cat1"], 48, 0, 48, "c1c")
        self._conv(B, S, t["dd1"], 16, 0, 16, "c1c", 48, t["dcat1"], 48, 0, relu=False, mask=t["cat1"], mcs=48,
                   dgrad=True)
        self._check(L.dsmc_sg_up2_bwd(s, B, S, self._ptr(t["dcat1"]), 48, 0, self._ptr(t["e2"]), 32, 0, 32,
                                      self._ptr(t["de2"]), 32, 0))
        # level 1 decoder
        self._wgrad(B, H, t["de2"], 32, 0, 32, t["d2"], 32, 0, 32, "c2d")
        self._conv(B, H, t["de2"], 32, 0, 32, "c2d", 32, t["dd2"], 32, 0, relu=False, mask=t["d2"], mcs=32,
                   dgrad=True)
        self._wgrad(B, H, t["dd2"], 32, 0, 32, t["cat2"], 96, 0, 96, "c2c")
        self._conv(B, H, t["dd2"], 32, 0, 32, "c2c", 96, t["dcat2"], 96, 0, relu=False, mask=t["cat2"], mcs=96,
                   dgrad=True)
        self._check(L.dsmc_sg_up2_bwd(s, B, H, self._ptr(t["dcat2"]), 96, 0, self._ptr(t["b3"]), 64, 0, 64,
                                      self._ptr(t["db3"]), 64, 0))
        # bottom
        self._wgrad(B, Q, t["db3"], 64, 0, 64, t["a3"], 64, 0, 64, "c3b")
        self._conv(B, Q, t["db3"], 64, 0, 64, "c3b", 64, t["da3"], 64, 0, relu=False, mask=t["a3"], mcs=64,
                   dgrad=True)
        self._wgrad(B, Q, t["da3"], 64, 0, 64, t["p2"], 32, 0, 32, "c3a")
        self._conv(B, Q, t["da3"], 64, 0, 64, "c3a", 32, t["dp2"], 32, 0, relu=False, dgrad=True)
        # level 1 encoder: pool backward + skip gradient + ReLU mask of c2b
        self._check(L.dsmc_sg_pool2_bwd(s, B, H, self._ptr(t["dp2"]), 32, 0, self._ptr(t["dcat2"]), 96, 64,
                                        self._ptr(t["cat2"]), 96, 64, 32, self._ptr(t["dc2b"]), 32, 0))
        self._wgrad(B, H, t["dc2b"], 32, 0, 32, t["a2"], 32, 0, 32, "c2b")
        self._conv(B, H, t["dc2b"], 32, 0, 32, "c2b", 32, t["da2"], 32, 0, relu=False, mask=t["a2"], mcs=32,
                   dgrad=True)
        self._wgrad(B, H, t["da2"], 32, 0, 32, t["p1"], 16, 0, 16, "c2a")
        self._conv(B, H, t["da2"], 32, 0, 32, "c2a", 16, t["dp1"], 16, 0, relu=False, dgrad=True)
        # level 0 encoder
        self._check(L.dsmc_sg_pool2_bwd(s, B, S, self._ptr(t["dp1"]), 16, 0, self._ptr(t["dcat1"]), 48, 32,
                                        self._ptr(t["cat1"]), 48, 32, 16, self._ptr(t["dc1b"]), 16, 0))
        self._wgrad(B, S, t["dc1b"], 16, 0, 16, t["a1"], 16, 0, 16, "c1b")
        self._conv(B, S, t["dc1b"], 16, 0, 16, "c1b", 16, t["da1"], 16, 0, relu=False, mask=t["a1"], mcs=16,
                   dgrad=True)
        self._wgrad(B, S, t["da1"], 16, 0, 16, t["x0"], 16, 0, 16, "c1a")

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.adam_step += 1
        self._check(self.lib.dsmc_sg_adam(self._s(), self._ptr(self.p), self._ptr(self.g), self._ptr(self.m),
                                          self._ptr(self.v), self.nparams, C.c_float(lr), C.c_float(beta1),
                                          C.c_float(beta2), C.c_float(eps), self.adam_step))
        self.pack_weights()

    def status(self, clear: bool = True) -> int:
        f = C.c_uint()
        self._check(self.lib.dsmc_sg_status(C.byref(f), 1 if clear else 0))
        return f.value

    def grads_host(self) -> dict:
        g = self.g.detach().cpu().numpy()
        return {k: g[o:o + int(np.prod(sh))].reshape(sh) for k, (o, sh) in self.layout.items()}


def benchmark(batch: int = 8, S: int = 64, repeats: int = 5, device: int = 0) -> dict:
    """Times one training step of the network (forward, backward, Adam) and
    each 3x3x3 convolution of it (forward, input gradient, weight gradient)
    with CUDA events on the current stream; returns milliseconds and the
    achieved dense bf16 TFLOP/s (2 * voxels * 27 * cin * cout per call)."""
    import torch
    dev = torch.device("cuda", device)
    net = UNet(device, seed=0)
    rng = np.random.default_rng(0)
    solid = torch.tensor((rng.random((batch, S, S, S)) < 0.4).astype(np.uint8), device=dev)
    feat = torch.zeros(batch, dtype=torch.float32, device=dev)
    target = torch.zeros((batch, S, S, S, 4), dtype=torch.float32, device=dev)
    valid = (solid == 0).to(torch.uint8)
    cw = [1.0, 1.0, 1.0, 1.0]
    for _ in range(2):
        net.forward(solid, feat)
        net.backward(target, valid, cw)
        net.adam()
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(st)
    for _ in range(repeats):
        net.forward(solid, feat)
        net.backward(target, valid, cw)
        net.adam()
    e1.record(st)
    e1.synchronize()
    step_ms = e0.elapsed_time(e1) / repeats
    t = net.buf.t
    L = net.lib
    layers = {}
    levels = {0: S, 1: S // 2, 2: S // 4}
    src = {"c1a": ("x0", 16), "c1b": ("a1", 16), "c2a": ("p1", 16), "c2b": ("a2", 32), "c3a": ("p2", 32),
           "c3b": ("a3", 64), "c2c": ("cat2", 96), "c2d": ("d2", 32), "c1c": ("cat1", 48), "c1d": ("d1", 16)}
    flops_total = 0.0
    for name, cin, cout, lev in LAYERS:
        E = levels[lev]
        x, xcs = src[name]
        y = torch.empty((batch, E, E, E, cout), dtype=torch.int16, device=dev)
        dy = torch.zeros((batch, E, E, E, cout), dtype=torch.int16, device=dev)
        dx = torch.empty((batch, E, E, E, cin), dtype=torch.int16, device=dev)
        flops = 2.0 * batch * E ** 3 * 27 * cin * cout
        res = {}
        for kind in ("forward", "dgrad", "wgrad"):
            torch.cuda.synchronize(dev)
            e0.record(st)
            for _ in range(repeats):
                if kind == "forward":
                    net._conv(batch, E, t[x], xcs, 0, cin, name, cout, y, cout, 0)
                elif kind == "dgrad":
                    net._conv(batch, E, dy, cout, 0, cout, name, cin, dx, cin, 0, relu=False, dgrad=True)
                else:
                    capi.check(L.dsmc_sg_conv3_wgrad(net._s(), batch, E, net._ptr(dy), cout, 0, cout, net._ptr(t[x]),
                                                     xcs, 0, cin, net._gp(name + ".w")))
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / repeats
            res[kind] = {"ms": ms, "tflops": flops / (ms / 1e3) / 1e12}
        layers[name] = {"cin": cin, "cout": cout, "edge": E, "gflop": flops / 1e9, **res}
        flops_total += 3 * flops
    return {"batch": batch, "edge": S, "train_step_ms": step_ms,
            "train_step_tflops": flops_total / (step_ms / 1e3) / 1e12, "layers": layers,
            "status": net.status()}


def _one_step(batch: int = 8, S: int = 64, device: int = 0) -> None:
    """One forward and backward pass of a random-init network on random
    masks (the small case its kernels are profiled on)."""
    import torch
    dev = torch.device("cuda", device)
    net = UNet(device, seed=0)
    rng = np.random.default_rng(0)
    solid = torch.tensor((rng.random((batch, S, S, S)) < 0.4).astype(np.uint8), device=dev)
    feat = torch.zeros(batch, dtype=torch.float32, device=dev)
    tgt = torch.zeros((batch, S, S, S, 4), dtype=torch.float32, device=dev)
    out = net.forward(solid, feat)
    net.backward(tgt, (solid == 0).to(torch.uint8), [1.0, 1.0, 1.0, 1.0])
    torch.cuda.synchronize(dev)
    print("one training step", batch, S, float(out.abs().mean()), "status", net.status())


if __name__ == "__main__":
    import sys
    _one_step(*(int(x) for x in sys.argv[1:3]))
