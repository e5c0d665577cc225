"""TEST INFRASTRUCTURE: CPU reference of the warm-start surrogate network
(master_b200/surrogate.py), the checker of its GPU forward and backward
kernels.  Never imported by the library.

The reference project has no surrogate (it always starts from a Maxwellian at
rest, dsmc/system.cpp:398-430), so there is nothing of it to pin against;
this restatement is built from torch's CPU conv3d / avg_pool3d / autograd in
fp64.  With `emulate_bf16` it rounds to bf16 at exactly the points where the
GPU path stores a bf16 tensor, in the forward pass (weights, every
activation, pooled volumes) and in the backward pass (the gradient of every
convolution's pre-activation, of the concatenated skip volumes and of the
pooled volumes), so the two can be compared tightly.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

LAYERS = [
    ("c1a", 16, 16), ("c1b", 16, 16), ("c2a", 16, 32), ("c2b", 32, 32), ("c3a", 32, 64), ("c3b", 64, 64),
    ("c2c", 96, 32), ("c2d", 32, 32), ("c1c", 48, 16), ("c1d", 16, 16),
]


def bf16(x: torch.Tensor) -> torch.Tensor:
    return x.to(torch.bfloat16).to(x.dtype)


class _RoundGrad(torch.autograd.Function):
    """Identity forward; rounds the incoming gradient to bf16."""

    @staticmethod
    def forward(ctx, x):
        return x.view_as(x)

    @staticmethod
    def backward(ctx, g):
        return bf16(g)


def unpack(params: np.ndarray):
    """The flat parameter vector (master_b200.surrogate.parameter_layout)."""
    out, off = {}, 0
    for name, cin, cout in LAYERS:
        n = cout * 27 * cin
        out[name + ".w"] = params[off:off + n].reshape(cout, 27, cin)
        off += n
        out[name + ".b"] = params[off:off + cout]
        off += cout
    out["head.w"] = params[off:off + 64].reshape(4, 16)
    off += 64
    out["head.b"] = params[off:off + 4]
    off += 4
    assert off == params.size
    return out


class UNetRef:
    def __init__(self, params: np.ndarray, emulate_bf16: bool = True):
        self.emulate = emulate_bf16
        self.t = {k: torch.tensor(np.asarray(v, np.float64), requires_grad=True) for k, v in unpack(params).items()}

    def _act(self, x):
        """Stored activation: rounded to bf16 (straight-through gradient)."""
        if not self.emulate:
            return x
        return x + (bf16(x) - x).detach()

    def _rg(self, x):
        return _RoundGrad.apply(x) if self.emulate else x

    def _conv(self, x, name, relu=True):
        w = self.t[name + ".w"]
        cout, _, cin = w.shape
        if self.emulate:
            w = w + (bf16(w) - w).detach()
        W = w.reshape(cout, 3, 3, 3, cin).permute(0, 4, 1, 2, 3)
        y = F.conv3d(F.pad(x, (1, 1, 1, 1, 1, 1), mode="circular"), W) + self.t[name + ".b"].view(1, -1, 1, 1, 1)
        y = self._rg(y)
        if relu:
            y = torch.relu(y)
        return self._act(y)

    def _pool(self, x):
        return self._rg(self._act(F.avg_pool3d(x, 2)))

    @staticmethod
    def _up(x):
        return x.repeat_interleave(2, 2).repeat_interleave(2, 3).repeat_interleave(2, 4)

    def forward(self, solid: np.ndarray, feature: np.ndarray) -> torch.Tensor:
        """solid (B, S, S, S) uint8, feature (B,) -> output (B, S, S, S, 4) fp64."""
        B, S = solid.shape[0], solid.shape[1]
        x = torch.zeros((B, 16, S, S, S), dtype=torch.float64)
        x[:, 0] = torch.tensor((solid == 0).astype(np.float64))
        x[:, 1] = torch.tensor(np.asarray(feature, np.float64)).view(B, 1, 1, 1)
        if self.emulate:
            x = bf16(x)
        a1 = self._conv(x, "c1a")
        s1 = self._conv(a1, "c1b")
        p1 = self._pool(s1)
        a2 = self._conv(p1, "c2a")
        s2 = self._conv(a2, "c2b")
        p2 = self._pool(s2)
        a3 = self._conv(p2, "c3a")
        b3 = self._conv(a3, "c3b")
        cat2 = self._rg(torch.cat([self._up(b3), s2], 1))
        d2 = self._conv(cat2, "c2c")
        e2 = self._conv(d2, "c2d")
        cat1 = self._rg(torch.cat([self._up(e2), s1], 1))
        d1 = self._conv(cat1, "c1c")
        e1 = self._conv(d1, "c1d")
        out = torch.einsum("bkzyx,ck->bzyxc", e1, self.t["head.w"]) + self.t["head.b"]
        return out

    def loss(self, out, target: np.ndarray, valid: np.ndarray, channel_weight, flux_weight: float = 0.0):
        """sum over valid voxels and channels of cw (out - target)^2 / count,
        plus flux_weight * the batch mean of (each sample's mean over its
        valid voxels of out - target in channel 1)^2."""
        tg = torch.tensor(np.asarray(target, np.float64))
        m = torch.tensor(np.asarray(valid, bool))
        cw = torch.tensor(np.asarray(channel_weight, np.float64))
        count = max(1, int(m.sum()))
        d = (out - tg) ** 2 * cw
        loss = d[m].sum() / count
        if flux_weight:
            B = out.shape[0]
            mf = m.reshape(B, -1).to(out.dtype)
            diff = (out[..., 1] - tg[..., 1]).reshape(B, -1)
            mean = (diff * mf).sum(1) / mf.sum(1).clamp(min=1)
            loss = loss + flux_weight * (mean ** 2).mean()
        return loss

    def grads(self) -> dict:
        return {k: v.grad.detach().numpy().copy() for k, v in self.t.items()}
