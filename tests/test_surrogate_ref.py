"""The CPU reference of the surrogate network (oracle/unet_ref.py) and the
host-side parameter layout, without a GPU."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from master_b200 import surrogate as sgm
from oracle import unet_ref


def test_parameter_layouts_agree():
    layout, n = sgm.parameter_layout()
    p = np.arange(n, dtype=np.float64)
    u = unet_ref.unpack(p)
    assert set(u) == set(layout)
    for k, (o, shape) in layout.items():
        assert u[k].shape == shape
        assert u[k].flat[0] == o
    assert [(a, b, c) for a, b, c, _ in sgm.LAYERS] == unet_ref.LAYERS
    assert n == 359_812


def test_reference_gradient_matches_finite_differences():
    """fp64 without bf16 emulation: the analytic gradient of the loss (the
    per-sample flux term included) equals central differences along random
    directions (periodic padding, pooling, upsampling, skips and the head
    included)."""
    rng = np.random.default_rng(0)
    B, S = 1, 16
    solid = (rng.random((B, S, S, S)) < 0.3).astype(np.uint8)
    feature = np.array([0.3])
    target = rng.normal(0, 1, (B, S, S, S, 4))
    valid = 1 - solid
    cw = [1.0, 0.5, 0.5, 0.5]
    p = sgm.init_parameters(seed=2).astype(np.float64)
    for k, (o, sh) in sgm.parameter_layout()[0].items():
        if k.endswith(".b"):
            p[o:o + int(np.prod(sh))] = rng.normal(0, 0.05, int(np.prod(sh)))
    ref = unet_ref.UNetRef(p, emulate_bf16=False)
    loss = ref.loss(ref.forward(solid, feature), target, valid, cw, flux_weight=2.0)
    loss.backward()
    g = ref.grads()
    flat = np.concatenate([g[k].ravel() for k in unet_ref.unpack(p)])  # layout order
    layout, n = sgm.parameter_layout()
    gvec = np.zeros(n)
    for k, (o, sh) in layout.items():
        gvec[o:o + int(np.prod(sh))] = g[k].ravel()
    assert flat.shape == gvec.shape

    def f(q):
        r = unet_ref.UNetRef(q, emulate_bf16=False)
        with torch.no_grad():
            return r.loss(r.forward(solid, feature), target, valid, cw, flux_weight=2.0).item()

    for trial in range(3):
        d = rng.normal(0, 1, n)
        d /= np.linalg.norm(d)
        h = 1e-4
        fd = (f(p + h * d) - f(p - h * d)) / (2 * h)
        # ReLU kinks within the step keep central differences from O(h^2) accuracy
        assert fd == pytest.approx(float(gvec @ d), rel=1e-3, abs=1e-9)


def test_bf16_emulation_changes_the_loss_by_rounding_only():
    rng = np.random.default_rng(1)
    B, S = 1, 16
    solid = (rng.random((B, S, S, S)) < 0.3).astype(np.uint8)
    p = sgm.init_parameters(seed=5).astype(np.float64)
    a = unet_ref.UNetRef(p, emulate_bf16=True).forward(solid, [0.1]).detach().numpy()
    b = unet_ref.UNetRef(p, emulate_bf16=False).forward(solid, [0.1]).detach().numpy()
    err = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert 1e-5 < err < 5e-2


def test_committed_weights_predict_a_plausible_field():
    """The trained weights shipped with the library (master_b200/weights/),
    run through the CPU reference on two unseen 64^3 packs: a finite field
    whose density averages 1 over the empty voxels (the targets are density
    over the box mean) and whose mean drift points along the body force (x),
    with the cross-stream means small against it."""
    from pathlib import Path
    from master_b200 import fields
    z = np.load(Path(sgm.__file__).resolve().parent / "weights" / "surrogate_64.npz")
    assert z["params"].shape == (sgm.parameter_layout()[1],)
    net = unet_ref.UNetRef(z["params"].astype(np.float64), emulate_bf16=False)
    for sp in fields.random_specs(2, 64, seed=9, porosity=(0.45, 0.75), knudsen=(0.3, 3.0)):
        solid = (sp.geometry().voxels > 0).astype(np.uint8)
        with torch.no_grad():
            out = net.forward(solid[None], np.array([np.log10(sp.knudsen)])).numpy()[0].reshape(-1, 4)
        empty = solid.ravel() == 0
        assert np.isfinite(out).all()
        assert abs(out[empty, 0].mean() - 1.0) < 0.05
        drift = out[empty, 1:].mean(axis=0)
        assert drift[0] > 0
        assert np.abs(drift[1:]).max() < 0.2 * drift[0]
