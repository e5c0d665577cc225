"""The field entry points: per-voxel particle sums (dsmc_field_accumulate)
against the same sums from the particles read back, and the field-seeded
initialisation (dsmc_particles_init_field) against its definition: voxels
drawn by weight, only empty ones, velocities a Maxwellian about each voxel's
drift."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from master_b200 import capi, fields, workloads
from master_b200.system import T0_TEMP, System

pytestmark = pytest.mark.gpu


def voxel_index(r, g, L):
    n = np.array(g.shape)
    c = np.floor(r / (L / n)).astype(np.int64)
    c = np.clip(c, 0, n - 1)
    return (c[:, 0] * n[1] + c[:, 1]) * n[2] + c[:, 2]


@pytest.mark.parametrize("precision", [capi.PREC_SPLIT32, capi.PREC_FP64])
@pytest.mark.parametrize("device", [0, 1])
def test_field_sums_equal_the_particles(precision, device):
    w = workloads.PACKED_64
    s = w.settings(rng_seed=4, statistics_interval=10 ** 9)
    g = w.geometry()
    S = System(s, g, precision=precision)
    S.step(3)
    V = int(np.prod(g.shape))
    if device:
        f = torch.zeros((V, 4), dtype=torch.float32, device="cuda")
        for _ in range(2):
            S.ctx.check(S.ctx.lib.dsmc_field_accumulate(S.ctx.handle, S.id, C.c_void_p(f.data_ptr()), 1))
        S.ctx.sync()  # device mode is asynchronous on the context's stream
        got = f.cpu().numpy().astype(np.float64) / 2
    else:
        f = np.zeros((V, 4), np.float32)
        S.ctx.check(S.ctx.lib.dsmc_field_accumulate(S.ctx.handle, S.id, C.c_void_p(f.ctypes.data), 0))
        got = f.astype(np.float64)
    r, v = S.get_particles()
    idx = voxel_index(r, g, s.Lx)
    ref = np.zeros((V, 4))
    np.add.at(ref[:, 0], idx, 1.0)
    for d in range(3):
        np.add.at(ref[:, 1 + d], idx, v[:, d])
    assert np.array_equal(got[:, 0], ref[:, 0])
    assert np.allclose(got[:, 1:], ref[:, 1:], rtol=1e-5, atol=1e-5)
    assert got[g.voxels.ravel() > 0, 0].sum() <= 1e-3 * len(r)  # boundary voxels hold a few


def test_field_seeded_particles_follow_the_field():
    w = workloads.PACKED_64
    s = w.settings(rng_seed=8, statistics_interval=10 ** 9)
    g = w.geometry()
    V = int(np.prod(g.shape))
    empty = g.voxels.ravel() == 0
    # weights: twice as dense in the upper half along x; drift +u in the lower, -u in the upper
    i = np.arange(V) // (g.shape[1] * g.shape[2])
    upper = i >= g.shape[0] // 2
    weight = np.where(empty, np.where(upper, 2.0, 1.0), 5.0).astype(np.float32)  # solid weight ignored
    u = 0.05
    drift = np.zeros((V, 3), np.float32)
    drift[:, 0] = np.where(upper, -u, u)
    S = System(s, g, init_particles=False)
    n = 2_000_000
    S.ctx.check(S.ctx.lib.dsmc_particles_init_field(S.ctx.handle, S.id, n, weight.ctypes.data, drift.ctypes.data, 0))
    assert S.num_molecules == n
    r, v = S.get_particles()
    idx = voxel_index(r, g, s.Lx)
    assert empty[idx].all()
    up = upper[idx]
    # expected share of the upper half: its weight over the total
    w_up = (2.0 * (empty & upper)).sum()
    w_lo = (1.0 * (empty & ~upper)).sum()
    frac = w_up / (w_up + w_lo)
    assert abs(up.mean() - frac) < 5 * np.sqrt(frac * (1 - frac) / n)
    sig = np.sqrt(s.temperature / T0_TEMP / s.mass)  # sqrt(T/m) in reduced units
    for sel, ux in ((up, -u), (~up, u)):
        m = v[sel].mean(0)
        se = sig / np.sqrt(sel.sum())
        assert abs(m[0] - ux) < 5 * se and abs(m[1]) < 5 * se and abs(m[2]) < 5 * se
        assert v[sel].std(0) == pytest.approx([sig] * 3, rel=0.01)
    # the seeded state steps like any other
    S.step(2)
    assert S.ctx.device_status()[0] & capi.EBIT_FATAL == 0


def test_field_seeding_rejects_a_field_without_weight():
    w = workloads.PACKED_64
    g = w.geometry()
    S = System(w.settings(), g, init_particles=False)
    V = int(np.prod(g.shape))
    weight = np.where(g.voxels.ravel() == 0, 0.0, 1.0).astype(np.float32)
    drift = np.zeros((V, 3), np.float32)
    with pytest.raises(capi.DsmcError) as e:
        S.ctx.check(S.ctx.lib.dsmc_particles_init_field(S.ctx.handle, S.id, 100, weight.ctypes.data,
                                                       drift.ctypes.data, 0))
    assert e.value.code == capi.DSMC_ERR_STATE
