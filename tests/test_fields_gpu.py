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


def _synthetic_field(g, phase):
    """A weight and drift pattern over the voxels of g, as finish_field writes them."""
    V = int(np.prod(g.shape))
    i = np.arange(V) // (g.shape[1] * g.shape[2])
    out = np.zeros((V, 4))
    out[:, 0] = 1.0 + 0.5 * np.sin(2 * np.pi * i / g.shape[0] + phase)
    out[:, 1] = 30.0 * np.cos(2 * np.pi * i / g.shape[0] + phase)
    out[:, 2] = 5.0
    return out


def test_field_seeding_many_systems_at_once_equals_one_call_each():
    """dsmc_particles_init_field_many on systems of one context (one
    re-layout) gives each system the particles, and then the trajectory, of
    dsmc_particles_init_field on that system alone."""
    specs = fields.random_specs(4, 32, seed=44, per_cell=20)
    ens = fields.Ensemble(specs, rng_seed=60, cold=False)
    solids = [(g.voxels > 0).astype(np.uint8).ravel() for g in ens.geoms]
    outs = [_synthetic_field(g, k) for k, g in enumerate(ens.geoms)]
    counts = [30_000 + 1000 * k for k in range(len(specs))]
    fields.warm_start_many(ens.ctx, ens.systems, outs, solids, counts, group=3)  # two calls: 3 + 1
    ens.ctx.step(5)
    for k, S in enumerate(ens.systems):
        alone = System(ens.settings[k], ens.geoms[k], init_particles=False)
        fields.warm_start(alone, outs[k], solids[k], n=counts[k])
        alone.step(5)
        ra, va, ca = S.get_particles(with_cells=True)
        rb, vb, cb = alone.get_particles(with_cells=True)
        assert len(ra) == counts[k]
        assert np.array_equal(ra, rb) and np.array_equal(va, vb) and np.array_equal(ca, cb), k
        alone.ctx.close()
    # uniform density: the weight 1 in every empty voxel, the fields' drift
    ens2 = fields.Ensemble(specs[:2], rng_seed=60, cold=False)
    fields.warm_start_many(ens2.ctx, ens2.systems, outs[:2], solids[:2], counts[:2], uniform_density=True)
    for k, S in enumerate(ens2.systems):
        alone = System(ens2.settings[k], ens2.geoms[k], init_particles=False)
        flat = outs[k].copy()
        flat[:, 0] = 1.0
        fields.warm_start(alone, flat, solids[k], n=counts[k])
        ra, va = S.get_particles()
        rb, vb = alone.get_particles()
        assert np.array_equal(ra, rb) and np.array_equal(va, vb), k
        alone.ctx.close()
    ens2.close()
    assert ens.ctx.device_status()[0] & capi.EBIT_FATAL == 0
    ens.close()


def test_field_seeding_many_checks_every_field_first():
    specs = fields.random_specs(2, 32, seed=45, per_cell=20)
    ens = fields.Ensemble(specs, rng_seed=61)
    before = [S.get_particles() for S in ens.systems]
    solids = [(g.voxels > 0).astype(np.uint8).ravel() for g in ens.geoms]
    outs = [_synthetic_field(g, 0.0) for g in ens.geoms]
    outs[1][:, 0] = 0.0  # no weight anywhere in the second system
    with pytest.raises(capi.DsmcError) as e:
        fields.warm_start_many(ens.ctx, ens.systems, outs, solids, [1000, 1000])
    assert e.value.code == capi.DSMC_ERR_STATE
    for S, (r, v) in zip(ens.systems, before):  # nothing replaced
        r2, v2 = S.get_particles()
        assert np.array_equal(r, r2) and np.array_equal(v, v2)
    # a system listed twice
    ids = (C.c_int * 2)(ens.systems[0].id, ens.systems[0].id)
    with pytest.raises(capi.DsmcError) as e:
        ens.ctx.check(ens.ctx.lib.dsmc_particles_init_many(ens.ctx.handle, 2, ids, None))
    assert e.value.code == capi.DSMC_ERR_ARG
    ens.close()
