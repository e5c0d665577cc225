"""The production split-precision pass against the fp64 path at the
benchmark scales, one step from a common state.

The fp64 path reproduces the reference's own routines bit for bit
(tests/test_parity_gpu.py: positions identical, velocities within 1e-12,
integer voxel and cell indices and every counter identical).  The draws of
both precisions are keyed by particle id, cell and step, never by precision,
so the fp64 path serves as the yardstick of the production kernels at full size:

* packed_64: 64^3 voxels, r = 4 voxel spheres to porosity 0.6, 32^3 cells,
  ~3.9e5 particles (the plain-DSMC configuration);
* packed_128: 128^3 voxels, r = 6, porosity 0.5, 64^3 cells, ~3.9e6
  particles (the large-geometry physics at 1/8 of its volume).

Each case starts both paths from one state (the initial Maxwellian, and the
state after 30 fp64 steps with its cell bookkeeping) and runs one full step
(accelerate, move, re-bin, collide).  Bars, for every particle that meets no
wall in the step (its fp64 end point is the ballistic one):

* the voxel and cell indices are identical, except for a particle whose fp64
  end point lies within 1e-6 voxel of a voxel face, where the fp32 offset
  may round to the neighbour (counted; at most 1e-5 of the particles);
* positions agree within 1e-6 of the box length (MoleculeMover::move_molecule,
  dsmc/moleculemover.cpp:50-126; Grid::get_index_of_voxel, dsmc/grid.h:139-145).

Wall-hitting particles are reported (fraction whose voxel differs or whose
position strays beyond 1e-6 L) and held to 2 %; the collision count agrees
to 1e-4 (Cell::collide, dsmc/cell.cpp:75-111).
"""
from __future__ import annotations

import numpy as np
import pytest

from master_b200 import capi, workloads
from master_b200.system import System

pytestmark = pytest.mark.gpu

FACE_BAND = 1e-6      # voxel units
POS_TOL = 1e-6        # of the box length


def periodic_dist(a, b, L):
    d = np.abs(a - b)
    return np.minimum(d, L - d)


def ballistic(r0, v0, s):
    """The end point of a flight that meets no wall: accelerate along the
    flow axis, then r + v dt with one periodic wrap per axis
    (System::accelerate, dsmc/system.cpp:133-144; moleculemover.h:29-38)."""
    v = v0.copy()
    if s.flow_direction >= 0:
        v[:, s.flow_direction] += s.gravity * s.dt
    r = r0 + v * s.dt
    L = np.array([s.Lx, s.Ly, s.Lz])
    return np.mod(r, L)


def voxel_of(r, n, L):
    return np.floor(r * (n / L)).astype(np.int64) % n


def compare_one_step(w, r0, v0, cell_state=None):
    s = w.settings(rng_seed=7, statistics_interval=10 ** 9)
    g = w.geometry()
    out = {}
    for name, prec in (("fp64", capi.PREC_FP64), ("split", capi.PREC_SPLIT32)):
        S = System(s, g, precision=prec, init_particles=False)
        S.set_particles(r0, v0)
        if cell_state is not None:
            S.set_cell_state(*cell_state)
        S.step(1)
        r, v, cell = S.get_particles(with_cells=True)
        err, _ = S.ctx.device_status()
        assert err & capi.EBIT_FATAL == 0, (name, hex(err))
        out[name] = (r, v, cell, S.tallies())
        S.ctx.close()
    L = s.Lx
    rf, vf, cf, tf = out["fp64"]
    rs, vs, cs, ts = out["split"]
    n = w.n
    N = len(r0)
    wall_free = periodic_dist(rf, ballistic(r0, v0, s), L).max(1) <= 1e-9 * L
    scaled = rf * (n / L)
    frac = scaled - np.floor(scaled)
    near_face = (np.minimum(frac, 1 - frac) < FACE_BAND).any(1)
    vox_f, vox_s = voxel_of(rf, n, L), voxel_of(rs, n, L)
    same_vox = (vox_f == vox_s).all(1)
    pos_ok = periodic_dist(rf, rs, L).max(1) <= POS_TOL * L
    strict = wall_free & ~near_face
    # every wall-free particle away from a face: identical indices, close positions
    bad = strict & ~(same_vox & (cf == cs) & pos_ok)
    assert not bad.any(), f"{bad.sum()} wall-free particles differ, e.g. ids {np.flatnonzero(bad)[:5]}"
    # within the face band: at most one voxel apart, and rare
    band = wall_free & near_face
    assert (np.abs(vox_f[band] - vox_s[band]) % (n - 1) <= 1).all()
    band_flips = int((band & ~same_vox).sum())
    assert band_flips <= max(5, 1e-5 * N)
    assert pos_ok[wall_free].all()
    # wall hitters: reported, held to 2 %
    hit = ~wall_free
    hit_mismatch = int((hit & ~(same_vox & pos_ok)).sum())
    assert hit_mismatch <= 0.02 * max(1, hit.sum())
    # collisions and wall hits of the step
    assert abs(int(tf.collisions) - int(ts.collisions)) <= 1e-4 * tf.collisions + 5
    assert abs(int(tf.wall_collisions) - int(ts.wall_collisions)) <= 1e-3 * tf.wall_collisions + 5
    assert list(tf.count_periodic) == list(ts.count_periodic) or \
        np.abs(np.subtract(tf.count_periodic, ts.count_periodic)).max() <= 2
    # velocities of wall-free particles: fp32 state, fp64 bookkeeping
    vscale = np.sqrt((vf ** 2).mean())
    dv = np.abs(vf - vs).max(1)
    assert (dv[strict] <= 1e-5 * vscale).mean() >= 0.9999
    return {"particles": N, "wall_free": int(wall_free.sum()), "wall_hits": int(hit.sum()),
            "wall_hit_mismatch": hit_mismatch, "face_band": int(band.sum()), "face_band_flips": band_flips,
            "collisions": (int(tf.collisions), int(ts.collisions))}


def initial_state(w, seed=3):
    s = w.settings(rng_seed=seed)
    S = System(s, w.geometry(), precision=capi.PREC_FP64)
    r, v = S.get_particles()
    S.ctx.close()
    return r, v


def developed_state(w, steps=30, seed=5):
    s = w.settings(rng_seed=seed, statistics_interval=10 ** 9)
    S = System(s, w.geometry(), precision=capi.PREC_FP64)
    S.step(steps)
    r, v = S.get_particles()
    c = S.cells()
    S.ctx.close()
    return r, v, (c["vr_max"], c["rest"])


@pytest.mark.parametrize("name", ["packed_64", "packed_128"])
def test_production_pass_matches_fp64_from_initial_state(name):
    w = workloads.WORKLOADS[name]
    r0, v0 = initial_state(w)
    rep = compare_one_step(w, r0, v0)
    print(name, "initial", rep)


@pytest.mark.parametrize("name", ["packed_64", "packed_128"])
def test_production_pass_matches_fp64_from_developed_state(name):
    w = workloads.WORKLOADS[name]
    r0, v0, cells = developed_state(w)
    rep = compare_one_step(w, r0, v0, cells)
    print(name, "developed", rep)
