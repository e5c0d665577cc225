"""GPU parity of the timestep against the reference's own routines.

The golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py
from oracle/_ref, the reference built from its sources) hold the reference's
state after its setup_molecules, one accelerate+move, one cell re-binning,
one NTC collide and ten full steps, all fed the same counter-based draws as
the kernels.  Bar: integer voxel/cell indices and counters bit-exact; fp64
positions and velocities within 1e-12 (the only differences come from libm
vs CUDA log/cos in wall reflections and collisions, a few ulp).
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from master_b200 import capi
from master_b200.system import Geometry, Settings, System

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ["small_dt1", "small_dt5", "small_specular", "small_cl"]
WALL_MODELS = {"thermal": 0, "specular": 1, "cercignani_lampis": 2}
TOL = 1e-12


def load_case(case):
    z = np.load(GOLDEN / f"{case}.npz")
    meta = json.loads(str(z["meta"]))
    c = meta["params"]
    g = Geometry.packed_spheres(c["n"], c["radius_voxels"], wanted_porosity=c["porosity"], seed=c["geom_seed"])
    s = Settings()
    st = meta["settings"]
    for k in ("Lx", "Ly", "Lz", "cells_x", "cells_y", "cells_z", "dt", "diam", "atoms_per_molecule", "mass",
              "temperature", "wall_temperature", "gravity", "flow_direction", "density"):
        setattr(s, k, st[k])
    s.statistics_interval = 1
    s.max_molecules_per_node = st["max_molecules"]
    s.rng_seed = c["rng_seed"]
    s.surface_model = WALL_MODELS[st.get("surface", "thermal")]
    s.alpha_n = st.get("alpha_n", 0.5)
    s.alpha_t = st.get("alpha_t", 0.8)
    return z, meta, s, g


def thermal(meta) -> bool:
    """Only the reference's thermal collider counts wall collisions
    (dsmc/colliderthermal.cpp:45); this library counts them for every model."""
    return meta["settings"].get("surface", "thermal") == "thermal"


def voxel_of(r, n, L):
    """The reference's Grid::get_index_of_voxel for the fixture boxes
    (n/L exactly representable: 10 voxels per um)."""
    return np.floor(r * (n / L)).astype(np.int64) % n


@pytest.mark.parametrize("case", CASES)
def test_init_matches_reference(case):
    z, meta, s, g = load_case(case)
    S = System(s, g, precision=capi.PREC_FP64)
    assert S.num_molecules == meta["n"]
    r, v, cell = S.get_particles(with_cells=True)
    assert np.array_equal(r, z["r0"])
    assert np.abs(v - z["v0"]).max() <= TOL
    assert np.array_equal(cell, z["cell0"])


@pytest.mark.parametrize("case", CASES)
def test_stages_match_reference(case):
    """One timestep stage by stage: accelerate+move, re-bin, collide."""
    z, meta, s, g = load_case(case)
    S = System(s, g, precision=capi.PREC_FP64, init_particles=False)
    S.set_particles(z["r0"], z["v0"])
    S.accelerate_and_move()
    r1, v1 = S.get_particles()
    assert np.abs(r1 - z["r1"]).max() <= TOL
    assert np.abs(v1 - z["v1"]).max() <= TOL
    n, L = meta["params"]["n"], meta["settings"]["Lx"]
    assert np.array_equal(voxel_of(r1, n, L), voxel_of(z["r1"], n, L))
    t = S.tallies()
    ref = meta["counters_move"]
    assert t.wall_collisions == ref["wall_collisions"] or not thermal(meta)
    assert list(t.count_periodic) == ref["count_periodic"]
    assert t.reseeds == 0
    S.update_molecule_cells()
    _, _, cell1 = S.get_particles(with_cells=True)
    assert np.array_equal(cell1, z["cell1"])
    cells = S.cells()
    assert np.array_equal(cells["global_index"], z["cell_global"])
    assert np.array_equal(cells["count"], z["count1"])
    S.collide()
    _, v1c = S.get_particles()
    assert np.abs(v1c - z["v1c"]).max() <= TOL
    cells = S.cells()
    assert np.abs(cells["vr_max"] - z["vr_max1"]).max() <= TOL
    assert np.abs(cells["rest"] - z["rest1"]).max() <= TOL
    assert S.tallies().collisions == meta["counters_collide"]["collisions"]


@pytest.mark.parametrize("case", CASES)
def test_fused_steps_match_reference(case):
    """Ten fused timesteps (one kernel pass per step) against ten reference steps."""
    z, meta, s, g = load_case(case)
    S = System(s, g, precision=capi.PREC_FP64, init_particles=False)
    S.set_particles(z["r0"], z["v0"])
    K = meta["params"]["steps"]
    S.step(K)
    r, v, cell = S.get_particles(with_cells=True)
    assert np.abs(r - z["rK"]).max() <= 1e-10
    assert np.abs(v - z["vK"]).max() <= 1e-10
    assert np.array_equal(cell, z["cellK"])
    t = S.tallies()
    ref = meta["counters_final"]
    assert t.collisions == ref["collisions"]
    assert t.wall_collisions == ref["wall_collisions"] or not thermal(meta)
    assert list(t.count_periodic) == ref["count_periodic"]
    assert t.step == K
    cells = S.cells()
    assert np.array_equal(cells["count"], z["countK"])
    assert np.abs(cells["vr_max"] - z["vr_maxK"]).max() <= 1e-10


@pytest.mark.parametrize("case", CASES)
def test_split_precision_tracks_reference(case):
    """int voxel + fp32 offset state: one step against the fp64 reference."""
    z, meta, s, g = load_case(case)
    S = System(s, g, precision=capi.PREC_SPLIT32, init_particles=False)
    S.set_particles(z["r0"], z["v0"])
    r0, _ = S.get_particles()
    L = meta["settings"]["Lx"]
    assert np.abs(r0 - z["r0"]).max() <= 1e-7 * L
    S.accelerate_and_move()
    S.update_molecule_cells()
    r1, v1, cell1 = S.get_particles(with_cells=True)
    d = np.abs(r1 - z["r1"])
    d = np.minimum(d, L - d)  # periodic
    close = d.max(1) <= 1e-6 * L
    # every particle that did not meet a wall this step agrees to fp32 precision;
    # wall hits agree too unless an fp32 rounding flips which face is reached
    assert close.mean() >= 0.995
    assert (cell1 == z["cell1"]).mean() >= 0.995


def run_pair(case, capacity=None):
    z, meta, s, g = load_case(case)
    A = System(s, g, precision=capi.PREC_SPLIT32, init_particles=False)
    if capacity:
        A.ctx.check(A.ctx.lib.dsmc_ctx_set_capacity(A.ctx.handle, *capacity))
    A.set_particles(z["r0"], z["v0"])
    return A, z, meta


@pytest.mark.parametrize("case", CASES)
def test_fused_pass_equals_stage_calls(case):
    """The production pass (collide, move, place and wall kernels) and the four
    stand-alone stage kernels give bit-identical trajectories."""
    A, z, meta = run_pair(case)
    B, _, _ = run_pair(case)
    assert A.ctx.pass_info()["pipelined"] == 1
    K = 6
    A.step(K)
    for _ in range(K):
        B.accelerate_and_move()
        B.update_molecule_cells()
        B.collide()
    ra, va, ca = A.get_particles(with_cells=True)
    rb, vb, cb = B.get_particles(with_cells=True)
    assert np.array_equal(ra, rb)
    assert np.array_equal(va, vb)
    assert np.array_equal(ca, cb)
    ta, tb = A.tallies(), B.tallies()
    for k in ("collisions", "wall_collisions", "reseeds", "candidates"):
        assert getattr(ta, k) == getattr(tb, k), k
    assert list(ta.count_periodic) == list(tb.count_periodic)


def test_overflow_spills_and_repacks_without_loss():
    """Cells with no spare slots overflow every step; the spill list and the
    host repack must give the same trajectories as ample capacity."""
    A, z, meta = run_pair("small_dt5")
    B, _, _ = run_pair("small_dt5", capacity=(1.0, 0))
    assert A.ctx.pass_info()["pipelined"] == 1 and B.ctx.pass_info()["pipelined"] == 1
    A.step(5)
    B.step(5)
    ra, va = A.get_particles()
    rb, vb = B.get_particles()
    assert np.array_equal(ra, rb) and np.array_equal(va, vb)
    assert A.tallies().step == B.tallies().step == 5
    assert A.ctx.device_status()[0] & 0xbd == 0


def test_rerun_is_bit_identical():
    A, _, _ = run_pair("small_dt1")
    B, _, _ = run_pair("small_dt1")
    A.step(8)
    B.step(3)
    B.step(5)
    ra, va = A.get_particles()
    rb, vb = B.get_particles()
    assert np.array_equal(ra, rb) and np.array_equal(va, vb)


def test_geometry_gpu_matches_cpu():
    import ctypes as C
    from master_b200.capi import ptr
    g = Geometry.packed_spheres(64, 4, wanted_porosity=0.6, seed=1)
    solid = (g.voxels > 0).astype(np.uint8)
    a = Geometry.from_mask(solid)
    b = Geometry.empty(64, 64, 64)
    b.voxels[...] = solid
    capi.check(capi.load().dsmc_geometry_finish_gpu(0, 64, 64, 64, 1, ptr(b.voxels, C.c_uint8),
                                                      ptr(b.normals, C.c_float), ptr(b.tangents1, C.c_float),
                                                      ptr(b.tangents2, C.c_float)))
    for k in ("voxels", "normals", "tangents1", "tangents2"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


@pytest.mark.parametrize("capacity", [None, (1.3, 0)])
def test_fused_equals_stages_dense_cells(capacity):
    """~40 particles per cell: the pipelined pass against the stage kernels.
    The default capacity gives a ring of at least 128 slots per warp; with
    tight capacity the ring holds fewer than three of the largest cells, so
    staging stops on a full ring, and cells overflow into the spill list."""
    from master_b200 import workloads
    w = workloads.Workload("dense32", n=32, radius_voxels=3, porosity=0.5, geometry_seed=3, cells=16,
                           atoms_per_molecule=workloads.simulators_per_cell_weight(2.5e24, 0.1, 2, 40))
    s = w.settings(rng_seed=99, statistics_interval=1)
    g = w.geometry()
    A = System(s, g)
    if capacity:
        A.ctx.check(A.ctx.lib.dsmc_ctx_set_capacity(A.ctx.handle, *capacity))
        A.set_particles(*A.get_particles())  # re-lay the cells out at the tight capacity
    B = System(s, g)
    info = A.ctx.pass_info()
    assert info["pipelined"] == 1
    if capacity is None:
        assert info["stage_capacity"] >= 128
    else:
        assert info["stage_capacity"] < 3 * A.cells()["count"].max()
    A.step(4)
    for _ in range(4):
        B.accelerate_and_move()
        B.update_molecule_cells()
        B.collide()
        B.sample()
    ra, va = A.get_particles()
    rb, vb = B.get_particles()
    assert np.array_equal(ra, rb) and np.array_equal(va, vb)
    ma, mb = A.cells()["moments"], B.cells()["moments"]
    assert np.allclose(ma, mb, rtol=1e-12, atol=1e-12)
    assert A.tallies().samples == B.tallies().samples == 4
