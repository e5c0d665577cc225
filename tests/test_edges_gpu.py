"""Edge cases of the timestep on the GPU: an empty system, a single
particle, a crowded cell far above the mean occupancy, and particles on the
box faces.  Each runs the production pass against the stand-alone stage
kernels (bit-identical trajectories) and checks that no particle is lost."""
from __future__ import annotations

import numpy as np
import pytest

from master_b200 import capi
from master_b200.system import System
from test_parity_gpu import load_case

pytestmark = pytest.mark.gpu


def pair(case, r, v):
    z, meta, s, g = load_case(case)
    A = System(s, g, init_particles=False)
    B = System(s, g, init_particles=False)
    A.set_particles(r, v)
    B.set_particles(r, v)
    return A, B


def run_both(A, B, K):
    A.step(K)
    for _ in range(K):
        B.accelerate_and_move()
        B.update_molecule_cells()
        B.collide()
        B.sample()
    ra, va, ca = A.get_particles(with_cells=True)
    rb, vb, cb = B.get_particles(with_cells=True)
    assert np.array_equal(ra, rb) and np.array_equal(va, vb) and np.array_equal(ca, cb)
    ta, tb = A.tallies(), B.tallies()
    for k in ("collisions", "wall_collisions", "candidates", "reseeds"):
        assert getattr(ta, k) == getattr(tb, k), k
    return ra, va


def test_empty_system_steps():
    z, meta, s, g = load_case("small_dt1")
    S = System(s, g, init_particles=False)
    S.set_particles(np.zeros((0, 3)), np.zeros((0, 3)))
    S.step(4)
    t = S.tallies()
    assert S.num_molecules == 0
    assert t.step == 4 and t.collisions == 0 and t.wall_collisions == 0 and t.particle_steps == 0
    r, v = S.get_particles()
    assert r.shape == (0, 3)
    assert not S.profile_sums().any()


def test_single_particle():
    z, meta, s, g = load_case("small_dt5")
    A, B = pair("small_dt5", z["r0"][:1], z["v0"][:1])
    r, v = run_both(A, B, 20)
    assert A.num_molecules == 1 and A.tallies().collisions == 0


@pytest.mark.parametrize("crowd", [110, 230])
def test_crowded_cell_spills_and_keeps_every_particle(crowd):
    """One cell starts with `crowd` particles (the mean is 15): its members
    take the production pass's large-cell paths, its neighbours overflow as
    the crowd spreads and the host repacks, and both paths still agree and
    keep every particle."""
    z, meta, s, g = load_case("small_dt5")
    r = z["r0"].copy()
    v = z["v0"].copy()
    N = r.shape[0]
    cell = z["cell0"]
    target = np.bincount(cell).argmax()
    home = r[np.flatnonzero(cell == target)[0]]
    others = np.flatnonzero(cell != target)[: crowd - int((cell == target).sum())]
    r[others] = home
    A, B = pair("small_dt5", r, v)
    assert A.cells()["count"].max() >= crowd
    assert A.ctx.pass_info()["pipelined"] == 1
    run_both(A, B, 6)
    assert A.num_molecules == N


def test_particles_on_the_box_faces():
    """Positions at 0 and one ulp below L in each direction (in the first and
    last voxel layers) wrap and move exactly as the stage kernels do."""
    z, meta, s, g = load_case("small_dt1")
    r = z["r0"].copy()
    v = z["v0"].copy()
    L = np.array([s.Lx, s.Ly, s.Lz])
    n = np.array(g.shape)
    vox = L / n
    used = set()
    for d in range(3):
        for upper in (False, True):
            layer = r[:, d] >= L[d] - vox[d] if upper else r[:, d] < vox[d]
            i = next(int(j) for j in np.flatnonzero(layer) if int(j) not in used)
            used.add(i)
            r[i, d] = np.nextafter(L[d], 0) if upper else 0.0
            v[i, d] = abs(v[i, d]) if upper else -abs(v[i, d])  # heading out of the box
    A, B = pair("small_dt1", r, v)
    ra, _ = A.get_particles()
    for i in used:
        assert (ra[i] >= 0).all() and (ra[i] < L).all()
    run_both(A, B, 5)
    assert A.num_molecules == r.shape[0]


def test_graph_replay_equals_plain_launches():
    """The production pass replayed from captured CUDA graphs (the default)
    and launched kernel by kernel (as with the per-kernel timers on) give
    bit-identical trajectories."""
    z, meta, s, g = load_case("small_dt5")
    A = System(s, g, init_particles=False)
    B = System(s, g, init_particles=False)
    A.set_particles(z["r0"], z["v0"])
    B.set_particles(z["r0"], z["v0"])
    B.ctx.set_timing(True)
    for k in (1, 3, 7):  # batches of several passes, every buffer parity and occupancy set
        A.step(k)
        B.step(k)
    ra, va, ca = A.get_particles(with_cells=True)
    rb, vb, cb = B.get_particles(with_cells=True)
    assert np.array_equal(ra, rb) and np.array_equal(va, vb) and np.array_equal(ca, cb)
    assert A.tallies().collisions == B.tallies().collisions
    assert B.ctx.pass_times()["passes"] > 0


@pytest.mark.parametrize("capacity", [None, (1.5, 3), (1.0, 0)])
def test_device_layout_follows_the_capacity_rule(capacity):
    """Cell capacities are computed on the device whenever the buffers are
    laid out: ceil(factor * max(expected, present) + pad) per active cell,
    expected = particles * free voxels of the cell / free voxels of the
    system (rounded without fused multiply-add), and the slots total their
    sum.  The counts come back through the device table as well."""
    from master_b200.system import cells_layout
    z, meta, s, g = load_case("small_dt5")
    S = System(s, g, init_particles=False)
    factor, pad = capacity or (2.0, 24)
    if capacity:
        S.ctx.check(S.ctx.lib.dsmc_ctx_set_capacity(S.ctx.handle, factor, pad))
    S.set_particles(z["r0"], z["v0"])
    cells = S.cells()
    lay = cells_layout(s, g)
    assert np.array_equal(cells["global_index"], lay["global_index"])
    present = cells["count"].astype(np.float64)
    assert present.sum() == z["r0"].shape[0]
    pix = lay["pixels"].astype(np.float64)
    expect = (z["r0"].shape[0] * pix) / pix.sum()
    cap = np.maximum(np.ceil(factor * np.maximum(expect, present) + pad), 1.0)
    assert S.info().slots == int(cap.sum())


@pytest.mark.parametrize("precision", [capi.PREC_SPLIT32, capi.PREC_FP64])
@pytest.mark.parametrize("where", ["r_nan", "v_nan", "v_inf"])
def test_non_finite_state_is_refused_and_the_system_keeps_its_particles(precision, where):
    """A non-finite position or velocity handed to dsmc_particles_set is
    refused (DSMC_ERR_STATE, the message says why) before it reaches a
    kernel; the system keeps the particles it had and steps on."""
    z, meta, s, g = load_case("small_dt1")
    S = System(s, g, precision=precision, init_particles=False)
    S.set_particles(z["r0"], z["v0"])
    r_before, v_before = S.get_particles()
    r, v = z["r0"].copy(), z["v0"].copy()
    if where == "r_nan":
        r[len(r) // 2, 1] = np.nan
    elif where == "v_nan":
        v[3, 0] = np.nan
    else:
        v[-1, 2] = np.inf
    with pytest.raises(capi.DsmcError) as e:
        S.set_particles(r, v)
    assert e.value.code == capi.DSMC_ERR_STATE and "non-finite" in str(e.value)
    assert S.num_molecules == len(z["r0"])
    r_after, v_after = S.get_particles()
    assert np.array_equal(r_after, r_before) and np.array_equal(v_after, v_before)
    S.step(3)
    err, _ = S.ctx.device_status()
    assert err & capi.EBIT_FATAL == 0
    r3, v3 = S.get_particles()
    assert np.isfinite(r3).all() and np.isfinite(v3).all() and S.tallies().step == 3
