"""Checkpoint interop: the reference's own state file and Tocontinue
(dsmc/dsmc_io.cpp:82-159, dsmc/main.cpp:37-55), both directions against the
reference solver built from its sources, and the exact checkpoint of this
library (continuation gives the same trajectories)."""
from __future__ import annotations


import numpy as np
import pytest

from master_b200 import capi, workloads
from master_b200.system import (Geometry, System, read_state_file, read_tocontinue, write_state_file,
                                write_tocontinue)

from oracle import run_reference

needs_ref = pytest.mark.skipif(not run_reference.available(), reason="oracle/_ref/dsmc_ref is not built")

SMALL = workloads.Workload("ckpt32", n=32, radius_voxels=3, porosity=0.6, geometry_seed=4, cells=16,
                           atoms_per_molecule=workloads.simulators_per_cell_weight(2.5e24, 0.1, 2, 12))


def test_state_file_and_tocontinue_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    r, v = rng.random((57, 3)), rng.normal(size=(57, 3))
    write_state_file(tmp_path / "state0000.bin", r, v)
    raw = (tmp_path / "state0000.bin").read_bytes()
    assert np.frombuffer(raw[:4], np.int32)[0] == 57 and len(raw) == 4 + 57 * 48
    r2, v2 = read_state_file(tmp_path / "state0000.bin")
    assert np.array_equal(r, r2) and np.array_equal(v, v2)
    write_tocontinue(tmp_path / "Tocontinue", 0.1 + 0.2, 1234, 56, 78)
    assert read_tocontinue(tmp_path / "Tocontinue") == {"t": 0.1 + 0.2, "steps": 1234, "collisions": 56,
                                                        "wall_collisions": 78}
    (tmp_path / "bad").write_text("1.0 2")
    with pytest.raises(capi.DsmcError):
        read_tocontinue(tmp_path / "bad")


@needs_ref
def test_reference_state_file_read_and_ours_read_by_reference(tmp_path):
    s = SMALL.settings(statistics_interval=1)
    g = SMALL.geometry()
    run_reference.run_replicas(s, g, timesteps=3, replicas=1, workdir=tmp_path)
    run = tmp_path / "r000"
    r, v = read_state_file(run / "state_files" / "state0000.bin")
    n = len(r)
    assert n > 1000
    assert (r >= 0).all() and (r[:, 0] < s.Lx).all() and (r[:, 1] < s.Ly).all() and (r[:, 2] < s.Lz).all()
    # Maxwellian at 300 K: per-component rms sqrt(T/m) in reduced units
    t_red = s.temperature / (1.65088e-21 / 1.3806503e-23)
    assert np.isfinite(v).all() and np.sqrt((v ** 2).mean()) == pytest.approx(np.sqrt(t_red / s.mass), rel=0.05)
    cont = read_tocontinue(run / "Tocontinue")
    assert cont["steps"] == 3 and cont["collisions"] > 0 and cont["wall_collisions"] > 0
    # our writer, the reference's loader: it continues from the file we wrote
    write_state_file(run / "state_files" / "state0000.bin", r, -v)
    ini = (run / "dsmc.ini").read_text().replace("load_previous_state = false", "load_previous_state = true")
    (run / "dsmc.ini").write_text(ini)
    import subprocess
    res = subprocess.run([str(run_reference.DSMC_REF)], cwd=run, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout[-2000:]
    assert run_reference.parse_report(res.stdout)["molecules"] == n
    assert read_tocontinue(run / "Tocontinue")["steps"] == 6


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [capi.PREC_SPLIT32, capi.PREC_FP64])
def test_checkpoint_continues_bit_identically(tmp_path, precision):
    s = SMALL.settings(statistics_interval=2)
    g = SMALL.geometry()
    A = System(s, g, precision=precision)
    A.step(9)
    B = System(s, g, precision=precision)
    B.step(4)
    B.ctx.checkpoint_save(tmp_path / "ck.bin")
    B.step(5)
    C = System(s, g, precision=precision, init_particles=False)
    C.ctx.checkpoint_load(tmp_path / "ck.bin")
    C.step(5)
    for X in (B, C):
        ra, va = A.get_particles()
        rx, vx = X.get_particles()
        assert np.array_equal(ra, rx) and np.array_equal(va, vx)
        ta, tx = A.tallies(), X.tallies()
        for k in ("step", "collisions", "wall_collisions", "candidates", "samples", "particle_steps"):
            assert getattr(ta, k) == getattr(tx, k), k
        assert list(ta.count_periodic) == list(tx.count_periodic)
        # fp64 moment sums round by summation order, which depends on the
        # slot order and on the kernel that samples
        assert np.allclose(A.cells()["moments"], X.cells()["moments"], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_continue_from_reference_counters(tmp_path):
    s = SMALL.settings(statistics_interval=1)
    g = SMALL.geometry()
    A = System(s, g)
    A.step(2)
    r, v = A.get_particles()
    t0 = A.tallies()
    B = System(s, g, init_particles=False)
    B.set_particles(r, v)
    B.continue_from(t0.time, t0.step, t0.collisions, t0.wall_collisions)
    tb = B.tallies()
    assert tb.step == t0.step and tb.collisions == t0.collisions and tb.wall_collisions == t0.wall_collisions
    assert tb.time == pytest.approx(t0.time)
    B.step(3)
    assert B.tallies().step == t0.step + 3
