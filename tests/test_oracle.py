"""The C restatement oracle (oracle/dsmc_oracle.c), pinned against the
reference's own routines: the golden fixtures (tests/golden/, made from
oracle/_ref) and, where the reference build is present, a fresh run of it.
Also the published Philox4x32-10 known-answer vectors of the draw source."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from master_b200.system import Geometry

import oracle_c
import ref_harness as rh

GOLDEN = Path(__file__).resolve().parent / "golden"


def load(case):
    z = np.load(GOLDEN / f"{case}.npz")
    meta = json.loads(str(z["meta"]))
    c = meta["params"]
    g = Geometry.packed_spheres(c["n"], c["radius_voxels"], wanted_porosity=c["porosity"], seed=c["geom_seed"])
    return z, meta, g


@pytest.mark.parametrize("case", ["small_dt1", "small_dt5", "small_specular", "small_cl"])
def test_oracle_reproduces_reference_steps(case):
    z, meta, g = load(case)
    o = oracle_c.Oracle(g, meta["settings"], meta["params"]["rng_seed"])
    assert np.array_equal(o.global_index, z["cell_global"])
    assert np.array_equal(o.coeff, z["cell_coeff"]) and np.array_equal(o.volume, z["cell_volume"])
    o.init(meta["n"])
    assert np.array_equal(o.r, z["r0"]) and np.array_equal(o.v, z["v0"])
    o.move(1)
    assert np.array_equal(o.r, z["r1"]) and np.array_equal(o.v, z["v1"])
    c = o.counters()
    # only the reference's thermal collider counts wall collisions
    thermal = meta["settings"].get("surface", "thermal") == "thermal"
    assert c["wall_collisions"] == meta["counters_move"]["wall_collisions"] or not thermal
    assert c["count_periodic"] == meta["counters_move"]["count_periodic"]
    o.sort()
    assert np.array_equal(o.cell_global_of_particles, z["cell1"])
    assert np.array_equal(o.count, z["count1"])
    o.collide(1)
    assert np.array_equal(o.v, z["v1c"])
    assert np.array_equal(o.vr_max, z["vr_max1"]) and np.array_equal(o.rest, z["rest1"])
    for step in range(2, meta["params"]["steps"] + 1):
        o.step(step)
    assert np.array_equal(o.r, z["rK"]) and np.array_equal(o.v, z["vK"])
    assert np.array_equal(o.cell_global_of_particles, z["cellK"])
    c = o.counters()
    ref = meta["counters_final"]
    assert c["collisions"] == ref["collisions"]
    assert c["wall_collisions"] == ref["wall_collisions"] or not thermal
    assert c["count_periodic"] == ref["count_periodic"]


MEASURES = ("energy_eV", "temperature_K", "number_flow_rate", "volumetric_flow_rate", "pressure_Pa",
            "permeability_darcy")


@pytest.mark.parametrize("case", ["small_dt1", "small_dt5", "small_specular", "small_cl"])
def test_oracle_sampler_reproduces_reference_sampler(case, tmp_path):
    """The oracle's sampler over the fixture's steps (one sample after each,
    as the fixture's statistics_interval of 1 has it) gives the reference
    StatisticsSampler's profile sums and its scalar measurements of the
    last step, both bit for bit (the same operations in the same order)."""
    z, meta, g = load(case)
    st = meta["settings"]
    o = oracle_c.Oracle(g, st, meta["params"]["rng_seed"])
    o.init(meta["n"])
    for step in range(1, meta["params"]["steps"] + 1):
        o.step(step)
        o.sample()
    assert np.array_equal(o.r, z["rK"]) and np.array_equal(o.v, z["vK"])
    assert np.array_equal(o.profile_sums(), z["prof_sumsK"])
    # System::volume_global: the box times the world file's float porosity (dsmc/system.cpp:313-314)
    g.write_world(tmp_path)
    por = Geometry.read_world(tmp_path / "0000.bin").porosity_global
    got = o.measures(st["Lx"] * st["Ly"] * st["Lz"] * por)
    for k, x in zip(MEASURES, got):
        assert x == meta["measures_final"][k], k


KAT = [  # Salmon et al. (SC'11), Random123 kat_vectors: philox4x32, 10 rounds
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def philox_py(ctr, key):
    """Philox4x32-10 in Python, for the known-answer check of both C copies."""
    c = list(ctr)
    k = list(key)
    M = 0xFFFFFFFF
    for _ in range(10):
        p0 = 0xD2511F53 * c[0]
        p1 = 0xCD9E8D57 * c[2]
        c = [((p1 >> 32) ^ c[1] ^ k[0]) & M, p1 & M, ((p0 >> 32) ^ c[3] ^ k[1]) & M, p0 & M]
        k = [(k[0] + 0x9E3779B9) & M, (k[1] + 0xBB67AE85) & M]
    return tuple(c)


@pytest.mark.parametrize("ctr,key,out", KAT)
def test_philox_known_answers(ctr, key, out):
    assert philox_py(ctr, key) == out


def test_oracle_draws_follow_philox():
    """draw k of stream (id, step, tag): words of block k>>1, 52-bit fp64."""
    lib = C.CDLL(str(oracle_c.LIB))
    seed = 0x0123456789ABCDEF
    # oracle_init's first two draws of particle 5 build v_x via next_gauss;
    # check the uniform construction directly in Python against a draw-level
    # reimplementation of the stream layout
    w = philox_py((5, 0, 3, 0), (seed & 0xFFFFFFFF, seed >> 32))
    x0 = (w[0] << 20) | (w[1] >> 12)
    x1 = (w[2] << 20) | (w[3] >> 12)
    u0 = (x0 + 0.5) / 2 ** 52
    u1 = (x1 + 0.5) / 2 ** 52
    gauss = np.sqrt(-2.0 * np.log(1.0 - u0)) * np.cos(6.283185307 * u1)
    g = Geometry.empty(4, 4, 4)
    st = dict(cells_x=2, cells_y=2, cells_z=2, Lx=0.4, Ly=0.4, Lz=0.4, dt=0.01, gravity=0.0, flow_direction=-1,
              wall_temperature=300.0, temperature=300.0, mass=40.0, atoms_per_molecule=1, diam=3.66e-4)
    o = oracle_c.Oracle(g, st, seed)
    o.init(6)
    assert o.v[5, 0] == pytest.approx(gauss * o.s.sqrt_t_over_m, rel=1e-15)


LAYOUT_CASES = [  # (voxels per axis, cells per axis, solid fraction, seed)
    ((8, 8, 8), (4, 4, 4), 0.0, 1),          # all open
    ((8, 8, 8), (8, 8, 8), 0.5, 2),          # one voxel per cell: half the cells inactive
    ((12, 8, 16), (3, 4, 8), 0.6, 3),        # uneven box and cells
    ((16, 16, 16), (4, 4, 4), 0.97, 4),      # nearly solid: cells with one or two open voxels
    ((10, 10, 10), (5, 2, 10), 0.3, 5),
    ((4, 4, 4), (2, 2, 2), 1.0, 6),          # all solid: no active cell
]


@pytest.mark.parametrize("shape,cells,solid,seed", LAYOUT_CASES)
def test_cell_layout_of_the_library_equals_the_oracle(shape, cells, solid, seed):
    """System::setup_cells + Cell::update_volume (dsmc/system.cpp:432-490,
    dsmc/cell.cpp:27-40) restated twice, by the library's host code
    (dsmc_cells_layout) and by the C oracle: identical on random masks,
    uneven boxes and cells down to one voxel."""
    from master_b200.system import Settings, cells_layout
    rng = np.random.default_rng(seed)
    g = Geometry.empty(*shape)
    g.voxels[...] = (rng.random(shape) < solid).astype(np.uint8)
    st = dict(cells_x=cells[0], cells_y=cells[1], cells_z=cells[2], Lx=0.1 * shape[0], Ly=0.1 * shape[1],
              Lz=0.1 * shape[2], dt=0.00997, gravity=0.0, flow_direction=-1, wall_temperature=300.0,
              temperature=300.0, mass=39.948, atoms_per_molecule=1000, diam=3.66e-4)
    o = oracle_c.Oracle(g, st, 1)
    s = Settings()
    for k in ("Lx", "Ly", "Lz", "cells_x", "cells_y", "cells_z", "dt", "diam", "atoms_per_molecule"):
        setattr(s, k, st[k])
    lib = cells_layout(s, g)
    assert np.array_equal(lib["global_index"], o.global_index)
    assert np.array_equal(lib["volume"], o.volume)
    assert np.array_equal(lib["coeff"], o.coeff)
    open_voxels = (g.voxels == 0).sum()
    assert lib["pixels"].sum() == open_voxels and (lib["pixels"] > 0).all()


FRESH = {  # systems beyond the fixtures: other sizes, cells, timesteps, flow axes and walls
    "thermal_16": dict(n=16, radius_voxels=2, porosity=0.5, geom_seed=21, cells=8, dt_si=1e-11, flow=0,
                       rng_seed=0x51DE, surface="thermal"),
    "specular_20_flow_y": dict(n=20, radius_voxels=2.5, porosity=0.7, geom_seed=22, cells=10, dt_si=3e-11, flow=1,
                               rng_seed=0xF10F, surface="specular"),
    "thermal_box_16x12x20_no_flow": dict(n=(16, 12, 20), radius_voxels=2, porosity=0.55, geom_seed=24,
                                         cells=(8, 6, 10), dt_si=2e-11, flow=-1, rng_seed=0xB0C5,
                                         surface="thermal"),
    # alpha_n 0.8: at alpha_n <= ~0.4 the reference's Cercignani-Lampis
    # sampler needs ~1e6 trials for a particle that meets the wall at twice
    # the wall's most probable speed, past the 1e5 at which the tape draws
    # stop the process
    "cl_16_coarse_cells": dict(n=16, radius_voxels=3, porosity=0.65, geom_seed=23, cells=4, dt_si=2e-11, flow=2,
                               rng_seed=0xC0C0A, surface="cercignani_lampis", alpha_n=0.8, alpha_t=0.5),
}


@pytest.mark.skipif(not rh.available(), reason="oracle/_ref (the reference built from its sources) is not built")
@pytest.mark.parametrize("name", sorted(FRESH))
def test_oracle_matches_a_fresh_reference_run(name, tmp_path):
    """The oracle against the reference's own routines run now (the tape
    build, oracle/_ref/libdsmc_ref_tape.so), on systems the fixtures do not
    hold: the initial state, 25 full steps sampled after each, every
    position, velocity, cell, counter, profile sum and measurement bit for
    bit."""
    from master_b200.system import acceleration_from_si, time_from_si
    c = FRESH[name]
    g = Geometry.packed_spheres(c["n"], c["radius_voxels"], wanted_porosity=c["porosity"], seed=c["geom_seed"])
    n3 = (c["n"],) * 3 if np.isscalar(c["n"]) else c["n"]
    cells3 = (c["cells"],) * 3 if np.isscalar(c["cells"]) else c["cells"]
    L = [0.1 * k for k in n3]
    st = dict(max_molecules=200000, atoms_per_molecule=4000, temperature=300.0, wall_temperature=320.0,
              statistics_interval=1, sampling_bins=cells3[1], dt=time_from_si(c["dt_si"]),
              gravity=acceleration_from_si(1e9) if c["flow"] >= 0 else 0.0, flow_direction=max(c["flow"], 0),
              seed=c["geom_seed"], density=2.5e24, diam=3.66e-4, mass=6.63e-26 / 1.66053886e-27, Lx=L[0],
              Ly=L[1], Lz=L[2], cells_x=cells3[0], cells_y=cells3[1], cells_z=cells3[2], surface=c["surface"],
              alpha_n=c.get("alpha_n", 0.5), alpha_t=c.get("alpha_t", 0.8))
    compare_with_fresh_reference(g, st, c["rng_seed"], 25, tmp_path)


def compare_with_fresh_reference(g, st: dict, seed: int, steps: int, tmp_path) -> None:
    """Runs the reference's own routines (the tape build) and the oracle side
    by side from the same initial state for `steps` full steps, sampled
    after each, and requires every position, velocity, cell, counter,
    profile sum and measurement to be identical."""
    R, _ = rh.make_ref_system(g, st, tmp_path / "ref")
    n = R.n
    assert n > 100
    R.init_particles(seed, n)
    R.reset_counters()
    o = oracle_c.Oracle(g, st, seed)
    o.init(n)
    r, v, _ = R.get_particles()
    assert np.array_equal(o.r, r) and np.array_equal(o.v, v)
    cells = R.cells()
    assert np.array_equal(o.global_index, cells["global_index"]) and np.array_equal(o.coeff, cells["coeff"])
    for step in range(1, steps + 1):
        R.accelerate()
        R.move(seed, step)
        R.update_cells()
        R.canonicalize()
        R.collide(seed, step)
        R.sample(step)
        o.step(step)
        o.sample()
        r, v, cell = R.get_particles()
        assert np.array_equal(o.r, r), step
        assert np.array_equal(o.v, v), step
        assert np.array_equal(o.cell_global_of_particles, cell), step
    cells = R.cells()
    assert np.array_equal(o.vr_max, cells["vr_max"]) and np.array_equal(o.rest, cells["rest"])
    cnt = R.counters()
    mine = o.counters()
    assert mine["count_periodic"] == cnt["count_periodic"] and mine["collisions"] == cnt["collisions"]
    if st.get("surface", "thermal") == "thermal":  # only the thermal collider counts wall collisions
        assert mine["wall_collisions"] == cnt["wall_collisions"] > 0
    assert np.array_equal(o.profile_sums(), R.profile_sums())
    (tmp_path / "w").mkdir()
    g.write_world(tmp_path / "w")
    por = Geometry.read_world(tmp_path / "w" / "0000.bin").porosity_global
    got = o.measures(st["Lx"] * st["Ly"] * st["Lz"] * por)
    ref = R.measures()
    for k, x in zip(MEASURES, got):
        # without gravity the reference's permeability divides by zero
        assert x == ref[k] or (np.isnan(x) and np.isnan(ref[k])), k


@pytest.mark.skipif(not rh.available(), reason="oracle/_ref (the reference built from its sources) is not built")
def test_oracle_matches_the_reference_on_the_plain_dsmc_workload(tmp_path):
    """The same on the plain-DSMC workload itself (packed_64: 64^3 voxels of
    0.1 um, spheres of r = 4 voxels to porosity 0.6, 32^3 cells, F_N = 1000,
    about 3.9e5 particles, dt = 1e-11 s, g = 1e9 m/s^2 along x), three steps."""
    from master_b200 import workloads
    w = workloads.PACKED_64
    s = w.settings(rng_seed=1, statistics_interval=1)
    st = {k: getattr(s, k) for k in ("atoms_per_molecule", "temperature", "wall_temperature", "statistics_interval",
                                     "sampling_bins", "dt", "gravity", "flow_direction", "seed", "density", "diam",
                                     "mass", "Lx", "Ly", "Lz", "cells_x", "cells_y", "cells_z")}
    st["max_molecules"] = 1_000_000
    compare_with_fresh_reference(w.geometry(), st, 0x64C0F1, 3, tmp_path)
