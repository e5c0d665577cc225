"""Generates the golden parity fixtures under tests/golden/ by running the
reference's own routines (oracle/_ref/libdsmc_ref_tape.so, built from the
reference sources by oracle/Makefile) on small packed-sphere systems, fed
the counter-based draws the GPU kernels take.

    python tests/golden/make_golden.py

Each fixture holds, for one system: the initial state of
System::setup_molecules with per-particle draw streams, the state after one
accelerate + move (+ periodic wrap) and cell re-binning, the velocities and
cell bookkeeping after one NTC collide, and the state after several full
steps (every collide on id-ordered cell members), with the reference's
counters at each point, and the reference sampler's profiles over those
steps (sampled after every step).  It also records sha256 digests of the reference
geometry tool's world arrays for the config-1 geometry.
"""
from __future__ import annotations

import hashlib
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import ref_harness as rh  # noqa: E402
from master_b200.system import Geometry, time_from_si, acceleration_from_si  # noqa: E402

OUT = Path(__file__).resolve().parent

CASES = {
    # config-1 physics (dt = 1e-11 s) in a 24^3 box
    "small_dt1": dict(n=24, radius_voxels=2, porosity=0.6, geom_seed=7, cells=12, dt_si=1e-11, apm=10000,
                      rng_seed=0x1234ABCD5678, steps=10),
    # five times the timestep: multi-voxel flights and many wall hits
    "small_dt5": dict(n=24, radius_voxels=2, porosity=0.6, geom_seed=11, cells=12, dt_si=5e-11, apm=10000,
                      rng_seed=0x0BADC0FFEE, steps=10),
    # the other wall models of the reference (dsmc/system.cpp:345-352)
    "small_specular": dict(n=24, radius_voxels=2, porosity=0.6, geom_seed=11, cells=12, dt_si=5e-11, apm=10000,
                           rng_seed=0x5BEC, steps=10, surface="specular"),
    "small_cl": dict(n=24, radius_voxels=2, porosity=0.6, geom_seed=11, cells=12, dt_si=5e-11, apm=10000,
                     rng_seed=0xC1C1, steps=10, surface="cercignani_lampis", alpha_n=0.5, alpha_t=0.8),
}


def settings_dict(c):
    L = c["n"] * 0.1
    return dict(max_molecules=200000, atoms_per_molecule=c["apm"], temperature=300.0, wall_temperature=300.0,
                statistics_interval=1, sampling_bins=c["cells"], dt=time_from_si(c["dt_si"]),
                gravity=acceleration_from_si(1e9), flow_direction=0, seed=c["geom_seed"], density=2.5e24,
                diam=3.66e-4, mass=6.63e-26 / 1.66053886e-27, Lx=L, Ly=L, Lz=L, cells_x=c["cells"],
                cells_y=c["cells"], cells_z=c["cells"], surface=c.get("surface", "thermal"),
                alpha_n=c.get("alpha_n", 0.5), alpha_t=c.get("alpha_t", 0.8))


def make_case(name, c):
    g = Geometry.packed_spheres(c["n"], c["radius_voxels"], wanted_porosity=c["porosity"], seed=c["geom_seed"])
    s = settings_dict(c)
    R, wd = rh.make_ref_system(g, s)
    # the reference's own particle count (dsmc/system.cpp:323)
    n = R.n
    seed = c["rng_seed"]
    R.init_particles(seed, n)
    r0, v0, cell0 = R.get_particles()
    cells0 = R.cells()
    R.reset_counters()
    # step 1, stage by stage
    R.accelerate()
    R.move(seed, 1)
    r1, v1, _ = R.get_particles()
    R.update_cells()
    _, _, cell1 = R.get_particles()
    cnt_move = R.counters()
    R.canonicalize()
    R.collide(seed, 1)
    R.sample(1)
    _, v1c, _ = R.get_particles()
    cells1 = R.cells()
    cnt_col = R.counters()
    # further full steps
    for step in range(2, c["steps"] + 1):
        R.accelerate()
        R.move(seed, step)
        R.update_cells()
        R.canonicalize()
        R.collide(seed, step)
        R.sample(step)  # statistics_interval = 1: every step
    rK, vK, cellK = R.get_particles()
    # the sampler's profiles over steps 1..K (dsmc/statisticalproperty.cpp:229-478)
    prof = R.profile_sums()
    fin = R.profiles()
    measures = R.measures()
    cellsK = R.cells()
    cntK = R.counters()
    meta = dict(case=name, params=c, settings=s, n=n, counters_move=cnt_move, counters_collide=cnt_col,
                counters_final=cntK, porosity=float(g.porosity), measures_final=measures)
    np.savez_compressed(OUT / f"{name}.npz", r0=r0, v0=v0, cell0=cell0, r1=r1, v1=v1, cell1=cell1, v1c=v1c,
                        vr_max1=cells1["vr_max"], rest1=cells1["rest"], count1=cells1["count"], rK=rK, vK=vK,
                        cellK=cellK, vr_maxK=cellsK["vr_max"], restK=cellsK["rest"], countK=cellsK["count"],
                        cell_global=cells0["global_index"], cell_volume=cells0["volume"], cell_coeff=cells0["coeff"],
                        cell_pixels=cells0["pixels"], cell_total_pixels=cells0["total_pixels"],
                        prof_sumsK=prof, prof_vzK=fin["velocity_z"], prof_TK=fin["temperature"],
                        prof_PK=fin["pressure"], prof_vx_center=fin["vx_center"],
                        vr_max0=cells0["vr_max"], meta=np.array(json.dumps(meta)))
    print(name, "n", n, "move", cnt_move, "final", cntK)


def geometry_digests():
    """sha256 of the reference geometry tool's arrays for config 1 (64^3,
    r = 4 voxels, porosity 0.6, seed 1), read back without halo."""
    tool = ROOT / "oracle" / "_ref" / "geometry_ref"
    out = {}
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        (d / "worlds").mkdir()
        (d / "geometry_settings.ini").write_text("\n".join([
            "type = packed_spheres", "num_voxels_x = 64", "num_voxels_y = 64", "num_voxels_z = 64",
            "number_of_neighbor_averages = 1", "create_border = false", "save_file = true",
            "binary_output_folder = worlds", "num_processors_x = 1", "num_processors_y = 1",
            "num_processors_z = 1", "radius = 0.0625", "inverted = true", "spheres_num = 0",
            "prevent_overlap = false", "wanted_porosity = 0.6", "spheres_type = 1", "seed = 1",
            "screen_width = 1", "screen_height = 1", "Lx = 1", "Ly = 1", "Lz = 1", "visualize = false", ""]))
        subprocess.run([str(tool)], cwd=d, check=True, capture_output=True)
        g = Geometry.read_world(d / "worlds" / "0000.bin")
        for k in ("voxels", "normals", "tangents1", "tangents2"):
            out[k] = hashlib.sha256(np.ascontiguousarray(getattr(g, k)).tobytes()).hexdigest()
        out["porosity_global"] = float(g.porosity_global)
        out["params"] = dict(n=64, radius=0.0625, wanted_porosity=0.6, seed=1, number_of_neighbor_averages=1)
    (OUT / "geometry_packed64_digests.json").write_text(json.dumps(out, indent=1))
    print("geometry digests", out["porosity_global"])


if __name__ == "__main__":
    if not rh.available():
        raise SystemExit("build oracle/_ref first: make -C oracle ref REF=<reference project>/code/base_code/program/dsmc")
    only = sys.argv[1:]  # case names to (re)generate; all when none
    for name, c in CASES.items():
        if not only or name in only:
            make_case(name, c)
    if not only:
        geometry_digests()
