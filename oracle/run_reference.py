"""TEST / BASELINE INFRASTRUCTURE: runs the unmodified reference solver
(oracle/_ref/dsmc_ref, built from andeplane/master's sources by oracle/Makefile)
on a workload and reads back its own timing report (dsmc/main.cpp:77-109).

Used only by bench.py's CPU baseline legs and by tests.  Replicas run as
independent single-rank processes, one per core, each with its own seed.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
DSMC_REF = HERE / "_ref" / "dsmc_ref"

INI = """load_previous_state = false
create_movie = false
max_molecules_per_node = {max_molecules}
atoms_per_molecule = {atoms_per_molecule}
timesteps = {timesteps}
temperature = {temperature!r}
wall_temperature = {wall_temperature!r}
statistics_interval = {statistics_interval}
velocity_profile_type = other
sampling_bins = {sampling_bins}
movie_every_n_frame = 1
movie_molecules = 1
dt = {dt!r}
gravity = {gravity!r}
flow_direction = {flow_direction}
pressure_A = 100000
pressure_B = 100000
reservoir_fraction = 0
world = {world}
surface_interaction_model = thermal
alpha_n = 0.5
alpha_t = 0.8
seed = {seed}
density = {density!r}
diam = {diam!r}
mass = {mass!r}
viscosity = 2.23e-5
Lx = {Lx!r}
Ly = {Ly!r}
Lz = {Lz!r}
cells_x = {cells_x}
cells_y = {cells_y}
cells_z = {cells_z}
nx = 1
ny = 1
nz = 1
"""


def available() -> bool:
    return DSMC_REF.exists()


def ini_text(settings, timesteps: int, seed: int, world: str, porosity: float = 1.0) -> str:
    s = settings
    # System::setup_molecules sizes r and v as 3*max_molecules_per_node ints'
    # worth of doubles (dsmc/system.cpp:405-406): keep it near the need.
    expected = s.density * 1e-18 * s.Lx * s.Ly * s.Lz * porosity / s.atoms_per_molecule
    max_molecules = int(min(max(s.max_molecules_per_node, 1), 2 * expected + 1000))
    return INI.format(max_molecules=max_molecules, atoms_per_molecule=s.atoms_per_molecule,
                      timesteps=timesteps, temperature=s.temperature, wall_temperature=s.wall_temperature,
                      statistics_interval=s.statistics_interval, sampling_bins=s.sampling_bins, dt=s.dt,
                      gravity=s.gravity, flow_direction=s.flow_direction, world=world, seed=seed,
                      density=s.density, diam=s.diam, mass=s.mass, Lx=s.Lx, Ly=s.Ly, Lz=s.Lz,
                      cells_x=s.cells_x, cells_y=s.cells_y, cells_z=s.cells_z)


def parse_report(text: str) -> dict:
    """The reference's end-of-run report (dsmc/main.cpp:94-108)."""
    out = {}
    m = re.search(r"^(\d+) molecules \(", text, re.M)
    if m:
        out["molecules"] = int(m.group(1))
    for key, label in (("moving", "Moving"), ("colliding", "Colliding"), ("accelerating", "Accelerating"),
                       ("sampling", "Sampling"), ("initialize", "System initialize"), ("io", "Disk IO")):
        m = re.search(rf"{label}\s*:\s*([0-9.eE+-]+) s", text)
        if m:
            out[key] = float(m.group(1))
    m = re.search(r"([0-9.eE+-]+)k atom-timesteps / second\. \n", text)
    if m:
        out["k_atom_timesteps_per_s"] = float(m.group(1))
    for m in re.finditer(r"^(\d+)\s+t=.*?T=([0-9.eE+-]+)K\s+Collisions: (\d+)\s+Wall collisions: (\d+)", text, re.M):
        out.setdefault("samples", []).append((int(m.group(1)), float(m.group(2)), int(m.group(3)), int(m.group(4))))
    return out


def run_replicas(settings, geometry, timesteps: int, replicas: int, seeds=None, workdir: Path | None = None,
                 timeout: float = 600.0) -> dict:
    """Runs `replicas` single-rank reference solvers in parallel on one world.
    Returns per-replica reports plus the summed particle-steps per second of
    the timestep stages (moving + colliding + accelerating + sampling)."""
    if not available():
        raise RuntimeError("oracle/_ref/dsmc_ref is not built")
    own = workdir is None
    root = Path(workdir or tempfile.mkdtemp(prefix="dsmc_ref_run_"))
    try:
        world = root / "worlds"
        world.mkdir(parents=True, exist_ok=True)
        geometry.write_world(world)
        seeds = seeds or list(range(1, replicas + 1))

        def one(i):
            d = root / f"r{i:03d}"
            for sub in ("statistics/time", "state_files", "movie_files"):
                (d / sub).mkdir(parents=True, exist_ok=True)
            (d / "dsmc.ini").write_text(ini_text(settings, timesteps, seeds[i], str(world), geometry.porosity))
            (d / "Tocontinue").write_text("0.0 0 0 0")
            t0 = time.perf_counter()
            res = subprocess.run([str(DSMC_REF)], cwd=d, capture_output=True, text=True, timeout=timeout)
            wall = time.perf_counter() - t0
            if res.returncode != 0:
                raise RuntimeError(f"reference run failed: {res.stdout[-2000:]} {res.stderr[-2000:]}")
            rep = parse_report(res.stdout)
            rep["wall_s"] = wall
            rep["stdout_tail"] = res.stdout[-4000:]
            return rep

        with ThreadPoolExecutor(max_workers=replicas) as ex:
            reports = list(ex.map(one, range(replicas)))
    finally:
        if own:
            shutil.rmtree(root, ignore_errors=True)
    rate = 0.0
    for r in reports:
        step_s = r.get("moving", 0) + r.get("colliding", 0) + r.get("accelerating", 0) + r.get("sampling", 0)
        r["step_seconds"] = step_s
        if step_s > 0:
            rate += r["molecules"] * timesteps / step_s
    return {"reports": reports, "particle_steps_per_s": rate, "replicas": replicas, "timesteps": timesteps}
