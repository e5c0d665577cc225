"""TEST / BASELINE INFRASTRUCTURE: runs the unmodified reference solver
(oracle/_ref/dsmc_ref, built from andeplane/master's sources by oracle/Makefile)
on a workload and reads back its own timing report (dsmc/main.cpp:77-109).

Used only by bench.py's CPU baseline legs and by tests.  Replicas run as
independent single-rank processes, one per core, each with its own seed.

`RefWorkload` describes a benchmark workload with nothing but the reference's
own inputs: a geometry_settings.ini for the reference's geometry tool
(oracle/_ref/geometry_ref, dsmc/geometry.cpp:16-91 driving
ComplexGeometry::create_packed_spheres, dsmc/complexgeometry.cpp:401-513) and
a dsmc.ini for the solver.  Nothing here imports or loads the B200 library.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from pathlib import Path
from types import SimpleNamespace

HERE = Path(__file__).resolve().parent
DSMC_REF = HERE / "_ref" / "dsmc_ref"
GEOMETRY_REF = HERE / "_ref" / "geometry_ref"

# reduced units of the reference (dsmc/unitconverter.cpp:3-21)
_M0 = 1.66053886e-27
_L0 = 1e-6
_E0 = 1.65088e-21
_T0_TIME = _L0 * (_M0 / _E0) ** 0.5
_A0 = (_L0 / _T0_TIME) / _T0_TIME
ARGON_MASS_AMU = 6.63e-26 / _M0
ARGON_DIAM_UM = 3.66e-4

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


def geometry_tool_available() -> bool:
    return GEOMETRY_REF.exists()


class ToolGeometry:
    """A packed-sphere world written by the reference's own geometry tool.

    `write_world(folder)` runs oracle/_ref/geometry_ref with a
    geometry_settings.ini of `type = packed_spheres` (dsmc/geometry.cpp:18-47,
    dsmc/complexgeometry.cpp:401-513: inverted spheres, spheres_type 1 = until
    the porosity target, one neighbour average for the normals) and reads the
    global porosity back from the tool's porosity.txt (:306-318).  The world
    file holds the 3x3x3 periodic halo of a single rank: 27 n^3 voxels of
    37 bytes (16.8 GB at n = 256)."""

    def __init__(self, n: int, radius_voxels: float, porosity: float, seed: int):
        self.n, self.radius_voxels, self.wanted_porosity, self.seed = n, radius_voxels, porosity, seed
        self.porosity = porosity
        self.tool_seconds = None

    def ini(self, folder: Path) -> str:
        return "\n".join([
            "type = packed_spheres", f"num_voxels_x = {self.n}", f"num_voxels_y = {self.n}",
            f"num_voxels_z = {self.n}", "number_of_neighbor_averages = 1", "create_border = false",
            "save_file = true", f"binary_output_folder = {folder}", "num_processors_x = 1",
            "num_processors_y = 1", "num_processors_z = 1", f"radius = {self.radius_voxels / self.n!r}",
            "inverted = true", "spheres_num = 0", "prevent_overlap = false",
            f"wanted_porosity = {self.wanted_porosity!r}", "spheres_type = 1", f"seed = {self.seed}",
            "screen_width = 1", "screen_height = 1", "Lx = 1", "Ly = 1", "Lz = 1", "visualize = false", ""])

    def write_world(self, folder) -> None:
        if not geometry_tool_available():
            raise RuntimeError("oracle/_ref/geometry_ref is not built")
        folder = Path(folder).resolve()
        folder.mkdir(parents=True, exist_ok=True)
        with tempfile.TemporaryDirectory(prefix="geometry_ref_") as d:
            (Path(d) / "geometry_settings.ini").write_text(self.ini(folder))
            t0 = time.perf_counter()
            res = subprocess.run([str(GEOMETRY_REF)], cwd=d, capture_output=True, text=True)
            self.tool_seconds = time.perf_counter() - t0
        if res.returncode != 0 or not (folder / "0000.bin").exists():
            raise RuntimeError(f"geometry_ref failed: {res.stdout[-1000:]} {res.stderr[-1000:]}")
        self.porosity = float((folder / "porosity.txt").read_text().split()[0])

    def world_bytes(self) -> int:
        return 27 * self.n ** 3 * 37 + 32


@dataclass
class RefWorkload:
    """A benchmark workload in the reference's own inputs (the fields of a
    dsmc.ini, dsmc/settings.cpp:3-44, and of a geometry_settings.ini)."""
    name: str
    n: int
    radius_voxels: float
    porosity: float
    geometry_seed: int
    cells: int
    atoms_per_molecule: int
    voxel_um: float = 0.1
    density_si: float = 2.5e24
    temperature: float = 300.0
    dt_si: float = 1e-11
    gravity_si: float = 1e9
    flow_direction: int = 0

    def settings(self, statistics_interval: int = 100) -> SimpleNamespace:
        L = self.n * self.voxel_um
        return SimpleNamespace(
            Lx=L, Ly=L, Lz=L, cells_x=self.cells, cells_y=self.cells, cells_z=self.cells, mass=ARGON_MASS_AMU,
            diam=ARGON_DIAM_UM, density=self.density_si, temperature=self.temperature,
            wall_temperature=self.temperature, dt=self.dt_si / _T0_TIME, gravity=self.gravity_si / _A0,
            flow_direction=self.flow_direction, atoms_per_molecule=self.atoms_per_molecule,
            max_molecules_per_node=2 ** 31 - 1, statistics_interval=statistics_interval,
            sampling_bins=self.cells)

    def geometry(self) -> ToolGeometry:
        return ToolGeometry(self.n, self.radius_voxels, self.porosity, self.geometry_seed)

    def expected_particles(self, porosity: float | None = None) -> float:
        L = self.n * self.voxel_um
        return self.density_si * 1e-18 * L ** 3 * (porosity or self.porosity) / self.atoms_per_molecule

    def replica_bytes(self) -> int:
        """Host memory of one reference process: the halo grid (37 bytes per
        voxel of the 27 n^3 block, dsmc/dsmc_io.cpp:183-220) and r, v,
        molecule_index_in_cell, molecule_cell_index, steps_since_collision
        sized for max_molecules_per_node (dsmc/system.cpp:405-410; 60 bytes
        each), with max_molecules_per_node = 2 x expected + 1000, plus the
        cells' member lists (8 bytes per particle) and 10 % slack."""
        m = 2 * self.expected_particles() + 1000
        return int(1.1 * (27 * self.n ** 3 * 37 + 60 * m + 8 * self.expected_particles()))


def _weight(per_cell: float, voxel_um: float = 0.1, voxels_per_cell: int = 2, density_si: float = 2.5e24) -> int:
    return int(density_si * 1e-18 * (voxels_per_cell * voxel_um) ** 3 / per_cell)


# The benchmark workloads, stated in the reference's inputs (the same fields
# as the GPU side's workload table; tests/test_bench_reference.py checks that
# both say the same).
PACKED_64 = RefWorkload("packed_64", n=64, radius_voxels=4, porosity=0.6, geometry_seed=1, cells=32,
                        atoms_per_molecule=1000)
PACKED_256 = RefWorkload("packed_256", n=256, radius_voxels=6, porosity=0.5, geometry_seed=1, cells=128,
                         atoms_per_molecule=_weight(30))
PACKED_256_SAMPLE = RefWorkload("packed_256_sample64", n=64, radius_voxels=6, porosity=0.5, geometry_seed=1,
                                cells=32, atoms_per_molecule=_weight(30))
WORKLOADS = {w.name: w for w in (PACKED_64, PACKED_256, PACKED_256_SAMPLE)}


def host_memory_available() -> int:
    """MemAvailable of /proc/meminfo in bytes (0 when unreadable)."""
    try:
        for line in Path("/proc/meminfo").read_text().splitlines():
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def replicas_that_fit(w: RefWorkload, cores: int, fraction: float = 0.7) -> int:
    """As many single-rank replicas as the host cores and `fraction` of the
    available host memory hold (at least one)."""
    mem = host_memory_available()
    by_mem = int(fraction * mem // w.replica_bytes()) if mem else 1
    return max(1, min(cores, by_mem))


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
                 timeout: float = 600.0, world_dir: Path | None = None, workers: int | None = None) -> dict:
    """Runs `replicas` single-rank reference solvers in parallel on one world.
    Returns per-replica reports plus the summed particle-steps per second of
    the timestep stages (moving + colliding + accelerating + sampling).
    `world_dir`: a folder that already holds the geometry's world file (then
    `geometry` only supplies its porosity)."""
    if not available():
        raise RuntimeError("oracle/_ref/dsmc_ref is not built")
    own = workdir is None
    root = Path(workdir or tempfile.mkdtemp(prefix="dsmc_ref_run_"))
    try:
        if world_dir is None:
            world = root / "worlds"
            world.mkdir(parents=True, exist_ok=True)
            geometry.write_world(world)
        else:
            world = Path(world_dir).resolve()
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

        with ThreadPoolExecutor(max_workers=min(replicas, workers or replicas)) as ex:
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
