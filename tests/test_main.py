"""The reference-style executable (master_b200/dsmc_b200_main, the
counterpart of dsmc/main.cpp): usage on the CPU, a short run on the GPU."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

from master_b200.system import Geometry

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "master_b200" / "dsmc_b200_main"

INI = """load_previous_state = false
max_molecules_per_node = 1000000
atoms_per_molecule = 1000
timesteps = 6
temperature = 300
wall_temperature = 300
statistics_interval = 2
sampling_bins = 16
dt = 0.00997087
gravity = 0.00100585
flow_direction = 0
world = worlds/test
surface_interaction_model = thermal
alpha_n = 1
alpha_t = 1
seed = 3
density = 2.5e24
diam = 3.66e-4
mass = 39.948
viscosity = 2.23e-5
Lx = 3.2
Ly = 3.2
Lz = 3.2
cells_x = 16
cells_y = 16
cells_z = 16
nx = 1
ny = 1
nz = 1
"""


def test_executable_usage():
    assert EXE.exists(), "build() links the executable with the library"
    r = subprocess.run([str(EXE), "--bogus"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
def test_executable_runs_like_reference_main(tmp_path):
    g = Geometry.packed_spheres(32, 3, wanted_porosity=0.6, seed=2)
    (tmp_path / "worlds" / "test").mkdir(parents=True)
    g.write_world(tmp_path / "worlds" / "test")
    (tmp_path / "dsmc.ini").write_text(INI)
    r = subprocess.run([str(EXE)], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Time analysis" in r.stdout and "atom-timesteps / second" in r.stdout
    t, steps, collisions, walls = (tmp_path / "Tocontinue").read_text().split()
    assert int(steps) == 6 and int(walls) > 0 and float(t) > 0
    # the sampler's files (dsmc/dsmc_io.cpp:33-47): a line per sample (steps
    # 2, 4, 6) and the profiles at the end
    st = tmp_path / "statistics"
    for name in ("energy", "temperature", "pressure", "number_flow_rate", "volumetric_flow_rate"):
        rows = [line.split() for line in (st / f"{name}.txt").read_text().splitlines()]
        assert len(rows) == 3 and all(len(r) == 2 for r in rows), name
        assert float(rows[0][0]) < float(rows[1][0]) < float(rows[2][0])
    T = [float(r.split()[1]) for r in (st / "temperature.txt").read_text().splitlines()]
    assert all(250 < x < 350 for x in T)
    for name in ("velocity", "linear_temperature", "linear_pressure"):
        assert len((st / f"{name}.txt").read_text().split()) == 16, name
    hist = [line.split() for line in (st / "velocity_distribution.txt").read_text().splitlines()]
    assert len(hist) == 16 and sum(int(c) for _, c in hist) > 0
    assert len((st / "permeability.txt").read_text().split()) == 1
    assert sum("Molecules:" in line for line in r.stdout.splitlines()) == 3


@pytest.mark.gpu
def test_executable_continues_from_its_state_files(tmp_path):
    """load_previous_state: the second run reads state_files/state0000.bin and
    Tocontinue written by the first and carries the counters on."""
    g = Geometry.packed_spheres(32, 3, wanted_porosity=0.6, seed=2)
    (tmp_path / "worlds" / "test").mkdir(parents=True)
    g.write_world(tmp_path / "worlds" / "test")
    (tmp_path / "dsmc.ini").write_text(INI)
    r = subprocess.run([str(EXE)], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    first = (tmp_path / "Tocontinue").read_text().split()
    assert (tmp_path / "state_files" / "state0000.bin").exists()
    (tmp_path / "dsmc.ini").write_text(INI.replace("load_previous_state = false", "load_previous_state = true"))
    r = subprocess.run([str(EXE)], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    t, steps, collisions, walls = (tmp_path / "Tocontinue").read_text().split()
    assert int(steps) == 12 and int(collisions) >= int(first[2]) and int(walls) > int(first[3])
    assert float(t) > float(first[0])

