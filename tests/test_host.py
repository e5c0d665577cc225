"""CPU tests of the host side: the C ABI exports, settings/ini parsing, world
files, the packed-sphere generator and the cell layout, pinned against the
reference's own tool output and the golden fixtures (tests/golden/)."""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import re
from pathlib import Path

import numpy as np
import pytest

from master_b200 import capi
from master_b200.system import Geometry, Settings, cells_layout

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"


def header_functions(header="dsmc_b200.h"):
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dsmc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = capi.load()
    names = header_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    assert set(capi.EXPORTED) == set(names)
    sg = header_functions("dsmc_surrogate.h")
    for name in sg:
        assert hasattr(lib, name), name
    assert set(capi.EXPORTED_SURROGATE) == set(sg)
    headers = sorted(p.name for p in (ROOT / "include").glob("*.h"))
    assert headers == ["dsmc_b200.h", "dsmc_surrogate.h"]


def test_settings_defaults_match_python_driver():
    s = Settings()
    assert s.atoms_per_molecule == 1000 and s.statistics_interval == 100 and s.cells_x == 10
    assert s.mass == pytest.approx(39.948) and s.temperature == 300


INI = """load_previous_state = false
create_movie = false
max_molecules_per_node = 1000000
atoms_per_molecule = 1000
timesteps = 200
temperature = 300
wall_temperature = 310
statistics_interval = 100
velocity_profile_type = other
sampling_bins = 32
movie_every_n_frame = 1
movie_molecules = 1000
dt        = 0.00997087
# Gravity direction also determins which dimension we measure flux in
gravity = 0.00100585
flow_direction = 0
pressure_A = 100000
pressure_B = 100000
reservoir_fraction = 0
world = worlds/test
surface_interaction_model = thermal
alpha_n = 0.5
alpha_t = 0.8
seed = 7
density = 2.5e24
diam = 3.66e-4
mass = 39.9268
viscosity = 2.23e-5
Lx  = 6.4
Ly  = 6.4
Lz  = 6.4
cells_x = 32
cells_y = 32
cells_z = 32
nx = 1
ny = 1
nz = 1
"""


def test_ini_parsed_like_cinifile(tmp_path):
    p = tmp_path / "dsmc.ini"
    p.write_text(INI.replace("\n", "\r\n"))
    s = Settings.from_ini(p)
    assert s.dt == 0.00997087 and s.gravity == 0.00100585 and s.wall_temperature == 310
    assert s.cells_y == 32 and s.seed == 7 and s.world == "worlds/test" and s.Lx == 6.4
    assert s.density == 2.5e24 and s.flow_direction == 0


def test_ini_wall_models(tmp_path):
    p = tmp_path / "dsmc.ini"
    for name, code in (("thermal", 0), ("specular", 1), ("cercignani_lampis", 2)):
        p.write_text(INI.replace("= thermal", "= " + name))
        assert Settings.from_ini(p).surface_model == code


def test_ini_missing_key_and_unbuilt_model(tmp_path):
    p = tmp_path / "dsmc.ini"
    p.write_text(INI.replace("diam = 3.66e-4\n", ""))
    with pytest.raises(capi.DsmcError) as e:
        Settings.from_ini(p)
    assert e.value.code == capi.DSMC_ERR_NOT_FOUND and "diam" in str(e.value)
    p.write_text(INI.replace("= thermal", "= maxwell"))
    with pytest.raises(capi.DsmcError) as e:
        Settings.from_ini(p)
    assert e.value.code == capi.DSMC_ERR_CONFIG
    with pytest.raises(capi.DsmcError) as e:
        Settings.from_ini(tmp_path / "absent.ini")
    assert e.value.code == capi.DSMC_ERR_IO


def test_packed_spheres_identical_to_reference_tool():
    """ComplexGeometry::create_packed_spheres + normals/tangents/boundary, run by
    the reference's own geometry tool (digests in tests/golden/)."""
    d = json.loads((GOLDEN / "geometry_packed64_digests.json").read_text())
    g = Geometry.packed_spheres(64, 4, wanted_porosity=0.6, seed=1)
    for k in ("voxels", "normals", "tangents1", "tangents2"):
        assert hashlib.sha256(np.ascontiguousarray(getattr(g, k)).tobytes()).hexdigest() == d[k], k
    assert g.porosity_global == d["porosity_global"]


def test_world_file_roundtrip_and_halo(tmp_path):
    g = Geometry.packed_spheres(16, 2, wanted_porosity=0.6, seed=5)
    g.write_world(tmp_path)
    raw = (tmp_path / "0000.bin").read_bytes()
    hdr = np.frombuffer(raw[:32], np.uint32)
    assert tuple(hdr[2:8]) == (16, 16, 16, 48, 48, 48)
    assert len(raw) == 32 + 48 ** 3 * (1 + 36)
    # the halo holds periodic copies: voxel (i,j,k) of the stored grid is global (i-16, j-16, k-16) mod 16
    vox = np.frombuffer(raw[32:32 + 48 ** 3], np.uint8).reshape(48, 48, 48)
    assert np.array_equal(vox, np.tile(g.voxels, (3, 3, 3)))
    back = Geometry.read_world(tmp_path / "0000.bin")
    for k in ("voxels", "normals", "tangents1", "tangents2"):
        assert np.array_equal(getattr(back, k), getattr(g, k))
    assert (tmp_path / "porosity.txt").read_text().startswith("0.")


def test_world_file_errors(tmp_path):
    p = tmp_path / "short.bin"
    p.write_bytes(b"\0" * 10)
    with pytest.raises(capi.DsmcError) as e:
        Geometry.read_world(p)
    assert e.value.code == capi.DSMC_ERR_IO
    g = Geometry.packed_spheres(16, 2, wanted_porosity=0.6, seed=5)
    g.write_world(tmp_path)
    full = (tmp_path / "0000.bin").read_bytes()
    (tmp_path / "trunc.bin").write_bytes(full[: len(full) // 2])
    with pytest.raises(capi.DsmcError):
        Geometry.read_world(tmp_path / "trunc.bin")


def test_multi_rank_world_files(tmp_path):
    g = Geometry.packed_spheres(16, 2, wanted_porosity=0.6, seed=5)
    g.write_world(tmp_path, procs=(2, 1, 1))
    for rank in range(2):
        raw = (tmp_path / f"{rank:04d}.bin").read_bytes()
        hdr = np.frombuffer(raw[8:32], np.uint32)
        assert tuple(hdr) == (16, 16, 16, 24, 48, 48)
        vox = np.frombuffer(raw[32:32 + 24 * 48 * 48], np.uint8).reshape(24, 48, 48)
        # rank r's centre block is global x in [8r, 8r+8)
        assert np.array_equal(vox[8:16, 16:32, 16:32], g.voxels[8 * rank:8 * rank + 8])


@pytest.mark.parametrize("case", ["small_dt1", "small_dt5"])
def test_cells_layout_matches_reference(case):
    """System::setup_cells + Cell::update_volume of the reference."""
    z = np.load(GOLDEN / f"{case}.npz")
    meta = json.loads(str(z["meta"]))
    c = meta["params"]
    g = Geometry.packed_spheres(c["n"], c["radius_voxels"], wanted_porosity=c["porosity"], seed=c["geom_seed"])
    s = Settings()
    st = meta["settings"]
    for k in ("Lx", "Ly", "Lz", "cells_x", "cells_y", "cells_z", "dt", "diam", "atoms_per_molecule"):
        setattr(s, k, st[k])
    cl = cells_layout(s, g)
    assert np.array_equal(cl["global_index"], z["cell_global"])
    assert np.array_equal(cl["pixels"], z["cell_pixels"])
    assert np.array_equal(cl["total_pixels"], z["cell_total_pixels"])
    assert np.array_equal(cl["volume"], z["cell_volume"])
    assert np.array_equal(cl["coeff"], z["cell_coeff"])


def test_from_mask_normals():
    n = 16
    i, j, k = np.meshgrid(*(np.arange(n),) * 3, indexing="ij")
    solid = ((i - 7.5) ** 2 + (j - 7.5) ** 2 + (k - 7.5) ** 2) < 16
    g = Geometry.from_mask(solid.astype(np.uint8))
    b = g.voxels == 2
    assert b.any() and (g.voxels == 1).any()
    nn = np.linalg.norm(g.normals[b], axis=-1)
    assert np.allclose(nn, 1, atol=1e-6)
    # normals of a solid ball point outwards
    pos = np.stack([i, j, k], -1)[b] - 7.5
    assert (np.sum(pos * g.normals[b], -1) > 0).mean() > 0.99
    t1 = g.tangents1[b]
    assert np.abs(np.sum(t1 * g.normals[b], -1)).max() < 1e-5
