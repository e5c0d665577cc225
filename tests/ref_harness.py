"""ctypes driver of oracle/_ref/libdsmc_ref_tape.so: the reference's own
System / MoleculeMover / Cell routines, stage by stage, fed the counter-based
draws the GPU kernels take (see oracle/ref_harness.cpp).  Test infrastructure.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "oracle" / "_ref" / "libdsmc_ref_tape.so"

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def available() -> bool:
    return LIB.exists()


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


INI_TEMPLATE = """load_previous_state = false
create_movie = false
max_molecules_per_node = {max_molecules}
atoms_per_molecule = {atoms_per_molecule}
timesteps = 1
temperature = {temperature}
wall_temperature = {wall_temperature}
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
surface_interaction_model = {surface}
alpha_n = {alpha_n!r}
alpha_t = {alpha_t!r}
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


def write_ini(path: Path, **kw) -> None:
    kw.setdefault("surface", "thermal")
    kw.setdefault("alpha_n", 0.5)
    kw.setdefault("alpha_t", 0.8)
    path.write_text(INI_TEMPLATE.format(**kw))


class RefSystem:
    """The reference's System built from an ini in a scratch directory that
    also holds the world file (written by the caller)."""

    def __init__(self, workdir: Path):
        self.lib = C.CDLL(str(LIB))
        L = self.lib
        L.refh_create.restype = C.c_void_p
        L.refh_create.argtypes = [C.c_char_p]
        for name in ["refh_num_particles"]:
            getattr(L, name).restype = C.c_long
        for name in ["refh_dt", "refh_porosity"]:
            getattr(L, name).restype = C.c_double
        for name in ["refh_num_particles", "refh_num_active_cells", "refh_max_particles", "refh_dt", "refh_porosity",
                     "refh_accelerate", "refh_update_cells", "refh_canonicalize_cells", "refh_reset_counters"]:
            getattr(L, name).argtypes = [C.c_void_p]
        L.refh_set_particles.argtypes = [C.c_void_p, C.c_long, _D, _D]
        L.refh_get_particles.argtypes = [C.c_void_p, _D, _D, _I]
        L.refh_move.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32]
        L.refh_init_particles.argtypes = [C.c_void_p, C.c_uint64, C.c_long]
        L.refh_collide.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32]
        L.refh_counters.argtypes = [C.c_void_p, C.POINTER(C.c_long), C.POINTER(C.c_ulong), C.POINTER(C.c_ulong)]
        L.refh_cell_info.argtypes = [C.c_void_p, _I, _I, _I, _D, _D, _D, _D, _I]
        L.refh_set_cell_state.argtypes = [C.c_void_p, _D, _D]
        L.refh_cell_members.argtypes = [C.c_void_p, C.c_int, _I, C.c_int]
        L.refh_cell_index_map.argtypes = [C.c_void_p, _I, C.c_int]
        L.refh_grid_dims.argtypes = [C.c_void_p, C.POINTER(C.c_uint)]
        L.refh_grid_core.argtypes = [C.c_void_p, C.POINTER(C.c_ubyte), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                     C.POINTER(C.c_float)]
        L.refh_voxel_index.argtypes = [C.c_void_p, _D]
        L.refh_cell_index_of.argtypes = [C.c_void_p, C.c_long]
        L.refh_sampler_create.restype = C.c_void_p
        L.refh_sampler_create.argtypes = [C.c_void_p]
        L.refh_sample.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        L.refh_profile_sums.argtypes = [C.c_void_p, C.c_int, _D]
        L.refh_profiles_finish.argtypes = [C.c_void_p, C.c_void_p, C.c_int, _D, _D, _D, _D]
        L.refh_measures.argtypes = [C.c_void_p, C.c_void_p, _D]
        self._sampler = None
        cwd = os.getcwd()
        os.chdir(workdir)
        try:
            (workdir / "statistics" / "time").mkdir(parents=True, exist_ok=True)
            self.h = L.refh_create(b"dsmc.ini")
        finally:
            os.chdir(cwd)
        if not self.h:
            raise RuntimeError("reference System::initialize failed")

    @property
    def n(self) -> int:
        return self.lib.refh_num_particles(self.h)

    def set_particles(self, r: np.ndarray, v: np.ndarray) -> None:
        r = np.ascontiguousarray(r, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        rc = self.lib.refh_set_particles(self.h, r.shape[0], _p(r, C.c_double), _p(v, C.c_double))
        if rc:
            raise RuntimeError("too many particles for max_molecules_per_node")

    def get_particles(self):
        n = self.n
        r = np.empty((n, 3))
        v = np.empty((n, 3))
        cell = np.empty(n, np.int32)
        self.lib.refh_get_particles(self.h, _p(r, C.c_double), _p(v, C.c_double), _p(cell, C.c_int))
        return r, v, cell

    def cells(self):
        nc = self.lib.refh_num_active_cells(self.h)
        out = {k: np.empty(nc, np.int32) for k in ("global_index", "pixels", "total_pixels", "count")}
        for k in ("volume", "coeff", "vr_max", "rest"):
            out[k] = np.empty(nc)
        self.lib.refh_cell_info(self.h, _p(out["global_index"], C.c_int), _p(out["pixels"], C.c_int),
                                _p(out["total_pixels"], C.c_int), _p(out["volume"], C.c_double),
                                _p(out["coeff"], C.c_double), _p(out["vr_max"], C.c_double),
                                _p(out["rest"], C.c_double), _p(out["count"], C.c_int))
        return out

    def set_cell_state(self, vr_max, rest):
        vr_max = np.ascontiguousarray(vr_max, np.float64)
        rest = np.ascontiguousarray(rest, np.float64)
        self.lib.refh_set_cell_state(self.h, _p(vr_max, C.c_double), _p(rest, C.c_double))

    def members(self, cell: int) -> np.ndarray:
        buf = np.empty(4096, np.int32)
        n = self.lib.refh_cell_members(self.h, cell, _p(buf, C.c_int), buf.size)
        return buf[:n].copy()

    def init_particles(self, seed: int, n: int) -> None:
        if self.lib.refh_init_particles(self.h, seed, n):
            raise RuntimeError("too many particles for max_molecules_per_node")

    def accelerate(self):
        self.lib.refh_accelerate(self.h)

    def move(self, seed: int, step: int):
        self.lib.refh_move(self.h, seed, step)

    def update_cells(self):
        self.lib.refh_update_cells(self.h)

    def canonicalize(self):
        self.lib.refh_canonicalize_cells(self.h)

    def collide(self, seed: int, step: int):
        self.lib.refh_collide(self.h, seed, step)

    def counters(self):
        cp = (C.c_long * 3)()
        col = C.c_ulong()
        wall = C.c_ulong()
        self.lib.refh_counters(self.h, cp, C.byref(col), C.byref(wall))
        return {"count_periodic": list(cp), "collisions": col.value, "wall_collisions": wall.value}

    def reset_counters(self):
        self.lib.refh_reset_counters(self.h)

    def sample(self, step: int) -> None:
        """StatisticsSampler::sample at System::steps = step (the sampler is
        created on first use, as dsmc/main.cpp:30 does before the loop)."""
        if self._sampler is None:
            self._sampler = self.lib.refh_sampler_create(self.h)
        self.lib.refh_sample(self.h, self._sampler, step)

    def profile_sums(self) -> np.ndarray:
        """(4, bins): y-binned count, sum v_z, sum 1/2 m v_z^2; v_x histogram."""
        buf = np.zeros(4 * 4096)
        b = self.lib.refh_profile_sums(self._sampler, buf.size, _p(buf, C.c_double))
        assert b > 0
        y = buf[:3 * b].reshape(b, 3)
        return np.stack([y[:, 0], y[:, 1], y[:, 2], buf[3 * b:4 * b]])

    MEASURES = ("energy_eV", "temperature_K", "number_flow_rate", "volumetric_flow_rate", "pressure_Pa",
                "permeability_darcy")

    def measures(self) -> dict:
        """The sampler's scalar measurements at the last sample."""
        out = np.zeros(6)
        self.lib.refh_measures(self.h, self._sampler, _p(out, C.c_double))
        return dict(zip(self.MEASURES, out.tolist()))

    def profiles(self) -> dict:
        """The reference's finished profiles in SI units (full precision)."""
        out = {k: np.zeros(4096) for k in ("velocity_z", "temperature", "pressure", "vx_center")}
        b = self.lib.refh_profiles_finish(self.h, self._sampler, 4096, *(_p(out[k], C.c_double) for k in
                                                                       ("velocity_z", "temperature", "pressure",
                                                                        "vx_center")))
        assert b > 0
        return {k: v[:b].copy() for k, v in out.items()}

    def voxel_index(self, r3) -> int:
        r3 = np.ascontiguousarray(r3, np.float64)
        return self.lib.refh_voxel_index(self.h, _p(r3, C.c_double))


def make_ref_system(geometry, settings: dict, workdir: Path | None = None) -> tuple[RefSystem, Path]:
    """Writes the world file and ini into a scratch dir and builds the reference System."""
    workdir = Path(workdir or tempfile.mkdtemp(prefix="refsys_"))
    (workdir / "worlds").mkdir(parents=True, exist_ok=True)
    geometry.write_world(workdir / "worlds")
    kw = dict(settings)
    kw["world"] = "worlds"
    write_ini(workdir / "dsmc.ini", **kw)
    return RefSystem(workdir), workdir
