"""Host-side mirror of the reference's System / StatisticsSampler interface
(andeplane/master code/base_code/program/dsmc/system.h:29-120,
statisticssampler.h) over the C ABI of libdsmc_b200.

    settings = Settings.from_ini("dsmc.ini")          # Settings::Settings
    system = System(settings, geometry)               # System::initialize
    for _ in range(settings.timesteps):
        system.step()                                 # System::step + sample

`System.step(n)` runs n fused timesteps on the GPU.  The stage methods
(`accelerate_and_move`, `update_molecule_cells`, `collide`, `sample`) run
System::step's stages one at a time for callers that drive them.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import capi
from .capi import Settings as _CSettings, check, ptr

# reduced units of the reference (dsmc/unitconverter.cpp:3-21)
M0 = 1.66053886e-27
L0 = 1e-6
E0 = 1.65088e-21
KB = 1.3806503e-23
T0_TIME = L0 * (M0 / E0) ** 0.5
T0_TEMP = E0 / KB
A0 = (L0 / T0_TIME) / T0_TIME


def time_from_si(t: float) -> float:
    return t / T0_TIME


def acceleration_from_si(a: float) -> float:
    return a / A0


class Settings:
    """dsmc_settings with attribute access (fields of dsmc/settings.h:11-49)."""

    def __init__(self, raw: _CSettings | None = None):
        lib = capi.load()
        if raw is None:
            raw = _CSettings()
            check(lib.dsmc_settings_defaults(C.byref(raw)))
        object.__setattr__(self, "raw", raw)

    @classmethod
    def from_ini(cls, path: str | Path) -> "Settings":
        raw = _CSettings()
        check(capi.load().dsmc_settings_load_ini(str(path).encode(), C.byref(raw)))
        return cls(raw)

    def __getattr__(self, k):
        v = getattr(self.raw, k)
        return v.decode() if isinstance(v, bytes) else v

    def __setattr__(self, k, v):
        if k == "world":
            v = str(v).encode()
        setattr(self.raw, k, v)


@dataclass
class Geometry:
    """Voxel types (0 empty, 1 wall, 2 boundary) with normals and tangents, in
    the reference's i*ny*nz + j*nz + k order, without halo."""
    voxels: np.ndarray       # uint8 (nx, ny, nz)
    normals: np.ndarray      # float32 (nx, ny, nz, 3)
    tangents1: np.ndarray
    tangents2: np.ndarray
    porosity_global: float = -1.0

    @property
    def shape(self):
        return self.voxels.shape

    @classmethod
    def empty(cls, nx, ny, nz) -> "Geometry":
        return cls(np.zeros((nx, ny, nz), np.uint8), *(np.zeros((nx, ny, nz, 3), np.float32) for _ in range(3)))

    @classmethod
    def packed_spheres(cls, n, radius_voxels=None, *, radius=None, wanted_porosity=0.6, seed=1, spheres_type=1,
                       spheres_num=0, inverted=True, prevent_overlap=False, number_of_neighbor_averages=1):
        """ComplexGeometry::create_packed_spheres (dsmc/complexgeometry.cpp:401-513)."""
        nx, ny, nz = (n, n, n) if np.isscalar(n) else n
        if radius is None:
            radius = radius_voxels / nx
        g = cls.empty(nx, ny, nz)
        p = capi.SphereParams(nx, ny, nz, float(radius), spheres_type, spheres_num, float(wanted_porosity), seed,
                              int(inverted), int(prevent_overlap), number_of_neighbor_averages)
        por = C.c_float()
        check(capi.load().dsmc_geometry_packed_spheres(C.byref(p), ptr(g.voxels, C.c_uint8),
                                                       ptr(g.normals, C.c_float), ptr(g.tangents1, C.c_float),
                                                       ptr(g.tangents2, C.c_float), C.byref(por)))
        g.porosity_global = float(por.value)
        return g

    @classmethod
    def from_mask(cls, solid: np.ndarray, number_of_neighbor_averages=1) -> "Geometry":
        """Normals/tangents/boundary of a 0/1 solid mask (dsmc/complexgeometry.cpp:196-201)."""
        nx, ny, nz = solid.shape
        g = cls.empty(nx, ny, nz)
        g.voxels[...] = (solid != 0).astype(np.uint8)
        check(capi.load().dsmc_geometry_finish(nx, ny, nz, number_of_neighbor_averages, ptr(g.voxels, C.c_uint8),
                                               ptr(g.normals, C.c_float), ptr(g.tangents1, C.c_float),
                                               ptr(g.tangents2, C.c_float)))
        return g

    @classmethod
    def read_world(cls, path: str | Path) -> "Geometry":
        """DSMC_IO::read_grid_matrix (dsmc/dsmc_io.cpp:183-220), halo stripped."""
        lib = capi.load()
        h = capi.WorldHeader()
        check(lib.dsmc_world_read_header(str(path).encode(), C.byref(h)))
        g = cls.empty(h.global_nx, h.global_ny, h.global_nz)
        check(lib.dsmc_world_read(str(path).encode(), ptr(g.voxels, C.c_uint8), ptr(g.normals, C.c_float),
                                  ptr(g.tangents1, C.c_float), ptr(g.tangents2, C.c_float)))
        g.porosity_global = float(h.porosity_global)
        return g

    def write_world(self, folder: str | Path, procs=(1, 1, 1)) -> None:
        """ComplexGeometry::save_to_file (dsmc/complexgeometry.cpp:220-318)."""
        nx, ny, nz = self.shape
        check(capi.load().dsmc_world_write(str(folder).encode(), nx, ny, nz, ptr(self.voxels, C.c_uint8),
                                           ptr(self.normals, C.c_float), ptr(self.tangents1, C.c_float),
                                           ptr(self.tangents2, C.c_float), *procs))

    @property
    def porosity(self) -> float:
        return float((self.voxels == 0).mean())


def cells_layout(settings: Settings, geometry: Geometry) -> dict:
    """System::setup_cells' active cells for a geometry (host only)."""
    lib = capi.load()
    nx, ny, nz = geometry.shape
    n = C.c_int()
    check(lib.dsmc_cells_layout(C.byref(settings.raw), nx, ny, nz, ptr(geometry.voxels, C.c_uint8), 0, None, None,
                                None, None, None, C.byref(n)))
    out = {k: np.empty(n.value, np.int32) for k in ("global_index", "pixels", "total_pixels")}
    out["volume"] = np.empty(n.value)
    out["coeff"] = np.empty(n.value)
    check(lib.dsmc_cells_layout(C.byref(settings.raw), nx, ny, nz, ptr(geometry.voxels, C.c_uint8), n.value,
                                ptr(out["global_index"], C.c_int32), ptr(out["pixels"], C.c_int32),
                                ptr(out["total_pixels"], C.c_int32), ptr(out["volume"], C.c_double),
                                ptr(out["coeff"], C.c_double), C.byref(n)))
    return out


def read_state_file(path) -> tuple[np.ndarray, np.ndarray]:
    """The reference's state file (state_files/state%04d.bin,
    dsmc/dsmc_io.cpp:82-159) as (r, v), each (N, 3) float64."""
    lib = capi.load()
    n = C.c_int64()
    check(lib.dsmc_state_file_read(str(path).encode(), 0, None, None, C.byref(n)))
    r = np.empty((n.value, 3))
    v = np.empty((n.value, 3))
    check(lib.dsmc_state_file_read(str(path).encode(), n.value, ptr(r, C.c_double), ptr(v, C.c_double), C.byref(n)))
    return r, v


def write_state_file(path, r, v) -> None:
    r = np.ascontiguousarray(r, np.float64)
    v = np.ascontiguousarray(v, np.float64)
    check(capi.load().dsmc_state_file_write(str(path).encode(), len(r), ptr(r, C.c_double), ptr(v, C.c_double)))


def read_tocontinue(path) -> dict:
    """The reference's Tocontinue counters (dsmc/main.cpp:37-55)."""
    t = C.c_double()
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
    check(capi.load().dsmc_tocontinue_read(str(path).encode(), C.byref(t), C.byref(a), C.byref(b), C.byref(c)))
    return {"t": t.value, "steps": a.value, "collisions": b.value, "wall_collisions": c.value}


def write_tocontinue(path, t: float, steps: int, collisions: int, wall_collisions: int) -> None:
    check(capi.load().dsmc_tocontinue_write(str(path).encode(), t, steps, collisions, wall_collisions))


def finish_profiles(settings: Settings, volume_global: float, sums: np.ndarray, *, lib=None) -> dict:
    """Finishes raw sampler sums (shape (4, bins), e.g. summed over ranks) by
    dsmc_profiles_finish."""
    lib = lib or capi.load()
    sums = np.asarray(sums, np.float64)
    b = sums.shape[1]
    flat = np.ascontiguousarray(np.concatenate([sums[:3].T.reshape(-1), sums[3]]))
    out = {k: np.empty(b) for k in ("count", "velocity_z", "temperature", "pressure", "vx_center", "vx_count")}
    raw = settings.raw if isinstance(settings, Settings) else settings
    rc = lib.dsmc_profiles_finish(C.byref(raw), volume_global, b, ptr(flat, C.c_double),
                                  *(ptr(out[k], C.c_double) for k in ("count", "velocity_z", "temperature",
                                                                      "pressure", "vx_center", "vx_count")))
    if rc:
        raise capi.DsmcError(rc, "dsmc_profiles_finish")
    return out


class Context:
    """One GPU context holding any number of systems (geometry + gas)."""

    def __init__(self, device: int = 0, precision: int = capi.PREC_SPLIT32):
        self.lib = capi.load()
        h = C.c_void_p()
        check(self.lib.dsmc_ctx_create(device, precision, C.byref(h)))
        self.handle = h
        self.device = device
        self.precision = precision

    def close(self):
        if self.handle:
            self.lib.dsmc_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc):
        check(rc, self.handle)

    def add_system(self, settings: Settings, geometry: Geometry) -> int:
        sid = C.c_int()
        nx, ny, nz = geometry.shape
        self.check(self.lib.dsmc_system_add(self.handle, C.byref(settings.raw), nx, ny, nz,
                                            ptr(geometry.voxels, C.c_uint8), ptr(geometry.normals, C.c_float),
                                            ptr(geometry.tangents1, C.c_float), ptr(geometry.tangents2, C.c_float),
                                            C.c_float(geometry.porosity_global), C.byref(sid)))
        return sid.value

    def add_slab(self, settings: Settings, geometry: Geometry, cell_x0: int, cell_x1: int) -> int:
        """The x-slab of the geometry holding cells with x index in
        [cell_x0, cell_x1): the context's only system (master_b200.slab)."""
        sid = C.c_int()
        nx, ny, nz = geometry.shape
        self.check(self.lib.dsmc_system_add_slab(self.handle, C.byref(settings.raw), nx, ny, nz,
                                                 ptr(geometry.voxels, C.c_uint8), ptr(geometry.normals, C.c_float),
                                                 ptr(geometry.tangents1, C.c_float),
                                                 ptr(geometry.tangents2, C.c_float),
                                                 C.c_float(geometry.porosity_global), cell_x0, cell_x1,
                                                 C.byref(sid)))
        return sid.value

    def exchange_take(self) -> np.ndarray:
        """The records that left the slab in the last step, shape (n, 8)
        uint32 (dsmc_exchange_take's layout), now removed from the slab."""
        n = C.c_int64()
        rc = self.lib.dsmc_exchange_take(self.handle, 0, None, 0, C.byref(n))
        if rc not in (0, capi.DSMC_ERR_CAPACITY):
            self.check(rc)
        out = np.empty((n.value, 8), np.uint32)
        if n.value:
            self.check(self.lib.dsmc_exchange_take(self.handle, n.value, out.ctypes.data, 0, C.byref(n)))
        return out[:n.value]

    def exchange_take_device(self, torch_device):
        """exchange_take into a tensor on the context's GPU (int32 view of the records)."""
        import torch
        n = C.c_int64()
        rc = self.lib.dsmc_exchange_take(self.handle, 0, None, 1, C.byref(n))
        if rc not in (0, capi.DSMC_ERR_CAPACITY):
            self.check(rc)
        out = torch.empty((n.value, 8), dtype=torch.int32, device=torch_device)
        if n.value:
            torch.cuda.synchronize(torch_device)
            self.check(self.lib.dsmc_exchange_take(self.handle, n.value, C.c_void_p(out.data_ptr()), 1, C.byref(n)))
        return out

    def exchange_put(self, sys_id: int, records) -> None:
        """Records (n, 8) from other slabs into system sys_id: a numpy array
        on the host, or a tensor on the context's GPU."""
        if hasattr(records, "data_ptr") and getattr(records, "is_cuda", False):
            if records.shape[0]:
                import torch
                torch.cuda.synchronize(records.device)
                self.check(self.lib.dsmc_exchange_put(self.handle, sys_id, records.shape[0],
                                                      C.c_void_p(records.contiguous().data_ptr()), 1))
            return
        rec = np.ascontiguousarray(np.asarray(records).view(np.uint32).reshape(-1, 8))
        if rec.shape[0]:
            self.check(self.lib.dsmc_exchange_put(self.handle, sys_id, rec.shape[0], rec.ctypes.data, 0))

    def step(self, n: int = 1):
        self.check(self.lib.dsmc_step(self.handle, n))

    def sync(self):
        self.check(self.lib.dsmc_sync(self.handle))

    def pass_info(self) -> dict:
        vals = [C.c_int() for _ in range(4)]
        self.check(self.lib.dsmc_pass_info(self.handle, *(C.byref(v) for v in vals)))
        return dict(zip(("pipelined", "grid", "block", "stage_capacity"), (v.value for v in vals)))

    def checkpoint_save(self, path) -> None:
        """Exact checkpoint of every system of the context."""
        self.check(self.lib.dsmc_checkpoint_save(self.handle, str(path).encode()))

    def checkpoint_load(self, path) -> None:
        self.check(self.lib.dsmc_checkpoint_load(self.handle, str(path).encode()))

    def set_timing(self, on: bool) -> None:
        self.check(self.lib.dsmc_ctx_set_timing(self.handle, 1 if on else 0))

    def pass_times(self) -> dict:
        """Summed milliseconds per production kernel since timing was turned on."""
        ms = np.zeros(4)
        n = C.c_int64()
        self.check(self.lib.dsmc_pass_times_get(self.handle, ms.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)))
        out = dict(zip(("collide_cells", "move_cells", "place_movers", "place_walls"), ms.tolist()))
        out["passes"] = n.value
        return out

    def device_status(self):
        e, s = C.c_uint32(), C.c_uint32()
        self.check(self.lib.dsmc_device_status(self.handle, C.byref(e), C.byref(s)))
        return e.value, s.value


class System:
    """The reference's System over one context (its only system unless a
    shared Context is given)."""

    def __init__(self, settings: Settings, geometry: Geometry, *, context: Context | None = None, device: int = 0,
                 precision: int = capi.PREC_SPLIT32, init_particles: bool = True, num_particles: int = -1):
        self.settings = settings
        self.geometry = geometry
        self.ctx = context or Context(device, precision)
        self.id = self.ctx.add_system(settings, geometry)
        if init_particles:
            self.ctx.check(self.ctx.lib.dsmc_particles_init(self.ctx.handle, self.id, num_particles))

    # ---- state -------------------------------------------------------------
    def info(self) -> capi.SystemInfo:
        i = capi.SystemInfo()
        self.ctx.check(self.ctx.lib.dsmc_system_info_get(self.ctx.handle, self.id, C.byref(i)))
        return i

    @property
    def num_molecules(self) -> int:
        return int(self.info().num_particles)

    def set_particles(self, r: np.ndarray, v: np.ndarray) -> None:
        r = np.ascontiguousarray(r, np.float64).reshape(-1, 3)
        v = np.ascontiguousarray(v, np.float64).reshape(-1, 3)
        assert r.shape == v.shape
        self.ctx.check(self.ctx.lib.dsmc_particles_set(self.ctx.handle, self.id, r.shape[0], ptr(r, C.c_double),
                                                       ptr(v, C.c_double)))

    def get_particles(self, with_cells: bool = False):
        n = self.num_molecules
        r = np.empty((n, 3), np.float64)
        v = np.empty((n, 3), np.float64)
        cell = np.empty(n, np.int32) if with_cells else None
        got = C.c_int64()
        self.ctx.check(self.ctx.lib.dsmc_particles_get(self.ctx.handle, self.id, n, ptr(r, C.c_double),
                                                       ptr(v, C.c_double), ptr(cell, C.c_int32), C.byref(got)))
        return (r, v, cell) if with_cells else (r, v)

    def cells(self):
        info = self.info()
        n = info.num_active_cells
        out = {
            "global_index": np.empty(n, np.int32), "count": np.empty(n, np.int32), "vr_max": np.empty(n),
            "rest": np.empty(n), "moments": np.empty((n, 8)), "volume": np.empty(n),
        }
        nc = C.c_int()
        self.ctx.check(self.ctx.lib.dsmc_cells_get(
            self.ctx.handle, self.id, n, ptr(out["global_index"], C.c_int32), ptr(out["count"], C.c_int32),
            ptr(out["vr_max"], C.c_double), ptr(out["rest"], C.c_double), ptr(out["moments"], C.c_double),
            ptr(out["volume"], C.c_double), C.byref(nc)))
        return out

    def set_cell_state(self, vr_max: np.ndarray, rest: np.ndarray) -> None:
        vr_max = np.ascontiguousarray(vr_max, np.float64)
        rest = np.ascontiguousarray(rest, np.float64)
        self.ctx.check(self.ctx.lib.dsmc_cells_set_state(self.ctx.handle, self.id, ptr(vr_max, C.c_double),
                                                         ptr(rest, C.c_double)))

    def continue_from(self, t: float, steps: int, collisions: int, wall_collisions: int) -> None:
        """Carry over an earlier run's time and counters (dsmc/main.cpp:37-55)."""
        self.ctx.check(self.ctx.lib.dsmc_continue_from(self.ctx.handle, self.id, t, steps, collisions,
                                                       wall_collisions))

    def tallies(self) -> capi.Tallies:
        t = capi.Tallies()
        self.ctx.check(self.ctx.lib.dsmc_tallies_get(self.ctx.handle, self.id, C.byref(t)))
        return t

    def measures(self) -> capi.Measures:
        """The sampler's scalar measurements now (energy, temperature, flow
        rates, pressure, permeability), as StatisticsSampler::sample records them."""
        m = capi.Measures()
        self.ctx.check(self.ctx.lib.dsmc_measures_get(self.ctx.handle, self.id, C.byref(m)))
        return m

    def reset_tallies(self) -> None:
        """Zeroes the tallies, the cell moments and the sampler profiles."""
        self.ctx.check(self.ctx.lib.dsmc_tallies_reset(self.ctx.handle, self.id))

    def profile_sums(self) -> np.ndarray:
        """Raw sampler sums, shape (4, bins): per y bin the count, sum v_z and
        sum 1/2 m v_z^2, then the v_x histogram (reduced units).  Sums of
        several runs add before finish_profiles."""
        bins = C.c_int()
        self.ctx.check(self.ctx.lib.dsmc_profile_sums_get(self.ctx.handle, self.id, 0, ptr(None, C.c_double),
                                                          C.byref(bins)))
        flat = np.empty(4 * bins.value)
        self.ctx.check(self.ctx.lib.dsmc_profile_sums_get(self.ctx.handle, self.id, flat.size,
                                                          ptr(flat, C.c_double), C.byref(bins)))
        b = bins.value
        y = flat[:3 * b].reshape(b, 3)
        return np.stack([y[:, 0], y[:, 1], y[:, 2], flat[3 * b:]])

    def profiles(self) -> dict:
        """The sampler's profiles finished as the reference's finalize()
        writes them (dsmc/statisticalproperty.cpp:303-309, 364-371, 419-426,
        462-478): y-binned count, v_z (m/s), temperature (K), pressure (Pa),
        and the v_x histogram (bin centres in m/s, counts)."""
        return finish_profiles(self.settings, self.info().volume_global, self.profile_sums(), lib=self.ctx.lib)

    # ---- the timestep ------------------------------------------------------
    def step(self, n: int = 1) -> None:
        """n x (System::step + StatisticsSampler::sample), dsmc/main.cpp:57-64."""
        self.ctx.step(n)

    def accelerate_and_move(self) -> None:
        """steps += 1; System::accelerate + System::move (dsmc/system.cpp:107-144)."""
        self.ctx.check(self.ctx.lib.dsmc_stage_move(self.ctx.handle))

    def update_molecule_cells(self) -> None:
        """System::update_molecule_cells (dsmc/system.cpp:146-157)."""
        self.ctx.check(self.ctx.lib.dsmc_stage_sort(self.ctx.handle))

    def collide(self) -> None:
        """System::collide (dsmc/system.cpp:122-131)."""
        self.ctx.check(self.ctx.lib.dsmc_stage_collide(self.ctx.handle))

    def sample(self) -> None:
        """The per-cell moment tallies of StatisticsSampler::sample."""
        self.ctx.check(self.ctx.lib.dsmc_stage_sample(self.ctx.handle))
