"""Steady fields of porous sphere packs from the DSMC timestep itself: the
training data of the warm-start surrogate, and the warm start.

A field set is generated as the batched-ensemble configuration runs: many
packed-sphere geometries of one edge (porosity, sphere radius and Knudsen
number drawn per geometry) as systems of one context, all advanced by one
launch per stage, each started cold (System::setup_molecules,
dsmc/system.cpp:398-430), run through its transient, then its per-voxel
particle sums accumulated every few steps (dsmc_field_accumulate) over the
sampling window.  Per voxel the result is the density relative to the
geometry's mean over empty voxels and the mean drift velocity.

The Knudsen number is set through the density, as the reference's unit
converter does for its Knudsen input (bc/dsmc_unit_converter.py:112-116,
n = 1 / (sqrt(2) pi d^2 Kn l)), with the characteristic length l = the mean
pore chord of the geometry, 4 * porosity / (specific surface), the specific
surface counted as solid-empty voxel faces per volume.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import capi
from .system import Context, Geometry, System
from .workloads import ARGON_DIAM_UM, Workload

VELOCITY_SCALE = 1e-3  # reduced units (~1 m/s): the network's drift unit


def mean_pore_chord(solid: np.ndarray, voxel_um: float) -> float:
    """4 * porosity / S_v, S_v = solid/empty voxel faces (periodic) per volume, in um."""
    s = solid.astype(bool)
    faces = 0
    for ax in range(3):
        faces += int(np.count_nonzero(s != np.roll(s, 1, axis=ax)))
    V = s.size * voxel_um ** 3
    sv = faces * voxel_um ** 2 / V
    phi = 1.0 - s.mean()
    return 4.0 * phi / sv if sv > 0 else float("inf")


def density_for_knudsen(kn: float, chord_um: float, diam_um: float = ARGON_DIAM_UM) -> float:
    """n in m^-3 with mean free path 1/(sqrt(2) pi d^2 n) = kn * chord."""
    d = diam_um * 1e-6
    return 1.0 / (math.sqrt(2.0) * math.pi * d * d * kn * chord_um * 1e-6)


@dataclass
class PackSpec:
    """One geometry of a field set."""
    n: int
    porosity: float
    radius_voxels: float
    seed: int
    knudsen: float
    per_cell: float = 20.0           # simulators per open cell
    voxel_um: float = 0.1
    cells: int = 0                   # cells per axis (default n / 2)
    extra: dict = field(default_factory=dict)

    def geometry(self) -> Geometry:
        return Geometry.packed_spheres(self.n, self.radius_voxels, wanted_porosity=self.porosity, seed=self.seed)

    def workload(self, g: Geometry) -> Workload:
        solid = g.voxels > 0
        chord = mean_pore_chord(solid, self.voxel_um)
        dens = density_for_knudsen(self.knudsen, chord)
        cells = self.cells or self.n // 2
        vox_per_cell = self.n // cells
        weight = max(1, int(dens * 1e-18 * (vox_per_cell * self.voxel_um) ** 3 / self.per_cell))
        self.extra.update(chord_um=chord, density=dens, atoms_per_molecule=weight)
        return Workload(f"pack_{self.seed}", n=self.n, radius_voxels=self.radius_voxels, porosity=self.porosity,
                        geometry_seed=self.seed, cells=cells, atoms_per_molecule=weight, density_si=dens)


def random_specs(count: int, n: int, seed: int, porosity=(0.4, 0.8), radius=(3.0, 8.0), knudsen=(0.1, 10.0),
                 per_cell: float = 20.0) -> list[PackSpec]:
    """Porosity and radius uniform, Knudsen log-uniform (the batched-ensemble
    configuration's ranges); geometry seeds seed*10000 + i."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        out.append(PackSpec(n=n, porosity=float(rng.uniform(*porosity)), radius_voxels=float(rng.uniform(*radius)),
                            seed=seed * 10000 + i + 1,
                            knudsen=float(10 ** rng.uniform(math.log10(knudsen[0]), math.log10(knudsen[1]))),
                            per_cell=per_cell))
    return out


class Ensemble:
    """Geometries of a field set as systems of one context (one launch per stage)."""

    def __init__(self, specs: list[PackSpec], device: int = 0, rng_seed: int = 1, precision=capi.PREC_SPLIT32,
                 cold: bool = True, geoms: list | None = None, capacity: tuple | None = None):
        self.specs = specs
        self.ctx = Context(device, precision)
        if capacity is not None:  # slots per cell: ceil(factor * max(expected, present) + pad)
            self.ctx.check(self.ctx.lib.dsmc_ctx_set_capacity(self.ctx.handle, float(capacity[0]), int(capacity[1])))
        self.geoms, self.systems, self.settings = [], [], []
        for i, sp in enumerate(specs):
            g = geoms[i] if geoms is not None else sp.geometry()
            w = sp.workload(g)
            s = w.settings(rng_seed=rng_seed + i, statistics_interval=10 ** 9)
            self.geoms.append(g)
            self.settings.append(s)
            self.systems.append(System(s, g, context=self.ctx, init_particles=False))
        if cold:  # every system's cold start in one call: one re-layout, not one per system
            self.init_cold(self.systems)

    def init_cold(self, systems, counts=None) -> None:
        """System::setup_molecules for the given systems of this ensemble
        (counts: particles per system, None: the reference's count)."""
        if not systems:
            return
        ids = (C.c_int * len(systems))(*[S.id for S in systems])
        n = None if counts is None else (C.c_int64 * len(systems))(*[int(k) for k in counts])
        self.ctx.check(self.ctx.lib.dsmc_particles_init_many(self.ctx.handle, len(systems), ids, n))

    @property
    def particles(self) -> int:
        return sum(S.num_molecules for S in self.systems)

    def accumulate_fields(self, steps: int, every: int) -> list[np.ndarray]:
        """Runs `steps` steps and sums each system's per-voxel {count, vx, vy,
        vz} every `every` steps; returns one (n^3, 4) float64 array per system
        (sums over the samples) and leaves the number of samples in
        self.samples."""
        import torch
        fields = [torch.zeros((sp.n ** 3, 4), dtype=torch.float32, device=torch.device("cuda", self.ctx_device()))
                  for sp in self.specs]
        acc = [np.zeros((sp.n ** 3, 4)) for sp in self.specs]
        samples = 0
        for k in range(steps // every):
            self.ctx.step(every)
            for S, f in zip(self.systems, fields):
                self.ctx.check(self.ctx.lib.dsmc_field_accumulate(self.ctx.handle, S.id, C.c_void_p(f.data_ptr()), 1))
            samples += 1
            if samples % 64 == 0:  # fp32 partial sums folded into fp64 on the host
                self.ctx.sync()    # the sums are written on the context's stream
                for a, f in zip(acc, fields):
                    a += f.cpu().numpy()
                    f.zero_()
                torch.cuda.synchronize()  # zeroed before the next sums
        self.ctx.sync()
        for a, f in zip(acc, fields):
            a += f.cpu().numpy()
        self.samples = samples
        return acc

    def ctx_device(self) -> int:
        """The context's GPU (the CUDA current device may belong to another
        context by now)."""
        return self.ctx.device

    def close(self):
        self.ctx.close()


def finish_field(sums: np.ndarray, solid: np.ndarray) -> np.ndarray:
    """(V, 4) sums -> (V, 4): density / mean density over empty voxels, and
    the mean drift in VELOCITY_SCALE units (0 where no particle was seen)."""
    cnt = sums[:, 0]
    empty = solid.ravel() == 0
    mean = cnt[empty].mean() if empty.any() else 1.0
    out = np.zeros_like(sums)
    out[:, 0] = np.where(empty, cnt / max(mean, 1e-30), 0.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        for d in range(3):
            out[:, 1 + d] = np.where(cnt > 0, sums[:, 1 + d] / np.maximum(cnt, 1) / VELOCITY_SCALE, 0.0)
    return out


def _seed_arrays(field_out: np.ndarray, solid: np.ndarray, uniform_density: bool = False,
                 zero_drift: bool = False):
    empty = solid.ravel() == 0
    dens = np.ones(len(empty)) if uniform_density else np.maximum(field_out[:, 0], 0.0)
    w = np.ascontiguousarray(np.where(empty, dens, 0.0), np.float32)
    if zero_drift:
        drift = np.zeros((len(empty), 3), np.float32)
    else:
        drift = np.ascontiguousarray(field_out[:, 1:4] * VELOCITY_SCALE, np.float32)
    return w, drift


def warm_start_many(ctx: Context, systems, field_outs, solids, counts, uniform_density: bool = False,
                    group: int = 64, zero_drift: bool = False) -> None:
    """warm_start for many systems of one context, `group` systems per
    dsmc_particles_init_field_many call (each call re-lays the context out
    once).  uniform_density: seed uniformly over the empty voxels (the cold
    start's density) with the fields' drift; zero_drift: seed the fields'
    density at rest (a Maxwellian without drift, as the cold start)."""
    for g0 in range(0, len(systems), group):
        sl = slice(g0, g0 + group)
        arrs = [_seed_arrays(f, so, uniform_density, zero_drift) for f, so in zip(field_outs[sl], solids[sl])]
        k = len(arrs)
        ids = (C.c_int * k)(*[S.id for S in systems[sl]])
        n = (C.c_int64 * k)(*[int(c) for c in counts[sl]])
        w = (C.c_void_p * k)(*[a[0].ctypes.data for a in arrs])
        d = (C.c_void_p * k)(*[a[1].ctypes.data for a in arrs])
        ctx.check(ctx.lib.dsmc_particles_init_field_many(ctx.handle, k, ids, n, w, d, 0))
        del arrs


def warm_start(system: System, field_out: np.ndarray, solid: np.ndarray, n: int = -1) -> None:
    """Seeds the system's particles from a predicted field (V, 4) as
    finish_field writes it: density weights and drift * VELOCITY_SCALE."""
    w, drift = _seed_arrays(field_out, solid)
    ctx = system.ctx
    ctx.check(ctx.lib.dsmc_particles_init_field(ctx.handle, system.id, n, w.ctypes.data, drift.ctypes.data, 0))
