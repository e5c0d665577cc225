"""The synthetic porous-media workloads the timestep is measured and checked on.

Geometries come from the reference's own packed-sphere generator semantics
(ComplexGeometry::create_packed_spheres, dsmc/complexgeometry.cpp:401-513):
solid spheres placed uniformly in the first octant until the octant porosity
drops below the target, mirrored into all eight octants, normals averaged
over a 3^3 window.  Gas: hard-sphere argon, reduced units of
dsmc/unitconverter.cpp:3-21.

  packed_64  - 64^3 voxels of 0.1 um, spheres of r = 4 voxels to porosity 0.6,
               cells of 2^3 voxels, n = 2.5e24 m^-3, F_N = 1000
               (~20 simulators per active cell, 3.9e5 particles), dt = 1e-11 s,
               g = 1e9 m/s^2 along x, walls at 300 K.
  packed_256 - 256^3 voxels of 0.1 um, r = 6 voxels, porosity 0.5, cells of
               2^3 voxels, 30 simulators per cell volume (F_N = n V_cell / 30),
               ~3.1e7 particles, same gas, dt and g.
"""
from __future__ import annotations

from dataclasses import dataclass

from .system import Geometry, Settings, acceleration_from_si, time_from_si

ARGON_MASS_AMU = 6.63e-26 / 1.66053886e-27   # 6.63e-26 kg
ARGON_DIAM_UM = 3.66e-4                       # 3.66e-10 m


@dataclass
class Workload:
    name: str
    n: int                   # voxels per axis
    radius_voxels: float
    porosity: float
    geometry_seed: int
    cells: int               # cells per axis
    atoms_per_molecule: int
    voxel_um: float = 0.1
    density_si: float = 2.5e24
    temperature: float = 300.0
    dt_si: float = 1e-11
    gravity_si: float = 1e9
    flow_direction: int = 0

    def settings(self, rng_seed: int = 1, statistics_interval: int = 100, sample_begin: int = 0) -> Settings:
        s = Settings()
        s.Lx = s.Ly = s.Lz = self.n * self.voxel_um
        s.cells_x = s.cells_y = s.cells_z = self.cells
        s.mass = ARGON_MASS_AMU
        s.diam = ARGON_DIAM_UM
        s.density = self.density_si
        s.temperature = self.temperature
        s.wall_temperature = self.temperature
        s.dt = time_from_si(self.dt_si)
        s.gravity = acceleration_from_si(self.gravity_si)
        s.flow_direction = self.flow_direction
        s.atoms_per_molecule = self.atoms_per_molecule
        s.max_molecules_per_node = 2 ** 31 - 1
        s.statistics_interval = statistics_interval
        s.sample_begin = sample_begin
        s.sampling_bins = self.cells
        s.seed = self.geometry_seed
        s.rng_seed = rng_seed
        return s

    def geometry(self, gpu: bool = False) -> Geometry:
        return Geometry.packed_spheres(self.n, self.radius_voxels, wanted_porosity=self.porosity,
                                       seed=self.geometry_seed)


def simulators_per_cell_weight(density_si: float, voxel_um: float, voxels_per_cell: int, per_cell: float) -> int:
    """F_N giving `per_cell` simulators in a fully open cell (an int, as the reference's)."""
    cell_volume_um3 = (voxels_per_cell * voxel_um) ** 3
    return int(density_si * 1e-18 * cell_volume_um3 / per_cell)


PACKED_64 = Workload("packed_64", n=64, radius_voxels=4, porosity=0.6, geometry_seed=1, cells=32,
                     atoms_per_molecule=1000)
PACKED_256 = Workload("packed_256", n=256, radius_voxels=6, porosity=0.5, geometry_seed=1, cells=128,
                      atoms_per_molecule=simulators_per_cell_weight(2.5e24, 0.1, 2, 30))
# The CPU reference's bounded sample of packed_256: the same voxel size,
# sphere radius, porosity, gas and simulator weight in a 64^3 box.
PACKED_256_SAMPLE = Workload("packed_256_sample64", n=64, radius_voxels=6, porosity=0.5, geometry_seed=1, cells=32,
                             atoms_per_molecule=simulators_per_cell_weight(2.5e24, 0.1, 2, 30))

# packed_256 at 1/8 the volume (128^3 voxels, ~3.9e6 particles, ~0.5 GB of
# particle slots): above the 126 MB L2, small enough for full ncu captures.
PACKED_128 = Workload("packed_128", n=128, radius_voxels=6, porosity=0.5, geometry_seed=1, cells=64,
                      atoms_per_molecule=simulators_per_cell_weight(2.5e24, 0.1, 2, 30))

WORKLOADS = {w.name: w for w in (PACKED_64, PACKED_128, PACKED_256, PACKED_256_SAMPLE)}
