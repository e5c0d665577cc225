"""Known-answer test of the diffuse wall (ColliderThermal::collide,
dsmc/colliderthermal.cpp:13-46): particles that meet a flat wall leave it
with the flux-weighted Maxwellian of the wall temperature, that is a
Rayleigh-distributed normal speed of scale s = sqrt(T_wall / m) and normal
tangential components of deviation s.  Every particle of the test meets the
wall once in one move; the re-emitted velocities are checked with
Kolmogorov-Smirnov tests in both precisions."""
from __future__ import annotations

import numpy as np
import pytest
from scipy import stats

from master_b200 import capi, workloads
from master_b200.system import Geometry, System

pytestmark = pytest.mark.gpu

T0 = 1.65088e-21 / 1.3806503e-23  # reduced temperature unit (dsmc/unitconverter.cpp)


@pytest.mark.parametrize("precision", [capi.PREC_SPLIT32, capi.PREC_FP64])
def test_diffuse_wall_reemits_the_flux_weighted_maxwellian(precision):
    n, N = 32, 20000
    w = workloads.Workload("wall_kat", n=n, radius_voxels=2, porosity=0.9, geometry_seed=1, cells=16,
                           atoms_per_molecule=1000, gravity_si=0.0)
    s = w.settings()
    s.gravity = 0.0
    s.wall_temperature = 500.0
    solid = np.zeros((n, n, n), np.uint8)
    solid[14:18] = 1  # a wall four voxels thick across the box, faces at x = 14 and x = 18 voxels
    g = Geometry.from_mask(solid)
    vox = s.Lx / n
    rng = np.random.default_rng(5)
    r = np.empty((N, 3))
    r[:, 0] = (13 + 0.99) * vox                       # a hundredth of a voxel short of the face
    r[:, 1:] = rng.uniform(0, s.Ly, size=(N, 2))
    v = np.zeros((N, 3))
    v[:, 0] = 0.05 * vox / s.dt                       # reaches the face in a fifth of the step
    S = System(s, g, precision=precision, init_particles=False)
    S.set_particles(r, v)
    S.accelerate_and_move()
    r1, v1 = S.get_particles()
    assert S.tallies().wall_collisions == N
    scale = np.sqrt((s.wall_temperature / T0) / s.mass)
    assert (v1[:, 0] < 0).all()                       # every particle leaves the wall
    assert (r1[:, 0] < 14 * vox).all()                # on the gas side
    assert stats.kstest(-v1[:, 0] / scale, "rayleigh").pvalue > 1e-3
    for d in (1, 2):
        assert stats.kstest(v1[:, d] / scale, "norm").pvalue > 1e-3
