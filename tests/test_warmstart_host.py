"""Host side of the warm start, without a GPU: per-voxel sums finished into
the surrogate's fields (density relative to the empty-voxel mean, drift in
VELOCITY_SCALE units), the seeding arrays handed to
dsmc_particles_init_field(_many), and the per-geometry fallback to the cold
start (System::setup_molecules, dsmc/system.cpp:398-430)."""
from __future__ import annotations

import numpy as np
import pytest

from master_b200 import fields, warmstart
from master_b200.fields import VELOCITY_SCALE


def sums_and_solid():
    solid = np.array([0, 0, 1, 0, 1, 0], np.uint8)
    cnt = np.array([4.0, 2.0, 0.0, 6.0, 0.0, 0.0])
    vel = np.zeros((6, 3))
    vel[0] = [8e-3, 0.0, -4e-3]      # sums of v over the samples' particles
    vel[1] = [-2e-3, 2e-3, 0.0]
    vel[3] = [3e-3, 3e-3, 3e-3]
    return np.column_stack([cnt, vel]), solid


def test_finish_field_normalises_density_and_drift():
    sums, solid = sums_and_solid()
    out = fields.finish_field(sums, solid)
    mean = (4 + 2 + 6 + 0) / 4                 # over the four empty voxels
    np.testing.assert_allclose(out[:, 0], [4 / mean, 2 / mean, 0, 6 / mean, 0, 0])
    # mean drift per voxel in VELOCITY_SCALE units, 0 where no particle was seen
    np.testing.assert_allclose(out[0, 1:], np.array([8e-3, 0, -4e-3]) / 4 / VELOCITY_SCALE)
    np.testing.assert_allclose(out[1, 1:], np.array([-2e-3, 2e-3, 0]) / 2 / VELOCITY_SCALE)
    np.testing.assert_allclose(out[3, 1:], np.full(3, 3e-3 / 6 / VELOCITY_SCALE))
    assert not out[[2, 4, 5], 1:].any()
    assert np.isfinite(out).all()


def test_seed_arrays_zero_solid_weights_and_scale_the_drift():
    sums, solid = sums_and_solid()
    out = fields.finish_field(sums, solid)
    out[2, 0] = 5.0                              # a weight in a solid voxel is dropped
    out[5, 0] = -1.0                             # a negative density counts as zero
    w, drift = fields._seed_arrays(out, solid)
    assert w.dtype == np.float32 and drift.dtype == np.float32 and w.flags.c_contiguous and drift.flags.c_contiguous
    np.testing.assert_allclose(w, np.where(solid == 0, np.maximum(out[:, 0], 0), 0), rtol=1e-7)
    np.testing.assert_allclose(drift, out[:, 1:] * VELOCITY_SCALE, rtol=1e-6)
    wu, drift_u = fields._seed_arrays(out, solid, uniform_density=True)
    np.testing.assert_array_equal(wu, (solid == 0).astype(np.float32))
    np.testing.assert_array_equal(drift_u, drift)


@pytest.mark.parametrize("case,want", [
    ("good", True),
    ("none", False),
    ("nan", False),
    ("inf_drift", False),
    ("no_density", False),
    ("density_only_in_solid", False),
])
def test_fallback_to_the_cold_start(case, want):
    sums, solid = sums_and_solid()
    p = fields.finish_field(sums, solid)
    if case == "none":
        p = None
    elif case == "nan":
        p[1, 0] = np.nan
    elif case == "inf_drift":
        p[3, 2] = np.inf
    elif case == "no_density":
        p[:, 0] = 0.0
    elif case == "density_only_in_solid":
        p[:, 0] = np.where(solid == 1, 1.0, -0.5)
    assert warmstart.seedable(p, solid) is want


def test_uniform_density_needs_only_a_finite_drift():
    sums, solid = sums_and_solid()
    p = fields.finish_field(sums, solid)
    p[:, 0] = 0.0
    assert warmstart.seedable(p, solid, uniform_density=True)
    p[0, 1] = np.nan
    assert not warmstart.seedable(p, solid, uniform_density=True)
