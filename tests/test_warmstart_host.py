"""Host side of the warm start, without a GPU: per-voxel sums finished into
the surrogate's fields (density relative to the empty-voxel mean, drift in
VELOCITY_SCALE units), the seeding arrays handed to
dsmc_particles_init_field(_many), the per-geometry fallback to the cold
start (System::setup_molecules, dsmc/system.cpp:398-430), and the held-out
error summary whose field error decides that fallback."""
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


def test_held_out_summary_and_the_fallback_criterion():
    """train_surrogate.summarize: relative L2 errors over empty voxels, the
    targets' sampling noise from their two halves, and the field error the
    fallback reads: the flux error with that noise taken out in quadrature."""
    from master_b200 import train_surrogate as ts
    rng = np.random.default_rng(3)
    n, V = 4, 64
    solid = (rng.random((n, V)) < 0.3).astype(np.uint8)
    truth = np.zeros((n, V, 4))
    truth[..., 0] = 1.0 + 0.1 * rng.standard_normal((n, V))
    truth[..., 1] = 2.0 + 0.5 * rng.standard_normal((n, V))
    noise = 0.05 * rng.standard_normal((n, 2, V, 4))
    halves = truth[:, None] + noise
    target = halves.mean(axis=1)
    # a prediction equal to the target: no error, field error 0
    s, res = ts.summarize(target.copy(), solid, target, halves)
    assert s["density_rel_l2"] == 0 and s["drift_x_rel_l2"] == 0 and s["field_error"] == 0
    # noise estimate: half the difference of the halves
    m = solid[0] == 0
    d = halves[0, 0, m, 1] - halves[0, 1, m, 1]
    assert res["noise_drift_x_rel_l2"][0] == pytest.approx(0.5 * np.linalg.norm(d) / np.linalg.norm(halves[0, 1, m, 1]))
    # a prediction whose flux is 10 % high everywhere: the raw flux error is
    # 10 %, and the field error is that with the noise taken out in quadrature
    pred = target.copy()
    pred[..., 1] *= 1.1
    s, res = ts.summarize(pred, solid, target, halves)
    assert s["field_error_raw"] == pytest.approx(0.1, rel=1e-9)
    assert s["field_error"] == pytest.approx(np.sqrt(0.1 ** 2 - s["flux_target_noise"] ** 2), rel=1e-9)
    assert s["field_error"] < s["field_error_raw"]
    assert s["flux_rel_err_median"] == pytest.approx(0.1, rel=1e-9)
    # solid voxels do not count: a wild value there changes nothing
    pred2 = pred.copy()
    pred2[solid == 1] = 1e6
    assert ts.summarize(pred2, solid, target, halves)[0] == s


def test_density_only_seeding_has_no_drift():
    """zero_drift: the field's density at rest, the control that leaves the
    drift channel out."""
    sums, solid = sums_and_solid()
    out = fields.finish_field(sums, solid)
    w, drift = fields._seed_arrays(out, solid, zero_drift=True)
    w_field, _ = fields._seed_arrays(out, solid)
    np.testing.assert_array_equal(w, w_field)
    assert drift.dtype == np.float32 and drift.shape == (len(solid), 3) and not drift.any()
