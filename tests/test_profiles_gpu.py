"""The sampler's y-binned profiles and v_x histogram on the GPU
(MeasureCount, MeasureVelocityDistributionPoiseuille,
MeasureTemperatureDistribution, MeasurePressureDistribution,
MeasureVelocityDistribution: dsmc/statisticalproperty.cpp:229-478).

* fp64 path, ten fused steps sampled after every step, against the reference
  sampler run on the reference's own ten steps (golden fixtures): per-bin
  counts and the v_x histogram bit-exact, sums within the state tolerance;
  the finished profiles (v_z, temperature, pressure, bin centres) as well;
* production split-precision pass against a host binning of the sampled
  states, on the sampling cadence; reset and checkpoint carry the sums;
* at a larger size, the profile and the cell moments, two independent
  accumulations of the same samples, agree.
"""
from __future__ import annotations

import numpy as np
import pytest

from master_b200 import capi, workloads
from master_b200.system import System, finish_profiles
from test_parity_gpu import CASES, load_case

pytestmark = pytest.mark.gpu


def host_profile(r, v, L_y, bins, mass, vx_min, vx_bin):
    """MeasureCount & co. on one sampled state (the bin arithmetic of
    dsmc/statisticalproperty.cpp:236, 269, 325, 446-451)."""
    b = np.clip((r[:, 1] * (1.0 / L_y) * bins).astype(np.int64), 0, bins - 1)
    out = np.zeros((4, bins))
    out[0] = np.bincount(b, minlength=bins)
    out[1] = np.bincount(b, weights=v[:, 2], minlength=bins)
    out[2] = np.bincount(b, weights=0.5 * mass * v[:, 2] * v[:, 2], minlength=bins)
    hb = np.trunc((v[:, 0] - vx_min) / vx_bin).astype(np.int64)
    ok = (hb >= 0) & (hb < bins)
    out[3] = np.bincount(hb[ok], minlength=bins)
    return out


def vx_bins(s):
    sd = np.sqrt((s.temperature / T0()) / s.mass)
    return -4 * sd, (4 * sd - (-4 * sd)) / s.sampling_bins


def T0():
    return 1.65088e-21 / 1.3806503e-23


@pytest.mark.parametrize("case", CASES)
def test_fp64_profiles_match_reference_sampler(case):
    z, meta, s, g = load_case(case)
    s.sampling_bins = meta["settings"]["sampling_bins"]
    S = System(s, g, precision=capi.PREC_FP64, init_particles=False)
    S.set_particles(z["r0"], z["v0"])
    S.step(meta["params"]["steps"])
    got = S.profile_sums()
    ref = z["prof_sumsK"]
    assert np.array_equal(got[0], ref[0])  # counts per y bin
    assert np.array_equal(got[3], ref[3])  # v_x histogram
    assert np.allclose(got[1:3], ref[1:3], rtol=1e-9, atol=1e-8)
    fin = S.profiles()
    assert np.allclose(fin["velocity_z"], z["prof_vzK"], rtol=1e-8, atol=1e-6)
    assert np.allclose(fin["temperature"], z["prof_TK"], rtol=1e-9)
    assert np.allclose(fin["pressure"], z["prof_PK"], rtol=1e-9)
    assert np.allclose(fin["vx_center"], z["prof_vx_center"], rtol=1e-12)
    assert np.array_equal(fin["count"], ref[0])


@pytest.mark.parametrize("interval", [1, 3])
def test_split_profiles_match_host_binning(interval):
    z, meta, s, g = load_case("small_dt5")
    s.sampling_bins = 16
    s.statistics_interval = interval
    S = System(s, g, init_particles=False)
    S.set_particles(z["r0"], z["v0"])
    vmin, vbin = vx_bins(s)
    want = np.zeros((4, 16))
    for step in range(1, 8):
        S.step(1)
        r, v = S.get_particles()  # the state the step's sample saw
        if step % interval == 0:
            want += host_profile(r, v, s.Ly, 16, s.mass, vmin, vbin)
    got = S.profile_sums()
    assert np.array_equal(got[0], want[0])
    assert np.array_equal(got[3], want[3])
    assert np.allclose(got[1:3], want[1:3], rtol=1e-12, atol=1e-10)
    assert S.tallies().samples == 7 // interval


def test_reset_and_checkpoint_carry_the_profiles(tmp_path):
    z, meta, s, g = load_case("small_dt1")
    s.sampling_bins = 8
    S = System(s, g, init_particles=False)
    S.set_particles(z["r0"], z["v0"])
    S.step(4)
    before = S.profile_sums()
    assert before[0].sum() == 4 * S.num_molecules
    S.ctx.checkpoint_save(tmp_path / "c.bin")
    S.step(3)
    after = S.profile_sums()
    S.ctx.checkpoint_load(tmp_path / "c.bin")
    assert np.array_equal(S.profile_sums(), before)
    S.step(3)
    assert np.allclose(S.profile_sums(), after, rtol=1e-12, atol=1e-12)
    S.reset_tallies()
    assert not S.profile_sums().any()


def test_profiles_agree_with_cell_moments_at_size():
    """Two accumulations of the same samples: the y-binned sums and the cell
    moments (sum over cells of n and sum v_z)."""
    w = workloads.PACKED_256_SAMPLE
    s = w.settings(statistics_interval=5)
    g = w.geometry()
    S = System(s, g)
    S.step(20)
    p = S.profile_sums()
    m = S.cells()["moments"]
    samples = S.tallies().samples
    assert samples == 4
    assert p[0].sum() == m[:, 0].sum() == samples * S.num_molecules
    assert p[1].sum() == pytest.approx(m[:, 3].sum(), rel=1e-9, abs=1e-6)
    assert p[2].sum() == pytest.approx(0.5 * s.mass * m[:, 6].sum(), rel=1e-9)
    # the histogram over +-4 sigma holds all but the far tails of the Maxwellian
    assert 0.999 * p[0].sum() <= p[3].sum() <= p[0].sum()
    fin = finish_profiles(S.settings, S.info().volume_global, p)
    T = fin["temperature"][fin["count"] > 0]
    assert np.allclose(T, s.temperature / 3, rtol=0.1)  # 2/3 of 1/2 m v_z^2 per particle: T/3


@pytest.mark.parametrize("case", CASES)
def test_fp64_measures_match_reference_sampler(case):
    """Energy, temperature, flow rates, pressure and permeability after ten
    steps against the reference's Measure* current values."""
    z, meta, s, g = load_case(case)
    s.viscosity = meta["settings"].get("viscosity", s.viscosity)
    S = System(s, g, precision=capi.PREC_FP64, init_particles=False)
    S.set_particles(z["r0"], z["v0"])
    S.step(meta["params"]["steps"])
    m = S.measures()
    ref = meta["measures_final"]
    assert m.step == meta["params"]["steps"]
    for k, want in ref.items():
        assert getattr(m, k) == pytest.approx(want, rel=1e-9), k
