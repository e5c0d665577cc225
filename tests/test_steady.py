"""Windowed flux and steps-to-steady on synthetic crossing counts (no GPU)."""
from __future__ import annotations

import numpy as np

from master_b200 import steady


def test_windowed_flux_differences_the_cumulative_count():
    every, window = 10, 100
    t = np.arange(0, 1001, every)
    rate = 3.0  # crossings per step
    counts = np.stack([rate * t, 2 * rate * t], 1)
    f = steady.windowed_flux(counts, every, window, weight=5.0, dt=0.5)
    assert f.shape == (len(t) - window // every, 2)
    assert np.allclose(f[:, 0], 5.0 * rate / 0.5) and np.allclose(f[:, 1], 2 * 5.0 * rate / 0.5)


def test_steps_to_steady_of_an_exponential_approach():
    every, window, hold, tau = 10, 1000, 1000, 300.0
    t = np.arange(0, 8001, every, dtype=np.float64)
    # rate(t) = 1 - exp(-t/tau): count = t - tau (1 - exp(-t/tau))
    c = (t - tau * (1 - np.exp(-t / tau)))[:, None].repeat(4, 1)
    r = steady.steps_to_steady(c, every, 1.0, weight=1.0, dt=1.0, window=window, hold=hold, tol=0.02)
    # forward window mean deficit: tau/W * exp(-t0/tau) (1 - exp(-W/tau)) <= 0.02
    expect = tau * np.log(tau / window * (1 - np.exp(-window / tau)) / 0.02)
    assert abs(r.steps - expect) <= every
    # a start already at the steady rate is steady at once
    r2 = steady.steps_to_steady(t[:, None].repeat(4, 1), every, 1.0, 1.0, 1.0, window, hold)
    assert r2.steps == 0
    # never steady within the record
    r3 = steady.steps_to_steady(0.5 * t[:, None].repeat(4, 1), every, 1.0, 1.0, 1.0, window, hold)
    assert r3.steps is None


def test_steady_flux_and_its_error():
    every = 10
    t = np.arange(0, 2001, every, dtype=np.float64)
    rng = np.random.default_rng(0)
    rates = 2.0 + 0.1 * rng.standard_normal(64)
    c = t[:, None] * rates[None, :]
    m, se, per = steady.steady_flux(c, every, 1000, weight=1.0, dt=1.0)
    assert np.allclose(per, rates) and abs(m - rates.mean()) < 1e-12 and se > 0


def test_total_steps_to_steady_of_uneven_systems():
    """The ensemble criterion of the warm start: systems of different
    weight and steady flux, summed, against the summed steady flux."""
    every, window, hold, tau = 10, 1000, 1000, 300.0
    t = np.arange(0, 8001, every, dtype=np.float64)
    rates = np.array([1.0, 3.0, 0.5, 2.0])
    weights = np.array([2.0, 1.0, 4.0, 0.5])
    c = (t - tau * (1 - np.exp(-t / tau)))[:, None] * rates[None, :]
    sv = weights * rates
    r = steady.total_steps_to_steady(c, every, weights, sv, 1.0, window, hold, 0.02)
    # every system approaches its rate on the same exponential, so the
    # normalised total does too: the single-system answer
    expect = tau * np.log(tau / window * (1 - np.exp(-window / tau)) / 0.02)
    assert abs(r.steps - expect) <= every
    assert abs(r.total[-1] - 1.0) < 1e-9 and r.noise < 1e-9
    # a system that never settles holds the total off its steady value
    c2 = c.copy()
    c2[:, 1] *= 1.2
    assert steady.total_steps_to_steady(c2, every, weights, sv, 1.0, window, hold, 0.02).steps is None


def test_total_noise_estimates_the_spread_of_the_total():
    every, window = 10, 1000
    t = np.arange(0, 6001, every)
    rng = np.random.default_rng(1)
    n = 256
    # independent Poisson crossings, 2 per step on average, per system
    c = np.vstack([np.zeros(n), rng.poisson(2.0 * every, (len(t) - 1, n)).cumsum(0)])
    sv = np.full(n, 2.0)
    r = steady.total_steps_to_steady(c, every, np.ones(n), sv, 1.0, window, 1000, 0.02)
    # a window holds 2000 crossings per system: relative sd sqrt(2000)/2000
    # per system, over sqrt(n) for the total
    expect = np.sqrt(2000.0) / 2000.0 / np.sqrt(n)
    assert 0.85 * expect < r.noise < 1.15 * expect
    assert r.steps == 0
