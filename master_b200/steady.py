"""Steps to steady state of the x mass flux, and the ensembles that measure it.

The reference reports the number flow rate as a cumulative mean since the
start of its sampling (MeasureNumberFlowRate::update,
dsmc/statisticalproperty.cpp:87-101: F_N * count_periodic[flow] / (t - t0)),
which cannot show when a run becomes steady.  The windowed flux here
differences the same crossing tally (MoleculeMover::count_periodic,
dsmc/moleculemover.h:29-38) over a sliding window instead:

    F_W(t) = F_N * (count(t + W) - count(t)) / (W * dt)

and a run is steady from step t0 when F_W(t) stays within `tol` of the
steady value for every window start t in [t0, t0 + hold].  One replica's
1000-step window is far too noisy for a 2 % criterion (the net crossings of
a few 1e5 particles in a weak flow), so every quantity here is the mean over
an ensemble of independent replicas advanced together in one context, and
its standard error comes with it.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def windowed_flux(counts: np.ndarray, every: int, window: int, weight: float, dt: float) -> np.ndarray:
    """counts: cumulative crossings sampled every `every` steps, shape
    (samples, replicas) with counts[0] at step 0.  Returns F_W at every
    sampled window start, shape (samples - window/every, replicas)."""
    assert window % every == 0
    k = window // every
    c = np.asarray(counts, np.float64)
    return weight * (c[k:] - c[:-k]) / (window * dt)


@dataclass
class Steady:
    steps: int | None        # first window start from which the flux stays within tol (None: never)
    value: float             # the steady value it was compared against
    series: np.ndarray       # ensemble-mean windowed flux per sampled window start
    stderr: np.ndarray       # its standard error over the replicas
    every: int


def steps_to_steady(counts: np.ndarray, every: int, steady_value: float, weight: float, dt: float,
                    window: int = 1000, hold: int = 1000, tol: float = 0.02) -> Steady:
    """The first step t0 (a multiple of `every`) such that the ensemble-mean
    windowed flux over [t, t + window) lies within tol * |steady_value| of
    steady_value for every sampled t in [t0, t0 + hold]."""
    f = windowed_flux(counts, every, window, weight, dt)
    mean = f.mean(axis=1)
    se = f.std(axis=1, ddof=1) / np.sqrt(f.shape[1]) if f.shape[1] > 1 else np.zeros_like(mean)
    ok = np.abs(mean - steady_value) <= tol * abs(steady_value)
    return Steady(first_steady(ok, every, hold), steady_value, mean, se, every)


def first_steady(ok: np.ndarray, every: int, hold: int) -> int | None:
    """The first sampled step t0 with ok[t] for every sampled t in [t0, t0 + hold]."""
    h = hold // every
    for i in range(0, len(ok) - h):
        if ok[i:i + h + 1].all():
            return i * every
    return None


@dataclass
class TotalSteady:
    steps: int | None        # steps to steady of the total (None: never within the record)
    total: np.ndarray        # the systems' summed windowed flux over their summed steady flux
    noise: float             # median standard error of `total` per window start


def total_steps_to_steady(counts: np.ndarray, every: int, weights: np.ndarray, steady_values: np.ndarray,
                          dt: float, window: int = 1000, hold: int = 1000, tol: float = 0.02) -> TotalSteady:
    """Steps to steady of an ensemble of different systems (one geometry
    each): the summed windowed flux sum_j F_W,j(t), normalised by the summed
    steady flux sum_j s_j, must stay within `tol` of 1.  weights: F_N of
    each system.  The systems' windowed fluxes are independent, so the
    variance of the total is the sum of theirs, estimated from the spread of
    F_W,j / s_j over the systems."""
    f = windowed_flux(counts, every, window, 1.0, dt) * np.asarray(weights, np.float64)
    sv = np.asarray(steady_values, np.float64)
    tot = f.sum(axis=1) / sv.sum()
    fn = f / sv
    se = np.sqrt(((fn - fn.mean(axis=1, keepdims=True)) ** 2).sum(axis=1)) / f.shape[1]
    return TotalSteady(first_steady(np.abs(tot - 1.0) <= tol, every, hold), tot, float(np.median(se)))


def steady_flux(counts: np.ndarray, every: int, start: int, weight: float, dt: float):
    """Mean flux of each replica from step `start` to the end of the record
    and the ensemble mean with its standard error: (mean, stderr, per_replica)."""
    c = np.asarray(counts, np.float64)
    i0 = start // every
    steps = (c.shape[0] - 1 - i0) * every
    per = weight * (c[-1] - c[i0]) / (steps * dt)
    se = per.std(ddof=1) / np.sqrt(len(per)) if len(per) > 1 else 0.0
    return float(per.mean()), float(se), per


def run_counts(ctx, systems, steps: int, every: int, axis: int = 0) -> np.ndarray:
    """Advances every system of the context `steps` steps and records each
    system's cumulative crossing count along `axis` every `every` steps
    (row 0: before the first step).  Reads the raw device counters only."""
    import ctypes as C
    out = np.zeros((steps // every + 1, len(systems)), np.int64)
    buf = (C.c_int64 * 8)()

    def read(row):
        for j, S in enumerate(systems):
            ctx.check(ctx.lib.dsmc_counters_get(ctx.handle, S.id, buf))
            out[row, j] = buf[4 + axis]
    read(0)
    for k in range(1, steps // every + 1):
        ctx.step(every)
        read(k)
    return out
