"""Statistical parity with the reference's FP64 CPU solver: an ensemble of
independently seeded runs of the production split-precision pass against
the reference solver's own ensemble on the same workload
(tests/golden/ensemble_ref.json, made by tests/golden/make_ensemble.py from
oracle/_ref/dsmc_ref).  Collisions, wall collisions, the number flow rate,
the temperature and the y-binned temperature and v_z profiles must agree
within ensemble 95 % confidence intervals (the two intervals overlap).  All
replicas run as systems of one context: one launch per stage advances them
all."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from master_b200 import workloads
from master_b200.system import Context, System

pytestmark = pytest.mark.gpu

REF = json.loads((Path(__file__).resolve().parent / "golden" / "ensemble_ref.json").read_text())
Z95 = 1.96


def overlap(mean_a, std_a, n_a, mean_b, std_b, n_b):
    """True where the two means' 95 % confidence intervals overlap."""
    mean_a, std_a, mean_b, std_b = map(np.asarray, (mean_a, std_a, mean_b, std_b))
    return np.abs(mean_a - mean_b) <= Z95 * (std_a / np.sqrt(n_a) + std_b / np.sqrt(n_b))


@pytest.fixture(scope="module")
def ours():
    wl = REF["workload"]
    w = workloads.Workload(wl["name"], n=wl["n"], radius_voxels=wl["radius_voxels"], porosity=wl["porosity"],
                           geometry_seed=wl["geometry_seed"], cells=wl["cells"],
                           atoms_per_molecule=wl["atoms_per_molecule"])
    g = w.geometry()
    ctx = Context(0)
    systems = [System(w.settings(rng_seed=7000 + k, statistics_interval=REF["statistics_interval"]), g, context=ctx)
               for k in range(16)]
    ctx.step(REF["steps"])
    rows = {k: [] for k in ("collisions", "wall_collisions", "flux", "temperature_K", "molecules")}
    prof_T, prof_vz = [], []
    for S in systems:
        t = S.tallies()
        m = S.measures()
        rows["collisions"].append(t.collisions)
        rows["wall_collisions"].append(t.wall_collisions)
        rows["flux"].append(m.number_flow_rate)
        rows["temperature_K"].append(m.temperature_K)
        rows["molecules"].append(S.num_molecules)
        p = S.profiles()
        prof_T.append(p["temperature"])
        prof_vz.append(p["velocity_z"])
        assert t.step == REF["steps"]
    return {k: np.asarray(v, np.float64) for k, v in rows.items()}, np.asarray(prof_T), np.asarray(prof_vz)


def test_same_particle_count(ours):
    rows, _, _ = ours
    assert (rows["molecules"] == REF["scalars"]["molecules"]["mean"]).all()


@pytest.mark.parametrize("key", ["collisions", "wall_collisions", "flux", "temperature_K"])
def test_scalars_within_confidence_intervals(ours, key):
    rows, _, _ = ours
    r = REF["scalars"][key]
    x = rows[key]
    assert overlap(x.mean(), x.std(ddof=1), x.size, r["mean"], r["std"], r["n"]), (key, x.mean(), r["mean"])


@pytest.mark.parametrize("key,idx", [("profile_temperature_K", 1), ("profile_velocity_z", 2)])
def test_profiles_within_confidence_intervals(ours, key, idx):
    prof = ours[idx]
    r = REF[key]
    ok = overlap(prof.mean(0), prof.std(0, ddof=1), prof.shape[0], r["mean"], r["std"], r["n"])
    # independent bins: allow one of sixteen outside its interval by chance
    assert (~ok).sum() <= 1, (key, np.flatnonzero(~ok))


def test_windowed_flux_matches_the_reference_ensemble():
    """The number flow rate past the transient (steps 1000-3000) of 128
    independent runs against the reference solver's own 128 runs
    (tests/golden/ensemble_ref.json "flux_window", differenced from its
    cumulative rate): the two means must agree within a two-sample 95 %
    interval (about 13 % of the flux here), which an x flux off by a sign,
    a factor or a lost crossing tally fails."""
    from master_b200 import steady
    fw = REF["flux_window"]
    wl = REF["workload"]
    w = workloads.Workload(wl["name"], n=wl["n"], radius_voxels=wl["radius_voxels"], porosity=wl["porosity"],
                           geometry_seed=wl["geometry_seed"], cells=wl["cells"],
                           atoms_per_molecule=wl["atoms_per_molecule"])
    g = w.geometry()
    ctx = Context(0)
    systems = [System(w.settings(rng_seed=9000 + k, statistics_interval=10 ** 9), g, context=ctx)
               for k in range(fw["replicas"])]
    counts = steady.run_counts(ctx, systems, fw["steps"], fw["interval"])
    s = systems[0].settings
    i1 = fw["from"] // fw["interval"]
    rate = s.atoms_per_molecule * (counts[-1] - counts[i1]) / ((fw["steps"] - fw["from"]) * s.dt)
    se = np.hypot(rate.std(ddof=1) / np.sqrt(rate.size), fw["std"] / np.sqrt(fw["n"]))
    assert abs(rate.mean() - fw["mean"]) <= Z95 * se, (rate.mean(), fw["mean"], se)
    # and the interval is tight enough to mean something
    assert Z95 * se < 0.2 * abs(fw["mean"])
    ctx.close()
