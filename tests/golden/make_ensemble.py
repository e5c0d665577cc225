"""Generates tests/golden/ensemble_ref.json: the reference solver's own FP64
CPU run (oracle/_ref/dsmc_ref, built from the reference sources by
oracle/Makefile) as an ensemble of independently seeded runs on a small
flowing-gas workload, with the statistics that the GPU timestep must
reproduce within ensemble 95 % confidence intervals
(tests/test_ensemble_gpu.py):

* collisions and wall collisions over the run (Tocontinue, dsmc/main.cpp:110-112),
* the number flow rate and the temperature at the last step
  (statistics/number_flow_rate.txt, temperature.txt: MeasureNumberFlowRate,
  MeasureTemperature, dsmc/statisticalproperty.cpp:57-101),
* the y-binned temperature and v_z profiles over every sample
  (statistics/linear_temperature.txt, velocity.txt: finalize(),
  dsmc/statisticalproperty.cpp:303-371).

Both codes start from a Maxwellian at rest in the empty voxels, so the whole
run, transient included, is compared.

A second, longer ensemble ("flux_window") pins the number flow rate itself:
FLUX_REPLICAS runs of FLUX_STEPS steps sampled every FLUX_INTERVAL steps.
The reference prints the cumulative rate F(t) = F_N count_periodic / t
(MeasureNumberFlowRate::update, dsmc/statisticalproperty.cpp:87-101), so the
rate over the window [FLUX_FROM, FLUX_STEPS], past the transient, is the
difference (F(t2) t2 - F(t1) t1) / (t2 - t1) of two printed values.

    python tests/golden/make_ensemble.py
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from master_b200 import workloads  # noqa: E402
from oracle import run_reference  # noqa: E402

OUT = Path(__file__).resolve().parent / "ensemble_ref.json"

# 32^3 voxels of 0.1 um, spheres of r = 3 voxels to porosity 0.6, cells of
# 2^3 voxels with 20 simulators in an open cell, argon at 300 K, dt = 1e-11 s,
# g = 1e9 m/s^2 along x (the cfg1 physics in a smaller box)
WORKLOAD = workloads.Workload("ensemble_32", n=32, radius_voxels=3, porosity=0.6, geometry_seed=4, cells=16,
                              atoms_per_molecule=workloads.simulators_per_cell_weight(2.5e24, 0.1, 2, 20))
STEPS = 400
INTERVAL = 10
REPLICAS = 16
FLUX_REPLICAS = 128
FLUX_STEPS = 3000
FLUX_INTERVAL = 500
FLUX_FROM = 1000


def summarize(rows):
    a = np.asarray(rows, np.float64)
    return {"mean": a.mean(axis=0).tolist(), "std": a.std(axis=0, ddof=1).tolist(), "n": int(a.shape[0])}


def flux_window(g):
    """Windowed number flow rate of FLUX_REPLICAS long reference runs."""
    s = WORKLOAD.settings(statistics_interval=FLUX_INTERVAL)
    seeds = list(range(1001, 1001 + FLUX_REPLICAS))
    rates = []
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        run_reference.run_replicas(s, g, timesteps=FLUX_STEPS, replicas=FLUX_REPLICAS, seeds=seeds, workdir=d,
                                   timeout=3600, workers=os.cpu_count())
        for i in range(FLUX_REPLICAS):
            rows = [ln.split() for ln in (d / f"r{i:03d}" / "statistics" / "number_flow_rate.txt").read_text()
                    .splitlines() if ln.strip()]
            # one line per sample, at steps FLUX_INTERVAL, 2 FLUX_INTERVAL, ...
            F = {FLUX_INTERVAL * (k + 1): float(r[1]) for k, r in enumerate(rows)}
            t1, t2 = FLUX_FROM, FLUX_STEPS
            rates.append((F[t2] * t2 - F[t1] * t1) / (t2 - t1))
    r = np.asarray(rates)
    return {"replicas": FLUX_REPLICAS, "steps": FLUX_STEPS, "from": FLUX_FROM, "interval": FLUX_INTERVAL,
            "seeds": seeds, "mean": float(r.mean()), "std": float(r.std(ddof=1)), "n": int(r.size)}


def main():
    if not run_reference.available():
        raise SystemExit("build oracle/_ref first: make -C oracle ref REF=<reference project>/code/base_code/program/dsmc")
    s = WORKLOAD.settings(statistics_interval=INTERVAL)
    g = WORKLOAD.geometry()
    stats = {k: [] for k in ("collisions", "wall_collisions", "flux", "temperature_K", "molecules")}
    prof_T, prof_vz = [], []
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        res = run_reference.run_replicas(s, g, timesteps=STEPS, replicas=REPLICAS,
                                         seeds=list(range(101, 101 + REPLICAS)), workdir=d)
        for i, rep in enumerate(res["reports"]):
            rd = d / f"r{i:03d}"
            t, steps, col, walls = (rd / "Tocontinue").read_text().split()
            assert int(steps) == STEPS
            stats["collisions"].append(float(col))
            stats["wall_collisions"].append(float(walls))
            stats["flux"].append(float((rd / "statistics" / "number_flow_rate.txt").read_text().split()[-1]))
            stats["temperature_K"].append(float((rd / "statistics" / "temperature.txt").read_text().split()[-1]))
            stats["molecules"].append(float(rep["molecules"]))
            prof_T.append([float(x) for x in (rd / "statistics" / "linear_temperature.txt").read_text().split()])
            prof_vz.append([float(x) for x in (rd / "statistics" / "velocity.txt").read_text().split()])
    out = {
        "workload": {"name": WORKLOAD.name, "n": WORKLOAD.n, "radius_voxels": WORKLOAD.radius_voxels,
                     "porosity": WORKLOAD.porosity, "geometry_seed": WORKLOAD.geometry_seed,
                     "cells": WORKLOAD.cells, "atoms_per_molecule": WORKLOAD.atoms_per_molecule},
        "steps": STEPS, "statistics_interval": INTERVAL, "seeds": list(range(101, 101 + REPLICAS)),
        "scalars": {k: summarize(v) for k, v in stats.items()},
        "profile_temperature_K": summarize(prof_T),
        "profile_velocity_z": summarize(prof_vz),
    }
    out["flux_window"] = flux_window(g)
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    for k, v in out["scalars"].items():
        print(k, v["mean"], "+-", v["std"])


if __name__ == "__main__":
    main()
