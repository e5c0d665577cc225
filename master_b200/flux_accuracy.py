"""Long-run accuracy of the split-precision production pass: its x mass flux
against the fp64 path's on the same workload.

    python -m master_b200.flux_accuracy --workload packed_64 --replicas 256 --steps 16000 --out DIR

The fp64 path reproduces the reference's own routines operation by operation
(positions bit-identical, velocities within 1e-12, every integer index and
counter identical), so it is the yardstick at sizes the reference cannot run.
Both precisions run the same `replicas` draw seeds as systems of one context
each; the flux of each replica is its crossing count over [from, steps]
(MoleculeMover::count_periodic, dsmc/moleculemover.h:29-38) times F_N over
the elapsed time (MeasureNumberFlowRate::update,
dsmc/statisticalproperty.cpp:87-101).  After the first ~1000 steps the two
precisions' trajectories are uncorrelated (a rounding that moves one
particle across a cell face changes its cell's collision partners), so the
two ensemble means are compared as independent samples:
  rel_diff = (split - fp64) / fp64, with a 95 % interval 1.96 * se_rel.
The split precision is held to |rel_diff| within 2 % with that interval inside 2 %.
Collision rates and temperatures are compared the same way.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import capi, steady, workloads
from .system import Context, System


def run(workload, precision, replicas: int, steps: int, every: int, seed0: int = 1):
    g = workload.geometry()
    ctx = Context(0, precision)
    systems = [System(workload.settings(rng_seed=seed0 + i, statistics_interval=10 ** 9), g, context=ctx)
               for i in range(replicas)]
    t0 = time.perf_counter()
    counts = steady.run_counts(ctx, systems, steps, every)
    ctx.sync()
    secs = time.perf_counter() - t0
    tal = [S.tallies() for S in systems]
    out = {"counts": counts, "seconds": secs, "particles": sum(S.num_molecules for S in systems),
           "collisions": np.array([t.collisions for t in tal], np.float64),
           "temperature": np.array([t.temperature for t in tal], np.float64),
           "error_bits": ctx.device_status()[0], "settings": systems[0].settings}
    ctx.close()
    return out


def compare(workload, replicas: int, steps: int, start: int, every: int = 100) -> dict:
    res = {"workload": workload.name, "replicas": replicas, "steps": steps, "from": start, "every": every}
    runs = {}
    for name, prec in (("split", capi.PREC_SPLIT32), ("fp64", capi.PREC_FP64)):
        runs[name] = run(workload, prec, replicas, steps, every)
        r = runs[name]
        s = r["settings"]
        m, se, per = steady.steady_flux(r["counts"], every, start, s.atoms_per_molecule, s.dt)
        res[name] = {"flux_mean": m, "flux_se": se, "seconds": r["seconds"], "particles": r["particles"],
                     "particle_steps_per_s": r["particles"] * steps / r["seconds"],
                     "collisions_mean": float(r["collisions"].mean()),
                     "collisions_se": float(r["collisions"].std(ddof=1) / np.sqrt(replicas)),
                     "temperature_mean": float(r["temperature"].mean()),
                     "temperature_se": float(r["temperature"].std(ddof=1) / np.sqrt(replicas)),
                     "error_bits": r["error_bits"]}
    a, b = res["split"], res["fp64"]
    rel = (a["flux_mean"] - b["flux_mean"]) / b["flux_mean"]
    se_rel = np.hypot(a["flux_se"], b["flux_se"]) / abs(b["flux_mean"])
    res["flux_rel_diff"] = rel
    res["flux_rel_ci95"] = 1.96 * se_rel
    res["flux_within_2pct"] = bool(abs(rel) + 1.96 * se_rel <= 0.02)
    res["flux_consistent_with_2pct"] = bool(abs(rel) <= 0.02 + 1.96 * se_rel)
    res["collisions_rel_diff"] = (a["collisions_mean"] - b["collisions_mean"]) / b["collisions_mean"]
    res["collisions_rel_ci95"] = 1.96 * np.hypot(a["collisions_se"], b["collisions_se"]) / b["collisions_mean"]
    res["temperature_diff_K"] = a["temperature_mean"] - b["temperature_mean"]
    res["temperature_ci95_K"] = 1.96 * np.hypot(a["temperature_se"], b["temperature_se"])
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="packed_64")
    ap.add_argument("--replicas", type=int, default=256)
    ap.add_argument("--steps", type=int, default=16000)
    ap.add_argument("--from", dest="start", type=int, default=1000)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    res = compare(workloads.WORKLOADS[a.workload], a.replicas, a.steps, a.start)
    text = json.dumps(res, indent=1, default=float)
    if a.out:
        Path(a.out).mkdir(parents=True, exist_ok=True)
        (Path(a.out) / "flux_accuracy.json").write_text(text)
    print(text)


if __name__ == "__main__":
    main()
