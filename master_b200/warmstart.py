"""Warm-started production runs against cold starts: steps and wall time
until the x mass flux is steady.

For a set of unseen packed-sphere geometries the surrogate (a trained
surrogate.UNet) predicts each one's steady density and drift from its solid
mask and Knudsen number; `dsmc_particles_init_field_many` seeds the particles
of every geometry from the local drifting Maxwellian of its field.  The cold start is the
reference's own (System::setup_molecules, dsmc/system.cpp:398-430: uniform in
the empty voxels, Maxwellian at rest).  Both ensembles hold the same
geometries, particle counts and draw seeds as systems of one context each,
and run the split-precision production pass.

Steady value: each geometry's mean flux over the second half of its cold run
(the plain method's own steady state).  The geometries' windowed fluxes
(steady.windowed_flux) are summed and normalised by the sum of their steady
values, which divides the sampling noise of one geometry's flux by about
the square root of their number; steps to steady is
steady.total_steps_to_steady of that normalised total against 1.

Fallback: when the surrogate's held-out field error (train_surrogate's
"field_error", the relative error of the predicted mean x flux over the
held-out geometries) exceeds `max_field_error` (10 %), or a prediction is not
finite, that geometry starts cold.
"""
from __future__ import annotations

import json
import time

import numpy as np

from . import fields, steady


def predict_fields(net, specs, geoms):
    """The surrogate's output (V, 4) for each geometry (edge a power of two)."""
    import torch
    dev = net.dev
    out = []
    for sp, g in zip(specs, geoms):
        solid = torch.tensor((g.voxels > 0).astype(np.uint8), device=dev).reshape(1, sp.n, sp.n, sp.n)
        feat = torch.tensor([np.log10(sp.knudsen)], dtype=torch.float32, device=dev)
        o = net.forward(solid, feat)
        out.append(o.detach().cpu().numpy().reshape(-1, 4).astype(np.float64))
    torch.cuda.synchronize(dev)
    return out


def seedable(pred, solid, uniform_density: bool = False) -> bool:
    """Whether a predicted field (V, 4) can seed its geometry: present, finite
    everywhere, and (unless the density is taken uniform) with positive
    density in some empty voxel of `solid` (V,).  Otherwise the geometry
    starts cold."""
    if pred is None or not np.isfinite(pred).all():
        return False
    return uniform_density or float(np.maximum(pred[solid == 0, 0], 0).sum()) > 0


def compare(net, specs, steps: int, every: int = 10, window: int = 1000, hold: int = 1000, tol: float = 0.02,
            field_error: float = 0.0, max_field_error: float = 0.10, device: int = 0, rng_seed: int = 500,
            capacity: tuple | None = None, force: bool = False, measured: tuple | None = None,
            uniform_density: bool = False, zero_drift: bool = False, log=print) -> dict:
    """Runs the cold ensemble, then the warm one (one context at a time, so
    the two never share the device memory), `steps` steps each, and returns
    the steps and wall time to steady of both.  uniform_density: seed the
    particles uniformly over the empty voxels, as the cold start does, with
    the predicted drift (the density channel left out); zero_drift: seed the
    predicted density at rest (the drift channel left out).  With
    `measured`, the same two switches seed one channel of the DSMC's own
    steady fields alone."""
    import torch
    rep = {"geometries": len(specs), "steps": steps, "every": every, "window": window, "hold": hold, "tol": tol,
           "surrogate_field_error": field_error, "max_field_error": max_field_error,
           "specs": [{"n": sp.n, "porosity": sp.porosity, "radius_voxels": sp.radius_voxels, "knudsen": sp.knudsen,
                      "seed": sp.seed} for sp in specs]}
    t0 = time.perf_counter()
    geoms = [sp.geometry() for sp in specs]
    rep["geometry_s"] = time.perf_counter() - t0
    out = {}
    # cold: the reference's start
    t0 = time.perf_counter()
    cold = fields.Ensemble(specs, device=device, rng_seed=rng_seed, cold=True, geoms=geoms, capacity=capacity)
    rep["cold_setup_s"] = time.perf_counter() - t0
    counts_n = [S.num_molecules for S in cold.systems]
    weights = np.array([s.atoms_per_molecule for s in cold.settings], np.float64)
    dt = cold.settings[0].dt
    t0 = time.perf_counter()
    c = steady.run_counts(cold.ctx, cold.systems, steps, every)
    cold.ctx.sync()
    out["cold"] = {"counts": c, "seconds": time.perf_counter() - t0, "error_bits": cold.ctx.device_status()[0]}
    cold.close()
    log("cold", out["cold"]["seconds"], "s")
    # warm: same geometries, seeds and particle counts, seeded from the surrogate
    warm = fields.Ensemble(specs, device=device, rng_seed=rng_seed, cold=False, geoms=geoms, capacity=capacity)
    use_net = force or field_error <= max_field_error
    rep["forced"] = bool(force and field_error > max_field_error)
    t0 = time.perf_counter()
    if measured is not None:
        # control: seed from the steady fields measured by the DSMC itself (a
        # separate cold ensemble, other seeds: `measured` = (transient steps,
        # sampling steps)) instead of the network's prediction
        warm.close()
        ref = fields.Ensemble(specs, device=device, rng_seed=rng_seed + 100000, cold=True, geoms=geoms,
                              capacity=capacity)
        ref.ctx.step(measured[0])
        sums = ref.accumulate_fields(measured[1], 20)
        ref.close()
        preds = [fields.finish_field(sm, (g.voxels > 0).astype(np.uint8).ravel()) for sm, g in zip(sums, geoms)]
        rep["seeded_from"] = f"DSMC-measured fields ({measured[0]} + {measured[1]} steps)"
        warm = fields.Ensemble(specs, device=device, rng_seed=rng_seed, cold=False, geoms=geoms, capacity=capacity)
    else:
        preds = predict_fields(net, specs, geoms) if use_net else [None] * len(specs)
        rep["seeded_from"] = "surrogate" if use_net else "cold (fallback)"
    torch.cuda.synchronize()
    rep["inference_s"] = time.perf_counter() - t0
    fallback, seeded = [], []
    t0 = time.perf_counter()
    solids = [(g.voxels > 0).astype(np.uint8).ravel() for g in geoms]
    for i, (p, solid) in enumerate(zip(preds, solids)):
        (seeded if seedable(p, solid, uniform_density) else fallback).append(i)
    fields.warm_start_many(warm.ctx, [warm.systems[i] for i in seeded], [preds[i] for i in seeded],
                           [solids[i] for i in seeded], [counts_n[i] for i in seeded], uniform_density=uniform_density,
                           zero_drift=zero_drift)
    warm.init_cold([warm.systems[i] for i in fallback], [counts_n[i] for i in fallback])
    rep["seed_s"] = time.perf_counter() - t0
    rep["density"] = "uniform" if uniform_density else "field"
    rep["drift"] = "zero" if zero_drift else "field"
    rep["fallback"] = fallback
    if preds[0] is not None:
        rep["predicted_mean_drift_x"] = [float(p[(g.voxels.ravel() == 0), 1].mean()) for p, g in zip(preds, geoms)]
    del preds
    t0 = time.perf_counter()
    c = steady.run_counts(warm.ctx, warm.systems, steps, every)
    warm.ctx.sync()
    out["warm"] = {"counts": c, "seconds": time.perf_counter() - t0, "error_bits": warm.ctx.device_status()[0]}
    warm.close()
    log("warm", out["warm"]["seconds"], "s")
    # steady value of each geometry: its cold run's second half
    cc = out["cold"]["counts"].astype(np.float64)
    i0 = (steps // 2) // every
    steady_val = weights * (cc[-1] - cc[i0]) / ((steps - i0 * every) * dt)
    rep["steady_flux"] = steady_val.tolist()
    res = {}
    for name in ("cold", "warm"):
        c = out[name]["counts"].astype(np.float64)
        # the ensemble's total flux over its total steady flux
        r = steady.total_steps_to_steady(c, every, weights, steady_val, dt, window, hold, tol)
        first = r.steps
        ms_step = 1e3 * out[name]["seconds"] / steps
        # short windows resolve the transient itself
        f100 = steady.windowed_flux(c, every, 100, 1.0, dt) * weights
        res[name] = {"steps_to_steady": first, "ms_per_step": ms_step,
                     "wall_s_to_steady": None if first is None else first * ms_step / 1e3,
                     "flux_over_steady_window": r.total[::max(1, 100 // every)].tolist(),
                     "flux_over_steady_100step": (f100.sum(axis=1) / steady_val.sum())[::max(1, 100 // every)].tolist(),
                     "window_noise": r.noise,
                     "error_bits": out[name]["error_bits"]}
    if res["warm"]["wall_s_to_steady"] is not None:
        res["warm"]["wall_s_to_steady"] += rep["inference_s"] + rep["seed_s"]
    c_, w_ = res["cold"]["steps_to_steady"], res["warm"]["steps_to_steady"]
    rep["ratio_steps"] = (c_ / max(w_, every)) if (c_ is not None and w_ is not None) else None
    rep.update(res)
    rep["particles"] = int(sum(counts_n))
    return rep


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="cold against surrogate-warm-started ensembles: steps to steady flux")
    ap.add_argument("--weights", required=True, help="surrogate.npz from master_b200.train_surrogate")
    ap.add_argument("--geometries", type=int, default=16)
    ap.add_argument("--edge", type=int, default=256)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--per-cell", type=float, default=30.0)
    ap.add_argument("--knudsen", type=float, nargs=2, default=(0.3, 3.0))
    ap.add_argument("--capacity", type=float, nargs=2, default=None, metavar=("FACTOR", "PAD"))
    ap.add_argument("--force", action="store_true",
                    help="seed from the surrogate even when its field error is above the fallback threshold")
    ap.add_argument("--measured", type=int, nargs=2, default=None, metavar=("TRANSIENT", "SAMPLING"),
                    help="control: seed from fields the DSMC measures itself instead of the network's")
    ap.add_argument("--density", choices=("field", "uniform"), default="field",
                    help="seed density: the field's, or uniform over the empty voxels with the field's drift")
    ap.add_argument("--drift", choices=("field", "zero"), default="field",
                    help="seed drift: the field's, or none (the field's density at rest)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    net, held = load_net(a.weights)
    specs = fields.random_specs(a.geometries, a.edge, seed=5, porosity=(0.45, 0.75), knudsen=tuple(a.knudsen),
                                per_cell=a.per_cell)
    rep = compare(net, specs, a.steps, every=a.every, field_error=float(held.get("field_error", 0.0)),
                  capacity=tuple(a.capacity) if a.capacity else None, force=a.force,
                  measured=tuple(a.measured) if a.measured else None, uniform_density=a.density == "uniform",
                  zero_drift=a.drift == "zero")
    rep["surrogate_held_out"] = held
    if a.out:
        from pathlib import Path
        Path(a.out).mkdir(parents=True, exist_ok=True)
        (Path(a.out) / "warmstart.json").write_text(json.dumps(rep, indent=1, default=float))
    print(json.dumps({k: v for k, v in rep.items() if k in ("ratio_steps", "fallback", "particles", "forced")} |
                     {n: {k: rep[n][k] for k in ("steps_to_steady", "wall_s_to_steady", "ms_per_step",
                                                  "window_noise")} for n in ("cold", "warm")}))


def load_net(path, device: int = 0):
    """A trained surrogate from train_surrogate's surrogate.npz, with its
    held-out field error."""
    from . import surrogate
    z = np.load(path)
    net = surrogate.UNet(device, params=z["params"].astype(np.float32))
    held = json.loads(str(z["held_out"])) if "held_out" in z else {}
    return net, held


if __name__ == "__main__":
    main()
