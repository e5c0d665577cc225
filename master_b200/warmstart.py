"""Warm-started production runs against cold starts: steps and wall time
until the x mass flux is steady.

For a set of unseen packed-sphere geometries the surrogate (a trained
surrogate.UNet) predicts each one's steady density and drift from its solid
mask and Knudsen number; `dsmc_particles_init_field` seeds the particles from
the local drifting Maxwellian of that field.  The cold start is the
reference's own (System::setup_molecules, dsmc/system.cpp:398-430: uniform in
the empty voxels, Maxwellian at rest).  Both ensembles hold the same
geometries, particle counts and draw seeds as systems of one context each,
and run the split-precision production pass.

Steady value: each geometry's mean flux over the second half of its cold run
(the plain method's own steady state).  The per-geometry windowed flux
(steady.windowed_flux) is normalised by it and averaged over the geometries,
which divides the sampling noise of one geometry's flux by the square root
of their number; steps to steady is steady.steps_to_steady of that
normalised curve against 1.

Fallback: when the surrogate's held-out field error (train_surrogate's
"field_error", the relative error of the predicted mean x flux over the
held-out geometries) exceeds `max_field_error` (10 %), or a prediction is not
finite, that geometry starts cold.
"""
from __future__ import annotations

import json
import time

import numpy as np

from . import capi, fields, steady


def predict_fields(net, specs, geoms, batch: int = 1):
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


def compare(net, specs, steps: int, every: int = 10, window: int = 1000, hold: int = 1000, tol: float = 0.02,
            field_error: float = 0.0, max_field_error: float = 0.10, device: int = 0, rng_seed: int = 500,
            log=print) -> dict:
    """Runs the cold and warm ensembles `steps` steps each and returns the
    steps and wall time to steady of both."""
    import torch
    rep = {"geometries": len(specs), "steps": steps, "every": every, "window": window, "hold": hold, "tol": tol,
           "surrogate_field_error": field_error, "max_field_error": max_field_error}
    # cold ensemble
    t0 = time.perf_counter()
    cold = fields.Ensemble(specs, device=device, rng_seed=rng_seed, cold=True)
    rep["cold_setup_s"] = time.perf_counter() - t0
    counts_n = [S.num_molecules for S in cold.systems]
    # warm ensemble: same geometries, seeds and particle counts
    warm = fields.Ensemble(specs, device=device, rng_seed=rng_seed, cold=False)
    t0 = time.perf_counter()
    use_net = field_error <= max_field_error
    preds = predict_fields(net, specs, warm.geoms) if use_net else [None] * len(specs)
    torch.cuda.synchronize()
    rep["inference_s"] = time.perf_counter() - t0
    fallback = []
    t0 = time.perf_counter()
    for i, (S, g, p) in enumerate(zip(warm.systems, warm.geoms, preds)):
        solid = (g.voxels > 0).astype(np.uint8).ravel()
        if p is None or not np.isfinite(p).all() or not (np.maximum(p[solid == 0, 0], 0).sum() > 0):
            fallback.append(i)
            S.ctx.check(S.ctx.lib.dsmc_particles_init(S.ctx.handle, S.id, counts_n[i]))
        else:
            fields.warm_start(S, p, solid, n=counts_n[i])
    rep["seed_s"] = time.perf_counter() - t0
    rep["fallback"] = fallback

    out = {}
    for name, ens in (("cold", cold), ("warm", warm)):
        t0 = time.perf_counter()
        c = steady.run_counts(ens.ctx, ens.systems, steps, every)
        ens.ctx.sync()
        out[name] = {"counts": c, "seconds": time.perf_counter() - t0,
                     "error_bits": ens.ctx.device_status()[0]}
        log(name, out[name]["seconds"], "s")
    s0 = cold.settings[0]
    dt = s0.dt
    weights = np.array([s.atoms_per_molecule for s in cold.settings], np.float64)
    cold.close()
    warm.close()
    # steady value of each geometry: its cold run's second half
    cc = out["cold"]["counts"].astype(np.float64)
    i0 = (steps // 2) // every
    steady_val = weights * (cc[-1] - cc[i0]) / ((steps - i0 * every) * dt)
    rep["steady_flux"] = steady_val.tolist()
    res = {}
    for name in ("cold", "warm"):
        c = out[name]["counts"].astype(np.float64)
        f = steady.windowed_flux(c, every, window, 1.0, dt) * weights / steady_val
        mean = f.mean(axis=1)
        se = f.std(axis=1, ddof=1) / np.sqrt(f.shape[1]) if f.shape[1] > 1 else np.zeros_like(mean)
        ok = np.abs(mean - 1.0) <= tol
        h = hold // every
        first = None
        for i in range(0, len(ok) - h):
            if ok[i:i + h + 1].all():
                first = i * every
                break
        ms_step = 1e3 * out[name]["seconds"] / steps
        res[name] = {"steps_to_steady": first, "ms_per_step": ms_step,
                     "wall_s_to_steady": None if first is None else first * ms_step / 1e3,
                     "normalised_flux": mean[::max(1, 100 // every)].tolist(),
                     "stderr_first_window": float(se[0]) if len(se) else None,
                     "stderr_median": float(np.median(se)) if len(se) else None,
                     "error_bits": out[name]["error_bits"]}
    if res["warm"]["wall_s_to_steady"] is not None:
        res["warm"]["wall_s_to_steady"] += (rep["inference_s"] + rep["seed_s"]) / 1.0
    c_, w_ = res["cold"]["steps_to_steady"], res["warm"]["steps_to_steady"]
    rep["ratio_steps"] = (c_ / max(w_, every)) if (c_ is not None and w_ is not None) else None
    rep.update(res)
    rep["particles"] = int(sum(counts_n))
    return rep


def load_net(path, device: int = 0):
    """A trained surrogate from train_surrogate's surrogate.npz, with its
    held-out field error."""
    from . import surrogate
    z = np.load(path)
    net = surrogate.UNet(device, params=z["params"].astype(np.float32))
    held = json.loads(str(z["held_out"])) if "held_out" in z else {}
    return net, held
