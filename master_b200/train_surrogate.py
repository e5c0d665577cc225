"""Trains the warm-start surrogate on steady fields that the DSMC timestep
generates, with the library's own forward and backward kernels.

    python -m master_b200.train_surrogate --out DIR [--train 512 --test 64 ...]

1. Field sets: `--train` and `--test` packed-sphere geometries of edge
   `--edge` (porosity U(0.4, 0.8), radius U(3, 8) voxels, Knudsen log-U(0.1,
   10) through the density), all systems of one context, advanced together
   by the production pass: `--warmup` steps of transient from a cold start,
   then per-voxel sums every `--every` steps over `--steps` steps, in two
   halves whose difference estimates the sampling noise of the targets.
2. Training: Adam (lr `--lr` decayed on a cosine to 5 % of it, batch
   `--batch`) on the weighted squared error, plus FLUX_WEIGHT times the
   squared error of each box's mean x drift (the per-voxel drift targets are
   mostly sampling noise; their mean over a box, the flux, is not),
   over empty voxels of density (relative to the mean) and drift (in units of
   fields.VELOCITY_SCALE); each batch is shifted by a random periodic offset
   (an exact symmetry of the periodic boxes).
3. Held-out error: relative L2 error of the predicted density and x drift
   over the empty voxels of the test geometries, next to the same error of
   the targets' own sampling noise, plus the error of the predicted mean x
   drift (the flux) per geometry.

Writes DIR/surrogate.npz (parameters and the field-set description) and
DIR/surrogate.json (losses, errors, timings).
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import fields, surrogate

CHANNEL_WEIGHT = [1.0, 4.0, 1.0, 1.0]  # density, drift x, y, z
# weight of each sample's mean x drift error (its flux): the per-voxel drift
# targets are mostly sampling noise, their mean over a box is not
FLUX_WEIGHT = 100.0


def generate(specs, warmup: int, steps: int, every: int, device: int = 0, log=print):
    """Steady fields of each spec: (targets (n,V,4), halves (n,2,V,4), solid (n,V), info)."""
    t0 = time.perf_counter()
    ens = fields.Ensemble(specs, device=device)
    t_setup = time.perf_counter() - t0
    N = ens.particles
    t0 = time.perf_counter()
    ens.ctx.step(warmup)
    ens.ctx.sync()
    t_warm = time.perf_counter() - t0
    t0 = time.perf_counter()
    half = steps // 2
    s1 = ens.accumulate_fields(half, every)
    n1 = ens.samples
    s2 = ens.accumulate_fields(steps - half, every)
    t_samp = time.perf_counter() - t0
    err, spill = ens.ctx.device_status()
    solid = np.stack([(g.voxels > 0).astype(np.uint8).ravel() for g in ens.geoms])
    tg, hv = [], []
    for i in range(len(specs)):
        tg.append(fields.finish_field(s1[i] + s2[i], solid[i]))
        hv.append(np.stack([fields.finish_field(s1[i], solid[i]), fields.finish_field(s2[i], solid[i])]))
    info = {"systems": len(specs), "particles": N, "setup_s": t_setup, "warmup_s": t_warm, "sampling_s": t_samp,
            "particle_steps_per_s": N * (warmup + steps) / (t_warm + t_samp), "error_bits": err,
            "samples": n1 + ens.samples}
    ens.close()
    log("fields", json.dumps(info))
    return np.stack(tg).astype(np.float32), np.stack(hv).astype(np.float32), solid, info


def features(specs) -> np.ndarray:
    """Scalar input of each geometry: log10 of its Knudsen number."""
    return np.array([np.log10(sp.knudsen) for sp in specs], np.float32)


def rel_err(pred, tgt, mask):
    m = mask.astype(bool)
    d = pred[m] - tgt[m]
    return float(np.linalg.norm(d) / max(np.linalg.norm(tgt[m]), 1e-30))


def predict(net, solid, feat, edge, batch, device):
    import torch
    dev = torch.device("cuda", device)
    preds = []
    for b0 in range(0, len(solid), batch):
        sl = slice(b0, b0 + batch)
        s = torch.tensor(solid[sl].reshape(-1, edge, edge, edge), device=dev)
        out = net.forward(s, torch.tensor(feat[sl], device=dev))
        preds.append(out.detach().cpu().numpy().reshape(-1, edge ** 3, 4))
    return np.concatenate(preds)


def evaluate(net, solid, feat, target, halves, edge, batch, device):
    pred = predict(net, solid, feat, edge, batch, device)
    summary, res = summarize(pred, solid, target, halves)
    return summary, pred, res


def summarize(pred, solid, target, halves):
    """Held-out errors of predictions pred (n, V, 4) against targets (n, V, 4)
    whose two half-window estimates are halves (n, 2, V, 4), over the empty
    voxels of solid (n, V): per geometry and summarised; "field_error" is
    the warm start's fallback criterion."""
    empty = solid == 0
    res = {"density_rel_l2": [], "drift_x_rel_l2": [], "noise_density_rel_l2": [], "noise_drift_x_rel_l2": [],
           "flux_pred": [], "flux_target": [], "flux_half_diff": []}
    for i in range(len(solid)):
        m = empty[i]
        res["density_rel_l2"].append(rel_err(pred[i, :, 0], target[i, :, 0], m))
        res["drift_x_rel_l2"].append(rel_err(pred[i, :, 1], target[i, :, 1], m))
        # sampling noise of the full-window target: half the difference of the halves
        res["noise_density_rel_l2"].append(0.5 * rel_err(halves[i, 0, :, 0], halves[i, 1, :, 0], m))
        res["noise_drift_x_rel_l2"].append(0.5 * rel_err(halves[i, 0, :, 1], halves[i, 1, :, 1], m))
        # mean x flux (density-weighted drift over the empty voxels)
        res["flux_pred"].append(float((np.maximum(pred[i, m, 0], 0) * pred[i, m, 1]).mean()))
        res["flux_target"].append(float((target[i, m, 0] * target[i, m, 1]).mean()))
        res["flux_half_diff"].append(float((halves[i, 0, m, 0] * halves[i, 0, m, 1]).mean()
                                           - (halves[i, 1, m, 0] * halves[i, 1, m, 1]).mean()))
    fp, ft = np.array(res["flux_pred"]), np.array(res["flux_target"])
    hd = np.array(res["flux_half_diff"])
    summary = {k: float(np.mean(v)) for k, v in res.items() if k.endswith("l2")}
    summary["flux_rel_err_median"] = float(np.median(np.abs(fp - ft) / np.maximum(np.abs(ft), 1e-30)))
    summary["flux_rel_err_mean"] = float(np.mean(np.abs(fp - ft) / np.maximum(np.abs(ft), 1e-30)))
    # field error as the warm start's fallback rule reads it: the relative
    # error of the predicted mean x flux over the held-out geometries, with
    # the targets' own sampling noise (half the difference of the two halves'
    # fluxes, per geometry) taken out in quadrature
    err2 = float(np.sum((fp - ft) ** 2))
    noise2 = float(np.sum((hd / 2) ** 2))
    norm2 = max(float(np.sum(ft ** 2)), 1e-30)
    summary["field_error_raw"] = float(np.sqrt(err2 / norm2))
    summary["flux_target_noise"] = float(np.sqrt(noise2 / norm2))
    summary["field_error"] = float(np.sqrt(max(0.0, err2 - noise2) / norm2))
    return summary, res


def train(net, solid, feat, target, edge, epochs, batch, lr, device, seed=0, lr_min=None, flux_weight=FLUX_WEIGHT,
          log=print):
    import torch
    dev = torch.device("cuda", device)
    n = len(solid)
    S_all = torch.tensor(solid.reshape(n, edge, edge, edge), device=dev)
    T_all = torch.tensor(target.reshape(n, edge, edge, edge, 4), device=dev)
    F_all = torch.tensor(feat, device=dev)
    cw = torch.tensor(CHANNEL_WEIGHT, dtype=torch.float32, device=dev)
    rng = np.random.default_rng(seed)
    hist = []
    t0 = time.perf_counter()
    steps = 0
    total = epochs * (n // batch)
    lr_min = lr * 0.05 if lr_min is None else lr_min
    for ep in range(epochs):
        order = rng.permutation(n)
        net.loss_acc.zero_()
        nb = 0
        for b0 in range(0, n - batch + 1, batch):
            idx = torch.tensor(order[b0:b0 + batch], device=dev)
            sh = [int(x) for x in rng.integers(0, edge, 3)]
            s = torch.roll(S_all[idx], sh, dims=(1, 2, 3))
            t = torch.roll(T_all[idx], sh, dims=(1, 2, 3))
            valid = (s == 0).to(torch.uint8)
            net.forward(s, F_all[idx])
            net.backward(t, valid, cw, flux_weight=flux_weight)
            # cosine decay from lr to lr_min over the run
            net.adam(lr=lr_min + 0.5 * (lr - lr_min) * (1.0 + np.cos(np.pi * steps / max(total, 1))))
            nb += 1
            steps += 1
        torch.cuda.synchronize(dev)
        loss = net.loss_acc.item() / max(nb, 1)
        hist.append(loss)
        if ep % 10 == 0 or ep == epochs - 1:
            log(f"epoch {ep} loss {loss:.5f} ({time.perf_counter() - t0:.1f} s)")
    dt = time.perf_counter() - t0
    return hist, {"seconds": dt, "adam_steps": steps, "ms_per_step": 1e3 * dt / max(steps, 1)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--train", type=int, default=512)
    ap.add_argument("--test", type=int, default=64)
    ap.add_argument("--edge", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=2000)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--per-cell", type=float, default=60.0)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--chunk", type=int, default=128, help="geometries per context while generating")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    import torch
    torch.cuda.set_device(a.device)
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    rep = {"args": vars(a)}

    def gen(specs):
        parts = [generate(specs[i:i + a.chunk], a.warmup, a.steps, a.every, a.device)
                 for i in range(0, len(specs), a.chunk)]
        return (np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts]),
                np.concatenate([p[2] for p in parts]), [p[3] for p in parts])

    tr_specs = fields.random_specs(a.train, a.edge, seed=1, per_cell=a.per_cell)
    te_specs = fields.random_specs(a.test, a.edge, seed=2, per_cell=a.per_cell)
    tr_t, tr_h, tr_s, tr_info = gen(tr_specs)
    te_t, te_h, te_s, te_info = gen(te_specs)
    rep["fields_train"], rep["fields_test"] = tr_info, te_info
    net = surrogate.UNet(a.device, seed=0)
    hist, tinfo = train(net, tr_s, features(tr_specs), tr_t, a.edge, a.epochs, a.batch, a.lr, a.device)
    rep["loss"] = hist
    rep["training"] = tinfo
    rep["surrogate_status"] = net.status()
    summ, pred, per = evaluate(net, te_s, features(te_specs), te_t, te_h, a.edge, a.batch, a.device)
    rep["held_out"] = summ
    rep["held_out_per_geometry"] = per
    rep["train_fit"] = evaluate(net, tr_s[:64], features(tr_specs[:64]), tr_t[:64], tr_h[:64], a.edge, a.batch,
                                a.device)[0]
    np.savez_compressed(out / "surrogate.npz", params=net.parameters_host(),
                        specs=json.dumps([vars(sp) for sp in tr_specs]), channel_weight=np.array(CHANNEL_WEIGHT),
                        velocity_scale=fields.VELOCITY_SCALE, held_out=json.dumps(summ))
    (out / "surrogate.json").write_text(json.dumps(rep, indent=1, default=float))
    print(json.dumps({"held_out": summ, "training": tinfo}))


if __name__ == "__main__":
    main()
