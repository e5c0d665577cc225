"""Autotuner of the production pass's launch shape, with a JSON cache.

The production pass is four persistent kernels per step (collide_cells,
move_cells, place_movers, place_walls; sample_cells on sampled steps), each a
grid of resident blocks.  Their shapes are searched on the workload itself:

* blocks per SM of each kernel, from one up to the most that are resident;
  the kernels run one after another, so each is timed alone by the library's
  per-kernel CUDA events (dsmc_ctx_set_timing) while the others keep theirs;
* move_cells' staging ring: the smallest that holds the largest cell, and
  the next larger rings (more staging per warp, fewer resident blocks);
* collide_cells' chunk claims: a fixed stride or a pass-wide counter.

Each candidate runs `steps` production steps `repeats` times and keeps the
median per-kernel time; the choice must also not lose on the whole step
against the default (else the default is kept).  Trials advance the
simulation (they are ordinary timesteps; every shape gives the same
trajectory).  The choice is cached per GPU model, SM count and workload
signature (active cells, particles, the ring needed, rounded to powers of
two) in a JSON file, DSMC_TUNE_CACHE or ~/.cache/dsmc_b200/tuning.json, and
applied to a context whose signature matches (`apply_cached`).

The reference has no counterpart: its stages are loops on one CPU core.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import statistics
from pathlib import Path

from . import capi

KERNELS = ("collide_cells", "move_cells", "place_movers", "place_walls")
RINGS = (64, 96, 128, 160, 192, 224, 256, 320, 384, 448, 512)


def cache_path() -> Path:
    p = os.environ.get("DSMC_TUNE_CACHE")
    if p:
        return Path(p)
    return Path(os.environ.get("XDG_CACHE_HOME", Path.home() / ".cache")) / "dsmc_b200" / "tuning.json"


def get(ctx) -> tuple[capi.Tuning, capi.Tuning]:
    cur, lim = capi.Tuning(), capi.Tuning()
    ctx.check(ctx.lib.dsmc_tuning_get(ctx.handle, C.byref(cur), C.byref(lim)))
    return cur, lim


def set_tuning(ctx, bps=(0, 0, 0, 0, 0), ring=0, claim=0) -> None:
    t = capi.Tuning()
    for k in range(5):
        t.blocks_per_sm[k] = int(bps[k])
    t.ring = int(ring)
    t.collide_claim = int(claim)
    ctx.check(ctx.lib.dsmc_tuning_set(ctx.handle, C.byref(t)))


def as_dict(t: capi.Tuning) -> dict:
    return {"blocks_per_sm": list(t.blocks_per_sm), "ring": t.ring, "collide_claim": t.collide_claim}


def signature(ctx) -> dict:
    """GPU and workload shape the cached choice applies to."""
    import torch
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    cells = parts = 0
    # every system's active cells and particles
    sid = 0
    info = capi.SystemInfo()
    while ctx.lib.dsmc_system_info_get(ctx.handle, sid, C.byref(info)) == 0:
        cells += info.num_active_cells
        parts += info.num_particles
        sid += 1
    pipelined = C.c_int()
    grid, block, cap = C.c_int(), C.c_int(), C.c_int()
    ctx.check(ctx.lib.dsmc_pass_info(ctx.handle, C.byref(pipelined), C.byref(grid), C.byref(block), C.byref(cap)))
    return {"gpu": props.name, "sms": props.multi_processor_count, "cells": _pow2(cells), "particles": _pow2(parts),
            "min_ring": cap.value, "pipelined": pipelined.value}


def _pow2(x: int) -> int:
    """x rounded to the nearest power of two in log scale (0 for x <= 0)."""
    return 0 if x <= 0 else 2 ** round(math.log2(x))


def _key(sig: dict) -> str:
    return json.dumps(sig, sort_keys=True)


def load_cache() -> dict:
    p = cache_path()
    try:
        return json.loads(p.read_text())
    except (OSError, ValueError):
        return {}


def save_cache(entries: dict) -> None:
    p = cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(".tmp")
    tmp.write_text(json.dumps(entries, indent=1, sort_keys=True))
    tmp.replace(p)


def apply_cached(ctx) -> dict | None:
    """Applies the cached choice for this context's signature; returns it (None: no entry)."""
    entry = load_cache().get(_key(signature(ctx)))
    if not entry:
        return None
    ch = entry["choice"]
    set_tuning(ctx, ch["blocks_per_sm"], ch["ring"], ch["collide_claim"])
    return entry


def _time(ctx, steps: int, repeats: int) -> dict:
    """Median per-kernel milliseconds per pass over `repeats` runs of `steps`."""
    runs = []
    for _ in range(repeats):
        ctx.set_timing(True)
        ctx.step(steps)
        t = ctx.pass_times()
        ctx.set_timing(False)
        runs.append({k: t[k] / max(t["passes"], 1) for k in KERNELS})
    out = {k: statistics.median(r[k] for r in runs) for k in KERNELS}
    out["step"] = sum(out[k] for k in KERNELS)
    return out


def tune(ctx, steps: int = 10, repeats: int = 3, extra_rings: int = 2, store: bool = True, log=None) -> dict:
    """Searches the launch shape on the context's current workload, applies
    the best and (store) caches it.  Returns the report: default and chosen
    times, every trial."""
    if ctx.pass_info()["pipelined"] != 1:
        return {"skipped": "the production pass does not run this context"}
    set_tuning(ctx)
    _, lim = get(ctx)
    max_bps = list(lim.blocks_per_sm)
    base_ring = lim.ring
    trials = []
    ctx.step(2)  # settle (graphs, first pass after a repack)
    default = _time(ctx, steps, repeats)
    trials.append({"config": "default", **default})
    best = {"bps": [0] * 5, "ring": 0, "claim": 0}

    def run(bps, ring, claim, label):
        set_tuning(ctx, bps, ring, claim)
        t = _time(ctx, steps, repeats)
        trials.append({"config": label, "bps": list(bps), "ring": ring, "claim": claim, **t})
        if log:
            log(label, {k: round(v, 4) for k, v in t.items()})
        return t

    # move_cells: ring x blocks per SM
    rings = [r for r in RINGS if r >= base_ring][:1 + extra_rings]
    best_move = (default["move_cells"], 0, 0)
    for ring in rings:
        set_tuning(ctx, [0] * 5, ring if ring != base_ring else 0, 0)
        _, l2 = get(ctx)
        for b in range(1, l2.blocks_per_sm[1] + 1):
            bps = [0, b, 0, 0, 0]
            t = run(bps, ring if ring != base_ring else 0, 0, f"move ring {ring} bps {b}")
            if t["move_cells"] < best_move[0]:
                best_move = (t["move_cells"], b, ring if ring != base_ring else 0)
    best["bps"][1], best["ring"] = best_move[1], best_move[2]
    # collide_cells: claims x blocks per SM
    best_col = (default["collide_cells"], 0, 0)
    for claim in (1, 2):
        for b in range(1, max_bps[0] + 1):
            t = run([b, 0, 0, 0, 0], 0, claim, f"collide claim {claim} bps {b}")
            if t["collide_cells"] < best_col[0]:
                best_col = (t["collide_cells"], b, claim)
    best["bps"][0], best["claim"] = best_col[1], best_col[2]
    # place_movers and place_walls
    for k, name in ((2, "place_movers"), (3, "place_walls")):
        bk = (default[name], 0)
        for b in range(1, max_bps[k] + 1):
            bps = [0] * 5
            bps[k] = b
            t = run(bps, 0, 0, f"{name} bps {b}")
            if t[name] < bk[0]:
                bk = (t[name], b)
        best["bps"][k] = bk[1]
    # the combination, against the default on the whole step
    chosen = run(best["bps"], best["ring"], best["claim"], "chosen")
    set_tuning(ctx)
    again = _time(ctx, steps, repeats)
    if chosen["step"] >= again["step"]:
        best = {"bps": [0] * 5, "ring": 0, "claim": 0}
    set_tuning(ctx, best["bps"], best["ring"], best["claim"])
    choice = {"blocks_per_sm": best["bps"], "ring": best["ring"], "collide_claim": best["claim"]}
    report = {"signature": signature(ctx), "choice": choice, "default_ms": again, "chosen_ms": chosen,
              "limits": {"blocks_per_sm": max_bps, "ring": base_ring}, "trials": trials,
              "steps_per_trial": steps, "repeats": repeats}
    if store:
        entries = load_cache()
        entries[_key(report["signature"])] = {"choice": choice, "default_ms": again, "chosen_ms": chosen}
        save_cache(entries)
    return report
