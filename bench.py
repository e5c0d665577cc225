#!/usr/bin/env python
"""Throughput of the B200 DSMC timestep: particle-steps per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one full timestep of the reference (System::step + sampler,
dsmc/main.cpp:57-64: accelerate, move with diffuse walls, cell re-binning,
NTC collide, sampling) over every particle of the workload, which is the
packed_256 geometry (256^3 voxels, r = 6 voxel spheres to porosity 0.5,
2^3-voxel cells, 30 simulators per cell, ~3.1e7 particles; seeded synthetic
geometry from the reference's own generator semantics).  Multi-GPU runs are
independent replicas (different draw seeds), one per rank: weak scaling.

--impl reference runs the reference's own CPU solver (oracle/_ref/dsmc_ref,
built from the reference sources) on the same workload, its world written by
the reference's own geometry tool, as single-rank replicas on the host cores
(rank 0 only), each timing a bounded number of timesteps (--ref-steps).  It
imports nothing of the B200 library.  A second leg times the 64^3 sample of
the workload that the GPU arm's cpu_baseline also runs.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DSMC particle-steps/s on 1 B200"
UNIT = "particle-steps/s"
BYTES_PER_PARTICLE_STEP = 64  # read + write of the 32-byte particle record


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = None
        fd, name = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        self.path = Path(name)

    def __enter__(self):
        self.out = open(self.path, "w")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
        self.out.close()

    def summary(self):
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        self.path.unlink(missing_ok=True)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def allreduce_max(pg, x: float) -> float:
    from master_b200 import ensemble
    return ensemble.reduce_max(pg, x)


def allreduce_sum(pg, x: float) -> float:
    from master_b200 import ensemble
    return ensemble.reduce_sum(pg, x)


def barrier(pg):
    from master_b200 import ensemble
    ensemble.barrier(pg)


def _host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_reference_sample(steps: int, replicas: int | None = None):
    """The reference's own CPU solver on the bounded 64^3 sample of the
    workload (same voxel size, sphere radius, porosity, gas and simulator
    weight), its world written by the reference's own geometry tool."""
    from oracle import run_reference
    w = run_reference.PACKED_256_SAMPLE
    cores = replicas or max(1, min(_host_cores(), 32))
    res = run_reference.run_replicas(w.settings(statistics_interval=100), w.geometry(), timesteps=steps,
                                     replicas=cores)
    mol = res["reports"][0].get("molecules")
    return {
        "value": res["particle_steps_per_s"], "unit": UNIT, "cores": cores, "kind": "reference",
        "particles_per_replica": mol, "workload": w.name, "steps": steps,
        "sample": (f"{cores} independent single-rank runs of the reference solver (oracle/_ref/dsmc_ref, g++ -O3) on "
                   f"a 64^3 box of the same voxel size, sphere radius, porosity, gas and simulator weight "
                   f"({mol} particles each; world from the reference's geometry tool), {steps} timesteps; its own "
                   f"stage timers (moving+colliding+accelerating+sampling)"),
    }


def cpu_reference_full(workload: str, steps: int):
    """The reference's own CPU solver on the benchmark workload itself: the
    world written by the reference's geometry tool (a single-rank world file
    with its 27x periodic halo, 16.8 GB at 256^3), then as many single-rank
    replicas as the host cores and 70 % of the available host memory hold
    (about 23 GB each at 256^3), each timing `steps` timesteps with its own
    stage timers.  Setup (geometry tool, world read, particle creation) is
    outside the timers, as in the reference's report."""
    from oracle import run_reference
    w = run_reference.WORKLOADS[workload]
    g = w.geometry()
    need = g.world_bytes()
    # a scratch folder with room for the world file and every replica's final
    # state file (48 bytes per particle)
    replicas = run_reference.replicas_that_fit(w, _host_cores())
    state_bytes = int(48 * 1.05 * w.expected_particles())
    cands = [os.environ.get("TMPDIR"), "/tmp", "/var/tmp", "/dev/shm"]
    base = None
    for c in cands:
        if c and os.path.isdir(c):
            free = shutil.disk_usage(c).free
            fit = int((free - 1.1 * need) // state_bytes) if free > 1.1 * need else 0
            if fit >= 1:
                base, replicas = c, max(1, min(replicas, fit))
                break
    if base is None:
        raise RuntimeError(f"no scratch folder with {need / 1e9:.1f} GB free for the reference's world file")
    root = Path(tempfile.mkdtemp(prefix="dsmc_ref_full_", dir=base))
    try:
        t0 = time.perf_counter()
        g.write_world(root / "worlds")
        tool_s = time.perf_counter() - t0
        res = run_reference.run_replicas(w.settings(statistics_interval=100), g, timesteps=steps, replicas=replicas,
                                         workdir=root / "runs", world_dir=root / "worlds", timeout=1800)
    finally:
        shutil.rmtree(root, ignore_errors=True)
    reps = res["reports"]
    mol = reps[0].get("molecules")
    init_s = statistics.median(r.get("initialize", 0.0) for r in reps)
    return {
        "value": res["particle_steps_per_s"], "unit": UNIT, "cores": replicas, "kind": "reference",
        "particles_per_replica": mol, "workload": w.name, "steps": steps,
        "step_seconds_median": statistics.median(r["step_seconds"] for r in reps),
        "geometry_tool_s": tool_s, "initialize_s_median": init_s,
        "host_cores": _host_cores(), "host_mem_available_gb": run_reference.host_memory_available() / 1e9,
        "sample": (f"{replicas} independent single-rank runs of the reference solver (oracle/_ref/dsmc_ref, g++ -O3) "
                   f"on the {w.name} workload itself ({w.n}^3 voxels, {mol} particles each; world from the "
                   f"reference's geometry tool), {steps} timesteps each; replica count limited by host cores "
                   f"({_host_cores()}) and 70 % of available host memory at ~{w.replica_bytes() / 1e9:.0f} GB per "
                   f"replica; its own stage timers (moving+colliding+accelerating+sampling)"),
    }


def run_reference_arm(args, world, rank, pg):
    """The reference's own CPU solver on this arm's workload and metric.  Imports
    nothing of the B200 library: worlds come from the reference's geometry
    tool, settings from the oracle's own workload table."""
    if rank != 0:
        return 0
    t0 = time.time()
    # a bounded sample of the workload per replica: a few of its timesteps
    steps = max(1, min(args.steps, args.ref_steps))
    try:
        full = cpu_reference_full(args.workload, steps)
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU solver could not run: {e}"}))
        return 0
    sample = None
    if not args.no_cpu_baseline:
        try:
            sample = cpu_reference_sample(steps=args.cpu_steps)
        except Exception as e:  # noqa: BLE001
            sample = {"value": None, "unavailable": str(e)}
    per_replica = full.get("particles_per_replica")
    ms = 1e3 * full["step_seconds_median"] / steps if full.get("step_seconds_median") else None
    line = {
        "metric": METRIC, "value": full["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
        "warmup": 0, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        # the reference's timers cover every step of its run: no warm-up to leave out
        "config": {"workload": full["workload"], "particles_per_replica": per_replica,
                   "parallelism": f"{full['cores']} replicas on host cores",
                   "sample": f"{steps} timesteps of the workload per replica (cpu_baseline.sample)"},
        "cpu_baseline": full,
        "sample_leg_64": sample,
        "e2e": {"value": full["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.time() - t0,
    }
    print(json.dumps(line))
    return 0


def _timed_steps(ctx, steps: int) -> float:
    """Milliseconds of `steps` timesteps of a context, CUDA events on its stream."""
    import torch
    from master_b200 import capi
    lib = capi.load()
    st = torch.cuda.ExternalStream(lib.dsmc_stream(ctx.handle))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ctx.sync()
    e0.record(st)
    ctx.step(steps)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1)


def other_configs(args, device):
    """The plain-DSMC configuration (packed_64: 64^3, r = 4, porosity 0.6,
    ~3.9e5 particles) in the fp64 reference arithmetic and in split
    precision, the large geometry (packed_256) in fp64, and the batched ensemble (64 packed-sphere geometries of edges
    32-128, porosity 0.4-0.8, radius 3-8, Knudsen 0.1-10, one context, one
    launch per stage), each timed over `steps` steps after a warm-up."""
    from master_b200 import capi, fields, workloads
    from master_b200.system import System
    out = {}
    w = workloads.PACKED_64
    g = w.geometry()
    for name, prec in (("packed_64_fp64", capi.PREC_FP64), ("packed_64_split", capi.PREC_SPLIT32)):
        S = System(w.settings(rng_seed=5, statistics_interval=100), g, device=device, precision=prec)
        S.step(max(args.warmup, 3))
        k = 100
        ms = _timed_steps(S.ctx, k)
        out[name] = {"value": S.num_molecules * k / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / k, "steps": k,
                     "particles": S.num_molecules, "dtype": "f64" if prec == capi.PREC_FP64 else
                     "fp32 state + fp64 tallies"}
        S.ctx.close()
    # the large geometry in the fp64 reference arithmetic (the yardstick of the
    # split-precision numbers above)
    w256 = workloads.PACKED_256
    S = System(w256.settings(rng_seed=5, statistics_interval=100), w256.geometry(), device=device,
               precision=capi.PREC_FP64)
    S.step(3)
    k = 10
    ms = _timed_steps(S.ctx, k)
    out["packed_256_fp64"] = {"value": S.num_molecules * k / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / k,
                              "steps": k, "particles": S.num_molecules, "dtype": "f64"}
    S.ctx.close()
    # batched ensemble of uneven geometries
    rng = np.random.default_rng(3)
    specs = fields.random_specs(64, 32, seed=3, per_cell=30.0)
    for sp in specs:
        sp.n = int(rng.choice([32, 48, 64, 96, 128]))
    ens = fields.Ensemble(specs, device=device, rng_seed=77)
    ens.ctx.step(max(args.warmup, 3))
    k = 20
    ms = _timed_steps(ens.ctx, k)
    counts = [S.num_molecules for S in ens.systems]
    by_edge = {}
    for sp, c in zip(specs, counts):
        by_edge.setdefault(str(sp.n), []).append(c)
    out["batched_64_uneven"] = {
        "value": sum(counts) * k / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / k, "steps": k,
        "systems": len(counts), "particles": sum(counts), "particles_min": min(counts), "particles_max": max(counts),
        "particles_by_edge": {e: sum(v) for e, v in sorted(by_edge.items(), key=lambda kv: int(kv[0]))},
        "systems_by_edge": {e: len(v) for e, v in sorted(by_edge.items(), key=lambda kv: int(kv[0]))},
        "launches_per_step": 4, "error_bits": ens.ctx.device_status()[0]}
    ens.close()
    return out


def surrogate_line(device):
    """The warm-start surrogate's training step (batch 8 of 64^3 boxes) and
    its convolutions on the tensor cores, against the measured dense bf16
    peak: the dominant convolution by time is the roofline kernel."""
    from master_b200 import surrogate
    b = surrogate.benchmark(batch=8, S=64, repeats=5, device=device)
    peak = None
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            peak = float(json.loads(p.read_text())["bf16_tflops"])
        except Exception:
            peak = None
    kind = "measured" if peak else "fallback"
    peak = peak or 1590.0
    top = max(((n, k, v) for n, L in b["layers"].items() for k, v in L.items() if isinstance(v, dict)),
              key=lambda x: x[2]["ms"])
    b["roofline"] = {"bound": "tensor", "kernel": f"conv3 {top[0]} {top[1]}", "achieved": top[2]["tflops"],
                     "peak": peak, "unit": "TFLOP/s", "frac": top[2]["tflops"] / peak, "peak_kind": kind}
    b["train_step_frac_of_peak"] = b["train_step_tflops"] / peak
    return b


def run_warmstart(args, rank):
    """The second half of the metric: steps and wall time until the x mass
    flux stays within 2 % of its steady value for 1000 steps, from the cold
    start (the reference's) and from the surrogate's warm start, on unseen
    packed-sphere boxes of 64^3 (master_b200/warmstart.py)."""
    if rank != 0:
        return 0
    import torch
    from master_b200 import fields, warmstart
    torch.cuda.set_device(0)
    net, held = warmstart.load_net(ROOT / "master_b200" / "weights" / "surrogate_64.npz")
    specs = fields.random_specs(args.warmstart_geometries, 64, seed=5, porosity=(0.45, 0.75), knudsen=(0.3, 3.0),
                                per_cell=60)
    rep = warmstart.compare(net, specs, 6000, every=10, field_error=float(held.get("field_error", 0.0)),
                            capacity=(1.6, 12), log=lambda *a: None)
    line = {"metric": "steps to steady x mass flux (2 % for 1000 steps), cold vs warm", "unit": "steps",
            "higher_is_better": False, "data": "synthetic", "n_gpus": 1,
            "config": {"workload": f"{len(specs)} unseen packed-sphere boxes of 64^3, porosity 0.45-0.75, "
                                   f"radius 3-8, Kn 0.3-3, 60 simulators per cell", "particles": rep["particles"],
                       "window": rep["window"], "hold": rep["hold"], "tol": rep["tol"]},
            "cold": {k: rep["cold"][k] for k in ("steps_to_steady", "wall_s_to_steady", "ms_per_step",
                                                 "window_noise")},
            "warm": {k: rep["warm"][k] for k in ("steps_to_steady", "wall_s_to_steady", "ms_per_step",
                                                 "window_noise")},
            "ratio_steps": rep["ratio_steps"], "seeded_from": rep.get("seeded_from"),
            "surrogate_field_error": rep["surrogate_field_error"], "inference_s": rep["inference_s"],
            "seed_s": rep["seed_s"],
            "cold_flux_over_steady": rep["cold"]["flux_over_steady_window"][:40:2],
            "warm_flux_over_steady": rep["warm"]["flux_over_steady_window"][:40:2]}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="packed_256")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--ref-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--no-configs", action="store_true", help="skip the packed_64 and batched-ensemble lines")
    ap.add_argument("--warmstart", action="store_true",
                    help="instead of the throughput line: steps and wall time to a steady flux, cold against "
                         "the surrogate's warm start, on unseen 64^3 packs (about 10 minutes)")
    ap.add_argument("--warmstart-geometries", type=int, default=384)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world, rank, local, pg = dist_setup(args)
    if args.warmstart:
        return run_warmstart(args, rank)
    if args.impl == "reference":
        rc = run_reference_arm(args, world, rank, pg)
        if pg is not None:
            pg.destroy_process_group()
        return rc

    import ctypes as C
    import torch
    from master_b200 import capi, workloads
    from master_b200.system import System

    torch.cuda.set_device(local)
    lib = capi.load()
    W = workloads.WORKLOADS[args.workload]
    # sampling on the reference's default cadence (every 100 steps), as in
    # the reference run that the CPU baseline times
    settings = W.settings(rng_seed=1000 + rank, statistics_interval=100)
    geometry = W.geometry()
    system = System(settings, geometry, device=local)
    N = system.num_molecules
    stream = torch.cuda.ExternalStream(lib.dsmc_stream(system.ctx.handle))

    # warm-up (untimed)
    system.step(args.warmup)
    system.ctx.sync()
    # launch shapes from the project's autotuner (trial passes are ordinary
    # untimed timesteps of this workload; the cache is applied when present)
    tuning = None
    if not args.no_tune and system.ctx.pass_info()["pipelined"] == 1:
        from master_b200 import autotune
        cached = autotune.apply_cached(system.ctx)
        if cached is not None:
            tuning = {"source": "cache", "choice": cached["choice"]}
        else:
            rep = autotune.tune(system.ctx, steps=10, repeats=3)
            tuning = {"source": "tuned here", "choice": rep["choice"], "default_ms_per_step": rep["default_ms"]["step"],
                      "chosen_ms_per_step": rep["chosen_ms"]["step"], "trials": len(rep["trials"])}
        system.step(3)
        system.ctx.sync()
    step_before = int(system.tallies().step)

    # ---- device-resident throughput ---------------------------------------
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier(pg)
        torch.cuda.synchronize()
        system.ctx.sync()
        ev0.record(stream)
        system.step(args.steps)
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        barrier(pg)
    clocks = clk.summary()
    step_after = int(system.tallies().step)
    ms_rank = ev0.elapsed_time(ev1)
    ms_max = allreduce_max(pg, ms_rank)
    n_total = allreduce_sum(pg, float(N))
    value = n_total * args.steps / (ms_max / 1e3)
    err, spill = system.ctx.device_status()

    # ---- per-kernel durations (CUDA events around each kernel of each pass,
    # recorded by the library on its stream), after the timed region -------
    pipelined = system.ctx.pass_info()["pipelined"] == 1
    kernels = None
    if pipelined:
        k_t = max(3, min(args.steps, 20))
        system.ctx.set_timing(True)
        system.step(k_t)
        pt = system.ctx.pass_times()
        system.ctx.set_timing(False)
        kernels = {k: pt[k] / pt["passes"] for k in ("collide_cells", "move_cells", "place_movers", "place_walls")}
        kernels["passes"] = pt["passes"]
    # ---- one whole sampler cadence (statistics_interval steps, one of them
    # sampled: sample_cells runs after its collide) -------------------------
    cad = settings.statistics_interval
    c0 = torch.cuda.Event(enable_timing=True)
    c1 = torch.cuda.Event(enable_timing=True)
    system.ctx.sync()
    c0.record(stream)
    system.step(cad)
    c1.record(stream)
    c1.synchronize()
    cad_ms = c0.elapsed_time(c1)
    cadence = {"steps": cad, "sampled_steps": 1, "ms_per_step": cad_ms / cad, "value": N * cad / (cad_ms / 1e3),
               "sampled_step_extra_ms": cad_ms - cad * (ms_rank / args.steps)}
    tal = system.tallies()

    # ---- end to end through the C ABI with host buffers --------------------
    k_e2e = args.e2e_steps or args.steps
    r_host, v_host = system.get_particles()
    r_pin = torch.from_numpy(r_host).pin_memory()
    v_pin = torch.from_numpy(v_host).pin_memory()
    r_out = torch.empty_like(r_pin).pin_memory()
    v_out = torch.empty_like(v_pin).pin_memory()
    counters = (C.c_int64 * 8)()
    got = C.c_int64()
    D = C.POINTER(C.c_double)
    # one untimed round trip first (the e2e path's own warm-up: staging and
    # output buffers reach their size)
    system.ctx.check(lib.dsmc_particles_set(system.ctx.handle, system.id, N, C.cast(r_pin.data_ptr(), D),
                                            C.cast(v_pin.data_ptr(), D)))
    system.ctx.check(lib.dsmc_step(system.ctx.handle, 1))
    system.ctx.check(lib.dsmc_particles_get(system.ctx.handle, system.id, N, C.cast(r_out.data_ptr(), D),
                                            C.cast(v_out.data_ptr(), D), None, C.byref(got)))
    barrier(pg)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    system.ctx.check(lib.dsmc_particles_set(system.ctx.handle, system.id, N, C.cast(r_pin.data_ptr(), D),
                                            C.cast(v_pin.data_ptr(), D)))
    for _ in range(k_e2e):
        system.ctx.check(lib.dsmc_step(system.ctx.handle, 1))
        system.ctx.check(lib.dsmc_counters_get(system.ctx.handle, system.id, counters))
    system.ctx.check(lib.dsmc_particles_get(system.ctx.handle, system.id, N, C.cast(r_out.data_ptr(), D),
                                            C.cast(v_out.data_ptr(), D), None, C.byref(got)))
    e2e_s = time.perf_counter() - t0
    e2e_s = allreduce_max(pg, e2e_s)
    e2e_value = n_total * k_e2e / e2e_s

    # the same with K steps per upload/download for a longer K: the state
    # crosses PCIe once each way per K steps, so e2e rises with K
    k_long = max(200, k_e2e)
    barrier(pg)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    system.ctx.check(lib.dsmc_particles_set(system.ctx.handle, system.id, N, C.cast(r_pin.data_ptr(), D),
                                            C.cast(v_pin.data_ptr(), D)))
    for _ in range(k_long):
        system.ctx.check(lib.dsmc_step(system.ctx.handle, 1))
        system.ctx.check(lib.dsmc_counters_get(system.ctx.handle, system.id, counters))
    system.ctx.check(lib.dsmc_particles_get(system.ctx.handle, system.id, N, C.cast(r_out.data_ptr(), D),
                                            C.cast(v_out.data_ptr(), D), None, C.byref(got)))
    e2e_long_s = allreduce_max(pg, time.perf_counter() - t0)

    # ---- roofline of the dominant kernel: move_cells streams every particle
    # record in and out once (32 B read + 32 B written per particle-step) ----
    peak, peak_kind = measured_peaks()
    if kernels:
        dominant = "move_cells"
        achieved = BYTES_PER_PARTICLE_STEP * N / (kernels["move_cells"] / 1e3) / 1e9
    else:
        dominant = "cell pass"
        achieved = BYTES_PER_PARTICLE_STEP * N * args.steps / (ms_rank / 1e3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "move_cells_traffic.json"
    if tfile.exists() and kernels:
        try:
            t = json.loads(tfile.read_text())
            traffic = float(t["dram_bytes_per_particle"]) * N
        except Exception:
            traffic = None

    # every rank's tallies on rank 0: one all-reduce over a table by rank
    from master_b200 import ensemble
    tot = ensemble.totals(ensemble.gather_tallies(pg, world, {rank: tal}))
    physics = {"temperature_K_rank0": tal.temperature, "collisions": int(tot["collisions"]),
               "wall_collisions": int(tot["wall_collisions"]), "reseeds": int(tot["reseeds"]),
               "stranded": int(tot["stranded"]), "ranks": world}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32 state + fp64 tallies", "data": "synthetic",
        "config": {"workload": W.name, "voxels": W.n, "cells": W.cells, "particles_per_gpu": N,
                   "particles_total": int(n_total), "atoms_per_molecule": W.atoms_per_molecule,
                   "parallelism": f"replicas x{world}", "l2": "particle state 2 x %.1f GB > 126 MB L2" % (
                       system.info().slots * 32 / 1e9)},
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": BYTES_PER_PARTICLE_STEP * N},
        "kernels_ms": kernels,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 48 * N / k_e2e,
                "d2h_bytes_per_step": (48 * N + 64 * k_e2e) / k_e2e, "steps": k_e2e,
                "note": "K dsmc_step(1) calls between one upload and one download of the fp64 state; rises with K"},
        "e2e_long": {"value": n_total * k_long / e2e_long_s, "unit": UNIT, "steps": k_long,
                     "h2d_bytes_per_step": 48 * N / k_long, "d2h_bytes_per_step": (48 * N + 64 * k_long) / k_long},
        "cadence": cadence,
        "tuning": tuning,
        # collide_cells + move_cells + place_movers + place_walls per step
        # (production pass) and sample_cells on the sampled steps the timed
        # passes collide; one pass kernel per step otherwise
        "gpu_launches": args.steps * (4 if pipelined else 1) + (sum(
            1 for st in range(step_before, step_after)
            if st > 0 and st % settings.statistics_interval == 0) if pipelined else 0),
        "clocks": clocks,
        "device_status": {"error_bits": err, "spill": spill},
        "pass": system.ctx.pass_info(),
        "physics": physics,
    }
    system.ctx.close()
    if rank == 0 and world == 1 and not args.no_configs:
        line["configs"] = other_configs(args, local)
        try:
            line["surrogate"] = surrogate_line(local)
        except Exception as e:  # noqa: BLE001
            line["surrogate"] = {"unavailable": str(e)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_reference_sample(steps=args.cpu_steps)
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if rank == 0:
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
