"""Runs over several ranks (master_b200/ensemble.py): systems sharded across
ranks, fp64 tallies gathered with one all-reduce, the slowest rank's time.
Two and three gloo ranks on the CPU, as a launch of one process per GPU
would run them."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from master_b200 import ensemble


def test_assign_covers_every_system_once():
    for world in (1, 2, 3, 8):
        seen = sorted(s for r in range(world) for s in ensemble.assign(13, r, world))
        assert seen == list(range(13))
    with pytest.raises(ValueError):
        ensemble.assign(4, 2, 2)


def fake_tallies(sid: int) -> dict:
    return {"collisions": 1000 + sid, "wall_collisions": 7 * sid, "reseeds": 0, "particle_steps": 10 ** 9 + sid,
            "count_periodic": [sid, -sid, 2 * sid], "samples": 3, "candidates": 4000 + sid,
            "kinetic_energy": 0.5 * sid, "stranded": 0}


def fake_profile(rank: int) -> np.ndarray:
    p = np.zeros((4, 6))
    p[0] = np.arange(6) + 10 * rank
    p[1] = 0.25 * (rank + 1)
    p[3, rank] = 3
    return p


def _rank(rank: int, world: int, port: int, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = ensemble.assign(5, rank, world)
        table = ensemble.gather_tallies(dist, 5, {s: fake_tallies(s) for s in mine})
        slowest = ensemble.reduce_max(dist, 10.0 + rank)
        total = ensemble.reduce_sum(dist, float(len(mine)))
        prof = ensemble.reduce_profile_sums(dist, fake_profile(rank))
        ensemble.barrier(dist)
        out.put((rank, table, slowest, total, prof))
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_gather_every_systems_tallies(world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = np.stack([ensemble.tally_row(fake_tallies(s)) for s in range(5)])
    for rank, table, slowest, total, prof in res:
        assert np.array_equal(table, expect)
        assert slowest == 10.0 + world - 1 and total == 5.0
        assert np.array_equal(prof, sum(fake_profile(r) for r in range(world)))
    tot = ensemble.totals(expect)
    assert tot["collisions"] == sum(1000 + s for s in range(5))
    assert tot["count_periodic_y"] == -sum(range(5))


def _rank_that_may_leave(rank: int, port: int, out):
    """Rank 1 leaves after joining, before the tally gather; rank 0 gathers."""
    import datetime
    import time as _time
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(0)   # leaves between steps: nothing of it in flight
    t0 = _time.monotonic()
    try:
        ensemble.gather_tallies(dist, 2, {0: fake_tallies(0)})
        out.put(("returned", _time.monotonic() - t0))
    except Exception as e:  # noqa: BLE001
        out.put((type(e).__name__, _time.monotonic() - t0))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:  # noqa: BLE001
            pass


def test_a_rank_that_left_makes_the_gather_fail_not_hang():
    """Failure detection on the host: a rank that exits between steps turns
    the survivors' next collective into an error within the process group's
    timeout, instead of a wait without end."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_that_may_leave, args=(r, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    what, secs = out.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert what != "returned", "the gather completed without the rank that left"
    assert secs < 60
