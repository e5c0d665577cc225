"""Host side of the x-slab decomposition (master_b200/slab.py): the
partition, record routing, and the all-to-all exchange over two and three gloo
ranks on the CPU with stand-in slabs (the records are the 32-byte layout of
dsmc_exchange_take; no GPU)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from master_b200 import slab as slabmod


def test_partition_covers_cells_in_balanced_ranges():
    for cells, world in ((12, 2), (12, 5), (128, 8), (7, 7)):
        parts = slabmod.partition(cells, world)
        assert parts[0][0] == 0 and parts[-1][1] == cells
        assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
        sizes = [x1 - x0 for x0, x1 in parts]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
        own = slabmod.owner_table(cells, world)
        for r, (x0, x1) in enumerate(parts):
            assert (own[x0:x1] == r).all()
    with pytest.raises(ValueError):
        slabmod.partition(3, 4)


class FakeCtx:
    """Stands in for a slab's context: take hands out the records given to
    it, put collects what arrives."""

    def __init__(self, records: np.ndarray):
        self.records = records
        self.got: list[np.ndarray] = []

    def exchange_take(self) -> np.ndarray:
        out, self.records = self.records, np.empty((0, 8), np.uint32)
        return out

    def exchange_put(self, sys_id: int, rec) -> None:
        self.got.append(np.asarray(rec).view(np.uint32).reshape(-1, 8).copy())


def fake_slab(rank: int, world: int, nx: int, cells_x: int, records: np.ndarray):
    s = object.__new__(slabmod.Slab)
    s.rank, s.world, s.id = rank, world, 0
    s.voxels_per_cell_x = nx // cells_x
    s.owner = slabmod.owner_table(cells_x, world)
    s.ctx = FakeCtx(records)
    return s


def records_for(rank: int, n: int, nx: int, seed: int) -> np.ndarray:
    """Records with random voxels (i | j << 11 | k << 22) and the sender's
    rank and row in the id word, so a receiver can tell where each came from."""
    rng = np.random.default_rng(seed)
    rec = rng.integers(0, 2 ** 32, size=(n, 8), dtype=np.uint64).astype(np.uint32)
    i = rng.integers(0, nx, n).astype(np.uint32)
    j = rng.integers(0, nx, n).astype(np.uint32)
    k = rng.integers(0, nx, n).astype(np.uint32)
    rec[:, 0] = i | (j << 11) | (k << 22)
    rec[:, 7] = (rank << 20) | np.arange(n, dtype=np.uint32)
    return rec


def test_destinations_follow_the_voxel_column():
    nx, cells_x, world = 24, 12, 3
    rec = records_for(0, 500, nx, 1)
    s = fake_slab(0, world, nx, cells_x, rec)
    dest = s.destinations(rec)
    i = rec[:, 0] & 0x7FF
    assert np.array_equal(dest, slabmod.owner_table(cells_x, world)[i // 2])


def _rank(rank: int, world: int, port: int, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nx, cells_x = 24, 12
        s = fake_slab(rank, world, nx, cells_x, records_for(rank, 300 + 50 * rank, nx, 10 + rank))
        got = slabmod.exchange_dist(dist, s)
        # a second exchange with nothing to send
        got2 = slabmod.exchange_dist(dist, s)
        out.put((rank, got, got2, np.concatenate(s.ctx.got) if s.ctx.got else np.empty((0, 8), np.uint32)))
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_exchange_records_to_their_owners(world):
    """Two ranks (each the other's only neighbour) and three (a middle
    slab with a neighbour on either side)."""
    nx, cells_x = 24, 12
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = {r: (got, got2, rec) for r, got, got2, rec in (out.get(timeout=120) for _ in procs)}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    own = slabmod.owner_table(cells_x, world)
    sent = [records_for(r, 300 + 50 * r, nx, 10 + r) for r in range(world)]
    for r in range(world):
        got, got2, rec = res[r]
        assert got2 == 0
        want = np.concatenate([s[own[(s[:, 0] & 0x7FF) // 2] == r] for s in sent])
        assert got == want.shape[0] == rec.shape[0]
        # every record arrives intact at its owner, once
        key = lambda a: a[np.lexsort(a.T[::-1])]
        assert np.array_equal(key(rec), key(want))
