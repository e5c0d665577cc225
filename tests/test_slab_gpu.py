"""x-slab decomposition on the GPU (master_b200/slab.py over
dsmc_system_add_slab / dsmc_exchange_take / dsmc_exchange_put).

Two or three slabs of one geometry, held by one process and advanced in lock
step (the exchange goes through the host), against the whole geometry as one
system: draws are keyed by particle id and cell, so every particle's position,
velocity and cell must agree bit for bit after the steps, and the tallies
must add up.  Slabs wait on nothing but the host, so several share one GPU
safely.
"""
from __future__ import annotations

import numpy as np
import pytest

from master_b200 import capi
from master_b200.slab import Slab, step_local, total_tallies
from master_b200.system import System
from test_parity_gpu import load_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", ["small_dt5", "small_cl"])
def test_slabs_follow_the_single_domain_trajectory(world, case):
    z, meta, s, g = load_case(case)
    K = 8
    one = System(s, g, init_particles=False)
    one.set_particles(z["r0"], z["v0"])
    one.step(K)
    r1, v1, c1 = one.get_particles(with_cells=True)
    t1 = one.tallies()

    slabs = [Slab(s, g, r, world, init_particles=False) for r in range(world)]
    for sl in slabs:
        sl.set_particles(z["r0"], z["v0"])
    N = z["r0"].shape[0]
    assert sum(sl.num_molecules for sl in slabs) == N
    step_local(slabs, K)
    assert sum(sl.num_molecules for sl in slabs) == N
    r = np.zeros((N, 3))
    v = np.zeros((N, 3))
    held = np.zeros(N, np.int64)
    cell = np.full(N, -1, np.int32)
    for sl in slabs:
        rs, vs, cs = sl.get_particles(N)
        hs = cs >= 0
        r[hs], v[hs], cell[hs] = rs[hs], vs[hs], cs[hs]
        held += hs
    assert (held == 1).all()  # every particle in exactly one slab
    assert np.array_equal(r, r1)
    assert np.array_equal(v, v1)
    assert np.array_equal(cell, c1)
    tot = total_tallies([sl.tallies() for sl in slabs])
    for k in ("collisions", "wall_collisions", "reseeds", "candidates", "stranded"):
        assert tot[k] == getattr(t1, k), k
    assert tot["count_periodic"] == list(t1.count_periodic)
    assert tot["step"] == t1.step == K
    assert tot["kinetic_energy"] == pytest.approx(t1.kinetic_energy, rel=1e-12)


def test_slab_cells_hold_the_right_particles():
    z, meta, s, g = load_case("small_dt5")
    world, N = 3, z["r0"].shape[0]
    slabs = [Slab(s, g, r, world, init_particles=False) for r in range(world)]
    for sl in slabs:
        sl.set_particles(z["r0"], z["v0"])
    step_local(slabs, 5)
    vpc = g.shape[0] // s.cells_x
    for sl in slabs:
        rs, _, cs = sl.get_particles(N)
        hs = cs >= 0
        assert (cs[hs] // (s.cells_y * s.cells_z) >= sl.x0).all() and (cs[hs] // (s.cells_y * s.cells_z) < sl.x1).all()
        i = np.floor(rs[hs, 0] * (g.shape[0] / s.Lx)).astype(np.int64) % g.shape[0]
        cx = i // vpc
        assert ((cx >= sl.x0) & (cx < sl.x1)).all()


def test_slab_init_splits_the_single_domain_init():
    z, meta, s, g = load_case("small_dt1")
    one = System(s, g)
    r1, v1 = one.get_particles()
    N = r1.shape[0]
    slabs = [Slab(s, g, r, 2) for r in range(2)]
    assert sum(sl.num_molecules for sl in slabs) == N
    held = np.zeros(N, np.int64)
    for sl in slabs:
        rs, vs, cs = sl.get_particles(N)
        hs = cs >= 0
        held += hs
        assert np.array_equal(rs[hs], r1[hs]) and np.array_equal(vs[hs], v1[hs])
    assert (held == 1).all()


def test_slab_rules():
    z, meta, s, g = load_case("small_dt1")
    sl = Slab(s, g, 0, 2)
    lib, h = sl.ctx.lib, sl.ctx.handle
    assert lib.dsmc_step(h, 2) == capi.DSMC_ERR_ARG            # one step between exchanges
    assert lib.dsmc_stage_move(h) == capi.DSMC_ERR_CONFIG       # moves go through the exchange
    assert lib.dsmc_exchange_put(h, 0, 0, None, 0) == 0
    sl.ctx.step(1)
    rec = sl.ctx.exchange_take()
    assert rec.shape[1] == 8
    # a record of the other slab's cells is refused
    other = Slab(s, g, 1, 2, init_particles=False)
    if rec.shape[0]:
        assert other.ctx.lib.dsmc_exchange_put(other.ctx.handle, 0, 0, None, 0) == 0
        rc = sl.ctx.lib.dsmc_exchange_put(h, 0, rec.shape[0], rec.ctypes.data, 0)
        assert rc == capi.DSMC_ERR_STATE
    from master_b200.system import Context
    c64 = Context(0, capi.PREC_FP64)
    with pytest.raises(capi.DsmcError):
        c64.add_slab(s, g, 0, 6)
    with pytest.raises(capi.DsmcError):
        sl.ctx.add_system(s, g)


def _slab_rank(rank: int, world: int, port: int, case: str, K: int, out):
    import os
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        z, meta, s, g = load_case(case)
        sl = Slab(s, g, rank, world, init_particles=False)
        sl.set_particles(z["r0"], z["v0"])
        sl.step_dist(dist, K)
        N = z["r0"].shape[0]
        r, v, cell = sl.get_particles(N)
        t = sl.tallies()
        out.put((rank, r, v, cell, int(t.collisions), int(t.wall_collisions), list(t.count_periodic)))
    finally:
        dist.destroy_process_group()


def test_two_processes_exchange_over_gloo():
    """Two ranks, one slab each (both on this GPU, exchanging through gloo on
    the host: no kernel waits on another), against one system."""
    import socket
    import torch.multiprocessing as mp
    case, K, world = "small_dt5", 6, 2
    z, meta, s, g = load_case(case)
    one = System(s, g, init_particles=False)
    one.set_particles(z["r0"], z["v0"])
    one.step(K)
    r1, v1, c1 = one.get_particles(with_cells=True)
    t1 = one.tallies()
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_slab_rank, args=(r, world, port, case, K, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    N = z["r0"].shape[0]
    r = np.zeros((N, 3))
    v = np.zeros((N, 3))
    cell = np.full(N, -1, np.int32)
    for _, rs, vs, cs, *_ in res:
        hs = cs >= 0
        assert not (cell[hs] >= 0).any()
        r[hs], v[hs], cell[hs] = rs[hs], vs[hs], cs[hs]
    assert np.array_equal(r, r1) and np.array_equal(v, v1) and np.array_equal(cell, c1)
    assert sum(x[4] for x in res) == t1.collisions
    assert sum(x[5] for x in res) == t1.wall_collisions
    assert [sum(x[6][d] for x in res) for d in range(3)] == list(t1.count_periodic)


def test_device_records_path_equals_host_path():
    """The exchange through device buffers (the nccl transport's path:
    exchange_take_device, owners on the device, exchange_put of CUDA
    tensors) moves the same records as the host path."""
    import torch
    case, K, world = "small_dt5", 6, 2
    z, meta, s, g = load_case(case)
    host = [Slab(s, g, r, world, init_particles=False) for r in range(world)]
    dev = [Slab(s, g, r, world, init_particles=False) for r in range(world)]
    for sl in host + dev:
        sl.set_particles(z["r0"], z["v0"])
    step_local(host, K)
    cuda = torch.device("cuda", 0)
    for _ in range(K):
        for sl in dev:
            sl.ctx.step(1)
        outs = [sl.ctx.exchange_take_device(cuda) for sl in dev]
        for sl in dev:
            parts = []
            for o, src in zip(outs, dev):
                if o.shape[0]:
                    d = src.destinations_device(o)  # owners computed on the GPU
                    assert np.array_equal(d.cpu().numpy(), src.destinations(o.cpu().numpy()))
                    parts.append(o[d == sl.rank])
            if parts:
                sl.ctx.exchange_put(sl.id, torch.cat(parts).contiguous())
    N = z["r0"].shape[0]
    for a, b in zip(host, dev):
        ra, va, ca = a.get_particles(N)
        rb, vb, cb = b.get_particles(N)
        assert np.array_equal(ca, cb) and np.array_equal(ra, rb) and np.array_equal(va, vb)
