"""One geometry over several GPUs in x-slabs: the reference's domain
decomposition (dsmc/topology.cpp, one MPI rank per processor box) and its
particle exchange System::mpi_move (dsmc/system.cpp:49-105), along x only.

Each rank holds the whole geometry (the mover follows a flight anywhere) and
owns the active cells of a contiguous range of cell x indices.  After every
step the particles that ended in another rank's cells leave their slab
(dsmc_exchange_take), travel to their owner in one all-to-all, and enter
their cells there (dsmc_exchange_put) before the next step's collide.  Draws
are keyed by particle id and cell index, not by rank, so a run over slabs
takes the same trajectory as the same geometry on one GPU.

Transports: `exchange_dist` over a torch.distributed group (nccl with the
records on the GPU from the take to the put, their owners computed there;
gloo through the host); `step_local` drives several
slabs held by one process (one GPU or several) in lock step.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from . import capi
from .system import Context, Geometry, Settings

VOXEL_I_MASK = 0x7FF  # voxel index i in the low 11 bits of a record's first word


def partition(cells_x: int, world: int) -> list[tuple[int, int]]:
    """Cell x ranges [x0, x1) of the ranks: contiguous, sizes differing by at
    most one cell."""
    if world < 1 or cells_x < world:
        raise ValueError(f"{cells_x} cell columns cannot make {world} slabs")
    return [(r * cells_x // world, (r + 1) * cells_x // world) for r in range(world)]


def owner_table(cells_x: int, world: int) -> np.ndarray:
    """Rank owning each cell x index."""
    own = np.empty(cells_x, np.int64)
    for r, (x0, x1) in enumerate(partition(cells_x, world)):
        own[x0:x1] = r
    return own


class Slab:
    """The slab of rank `rank` out of `world` for one geometry, on one GPU."""

    def __init__(self, settings: Settings, geometry: Geometry, rank: int, world: int, *, device: int = 0,
                 init_particles: bool = True, num_particles: int = -1):
        if not 0 <= rank < world:
            raise ValueError("rank outside the world")
        nx = geometry.shape[0]
        if nx % settings.cells_x:
            raise ValueError("voxels per cell must be whole")
        self.settings = settings
        self.geometry = geometry
        self.rank, self.world = rank, world
        self.x0, self.x1 = partition(settings.cells_x, world)[rank]
        self.voxels_per_cell_x = nx // settings.cells_x
        self.owner = owner_table(settings.cells_x, world)
        self.ctx = Context(device, capi.PREC_SPLIT32)
        self.id = self.ctx.add_slab(settings, geometry, self.x0, self.x1)
        if init_particles:
            self.ctx.check(self.ctx.lib.dsmc_particles_init(self.ctx.handle, self.id, num_particles))

    # ---- particles ---------------------------------------------------------
    def set_particles(self, r: np.ndarray, v: np.ndarray) -> None:
        """The geometry's particles (ids = row index); the slab keeps its own."""
        r = np.ascontiguousarray(r, np.float64).reshape(-1, 3)
        v = np.ascontiguousarray(v, np.float64).reshape(-1, 3)
        self.ctx.check(self.ctx.lib.dsmc_particles_set(self.ctx.handle, self.id, r.shape[0],
                                                       capi.ptr(r, capi.C.c_double), capi.ptr(v, capi.C.c_double)))

    @property
    def num_molecules(self) -> int:
        n = capi.C.c_int64()
        self.ctx.check(self.ctx.lib.dsmc_particles_count(self.ctx.handle, self.id, capi.C.byref(n)))
        return int(n.value)

    def get_particles(self, id_count: int):
        """(r, v, cell) over every id of the geometry: rows of the ids this
        slab holds are filled, with their cell's reference index; cell is -1
        for the other ids."""
        r = np.zeros((id_count, 3))
        v = np.zeros((id_count, 3))
        cell = np.empty(id_count, np.int32)
        n = capi.C.c_int64()
        self.ctx.check(self.ctx.lib.dsmc_particles_get(self.ctx.handle, self.id, id_count,
                                                       capi.ptr(r, capi.C.c_double), capi.ptr(v, capi.C.c_double),
                                                       capi.ptr(cell, capi.C.c_int32), capi.C.byref(n)))
        return r, v, cell

    def tallies(self) -> capi.Tallies:
        t = capi.Tallies()
        self.ctx.check(self.ctx.lib.dsmc_tallies_get(self.ctx.handle, self.id, capi.C.byref(t)))
        return t

    # ---- the exchange ------------------------------------------------------
    def destinations(self, records) -> np.ndarray:
        """Owner rank of each record, from its voxel index i."""
        rec = np.asarray(records).view(np.uint32).reshape(-1, 8)
        cx = (rec[:, 0] & VOXEL_I_MASK).astype(np.int64) // self.voxels_per_cell_x
        return self.owner[cx]

    def destinations_device(self, records):
        """destinations() on the device: records is an (n, 8) int32 tensor on
        the context's GPU; returns an int64 tensor there (no host copy)."""
        import torch
        own = getattr(self, "_owner_dev", None)
        if own is None or own.device != records.device:
            own = torch.as_tensor(self.owner, dtype=torch.int64, device=records.device)
            self._owner_dev = own
        cx = torch.bitwise_and(records[:, 0], VOXEL_I_MASK).to(torch.int64) // self.voxels_per_cell_x
        return own[cx]

    def step_dist(self, pg, n: int = 1) -> None:
        """n steps of this rank's slab, exchanging over `pg` after each."""
        for _ in range(n):
            self.ctx.step(1)
            exchange_dist(pg, self)


def exchange_dist(pg, slab: Slab) -> int:
    """One exchange over a torch.distributed group: the records that left
    every slab go to their owners in one all-to-all (counts first).  nccl
    keeps the records on the GPU; other backends go through the host.
    Returns the records this rank received."""
    import torch
    world = pg.get_world_size()
    if world != slab.world:
        raise ValueError("the group's size differs from the slab count")
    on_gpu = pg.get_backend() == "nccl"
    if on_gpu:
        # the records stay on the GPU: owners from their voxel column there
        dev = torch.device("cuda", getattr(slab.ctx, "device", torch.cuda.current_device()))
        out = slab.ctx.exchange_take_device(dev)
        dest = slab.destinations_device(out)
    else:
        dev = torch.device("cpu")
        rec_np = slab.ctx.exchange_take()
        out = torch.from_numpy(rec_np.view(np.int32).copy())
        dest = torch.from_numpy(slab.destinations(rec_np))
    order = torch.argsort(dest, stable=True)
    out = out[order].contiguous()
    send = torch.bincount(dest, minlength=world).to(torch.int64)
    recv = torch.empty_like(send)
    pg.all_to_all_single(recv, send)
    got = torch.empty((int(recv.sum().item()), 8), dtype=torch.int32, device=dev)
    pg.all_to_all_single(got, out, output_split_sizes=recv.tolist(), input_split_sizes=send.tolist())
    slab.ctx.exchange_put(slab.id, got if on_gpu else got.numpy())
    return int(got.shape[0])


def step_local(slabs: Sequence[Slab], n: int = 1) -> None:
    """n steps of slabs held by this process, in lock step: every slab
    steps, then the records that left each go straight to their owners."""
    world = len(slabs)
    if sorted(s.rank for s in slabs) != list(range(world)) or any(s.world != world for s in slabs):
        raise ValueError("step_local needs one slab per rank of the world")
    by_rank = sorted(slabs, key=lambda s: s.rank)
    for _ in range(n):
        for s in by_rank:
            s.ctx.step(1)
        inbox: list[list[np.ndarray]] = [[] for _ in range(world)]
        for s in by_rank:
            rec = s.ctx.exchange_take()
            if rec.shape[0]:
                dest = s.destinations(rec)
                for r in range(world):
                    part = rec[dest == r]
                    if part.shape[0]:
                        inbox[r].append(part)
        for s in by_rank:
            if inbox[s.rank]:
                s.ctx.exchange_put(s.id, np.concatenate(inbox[s.rank]))


def total_tallies(tallies: Sequence[capi.Tallies]) -> dict:
    """The geometry's tallies from its slabs': counts add; every slab
    samples on the same steps."""
    keys = ("collisions", "wall_collisions", "reseeds", "particle_steps", "candidates", "stranded")
    out = {k: sum(int(getattr(t, k)) for t in tallies) for k in keys}
    out["count_periodic"] = [sum(int(t.count_periodic[d]) for t in tallies) for d in range(3)]
    out["samples"] = max(int(t.samples) for t in tallies)
    out["step"] = max(int(t.step) for t in tallies)
    out["kinetic_energy"] = sum(float(t.kinetic_energy) for t in tallies)
    return out


__all__ = ("partition", "owner_table", "Slab", "exchange_dist", "step_local", "total_tallies")
