"""Runs over many ranks: one process per GPU, independent work per rank.

The timestep has no exchange step between independent systems, so a run over
N GPUs shards whole systems (geometries or replicas) across ranks and meets
only at reductions: the slowest rank's time and the sums of the fp64 tallies
at a sample flush: one all-reduce over a table indexed by system, the
counterpart of the reference's MPI_Reduce of per-rank energy, flux and
profile sums (dsmc/statisticalproperty.cpp:34, 95, 287-288).  No particle
exchange (the reference's mpi_move, dsmc/system.cpp:49-105) is needed
between independent systems.  Works with the "nccl" backend (tensors on the rank's GPU) and
with "gloo" (tensors on the host), so the same code is tested on CPUs.
"""
from __future__ import annotations

from typing import Iterable, Mapping, Sequence

import numpy as np

# tallies reduced by sum, in this order (dsmc_tallies fields)
TALLY_FIELDS = ("collisions", "wall_collisions", "reseeds", "particle_steps", "count_periodic_x",
                "count_periodic_y", "count_periodic_z", "samples", "candidates", "kinetic_energy", "stranded")


def _device(pg):
    import torch
    if pg is None:
        return torch.device("cpu")
    return torch.device("cuda", torch.cuda.current_device()) if pg.get_backend() == "nccl" else torch.device("cpu")


def assign(num_systems: int, rank: int, world: int) -> list[int]:
    """Systems this rank runs: round robin, so sizes that grow with the index
    spread evenly over ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    return list(range(rank, num_systems, world))


def reduce_max(pg, x: float) -> float:
    """The largest value over all ranks (e.g. the slowest rank's time)."""
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(pg, x: float) -> float:
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def tally_row(t) -> np.ndarray:
    """One system's tallies (a capi.Tallies or a mapping) as a row of TALLY_FIELDS."""
    get = (lambda k: t[k]) if isinstance(t, Mapping) else (lambda k: getattr(t, k))
    row = []
    for k in TALLY_FIELDS:
        if k.startswith("count_periodic_"):
            cp = get("count_periodic")
            row.append(float(cp["xyz".index(k[-1])]))
        else:
            row.append(float(get(k)))
    return np.array(row, dtype=np.float64)


def gather_tallies(pg, num_systems: int, local: Mapping[int, object]) -> np.ndarray:
    """Every system's tallies on every rank: each rank fills the rows of the
    systems it ran, the others stay zero, and one sum all-reduce completes the
    table (float64: counts below 2^53 are exact)."""
    table = np.zeros((num_systems, len(TALLY_FIELDS)), dtype=np.float64)
    for sid, t in local.items():
        if not 0 <= sid < num_systems:
            raise ValueError(f"system {sid} outside 0..{num_systems - 1}")
        table[sid] = tally_row(t)
    if pg is None:
        return table
    import torch
    t = torch.from_numpy(table).to(_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return t.cpu().numpy()


def reduce_profile_sums(pg, sums: np.ndarray) -> np.ndarray:
    """Sampler profile sums (System.profile_sums, shape (4, bins)) added over
    ranks: replicas of one system pool their samples, as the reference's
    get_average reduces count and sums over ranks before normalising
    (dsmc/statisticalproperty.cpp:287-288, 348-349).  Finish the result with
    system.finish_profiles."""
    sums = np.ascontiguousarray(sums, np.float64)
    if pg is None:
        return sums.copy()
    import torch
    t = torch.from_numpy(sums.copy()).to(_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return t.cpu().numpy()


def totals(table: np.ndarray, systems: Iterable[int] | None = None) -> dict:
    """Sums over systems of a gathered table, by field name."""
    rows = table if systems is None else table[list(systems)]
    return dict(zip(TALLY_FIELDS, rows.sum(axis=0).tolist()))


def barrier(pg) -> None:
    if pg is not None:
        pg.barrier()


__all__: Sequence[str] = ("assign", "reduce_max", "reduce_sum", "gather_tallies", "tally_row", "totals", "barrier",
                          "reduce_profile_sums", "TALLY_FIELDS")
