"""The batched-ensemble configuration: packed-sphere geometries of uneven
size (edges 32 to 96 voxels), porosity, sphere radius and Knudsen number as
systems of one context, advanced by one launch per stage.  Draws are keyed
by each system's seed, particle id, cell and step, never by its place in
the context, so every system follows exactly the trajectory it follows when
run alone."""
from __future__ import annotations

import numpy as np
import pytest

from master_b200 import capi, fields
from master_b200.system import System

pytestmark = pytest.mark.gpu


def test_uneven_batch_equals_each_system_run_alone():
    edges = [32, 48, 64, 96, 32, 48]
    specs = fields.random_specs(len(edges), 32, seed=7)
    for sp, e in zip(specs, edges):
        sp.n = e
    ens = fields.Ensemble(specs, rng_seed=50)
    assert ens.ctx.pass_info()["pipelined"] == 1
    K = 15
    ens.ctx.step(K)
    for i, S in enumerate(ens.systems):
        alone = System(ens.settings[i], ens.geoms[i])
        alone.step(K)
        ra, va, ca = S.get_particles(with_cells=True)
        rb, vb, cb = alone.get_particles(with_cells=True)
        assert np.array_equal(ra, rb) and np.array_equal(va, vb) and np.array_equal(ca, cb), i
        ta, tb = S.tallies(), alone.tallies()
        for k in ("collisions", "wall_collisions", "candidates", "reseeds", "step"):
            assert getattr(ta, k) == getattr(tb, k), (i, k)
        assert list(ta.count_periodic) == list(tb.count_periodic)
        alone.ctx.close()
    assert ens.ctx.device_status()[0] & capi.EBIT_FATAL == 0
    # the mix really is uneven
    counts = [S.num_molecules for S in ens.systems]
    assert max(counts) > 10 * min(counts)
