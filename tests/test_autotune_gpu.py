"""The production pass's launch tuning (dsmc_tuning_set) and the autotuner
(master_b200/autotune.py): any launch shape gives the same trajectories, and
the tuner's choice round-trips through its JSON cache."""
from __future__ import annotations

import numpy as np
import pytest

from master_b200 import autotune, capi, workloads
from master_b200.system import System

pytestmark = pytest.mark.gpu


def pair():
    w = workloads.PACKED_64
    s = w.settings(rng_seed=11, statistics_interval=5)
    g = w.geometry()
    A = System(s, g)
    r, v = A.get_particles()
    B = System(s, g, init_particles=False)
    B.set_particles(r, v)
    A.set_particles(r, v)
    return A, B


@pytest.mark.parametrize("bps,ring,claim", [((1, 1, 1, 1, 1), 0, 1), ((2, 0, 3, 0, 1), 256, 2), ((0, 2, 0, 2, 0), 512, 0)])
def test_any_launch_shape_gives_the_same_trajectory(bps, ring, claim):
    A, B = pair()
    autotune.set_tuning(B.ctx, bps, ring, claim)
    cur, lim = autotune.get(B.ctx)
    assert list(cur.blocks_per_sm) == list(bps) and cur.ring == ring and cur.collide_claim == claim
    assert lim.ring >= max(ring, A.ctx.pass_info()["stage_capacity"])
    A.step(12)
    B.step(12)
    ra, va, ca = A.get_particles(with_cells=True)
    rb, vb, cb = B.get_particles(with_cells=True)
    assert np.array_equal(ra, rb) and np.array_equal(va, vb) and np.array_equal(ca, cb)
    ta, tb = A.tallies(), B.tallies()
    for k in ("collisions", "wall_collisions", "candidates", "reseeds"):
        assert getattr(ta, k) == getattr(tb, k), k
    assert list(ta.count_periodic) == list(tb.count_periodic)
    assert B.ctx.device_status()[0] & capi.EBIT_FATAL == 0


def test_tuning_arguments_are_checked():
    A, _ = pair()
    with pytest.raises(capi.DsmcError):
        autotune.set_tuning(A.ctx, (0, 0, 0, 0, 0), 0, 3)
    with pytest.raises(capi.DsmcError):
        autotune.set_tuning(A.ctx, (0, -1, 0, 0, 0), 0, 0)
    with pytest.raises(capi.DsmcError):
        autotune.set_tuning(A.ctx, (0, 0, 0, 0, 0), 4096, 0)


def test_tuner_chooses_caches_and_reapplies(tmp_path, monkeypatch):
    monkeypatch.setenv("DSMC_TUNE_CACHE", str(tmp_path / "tuning.json"))
    A, B = pair()
    rep = autotune.tune(A.ctx, steps=3, repeats=1, extra_rings=1)
    assert rep["chosen_ms"]["step"] > 0 and len(rep["trials"]) > 5
    assert (tmp_path / "tuning.json").exists()
    entry = autotune.apply_cached(B.ctx)
    assert entry is not None and entry["choice"] == rep["choice"]
    cur, _ = autotune.get(B.ctx)
    assert autotune.as_dict(cur) == rep["choice"]
