"""The benchmark's reference arm drives the reference alone.

bench.py --impl reference times the reference's own solver on the bench's
own workload: the world comes from the reference's geometry tool and the
settings from the oracle's workload table, so that arm must load nothing of
the B200 library.  These tests check that the two workload tables describe
the same physics, and that a reference leg runs with no module of the
library imported."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

from oracle import run_reference

ROOT = Path(__file__).resolve().parents[1]


def test_reference_workloads_match_the_gpu_workloads():
    from master_b200 import workloads
    for name, rw in run_reference.WORKLOADS.items():
        gw = workloads.WORKLOADS[name]
        for k in ("n", "radius_voxels", "porosity", "geometry_seed", "cells", "atoms_per_molecule", "voxel_um",
                  "density_si", "temperature", "dt_si", "gravity_si", "flow_direction"):
            assert getattr(rw, k) == getattr(gw, k), (name, k)
        rs, gs = rw.settings(statistics_interval=100), gw.settings(statistics_interval=100)
        for k in ("Lx", "Ly", "Lz", "cells_x", "mass", "diam", "density", "temperature", "wall_temperature",
                  "flow_direction", "atoms_per_molecule", "sampling_bins"):
            assert getattr(rs, k) == pytest.approx(getattr(gs, k), rel=1e-15), (name, k)
        assert rs.dt == pytest.approx(gs.dt, rel=1e-15) and rs.gravity == pytest.approx(gs.gravity, rel=1e-15)


def test_replica_memory_estimate_covers_the_halo_grid():
    w = run_reference.PACKED_256
    assert w.replica_bytes() > 27 * 256 ** 3 * 37
    assert 20e9 < w.replica_bytes() < 30e9


@pytest.mark.skipif(not (run_reference.available() and run_reference.geometry_tool_available()),
                    reason="oracle/_ref is not built")
def test_reference_leg_imports_nothing_of_the_library():
    code = (
        "import sys, json; sys.path.insert(0, %r); import bench; "
        "r = bench.cpu_reference_sample(steps=1, replicas=1); "
        "print(json.dumps({'mods': sorted(m for m in sys.modules if m.startswith('master_b200')), "
        "'value': r['value'], 'mol': r['particles_per_replica']}))" % str(ROOT))
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    out = json.loads(res.stdout.strip().splitlines()[-1])
    assert out["mods"] == []
    assert out["value"] > 0 and out["mol"] > 100000
