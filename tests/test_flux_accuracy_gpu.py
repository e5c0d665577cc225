"""Split precision against fp64 over a long run: the x mass flux past the
transient, the collision count and the temperature of 64 replicas of the
plain-DSMC workload (packed_64) in each precision
(master_b200/flux_accuracy.py, which also runs the full-size measurement).

Bar: the flux difference is consistent with the 2 % the split precision is
held to (|difference| <= 2 % + its 95 % interval, here about 6 %), the
collision counts agree within 1 % plus their interval and the temperatures
within their interval plus 0.5 K."""
from __future__ import annotations

import pytest

from master_b200 import flux_accuracy, workloads

pytestmark = pytest.mark.gpu


def test_split_precision_flux_agrees_with_fp64():
    res = flux_accuracy.compare(workloads.PACKED_64, replicas=64, steps=3000, start=1000)
    print(res)
    assert res["split"]["error_bits"] == 0 and res["fp64"]["error_bits"] == 0
    assert res["flux_rel_ci95"] < 0.1
    assert res["flux_consistent_with_2pct"], res
    assert abs(res["collisions_rel_diff"]) <= 0.01 + res["collisions_rel_ci95"]
    assert abs(res["temperature_diff_K"]) <= 0.5 + res["temperature_ci95_K"]
