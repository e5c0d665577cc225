"""Unit conversions and the Knudsen-number density of the Python side,
against the reference's own unit converter (bc/dsmc_unit_converter.py)
evaluated by tests/golden/make_units.py."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from master_b200 import fields
from master_b200.system import acceleration_from_si, time_from_si
from master_b200.workloads import ARGON_DIAM_UM

REF = json.loads((Path(__file__).parent / "golden" / "units_ref.json").read_text())


def test_time_and_acceleration_match_the_reference_converter():
    for t, want in REF["time_from_si"]:
        assert time_from_si(t) == pytest.approx(want, rel=1e-15)
    for a, want in REF["acceleration_from_si"]:
        assert acceleration_from_si(a) == pytest.approx(want, rel=1e-15)


def test_knudsen_density_matches_the_reference_converter():
    assert REF["diam_um"] == ARGON_DIAM_UM
    for kn, length_um, want in REF["density_from_knudsen_number"]:
        assert fields.density_for_knudsen(kn, length_um) == pytest.approx(want, rel=1e-14)


def test_mean_pore_chord_of_a_slit():
    # a periodic slit of width w between solid plates: S_v = 2 n^2 faces over
    # n^3 voxels, porosity w / n, so 4 porosity / S_v = 2 w
    n, w = 16, 6
    solid = np.ones((n, n, n), bool)
    solid[:, :, :w] = False
    assert fields.mean_pore_chord(solid, 1.0) == pytest.approx(2.0 * w)
    assert fields.mean_pore_chord(solid, 0.1) == pytest.approx(0.2 * w)
    assert fields.mean_pore_chord(np.zeros((4, 4, 4), bool), 1.0) == float("inf")
