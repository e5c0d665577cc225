"""Host side of the sampler profiles: dsmc_profiles_finish against the
reference's own get_average / finalize (dsmc/statisticalproperty.cpp:280-301,
341-362, 393-426, 462-478) run on the reference sampler's sums in the golden
fixtures (tests/golden/make_golden.py), and its edge cases."""
from __future__ import annotations

import numpy as np
import pytest

from master_b200 import capi
from master_b200.system import Geometry, Settings, finish_profiles
from test_parity_gpu import CASES, load_case


def volume_global(s, g: Geometry, tmp_path) -> float:
    """L_x L_y L_z times the world file's porosity (dsmc/dsmc_io.cpp:189-193,
    dsmc/system.cpp:314)."""
    g.write_world(tmp_path)
    por = Geometry.read_world(tmp_path / "0000.bin").porosity_global
    return s.Lx * s.Ly * s.Lz * por


@pytest.mark.parametrize("case", CASES)
def test_finish_matches_reference_finalize(case, tmp_path):
    z, meta, s, g = load_case(case)
    fin = finish_profiles(s, volume_global(s, g, tmp_path), z["prof_sumsK"])
    assert np.array_equal(fin["count"], z["prof_sumsK"][0])
    assert np.array_equal(fin["vx_count"], z["prof_sumsK"][3])
    for k, ref in (("velocity_z", "prof_vzK"), ("temperature", "prof_TK"), ("pressure", "prof_PK"),
                   ("vx_center", "prof_vx_center")):
        assert np.array_equal(fin[k], z[ref]), k  # the same operations in the same order


def test_reference_sums_are_consistent():
    """Every sample counts every particle once in y; the v_x histogram holds
    the particles within +-4 sigma."""
    for case in CASES:
        z, meta, s, g = load_case(case)
        p = z["prof_sumsK"]
        assert p[0].sum() == meta["params"]["steps"] * meta["n"]
        assert 0.99 * p[0].sum() <= p[3].sum() <= p[0].sum()


def test_empty_bins_divide_by_one():
    s = Settings()
    sums = np.zeros((4, 5))
    sums[:, 2] = [4, 2.0, 6.0, 3]
    fin = finish_profiles(s, 10.0, sums)
    assert fin["velocity_z"][0] == 0 and fin["temperature"][0] == 0 and fin["pressure"][0] == 0
    assert np.isfinite(fin["temperature"]).all()
    assert fin["vx_count"][2] == 3


def test_finish_rejects_bad_arguments():
    lib = capi.load()
    s = Settings()
    buf = np.zeros(8)
    assert lib.dsmc_profiles_finish(None, 1.0, 2, capi.ptr(buf, capi.C.c_double), *([None] * 6)) == capi.DSMC_ERR_ARG
    rc = lib.dsmc_profiles_finish(capi.C.byref(s.raw), 1.0, 0, capi.ptr(buf, capi.C.c_double), *([None] * 6))
    assert rc == capi.DSMC_ERR_ARG
