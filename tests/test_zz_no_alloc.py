"""The allocation-free geometry entry point (dsmc_geometry_finish_gpu_noalloc).

It serves callers that must not allocate device memory: its working buffers
are a fixed array inside the library instead of cudaMalloc'd scratch.  Its
output must equal the allocating entry point's (dsmc_geometry_finish_gpu)
exactly, on consecutive calls that reuse the same fixed array.  Collected
last on purpose (file name), so a failure here leaves every other test run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from master_b200 import capi
from master_b200.capi import ptr
from master_b200.system import Geometry

pytestmark = pytest.mark.gpu


def finish(entry, solid):
    nx, ny, nz = solid.shape
    g = Geometry.empty(nx, ny, nz)
    g.voxels[...] = solid
    rc = getattr(capi.load(), entry)(0, nx, ny, nz, 1, ptr(g.voxels, C.c_uint8), ptr(g.normals, C.c_float),
                                     ptr(g.tangents1, C.c_float), ptr(g.tangents2, C.c_float))
    capi.check(rc)
    return g


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls():
    masks = [
        (Geometry.packed_spheres(64, 4, wanted_porosity=0.6, seed=1).voxels > 0).astype(np.uint8),
        (Geometry.packed_spheres((48, 32, 40), 3, wanted_porosity=0.5, seed=9).voxels > 0).astype(np.uint8),
    ]
    for solid in masks:
        a = finish("dsmc_geometry_finish_gpu", solid)
        b = finish("dsmc_geometry_finish_gpu_noalloc", solid)
        for k in ("voxels", "normals", "tangents1", "tangents2"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_noalloc_rejects_grids_beyond_its_fixed_scratch():
    solid = np.zeros((65, 64, 64), np.uint8)
    with pytest.raises(capi.DsmcError) as e:
        finish("dsmc_geometry_finish_gpu_noalloc", solid)
    assert e.value.code == capi.DSMC_ERR_CAPACITY and "64^3" in str(e.value)
