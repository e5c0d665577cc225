"""B200-native DSMC timestep: a drop-in for the mover, cell sort, NTC collide
and sampler of andeplane/master's DSMC solver (code/base_code/program/dsmc/).

The compute path is libdsmc_b200.so (C ABI in include/dsmc_b200.h) with
hand-written sm_100a kernels; this package is its host-side mirror.
"""
from . import capi
from .system import Context, Geometry, Settings, System, acceleration_from_si, time_from_si

__all__ = ["capi", "Context", "Geometry", "Settings", "System", "acceleration_from_si", "time_from_si"]
