"""Analytic known-answer tests of the timestep's physics on the GPU
(production split-precision pass):

* collision rate in a wall-free box at equilibrium against kinetic theory:
  collisions per step = 1/2 N n sigma <c_r> dt with <c_r> = sqrt(16 k T /
  (pi m)) (the NTC scheme of dsmc/cell.cpp:42-111 is unbiased for it);
* the temperature of a wall-free box at equilibrium stays put;
* diffuse walls (ColliderThermal) and fully accommodating Cercignani-Lampis
  walls bring the gas to the wall temperature; specular walls conserve the
  gas temperature.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from master_b200 import workloads
from master_b200.system import Geometry, System

pytestmark = pytest.mark.gpu

K_B = 1.3806503e-23
AMU = 1.66053886e-27


def box_settings(n_vox: int, cells: int, per_cell: float, dt_si: float):
    w = workloads.Workload("kat", n=n_vox, radius_voxels=2, porosity=0.6, geometry_seed=5, cells=cells,
                           atoms_per_molecule=workloads.simulators_per_cell_weight(2.5e24, 0.1, n_vox // cells,
                                                                                   per_cell),
                           dt_si=dt_si, gravity_si=0.0)
    s = w.settings(statistics_interval=10 ** 6)
    s.gravity = 0.0
    s.flow_direction = -1
    return w, s


def test_collision_rate_matches_kinetic_theory():
    w, s = box_settings(32, 16, 20, 1e-11)
    S = System(s, Geometry.empty(32, 32, 32))
    N = S.num_molecules
    S.step(5)  # let vr_max settle
    c0 = S.tallies().collisions
    K = 60
    S.step(K)
    measured = (S.tallies().collisions - c0) / K
    T, m = s.temperature, s.mass * AMU
    n_real = N * s.atoms_per_molecule / (s.Lx * s.Ly * s.Lz * 1e-18)  # the simulated density, m^-3
    sigma = math.pi * (s.diam * 1e-6) ** 2
    c_r = math.sqrt(16 * K_B * T / (math.pi * m))
    expected = 0.5 * N * n_real * sigma * c_r * 1e-11  # simulator collision events per step
    # relative statistical error ~ 1/sqrt(K * expected) ~ 0.5 %
    assert measured == pytest.approx(expected, rel=0.04), (measured, expected)


def test_equilibrium_temperature_is_conserved():
    w, s = box_settings(32, 16, 20, 1e-11)
    S = System(s, Geometry.empty(32, 32, 32))
    T = [S.tallies().temperature]
    for _ in range(5):
        S.step(20)
        T.append(S.tallies().temperature)
    assert np.allclose(T, s.temperature, rtol=0.01), T


@pytest.mark.parametrize("model,alpha,wall_T,expect",
                         [(0, 0.5, 500.0, 500.0),   # diffuse walls: the gas takes the wall temperature
                          (2, 1.0, 500.0, 500.0),   # Cercignani-Lampis, full accommodation: the same
                          (1, 0.5, 500.0, 300.0)])  # specular walls: no exchange with the wall
def test_walls_set_the_gas_temperature(model, alpha, wall_T, expect):
    w, s = box_settings(32, 16, 12, 5e-11)
    s.surface_model = model
    s.alpha_n = s.alpha_t = alpha
    s.wall_temperature = wall_T
    g = Geometry.packed_spheres(32, 3, wanted_porosity=0.6, seed=3)
    S = System(s, g)
    S.step(400)
    T = S.tallies().temperature
    assert T == pytest.approx(expect, rel=0.03), T
    assert S.tallies().wall_collisions > S.num_molecules  # every particle met the walls
