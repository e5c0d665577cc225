"""What the trained surrogate gains over the method without it: it predicts
the steady x flux (mean drift) of geometries it has never seen from their
solid mask and Knudsen number alone, where the plain method has to run the
DSMC to steady state to know it.

Twelve unseen 64^3 packed-sphere boxes (porosity 0.45-0.75, radius 3-8
voxels, Kn 0.3-3; seeds never used in training) are run by the DSMC from a
cold start, 1500 steps of transient and 3000 steps of measurement; each
box's mean x drift from its crossing tally is compared with the committed
network's prediction (master_b200/weights/surrogate_64.npz).  Bar: median
relative error below 25 % (the DSMC's own 3000-step estimate is noisy by
about 10 % per box) and below half that of the best constant predictor
(the boxes' own mean drift, which no method could know beforehand).  Also
the warm start seeds that field: the seeded particles carry the predicted
mean drift."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from master_b200 import fields, steady, warmstart

pytestmark = pytest.mark.gpu

WEIGHTS = Path(__file__).resolve().parents[1] / "master_b200" / "weights" / "surrogate_64.npz"


def test_trained_network_predicts_the_flux_of_unseen_geometries():
    net, held = warmstart.load_net(WEIGHTS)
    assert held["field_error"] < 0.10
    specs = fields.random_specs(12, 64, seed=31, porosity=(0.45, 0.75), knudsen=(0.3, 3.0), per_cell=60)
    ens = fields.Ensemble(specs, rng_seed=900)
    ens.ctx.step(1500)
    c = steady.run_counts(ens.ctx, ens.systems, 3000, 100)
    u_dsmc = []
    for j, (S, s) in enumerate(zip(ens.systems, ens.settings)):
        flux = s.atoms_per_molecule * (c[-1, j] - c[0, j]) / (3000 * s.dt)
        u_dsmc.append(flux * s.Lx / (S.num_molecules * s.atoms_per_molecule) / fields.VELOCITY_SCALE)
    u_dsmc = np.array(u_dsmc)
    preds = warmstart.predict_fields(net, specs, ens.geoms)
    u_net = np.array([p[g.voxels.ravel() == 0, 1].mean() for p, g in zip(preds, ens.geoms)])
    err_net = np.median(np.abs(u_net - u_dsmc) / np.abs(u_dsmc))
    err_const = np.median(np.abs(u_dsmc.mean() - u_dsmc) / np.abs(u_dsmc))
    print("net", np.round(u_net, 3), "dsmc", np.round(u_dsmc, 3), err_net, err_const)
    assert err_net < 0.25
    assert err_net < 0.5 * err_const
    ens.close()


def test_warm_start_seeds_the_predicted_drift():
    net, _ = warmstart.load_net(WEIGHTS)
    specs = fields.random_specs(2, 64, seed=32, porosity=(0.45, 0.75), knudsen=(0.3, 3.0), per_cell=60)
    ens = fields.Ensemble(specs, rng_seed=950, cold=False)
    preds = warmstart.predict_fields(net, specs, ens.geoms)
    for S, g, p in zip(ens.systems, ens.geoms, preds):
        solid = (g.voxels > 0).astype(np.uint8).ravel()
        fields.warm_start(S, p, solid, n=1_000_000)
        r, v = S.get_particles()
        w = np.maximum(p[solid == 0, 0], 0)
        expect = (w * p[solid == 0, 1]).sum() / w.sum() * fields.VELOCITY_SCALE
        sig = v[:, 1].std()
        assert abs(v[:, 0].mean() - expect) < 5 * sig / np.sqrt(len(v))
    ens.close()
