"""Skin-list evaluation (ghosts and an rcut + skin list reused between
rebuilds, as an MD engine passes them) against fresh lists every step:
the same energy, force and virial on perturbed water, compressed and FP64."""

import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(dpb):
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    mdl = importlib.import_module("deepmd_kit_lr_pt_b200.model")
    coord, atype, box = wl.water_frame(4, seed=2)
    params = mdl.prepare(mdl.init_params(mdl.SeAConfig(), seed=1), coord, atype, box)
    return mdl, coord, atype, box, params


@pytest.mark.parametrize("mode,tol_f,tol_e", [("compressed", 2e-5, 2e-6), ("plain", 1e-10, 1e-11)])
def test_skin_list_matches_fresh_lists(setup, mode, tol_f, tol_e):
    mdl, coord, atype, box, params = setup
    skin_ev = mdl.SeAEvaluator(params, atype, box, mode=mode, skin=2.0)
    fresh = mdl.SeAEvaluator(params, atype, box, mode=mode)
    rng = np.random.default_rng(0)
    c = coord.copy()
    nloc = atype.size
    for k in range(25):
        c = c + rng.normal(0.0, 0.01, size=c.shape)  # larger than c4's 0.002 A
        e1, f1, v1 = skin_ev.compute(c, rebuild=(k % 10 == 0))
        e0, f0, v0 = fresh.compute(c)
        assert abs(e1 - e0) / nloc < tol_e, (k, e1, e0)
        assert np.abs(f1 - f0).max() < tol_f, (k, np.abs(f1 - f0).max())
        assert np.abs(v1 - v0).max() < tol_f * 100, (k, np.abs(v1 - v0).max())
    skin_ev.check()


def test_repeated_driver(setup):
    mdl, coord, atype, box, params = setup
    rep = importlib.import_module("deepmd_kit_lr_pt_b200.repeated")
    ev = mdl.SeAEvaluator(params, atype, box, mode="compressed", skin=2.0)
    plain = mdl.SeAEvaluator(params, atype, box, mode="plain")
    out = rep.repeated_evaluation(ev, coord, steps=30, rebuild_every=10, sigma=0.002,
                                  check=plain.compute, check_every=10)
    assert out["rebuilds"] == 2 and len(out["checks"]) == 3
    for c in out["checks"]:
        assert c["force_rmse_ev_per_a"] < 1e-5 and c["energy_err_ev_per_atom"] < 1e-6


def test_rebuild_required(setup, dpb):
    mdl, coord, atype, box, params = setup
    ev = mdl.SeAEvaluator(params, atype, box, mode="compressed", skin=2.0)
    with pytest.raises(dpb._capi.DPBInvalidArgument):
        ev.step()
