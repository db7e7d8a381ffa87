"""Tile-shape knobs on the GPU: every option of every knob gives the same
energy, force, virial (and training gradient) as the default shapes, and the
autotuner leaves a working captured step behind."""

import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(dpb):
    return {m: importlib.import_module(f"deepmd_kit_lr_pt_b200.{m}")
            for m in ("model", "workload", "batch", "train", "autotune")}


@pytest.fixture()
def restore_knobs(mods):
    at = mods["autotune"]
    saved = at.current()
    yield
    at.apply(saved)


def _sweep(at, knob, run):
    """run() under every option of one knob, the others at their defaults."""
    out = {}
    old = at.get(knob)
    for v in at.options(knob):
        at.set_knob(knob, v)
        out[v] = run()
    at.set_knob(knob, old)
    return out


def test_batched_step_same_under_every_shape(mods, restore_knobs):
    mdl, wl, bt, at = mods["model"], mods["workload"], mods["batch"], mods["autotune"]
    rng = np.random.default_rng(5)
    frames = [wl.water_frame_density(96, rng), wl.cu_frame(64, rng),
              wl.water_frame_density(300, rng)]
    cfg = mdl.SeAConfig(sel=(46, 92, 60))
    params = mdl.prepare_frames(mdl.init_params(cfg, seed=3), frames)
    ev = bt.BatchEvaluator(params, frames)
    E0, F0, V0 = ev.compute()
    for knob in ("batch_atoms_per_cta", "desc_atoms_per_cta", "desc_coef_l1", "fit_n_tile",
                 "fit_split_b", "desc_tc"):
        for v, (E, F, V) in _sweep(at, knob, ev.compute).items():
            ev.check()
            # FP32 sums in another order: a few 1e-8 of the frame energies
            np.testing.assert_allclose(E, E0, rtol=3e-7, atol=1e-5, err_msg=f"{knob}={v}")
            np.testing.assert_allclose(F, F0, rtol=0, atol=1e-6, err_msg=f"{knob}={v}")
            np.testing.assert_allclose(V, V0, rtol=0, atol=1e-4, err_msg=f"{knob}={v}")


def test_frame_step_same_under_every_shape(mods, restore_knobs):
    mdl, wl, at = mods["model"], mods["workload"], mods["autotune"]
    coord, atype, box = wl.water_frame(4, seed=2)
    params = mdl.prepare(mdl.init_params(mdl.SeAConfig(), seed=1), coord, atype, box)
    ev = mdl.SeAEvaluator(params, atype, box, mode="compressed")
    E0, F0, V0 = ev.compute(coord)
    for knob in ("desc_atoms_per_cta", "desc_coef_l1", "fit_n_tile", "fit_split_b", "desc_tc"):
        for v, (E, F, V) in _sweep(at, knob, lambda: ev.compute(coord)).items():
            assert abs(E - E0) < 1e-4, (knob, v)
            np.testing.assert_allclose(F, F0, rtol=0, atol=1e-6, err_msg=f"{knob}={v}")
            np.testing.assert_allclose(V, V0, rtol=0, atol=1e-4, err_msg=f"{knob}={v}")


def test_training_gradient_same_under_every_shape(mods, restore_knobs):
    mdl, wl, tr, at = mods["model"], mods["workload"], mods["train"], mods["autotune"]
    frames = [wl.water_frame(4, seed=s) for s in (0, 1)]
    params = mdl.init_params(mdl.SeAConfig(), seed=3)
    params.davg, params.dstd, _ = mdl.env_stats_frames(params, frames[:1])
    loss = tr.EnergyStdLoss(start_pref_e=0.02, limit_pref_e=0.02, start_pref_f=1000,
                            limit_pref_f=1000, start_pref_v=0.02, limit_pref_v=0.02)
    t = tr.SeATrainer(params, frames, dtype=torch.float32, loss=loss)
    E, F, V = t.compute()
    t.set_labels(E + 1.0, 0.5 * F, V + 1.0)

    def grad():
        with torch.no_grad():
            E_, F_, V_ = t._forward()
            t._pref.copy_(torch.tensor(loss.prefactors(1.0), dtype=torch.float64))
            _, gE, gF, gV = tr.loss_grads(E_, F_, V_, *t.labels, t._natoms_inv, t._pref)
            return t._backward(gE, gF, gV).double().clone()

    g0 = grad()
    for knob in ("train_rows_per_group", "train_warps_per_cta", "batch_atoms_per_cta"):
        for v, g in _sweep(at, knob, grad).items():
            t.check()
            rel = float(torch.linalg.norm(g - g0) / torch.linalg.norm(g0))
            assert rel < 1e-5, (knob, v, rel)


def test_autotuner_leaves_a_working_step(mods, restore_knobs, tmp_path, monkeypatch):
    monkeypatch.setenv("DPB_TUNE_CACHE", str(tmp_path / "tune.json"))
    mdl, wl, bt, at = mods["model"], mods["workload"], mods["batch"], mods["autotune"]
    rng = np.random.default_rng(9)
    frames = [wl.water_frame_density(200, rng), wl.cu_frame(128, rng)]
    cfg = mdl.SeAConfig(sel=(46, 92, 60))
    params = mdl.prepare_frames(mdl.init_params(cfg, seed=3), frames)
    ev = bt.BatchEvaluator(params, frames)
    E0, F0, _ = ev.compute()
    res = ev.tune(reps=3)
    assert not res["cached"] and res["ms"] <= res["baseline_ms"]
    for k, v in res["knobs"].items():
        assert at.get(k) == v
    E1, F1, _ = ev.compute()
    np.testing.assert_allclose(E1, E0, rtol=0, atol=1e-5)
    np.testing.assert_allclose(F1, F0, rtol=0, atol=1e-6)
    again = ev.tune(reps=3)
    assert again["cached"] and again["knobs"] == res["knobs"]


@pytest.mark.parametrize("degree", [5, 3])
def test_tensor_core_contraction_matches(mods, restore_knobs, degree):
    """desc_tc = 1 (the forward contraction on the tensor cores, 3xTF32)
    against the CUDA-core contraction: xyz and D to FP32 resolution (3xTF32
    drops the lo x lo product, 2^-22 relative per product)."""
    mdl, wl, at = mods["model"], mods["workload"], mods["autotune"]
    coord, atype, box = wl.water_frame(5, seed=6)
    params = mdl.prepare(mdl.init_params(mdl.SeAConfig(), seed=1), coord, atype, box)
    ev = mdl.SeAEvaluator(params, atype, box, mode="compressed", table_degree=degree)
    out = {}
    for v in (0, 1):
        at.set_knob("desc_tc", v)
        ev.compute(coord)
        out[v] = (ev.xyz.double().cpu().numpy(), ev.D.double().cpu().numpy())
    for a, b in zip(out[1], out[0]):
        assert np.abs(a - b).max() <= 5e-6 * np.abs(b).max()
