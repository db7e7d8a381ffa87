"""CPU checks of the training-step oracle and of the loss mirror.

* The oracle's FP64 autograd restatement of the training gradient
  (oracle/model_ref.py: train_loss_grads) against the reference's own
  PyTorch model + EnergyStdLoss gradient (tests/golden/train_golden.npz,
  made by tests/golden/make_train_golden.py).
* The package's EnergyStdLoss against the reference loss value, and its
  closed-form gradient (train.loss_grads) against autograd.
"""

import importlib
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN


@pytest.fixture(scope="module")
def golden():
    with np.load(os.path.join(GOLDEN, "train_golden.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def case(dpb, golden):
    mdl = importlib.import_module("deepmd_kit_lr_pt_b200.model")
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    params = mdl.init_params(mdl.SeAConfig(), seed=int(golden["param_seed"]))
    params.davg, params.dstd = golden["davg"], golden["dstd"]
    frames = [wl.water_frame(4, seed=int(s)) for s in golden["seeds"]]
    labels = (golden["label_energy"], golden["label_force"], golden["label_virial"])
    return params, frames, labels


def check_against_golden(golden, grads, rtol=1e-8, atol=1e-9):
    """Compare a {name: gradient} dict with the golden summaries: relative to
    each tensor's scale, with an absolute floor for entries that are small
    sums of cancelling terms (the output bias: sum over frames of the energy
    residuals)."""
    names = [str(n) for n in golden["names"]]
    assert sorted(names) == sorted(grads)
    for k, name in enumerate(names):
        g = np.asarray(grads[name], np.float64)
        if f"full:{name}" in golden:
            ref = golden[f"full:{name}"]
            scale = np.abs(ref).max() + 1e-300
            assert np.abs(g.reshape(ref.shape) - ref).max() <= rtol * scale + atol, name
            continue
        g2 = g.reshape(g.shape[0], -1)
        rng = np.random.default_rng(1000 + k)
        V = rng.standard_normal((golden[f"proj:{name}"].size, g.size))
        norm = float(golden[f"norm:{name}"])
        assert abs(np.linalg.norm(g) - norm) <= rtol * norm, name
        for key, val in (("rows", g2.sum(1)), ("cols", g2.sum(0)), ("proj", V @ g.reshape(-1))):
            ref = golden[f"{key}:{name}"]
            assert np.abs(val - ref).max() <= rtol * norm * np.sqrt(g.size), (name, key)


def test_oracle_training_gradient_matches_reference_autograd(golden, case):
    from oracle import model_ref, oracle

    params, frames, labels = case
    lib = oracle.best()
    loss, E, F, V, grads = model_ref.train_loss_grads(lib, params, frames, labels,
                                                     tuple(golden["prefs"]))
    assert abs(loss - float(golden["loss"])) <= 1e-11 * abs(float(golden["loss"]))
    np.testing.assert_allclose(E, golden["energy"], rtol=1e-12)
    np.testing.assert_allclose(F, golden["force"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(V, golden["virial"], rtol=0, atol=1e-11)
    check_against_golden(golden, grads)


def test_energy_std_loss_matches_reference_value(golden, dpb):
    tr = importlib.import_module("deepmd_kit_lr_pt_b200.train")
    pe, pf, pv = golden["prefs"]
    loss_fn = tr.EnergyStdLoss(starter_learning_rate=1.0, start_pref_e=pe, limit_pref_e=pe,
                               start_pref_f=pf, limit_pref_f=pf, start_pref_v=pv,
                               limit_pref_v=pv)
    t = lambda k: torch.tensor(golden[k])  # noqa: E731
    pred = {"energy": t("energy"), "force": t("force"), "virial": t("virial")}
    label = {"energy": t("label_energy"), "force": t("label_force"),
             "virial": t("label_virial")}
    nat = [golden["force"].shape[0] // golden["energy"].size] * golden["energy"].size
    loss, more = loss_fn(pred, label, nat, 1.0)
    assert abs(float(loss) - float(golden["loss"])) <= 1e-12 * float(golden["loss"])
    assert set(more) >= {"rmse_e", "rmse_f", "rmse_v"}


def test_loss_closed_form_gradient_matches_autograd(dpb):
    tr = importlib.import_module("deepmd_kit_lr_pt_b200.train")
    rng = np.random.default_rng(4)
    nat = np.array([24, 57, 9])
    F, N = nat.size, int(nat.sum())
    mk = lambda *s: torch.tensor(rng.normal(size=s), requires_grad=True)  # noqa: E731
    E, Fo, V = mk(F), mk(N, 3), mk(F, 9)
    lab = {"energy": torch.tensor(rng.normal(size=F)), "force": torch.tensor(rng.normal(size=(N, 3))),
           "virial": torch.tensor(rng.normal(size=(F, 9)))}
    loss_fn = tr.EnergyStdLoss(starter_learning_rate=1e-3, start_pref_e=0.02, limit_pref_e=1.0,
                               start_pref_f=1000, limit_pref_f=1.0, start_pref_v=0.02,
                               limit_pref_v=1.0)
    lr = 4e-4
    loss, _ = loss_fn({"energy": E, "force": Fo, "virial": V}, lab, nat, lr)
    gE, gF, gV = torch.autograd.grad(loss, [E, Fo, V])
    inv = torch.tensor(1.0 / nat)
    pref = torch.tensor(loss_fn.prefactors(lr))
    l2, cE, cF, cV = tr.loss_grads(E.detach(), Fo.detach(), V.detach(), lab["energy"],
                                   lab["force"], lab["virial"], inv, pref)
    assert abs(float(l2) - float(loss)) <= 1e-13 * abs(float(loss))
    for a, b in ((gE, cE), (gF, cF), (gV, cV)):
        np.testing.assert_allclose(a.numpy(), b.numpy(), rtol=1e-13, atol=1e-15)
