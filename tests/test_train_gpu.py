"""Training step on the GPU (hand-written backward and double backward):

* FP64 energy/force/virial and the gradient of the EnergyStdLoss w.r.t.
  every weight against the reference's own PyTorch autograd gradient
  (tests/golden/train_golden.npz) and, entry by entry, against the oracle's
  FP64 autograd restatement;
* central finite differences in FP64 (h = 1e-5): the loss along a seeded
  direction in every weight tensor, and the energy along single coordinates
  (the force);
* FP32 against FP64; the fused Adam step against torch.optim.Adam through the
  autograd.Function path; the captured step against the eager one; a batch of
  16 water frames of 192 atoms trained for a few steps.
"""

import importlib
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from test_train_oracle import check_against_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden():
    with np.load(os.path.join(GOLDEN, "train_golden.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def mods(dpb):
    return (importlib.import_module("deepmd_kit_lr_pt_b200.model"),
            importlib.import_module("deepmd_kit_lr_pt_b200.workload"),
            importlib.import_module("deepmd_kit_lr_pt_b200.train"))


@pytest.fixture(scope="module")
def case(mods, golden):
    mdl, wl, tr = mods
    params = mdl.init_params(mdl.SeAConfig(), seed=int(golden["param_seed"]))
    params.davg, params.dstd = golden["davg"], golden["dstd"]
    frames = [wl.water_frame(4, seed=int(s)) for s in golden["seeds"]]
    labels = (golden["label_energy"], golden["label_force"], golden["label_virial"])
    pe, pf, pv = golden["prefs"]
    loss = tr.EnergyStdLoss(starter_learning_rate=1.0, start_pref_e=pe, limit_pref_e=pe,
                            start_pref_f=pf, limit_pref_f=pf, start_pref_v=pv, limit_pref_v=pv)
    return params, frames, labels, loss


def _trainer(mods, case, dtype):
    mdl, wl, tr = mods
    params, frames, labels, loss = case
    t = tr.SeATrainer(params, frames, dtype=dtype, loss=loss)
    t.set_labels(*labels)
    return t


def _autograd_grads(trainer, loss_fn):
    """flat gradient via the autograd.Function and the torch-side loss."""
    trainer.flat.grad = None
    E, F, V = trainer.energy_force_virial()
    Eh, Fh, Vh = trainer.labels
    loss, _ = loss_fn({"energy": E, "force": F, "virial": V},
                      {"energy": Eh, "force": Fh, "virial": Vh}, trainer.ft.counts, 1.0)
    loss.backward()
    trainer.check()
    return float(loss.detach()), trainer.flat.grad.detach().clone()


def _loss_value(trainer, loss_fn):
    E, F, V = trainer._forward()
    Eh, Fh, Vh = trainer.labels
    loss, _ = loss_fn({"energy": E, "force": F, "virial": V},
                      {"energy": Eh, "force": Fh, "virial": Vh}, trainer.ft.counts, 1.0)
    return float(loss.detach())


def test_fp64_energy_force_virial_match_reference(mods, case, golden):
    t = _trainer(mods, case, torch.float64)
    E, F, V = t.compute()
    t.check()
    np.testing.assert_allclose(E, golden["energy"], rtol=1e-12)
    np.testing.assert_allclose(F, golden["force"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(V, golden["virial"], rtol=0, atol=1e-10)


def test_fp64_gradient_matches_reference_autograd(mods, case, golden):
    t = _trainer(mods, case, torch.float64)
    loss, g = _autograd_grads(t, case[3])
    assert abs(loss - float(golden["loss"])) <= 1e-11 * float(golden["loss"])
    grads = {k: v.cpu().numpy() for k, v in t.named_grads(g).items()}
    check_against_golden(golden, grads, rtol=1e-8, atol=1e-9)


@pytest.mark.parametrize("shared_acc", [0, 1])
def test_fp64_gradient_matches_oracle_every_entry(mods, case, golden, shared_acc):
    """Every gradient entry against the oracle, with the reverse kernel's
    weight gradients in one copy per warp or one per block (shared-memory
    atomics, knob train_rev_shared_acc)."""
    from oracle import model_ref, oracle

    from deepmd_kit_lr_pt_b200 import autotune

    params, frames, labels, _ = case
    old = autotune.get("train_rev_shared_acc")
    autotune.set_knob("train_rev_shared_acc", shared_acc)
    try:
        t = _trainer(mods, case, torch.float64)
        _, g = _autograd_grads(t, case[3])
    finally:
        autotune.set_knob("train_rev_shared_acc", old)
    _, _, _, _, ref = model_ref.train_loss_grads(oracle.port(), params, frames, labels,
                                                 tuple(golden["prefs"]))
    for name, v in t.named_grads(g).items():
        r = ref[name].reshape(v.shape)
        err = np.abs(v.cpu().numpy() - r).max()
        assert err <= 1e-9 * np.abs(r).max() + 1e-9, (name, err)


def test_fp64_loss_gradient_finite_differences(mods, case):
    """(L(w + h v) - L(w - h v)) / 2h against <dL/dw, v> for a seeded unit
    direction v in every weight tensor, h = 1e-5, FP64."""
    t = _trainer(mods, case, torch.float64)
    _, g = _autograd_grads(t, case[3])
    flat = t.flat.detach()
    base = flat.clone()
    h = 1e-5
    rng = np.random.default_rng(21)
    for k, name in enumerate(t.names):
        a, b = int(t.offsets[k]), int(t.offsets[k + 1])
        v = rng.standard_normal(b - a)
        v /= np.linalg.norm(v)
        vt = torch.tensor(v, dtype=torch.float64, device=flat.device)
        flat[a:b] = base[a:b] + h * vt
        lp = _loss_value(t, case[3])
        flat[a:b] = base[a:b] - h * vt
        lm = _loss_value(t, case[3])
        flat.copy_(base)
        fd = (lp - lm) / (2 * h)
        an = float(torch.dot(g[a:b], vt))
        gn = float(torch.linalg.norm(g[a:b]))
        assert abs(fd - an) <= 1e-6 * gn + 1e-7, (name, fd, an)


def test_fp64_force_is_minus_energy_gradient(mods, case):
    t = _trainer(mods, case, torch.float64)
    c0 = t.coord.clone()
    E0, F0, _ = t.compute()
    h = 1e-5
    rng = np.random.default_rng(5)
    for _ in range(8):
        i, d = int(rng.integers(t.ft.N)), int(rng.integers(3))
        f = int(t.ft.row_frame_h[i])
        t.coord.copy_(c0)
        t.coord[i, d] += h
        Ep, _, _ = t.compute()
        t.coord.copy_(c0)
        t.coord[i, d] -= h
        Em, _, _ = t.compute()
        fd = -(Ep[f] - Em[f]) / (2 * h)
        assert abs(fd - F0[i, d]) <= 1e-6 * max(1.0, abs(F0[i, d])), (i, d, fd, F0[i, d])
    t.coord.copy_(c0)


def test_fp32_close_to_fp64(mods, case):
    t64 = _trainer(mods, case, torch.float64)
    t32 = _trainer(mods, case, torch.float32)
    E64, F64, V64 = t64.compute()
    E32, F32, V32 = t32.compute()
    t32.check()
    n = t64.ft.counts
    assert np.abs(E32 - E64).max() / n.min() < 1e-5
    assert np.sqrt(np.mean((F32 - F64) ** 2)) < 1e-4
    assert np.abs(V32 - V64).max() < 1e-3 * max(1.0, np.abs(V64).max())
    _, g64 = _autograd_grads(t64, case[3])
    _, g32 = _autograd_grads(t32, case[3])
    for name, v in t64.named_grads(g64).items():
        w = t32.named_grads(g32)[name].double()
        rel = float(torch.linalg.norm(w - v) / (torch.linalg.norm(v) + 1e-30))
        assert rel < 2e-3, (name, rel)


def test_fused_adam_step_matches_torch_adam(mods, case):
    """train_step (closed-form loss gradient + Adam kernel) against the
    autograd.Function path stepped by torch.optim.Adam."""
    a = _trainer(mods, case, torch.float64)
    b = _trainer(mods, case, torch.float64)
    opt = torch.optim.Adam([a.flat], lr=1e-3)
    for step in range(3):
        lr = 1e-3 * 0.9 ** step
        for gr in opt.param_groups:
            gr["lr"] = lr
        la, _ = _autograd_grads(a, case[3])  # leaves the gradient in a.flat.grad
        opt.step()
        lb = float(b.train_step(lr).item())
        assert abs(la - lb) <= 1e-10 * abs(la), (step, la, lb)
        diff = float((a.flat.detach() - b.flat.detach()).abs().max())
        assert diff <= 1e-12, (step, diff)


def test_captured_step_matches_eager(mods, case):
    a = _trainer(mods, case, torch.float32)
    b = _trainer(mods, case, torch.float32)
    b.capture()
    assert float((a.flat.detach() - b.flat.detach()).abs().max()) == 0.0
    for step in range(3):
        la = float(a.train_step(1e-3).item())
        lb = float(b.train_step(1e-3).item())
        assert abs(la - lb) <= 1e-4 * abs(la), (step, la, lb)
    diff = float((a.flat.detach() - b.flat.detach()).abs().max())
    assert diff <= 1e-5, diff
    b.check()


def test_water_batch_of_16_trains(mods):
    """16 frames x 192 atoms (the training batch), FP32: the loss goes down
    under Adam, and status words stay clean."""
    mdl, wl, tr = mods
    cfg = mdl.SeAConfig()
    frames = [wl.water_frame(4, seed=100 + s) for s in range(16)]
    params = mdl.prepare_frames(mdl.init_params(cfg, seed=9), frames[:1])
    loss = tr.EnergyStdLoss(starter_learning_rate=1e-3, start_pref_e=0.02, limit_pref_e=0.02,
                            start_pref_f=1000.0, limit_pref_f=1000.0, start_pref_v=0.02,
                            limit_pref_v=0.02)
    t = tr.SeATrainer(params, frames, dtype=torch.float32, loss=loss)
    E, F, V = t.compute()
    rng = np.random.default_rng(3)
    t.set_labels(E + rng.normal(0, 1.0, E.shape), 0.5 * F, V + rng.normal(0, 1.0, V.shape))
    # Adam moves every weight by about lr per step; 1e-5 keeps the steps in
    # the descent regime for these N(0, 1/fan_in) weights
    losses = [float(t.train_step(1e-5).item()) for _ in range(12)]
    t.check()
    assert np.all(np.isfinite(losses))
    assert losses[-1] < losses[0] and min(losses) < 0.9 * losses[0], losses


def test_fp64_uneven_three_species_batch_matches_oracle(mods):
    """Frames of different sizes and species (water 96 and 150 atoms, FCC Cu
    64 atoms; model O/H/Cu, sel [46, 92, 60]): the per-frame atom counts enter
    the loss and the ragged batch the kernels; every gradient entry against
    the oracle's FP64 autograd restatement."""
    from oracle import model_ref, oracle

    mdl, wl, tr = mods
    rng = np.random.default_rng(17)
    frames = [wl.water_frame_density(96, rng), wl.cu_frame(64, rng),
              wl.water_frame_density(150, rng)]
    cfg = mdl.SeAConfig(sel=(46, 92, 60))
    params = mdl.init_params(cfg, seed=5)
    params.davg, params.dstd, _ = mdl.env_stats_frames(params, frames)
    nat = np.array([a.size for _, a, _ in frames])
    labels = (rng.normal(0, 2.0, len(frames)), rng.normal(0, 0.5, (int(nat.sum()), 3)),
              rng.normal(0, 5.0, (len(frames), 9)))
    prefs = (0.02, 1000.0, 0.02)
    loss = tr.EnergyStdLoss(start_pref_e=prefs[0], limit_pref_e=prefs[0],
                            start_pref_f=prefs[1], limit_pref_f=prefs[1],
                            start_pref_v=prefs[2], limit_pref_v=prefs[2])
    t = tr.SeATrainer(params, frames, dtype=torch.float64, loss=loss)
    t.set_labels(*labels)
    lv, g = _autograd_grads(t, loss)
    ref_loss, E, F, V, ref = model_ref.train_loss_grads(oracle.port(), params, frames, labels,
                                                        prefs)
    assert abs(lv - ref_loss) <= 1e-10 * abs(ref_loss)
    for name, v in t.named_grads(g).items():
        r = ref[name].reshape(v.shape)
        err = np.abs(v.cpu().numpy() - r).max()
        assert err <= 1e-9 * np.abs(r).max() + 1e-9, (name, err)
