"""Batched uneven frames (water at 1.0 g/cm^3 and FCC Cu with vacancies,
3-species model O/H/Cu, sel [46, 92, 60]) evaluated together against the
single-frame evaluator frame by frame (ghost copies, its own cell grid): the
same energy, force and virial to FP32 precision; in both forms of the step
(one persistent launch, one launch per stage), and the two forms against
each other."""

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(dpb):
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    mdl = importlib.import_module("deepmd_kit_lr_pt_b200.model")
    bt = importlib.import_module("deepmd_kit_lr_pt_b200.batch")
    rng = np.random.default_rng(11)
    frames = [wl.water_frame_density(24, rng), wl.cu_frame(32, rng),
              wl.water_frame_density(300, rng), wl.cu_frame(107, rng),
              wl.water_frame_density(96, rng), wl.cu_frame(256, rng)]
    cfg = mdl.SeAConfig(sel=(46, 92, 60))
    params = mdl.prepare_frames(mdl.init_params(cfg, seed=3), frames)
    return mdl, bt, frames, params


@pytest.mark.parametrize("fused", [True, False])
def test_batch_matches_single_frames(setup, fused):
    mdl, bt, frames, params = setup
    ev = bt.BatchEvaluator(params, frames, fused=fused)
    assert (ev.plan is not None) == fused
    E, F, V = ev.compute()
    ev.check()
    for f, (coord, atype, box) in enumerate(frames):
        single = mdl.SeAEvaluator(params, atype, box, mode="compressed")
        e0, f0, v0 = single.compute(coord)
        n = atype.size
        assert abs(E[f] - e0) / n < 1e-6, (f, E[f], e0)
        assert np.abs(F[ev.frame_slice(f)] - f0).max() < 1e-5, f
        assert np.abs(V[f] - v0).max() < 1e-4 * max(1.0, np.abs(v0).max()), f


@pytest.mark.parametrize("fused", [True, False])
def test_batch_graph_replay_repeats(setup, fused):
    mdl, bt, frames, params = setup
    ev = bt.BatchEvaluator(params, frames, fused=fused)
    E0, F0, V0 = ev.compute()
    ev.capture()
    for _ in range(2):
        E1, F1, V1 = ev.compute()
        # atomic energies are FP32 sums of per-tile partials added atomically
        # (order varies run to run); forces and virials are FP64 sums
        np.testing.assert_allclose(E1, E0, rtol=0, atol=1e-5)
        np.testing.assert_allclose(F1, F0, rtol=0, atol=1e-9)
        np.testing.assert_allclose(V1, V0, rtol=0, atol=1e-7)


def test_fused_step_equals_staged_step(setup):
    """The one-launch step and the per-stage launches run the same device
    bodies: neighbor lists, env rows and descriptors identical; energies,
    forces and virials to FP32 accuracy (the one-launch step runs the short
    K = 240 fitting layers on the chunk-draining tile form, whose products
    are issued in another order, so the FP32 sums round differently)."""
    mdl, bt, frames, params = setup
    a = bt.BatchEvaluator(params, frames, fused=True)
    b = bt.BatchEvaluator(params, frames, fused=False)
    Ea, Fa, Va = a.compute()
    Eb, Fb, Vb = b.compute()
    a.check()
    b.check()
    assert np.array_equal(a.nlist.cpu().numpy(), b.nlist.cpu().numpy())
    assert np.array_equal(a.em.cpu().numpy(), b.em.cpu().numpy())
    assert np.array_equal(a.D.cpu().numpy(), b.D.cpu().numpy())
    np.testing.assert_allclose(Ea, Eb, rtol=0, atol=1e-5)
    np.testing.assert_allclose(Fa, Fb, rtol=0, atol=1e-6)
    np.testing.assert_allclose(Va, Vb, rtol=0, atol=1e-5 * max(1.0, float(np.abs(Vb).max())))
    # a second step of the fused form (accumulators re-zeroed in the launch)
    Ea2, Fa2, _ = a.compute()
    np.testing.assert_allclose(Ea2, Ea, rtol=0, atol=1e-5)
    np.testing.assert_allclose(Fa2, Fa, rtol=0, atol=1e-9)


def test_batch_rejects_small_or_skewed_boxes(setup, dpb):
    mdl, bt, frames, params = setup
    coord, atype, box = frames[0]
    skew = box.copy()
    skew[3] = 0.5
    with pytest.raises(dpb._capi.DPBInvalidArgument):
        bt.BatchEvaluator(params, [(coord, atype, skew)])
    small = np.diag([5.0, 5.0, 5.0]).reshape(9)
    with pytest.raises(dpb._capi.DPBInvalidArgument):
        bt.BatchEvaluator(params, [(coord % 5.0, atype, small)])
