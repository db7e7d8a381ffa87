"""Edge inputs of the whole evaluation against the FP64 oracle, with a model
whose statistics and tables come from an ordinary water frame: one molecule
in a large box (two neighbors per atom), atoms farther apart than the cutoff
(no neighbor at all: every env row is padding), a frame of one species only
(the other center type has no fitting rows), and a batch that mixes such
frames with an ordinary one."""

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(dpb):
    from oracle import oracle

    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    mdl = importlib.import_module("deepmd_kit_lr_pt_b200.model")
    bt = importlib.import_module("deepmd_kit_lr_pt_b200.batch")
    coord, atype, box = wl.water_frame(4, seed=31)
    params = mdl.prepare(mdl.init_params(mdl.SeAConfig(), seed=6), coord, atype, box)
    return wl, mdl, bt, params, (coord, atype, box), oracle.ref() or oracle.port()


def _cubic(L):
    return np.diag([L, L, L]).reshape(-1).astype(np.float64)


def _molecule(L=20.0):
    o = np.array([L / 2, L / 2, L / 2])
    c = np.stack([o, o + [0.9572, 0, 0], o + [-0.24, 0.9266, 0]])
    return c, np.array([0, 1, 1], np.int32), _cubic(L)


def _isolated(L=30.0):
    c = np.array([[1.0, 1.0, 1.0], [12.0, 1.5, 2.0], [1.0, 13.0, 14.0], [20.0, 20.0, 8.0]])
    return c, np.array([0, 1, 1, 0], np.int32), _cubic(L)


def _one_species(frame):
    coord, atype, box = frame
    keep = atype == 0
    return coord[keep].copy(), atype[keep].copy(), box


def _check(mdl, params, checker, frame, mode, etol, ftol):
    from oracle import model_ref

    coord, atype, box = frame
    ev = mdl.SeAEvaluator(params, atype, box, mode=mode)
    E, F, V = ev.compute(coord)
    ev.check()
    e0, f0, v0 = model_ref.evaluate(checker, params, coord, atype, box, mode=mode)
    n = atype.size
    assert abs(E - e0) / n <= etol, (E, e0)
    assert float(np.abs(F - f0).max()) <= ftol
    assert float(np.abs(V - v0).max()) <= 10 * ftol * max(1.0, float(np.abs(v0).max()))
    return E, F, V, e0


@pytest.mark.parametrize("mode,etol,ftol", [("compressed", 1e-6, 1e-5), ("plain", 1e-10, 1e-10)])
@pytest.mark.parametrize("case", ["molecule", "isolated", "one_species"])
def test_edge_frames_vs_oracle(env, mode, etol, ftol, case):
    wl, mdl, bt, params, water, checker = env
    frame = {"molecule": _molecule, "isolated": _isolated,
             "one_species": lambda: _one_species(water)}[case]()
    E, F, V, e0 = _check(mdl, params, checker, frame, mode, etol, ftol)
    if case == "isolated":  # no pair inside the cutoff: no force, no virial
        assert np.abs(F).max() == 0.0 and np.abs(V).max() == 0.0


def test_batch_with_edge_frames_vs_oracle(env):
    """Frames of 3, 4 and 64 atoms (molecule, isolated atoms, one species)
    batched with an ordinary water frame, in both forms of the step."""
    from oracle import model_ref

    wl, mdl, bt, params, water, checker = env
    frames = [_molecule(), water, _isolated(), _one_species(water)]
    for fused in (False, True):
        ev = bt.BatchEvaluator(params, frames, fused=fused)
        E, F, V = ev.compute()
        ev.check()
        for f, (coord, atype, box) in enumerate(frames):
            e0, f0, v0 = model_ref.evaluate(checker, params, coord, atype, box,
                                            mode="compressed")
            n = atype.size
            assert abs(E[f] - e0) / n <= 1e-6, (fused, f)
            assert float(np.abs(F[ev.frame_slice(f)] - f0).max()) <= 1e-5, (fused, f)
            assert float(np.abs(V[f] - v0).max()) <= 1e-4 * max(1.0, float(np.abs(v0).max()))
