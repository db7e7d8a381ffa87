"""forward_lower for an MD engine (engine.ForwardLower) and a compressed
model read from the reference's state-dict layout (checkpoint.load).

The engine's system is made as LAMMPS would hand it over: extended
coordinates with ghosts (copy_coord within rcut + skin), a neighbor list of
the local atoms within rcut + skin with every row in a random order. The
extended forces, folded onto their owners through the ghost mapping, and the
energy and virial must equal the single-frame compressed evaluator's (same
kernels: FP64 sums in a different order, 1e-9) and stay within the path's
tolerances of the FP64 oracle (|dE|/N <= 1e-6 eV/atom, force RMSE <= 1e-5
eV/A).
"""

import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
SKIN = 2.0


@pytest.fixture(scope="module")
def mods(dpb):
    imp = importlib.import_module
    return (imp("deepmd_kit_lr_pt_b200.workload"), imp("deepmd_kit_lr_pt_b200.model"),
            imp("deepmd_kit_lr_pt_b200.engine"), imp("deepmd_kit_lr_pt_b200.checkpoint"))


def _engine_system(dpb, coord, atype, box, rc_list, seed):
    ops = dpb.ops
    cx, tx, mx = ops.copy_coord(torch.tensor(coord, device=DEV), torch.tensor(atype, device=DEV),
                                rc_list, box)
    nloc = atype.size
    il, nn, rows, _ = ops.build_nlist(cx, nloc, rc_list, atype=tx)
    # engines hand over rows in no particular order
    r = rows.cpu().numpy()
    n = nn.cpu().numpy()
    rng = np.random.default_rng(seed)
    for i in range(nloc):
        r[i, :n[i]] = r[i, rng.permutation(n[i])]
    rows = torch.tensor(r, device=DEV)
    return cx, tx, mx, nn, rows


@pytest.mark.parametrize("case", ["water", "cu"])
def test_forward_lower_matches_evaluator_and_oracle(dpb, mods, case):
    from oracle import model_ref, oracle

    wl, mdl, eng, _ = mods
    rng = np.random.default_rng(4)
    if case == "water":
        coord, atype, box = wl.water_frame(5, seed=9)
        cfg = mdl.SeAConfig()
        frames = [(coord, atype, box)]
    else:
        coord, atype, box = wl.cu_frame(300, rng)
        cfg = mdl.SeAConfig(sel=(46, 92, 60))
        frames = [(coord, atype, box), wl.water_frame_density(150, rng)]
    params = mdl.prepare_frames(mdl.init_params(cfg, seed=2), frames)
    cx, tx, mx, nn, rows = _engine_system(dpb, coord, atype, box, cfg.rcut + SKIN, 7)
    nloc, nall = atype.size, cx.shape[0]
    fl = eng.ForwardLower(params, nloc, nall, max_nbor=rows.shape[1])
    fn = dpb.ops._row_pointers(rows)
    E, Fext, V = fl(cx, tx, nloc, nn, fn, rebuilt=True)
    fl.check()
    E = float(E.item())
    F = np.zeros((nloc, 3))
    np.add.at(F, mx.cpu().numpy(), Fext.cpu().numpy())
    V = V.cpu().numpy()
    e1, f1, v1 = mdl.SeAEvaluator(params, atype, box, mode="compressed").compute(coord)
    # the same kernels; each row's FP32 energy gets one partial sum per
    # column tile of the output layer, added atomically in whatever order the
    # tiles finish, so the totals agree to FP32 rounding per row
    assert abs(E - e1) <= 1e-8 * nloc
    np.testing.assert_allclose(F, f1, atol=1e-9, rtol=0)
    np.testing.assert_allclose(V, v1, atol=1e-8 * max(1.0, np.abs(v1).max()), rtol=0)
    e0, f0, v0 = model_ref.evaluate(oracle.ref() or oracle.port(), params, coord, atype, box,
                                    mode="compressed")
    assert abs(E - e0) / nloc <= 1e-6
    assert float(np.sqrt(np.mean((F - f0) ** 2))) <= 1e-5
    # a second call on moved atoms (the engine's list is reused)
    cx2 = cx + 0.01 * torch.tensor(np.random.default_rng(1).normal(size=cx.shape), device=DEV)
    cx2[nloc:] = cx2[mx[nloc:].long()] + (cx[nloc:] - cx[mx[nloc:].long()])
    E2, _, _ = fl(cx2, tx, nloc, nn, fn)
    assert abs(float(E2.item()) - E) > 0.0


def test_compressed_model_from_reference_layout(dpb, mods):
    """A compressed model written in the reference's state-dict layout and
    read back runs on the compressed path with the same results."""
    wl, mdl, _, ck = mods
    coord, atype, box = wl.water_frame(4, seed=12)
    params = mdl.prepare(mdl.init_params(mdl.SeAConfig(), seed=1), coord, atype, box)
    sd = ck.params_to_state_dict(params)
    p2 = ck.load({"model": {"model.Default." + k: v for k, v in sd.items()}}, sel=(46, 92))
    e0, f0, v0 = mdl.SeAEvaluator(params, atype, box).compute(coord)
    e1, f1, v1 = mdl.SeAEvaluator(p2, atype, box).compute(coord)
    # the same model: equal up to the order of the FP32 energy partial sums
    # (added atomically) and of the FP64 force sums
    assert abs(e0 - e1) <= 1e-8 * abs(e0)
    np.testing.assert_allclose(f1, f0, rtol=0, atol=1e-9)
    np.testing.assert_allclose(v1, v0, rtol=0, atol=1e-8 * max(1.0, np.abs(v0).max()))
