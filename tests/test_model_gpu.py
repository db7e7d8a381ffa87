"""Energy/force/virial of the GPU evaluators against the reference model.

* plain FP64 path vs the reference PyTorch model: 1e-10 (FP64 bar);
* compressed FP32 path vs the FP64 oracle of the same compressed model: energy
  within 1e-6 eV/atom and force RMSE within 1e-5 eV/A (the north-star
  tolerances), virial within 1e-5 relative;
* CUDA-graph replay reproduces the eager step exactly.
"""

import importlib
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "model_golden.npz")


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLD) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def mdl(dpb):
    return importlib.import_module("deepmd_kit_lr_pt_b200.model")


def _params(mdl, gold, case, tables=True):
    tab = importlib.import_module("deepmd_kit_lr_pt_b200.table")
    cfg = mdl.SeAConfig()
    p = mdl.init_params(cfg, seed=int(gold["param_seed"]))
    p.davg, p.dstd = gold[f"{case}:davg"], gold[f"{case}:dstd"]
    if tables:
        p.tables = tab.build_tables(p.emb, p.davg, p.dstd, cfg.sel,
                                    float(gold[f"{case}:min_nbor_dist"]), cfg.rcut_smth, cfg.rcut)
    return p


@pytest.mark.parametrize("case", ["w24", "w192"])
def test_env_stats_gpu(mdl, gold, case):
    cfg = mdl.SeAConfig()
    p = mdl.init_params(cfg, seed=1)
    davg, dstd, mind = mdl.env_stats(p, gold[f"{case}:coord"], gold[f"{case}:atype"],
                                     gold[f"{case}:box"])
    np.testing.assert_allclose(davg, gold[f"{case}:davg"], atol=1e-12)
    np.testing.assert_allclose(dstd, gold[f"{case}:dstd"], atol=1e-12)
    assert abs(mind - float(gold[f"{case}:min_nbor_dist"])) < 1e-12


@pytest.mark.parametrize("case", ["w24", "w192"])
def test_plain_fp64_matches_reference_model(mdl, gold, case):
    p = _params(mdl, gold, case, tables=False)
    ev = mdl.SeAEvaluator(p, gold[f"{case}:atype"], gold[f"{case}:box"], mode="plain")
    E, F, V = ev.compute(gold[f"{case}:coord"])
    ev.check()
    assert abs(E - float(gold[f"{case}:energy"])) < 1e-10 * max(1.0, abs(float(gold[f"{case}:energy"])))
    np.testing.assert_allclose(F, gold[f"{case}:force"], atol=1e-10)
    np.testing.assert_allclose(V, gold[f"{case}:virial"], atol=1e-9)


@pytest.mark.parametrize("case", ["w24", "w192"])
def test_compressed_fp32_within_tolerance(mdl, gold, case):
    p = _params(mdl, gold, case)
    atype = gold[f"{case}:atype"]
    ev = mdl.SeAEvaluator(p, atype, gold[f"{case}:box"], mode="compressed")
    E, F, V = ev.compute(gold[f"{case}:coord"])
    ev.check()
    n = atype.size
    e_err = abs(E - float(gold[f"{case}:energy_c"])) / n
    f_rmse = float(np.sqrt(np.mean((F - gold[f"{case}:force_c"]) ** 2)))
    v_err = float(np.abs(V - gold[f"{case}:virial_c"]).max())
    print(f"{case}: |dE|/N {e_err:.2e} eV/atom, force RMSE {f_rmse:.2e} eV/A, |dV| {v_err:.2e}")
    assert e_err <= 1e-6
    assert f_rmse <= 1e-5
    assert v_err <= 1e-5 * max(1.0, float(np.abs(gold[f"{case}:virial_c"]).max()))


@pytest.mark.parametrize("mode", ["compressed", "plain"])
def test_graph_replay_equals_eager(mdl, gold, mode):
    p = _params(mdl, gold, "w192", tables=(mode == "compressed"))
    ev = mdl.SeAEvaluator(p, gold["w192:atype"], gold["w192:box"], mode=mode)
    coord = gold["w192:coord"]
    E0, F0, V0 = ev.compute(coord)
    ev.capture()
    rng = np.random.default_rng(0)
    E1, F1, V1 = ev.compute(coord)
    assert abs(E1 - E0) <= (1e-12 if mode == "plain" else 1e-6) * abs(E0)
    # new coordinates through the captured graph vs a fresh eager evaluator
    c2 = coord + rng.normal(scale=0.01, size=coord.shape)
    E2, F2, V2 = ev.compute(c2)
    ev2 = mdl.SeAEvaluator(p, gold["w192:atype"], gold["w192:box"], mode=mode)
    E3, F3, V3 = ev2.compute(c2)
    tol = 1e-12 if mode == "plain" else 1e-5
    assert abs(E2 - E3) <= tol * abs(E3)
    np.testing.assert_allclose(F2, F3, atol=tol * max(1.0, np.abs(F3).max()))
    # order of atomic adds differs between runs: results agree to rounding only
    np.testing.assert_allclose(V1, V0, rtol=1e-9 if mode == "plain" else 1e-5, atol=1e-9)


@pytest.mark.parametrize("mode", ["compressed", "plain"])
def test_run_pinned_equals_compute(mdl, gold, mode):
    """The one-graph evaluation from pinned host input to pinned host output
    (run_pinned) gives compute()'s results, for new coordinates written into
    its input buffer between calls."""
    p = _params(mdl, gold, "w192", tables=(mode == "compressed"))
    ev = mdl.SeAEvaluator(p, gold["w192:atype"], gold["w192:box"], mode=mode)
    hc, hr = ev.io_buffers()
    rng = np.random.default_rng(5)
    for k in range(3):
        c = gold["w192:coord"] + rng.normal(scale=0.01, size=gold["w192:coord"].shape) * k
        hc.copy_(torch.tensor(c))
        E, F, V = ev.run_pinned()
        E0, F0, V0 = ev.compute(c)
        tol = 1e-12 if mode == "plain" else 1e-6
        assert abs(float(E[0]) - E0) <= tol * abs(E0)
        np.testing.assert_allclose(F.numpy(), F0, atol=1e-9 if mode == "plain" else 1e-6)
        np.testing.assert_allclose(V.numpy(), V0, rtol=1e-9 if mode == "plain" else 1e-5,
                                   atol=1e-9)


def _quintic_close(a, b, rows, info, M):
    """a0..a2 to 1e-12 and the quintic to 1e-12 across each interval (a3..a5
    carry the cancellation of their formulas, divided by up to h^5)."""
    a, b = a.reshape(-1, M, 6), b.reshape(-1, M, 6)
    assert np.abs(a[:, :, :3] - b[:, :, :3]).max() <= 1e-12
    first = int((info[1] - info[0]) / info[3])
    h = np.where(rows < first, info[3], info[4])[:, None]
    for frac in (0.0, 0.37, 0.999):
        pw = np.stack([(h * frac) ** k for k in range(6)], -1)
        assert np.abs(((a - b) * pw).sum(-1)).max() <= 1e-12, frac


def test_device_tables_match_host_builder_and_reference(dpb):
    """dpb_se_a_build_table_f64 against the FP64 host builder (every row) and
    the reference compressor's rows (tests/golden/table_golden.npz)."""
    mdl = importlib.import_module("deepmd_kit_lr_pt_b200.model")
    tab = importlib.import_module("deepmd_kit_lr_pt_b200.table")
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    with np.load(os.path.join(here, "table_golden.npz")) as z:
        g = {k: z[k] for k in z.files}
    cfg = mdl.SeAConfig()
    p = mdl.init_params(cfg, seed=1)
    args = (p.emb, g["davg"], g["dstd"], cfg.sel, float(g["min_nbor_dist"]), cfg.rcut_smth,
            cfg.rcut)
    host = tab.build_tables(*args)
    dev = tab.build_tables_device(*args)
    M = cfg.neuron[-1]
    for t in range(cfg.ntypes):
        td, info = dev[t][0].cpu().numpy(), dev[t][1]
        np.testing.assert_array_equal(info, host[t][1])
        np.testing.assert_array_equal(info, g[f"net{t}:info"])
        assert td.shape == host[t][0].shape == tuple(g[f"net{t}:shape"])
        _quintic_close(td, host[t][0], np.arange(td.shape[0]), info, M)
        rows = g[f"net{t}:rows"]
        _quintic_close(td[rows], g[f"net{t}:table_rows"], rows, info, M)
