"""Pins the FP64 energy/force/virial oracle (oracle/model_ref.py) against the
reference's own PyTorch model (tests/golden/model_golden.npz), and checks the
product's host-side model pieces that run without a GPU (seeded weights, FP64
table builder)."""

import importlib
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "model_golden.npz")


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLD) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def mdl(dpb):
    return importlib.import_module("deepmd_kit_lr_pt_b200.model")


@pytest.fixture(scope="module")
def tab(dpb):
    return importlib.import_module("deepmd_kit_lr_pt_b200.table")


def _params(mdl, tab, gold, case):
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_model_golden import weight_checksum

    cfg = mdl.SeAConfig()
    p = mdl.init_params(cfg, seed=int(gold["param_seed"]))
    assert abs(weight_checksum(p) - float(gold["weight_checksum"])) < 1e-9
    p.davg, p.dstd = gold[f"{case}:davg"], gold[f"{case}:dstd"]
    p.tables = tab.build_tables(p.emb, p.davg, p.dstd, cfg.sel, float(gold[f"{case}:min_nbor_dist"]),
                                cfg.rcut_smth, cfg.rcut)
    return p


@pytest.mark.parametrize("case", ["w24", "w192"])
def test_oracle_matches_reference_model(port, mdl, tab, gold, case):
    from oracle import model_ref

    p = _params(mdl, tab, gold, case)
    coord, atype, box = gold[f"{case}:coord"], gold[f"{case}:atype"], gold[f"{case}:box"]
    E, F, V = model_ref.evaluate(port, p, coord, atype, box, mode="plain")
    assert abs(E - float(gold[f"{case}:energy"])) < 1e-10
    np.testing.assert_allclose(F, gold[f"{case}:force"], atol=1e-10)
    np.testing.assert_allclose(V, gold[f"{case}:virial"], atol=1e-9)


def test_oracle_stats_match_golden(port, mdl, gold):
    from oracle import model_ref

    cfg = mdl.SeAConfig()
    davg, dstd, mind = model_ref.env_stats(port, cfg, gold["w192:coord"], gold["w192:atype"],
                                           gold["w192:box"])
    np.testing.assert_allclose(davg, gold["w192:davg"], atol=1e-12)
    np.testing.assert_allclose(dstd, gold["w192:dstd"], atol=1e-12)
    assert abs(mind - float(gold["w192:min_nbor_dist"])) < 1e-12


def test_compressed_fp64_close_to_plain(port, mdl, tab, gold):
    """The FP64 quintic table reproduces the MLP to ~1e-12 on this model."""
    from oracle import model_ref

    p = _params(mdl, tab, gold, "w24")
    coord, atype, box = gold["w24:coord"], gold["w24:atype"], gold["w24:box"]
    E, F, V = model_ref.evaluate(port, p, coord, atype, box, mode="compressed")
    assert abs(E - float(gold["w24:energy"])) < 1e-9
    np.testing.assert_allclose(F, gold["w24:force"], atol=1e-9)


def test_table_reproduces_embedding(mdl, tab):
    """Table value at random x vs the FP64 MLP (Hermite quintic interpolation)."""
    cfg = mdl.SeAConfig()
    p = mdl.init_params(cfg, seed=3)
    davg = np.zeros((2, cfg.nnei * 4))
    dstd = np.ones((2, cfg.nnei * 4))
    davg[:, 0::4] = 0.1
    dstd[:, 0::4] = 0.3
    (t0, info), _ = tab.build_tables(p.emb, davg, dstd, cfg.sel, 0.95, cfg.rcut_smth, cfg.rcut)
    x = np.random.default_rng(0).uniform(info[0], info[2] * 0.999, size=200)
    ref, _, _ = tab.embedding_derivatives(p.emb[0], x)
    first = int((info[1] - info[0]) / info[3])
    for k, xv in enumerate(x):
        if xv < info[1]:
            idx = int((xv - info[0]) / info[3])
            tt = xv - (idx * info[3] + info[0])
        else:
            idx = first + int((xv - info[1]) / info[4])
            tt = xv - ((idx - first) * info[4] + info[1])
        c = t0[idx].reshape(-1, 6)
        val = c[:, 0] + (c[:, 1] + (c[:, 2] + (c[:, 3] + (c[:, 4] + c[:, 5] * tt) * tt) * tt) * tt) * tt
        np.testing.assert_allclose(val, ref[k], atol=1e-7)


def test_tables_match_reference_compressor(mdl, tab):
    """The FP64 table builder against the reference's own compressor
    (tests/golden/table_golden.npz, made by enable_compression of the
    reference se_a descriptor on the same weights and statistics): identical
    table_info and shape, coefficients a0..a2 to 1e-12, a3..a5 within the
    cancellation their formulas amplify (differences of values divided by up to
    h^5 = 1e-10), and the polynomial itself to 1e-12 across each interval."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_model_golden import weight_checksum

    with np.load(os.path.join(os.path.dirname(GOLD), "table_golden.npz")) as z:
        g = {k: z[k] for k in z.files}
    cfg = mdl.SeAConfig()
    p = mdl.init_params(cfg, seed=1)
    assert abs(weight_checksum(p) - float(g["weight_checksum"])) < 1e-9
    tables = tab.build_tables(p.emb, g["davg"], g["dstd"], cfg.sel, float(g["min_nbor_dist"]),
                              cfg.rcut_smth, cfg.rcut)
    M = cfg.neuron[-1]
    tol = [1e-12, 1e-12, 1e-12, 1e-6, 1e-4, 2e-3]
    for t, (table, info) in enumerate(tables):
        np.testing.assert_array_equal(info, g[f"net{t}:info"])
        assert tuple(table.shape) == tuple(g[f"net{t}:shape"])
        rows = g[f"net{t}:rows"]
        mine, ref = table[rows].reshape(-1, M, 6), g[f"net{t}:table_rows"].reshape(-1, M, 6)
        for k in range(6):
            err = np.abs(mine[:, :, k] - ref[:, :, k]).max()
            assert err <= tol[k], (t, k, err)
        first = int((info[1] - info[0]) / info[3])
        h = np.where(rows < first, info[3], info[4])[:, None]  # [rows, 1]
        for frac in (0.0, 0.37, 0.999):
            x = h * frac
            pw = np.stack([x ** k for k in range(6)], -1)
            assert np.abs(((mine - ref) * pw).sum(-1)).max() <= 1e-12, (t, frac)


def test_oracle_table_builder_matches_reference_compressor(mdl):
    """The oracle's restatement of the reference compressor (used by the
    benchmark's reference arm instead of the product's builder) against the
    compressor's own output, with the bars of the product builder's test."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_model_golden import weight_checksum

    from oracle import table_ref

    with np.load(os.path.join(os.path.dirname(GOLD), "table_golden.npz")) as z:
        g = {k: z[k] for k in z.files}
    cfg = mdl.SeAConfig()
    p = mdl.init_params(cfg, seed=1)
    assert abs(weight_checksum(p) - float(g["weight_checksum"])) < 1e-9
    tables = table_ref.build_tables(p.emb, g["davg"], g["dstd"], cfg.sel,
                                    float(g["min_nbor_dist"]), cfg.rcut_smth, cfg.rcut)
    M = cfg.neuron[-1]
    tol = [1e-12, 1e-12, 1e-12, 1e-6, 1e-4, 2e-3]
    for t, (table, info) in enumerate(tables):
        np.testing.assert_array_equal(info, g[f"net{t}:info"])
        assert tuple(table.shape) == tuple(g[f"net{t}:shape"])
        rows = g[f"net{t}:rows"]
        mine, ref = table[rows].reshape(-1, M, 6), g[f"net{t}:table_rows"].reshape(-1, M, 6)
        for k in range(6):
            assert np.abs(mine[:, :, k] - ref[:, :, k]).max() <= tol[k], (t, k)
        first = int((info[1] - info[0]) / info[3])
        h = np.where(rows < first, info[3], info[4])[:, None]
        for frac in (0.0, 0.37, 0.999):
            pw = np.stack([(h * frac) ** k for k in range(6)], -1)
            assert np.abs(((mine - ref) * pw).sum(-1)).max() <= 1e-12, (t, frac)
