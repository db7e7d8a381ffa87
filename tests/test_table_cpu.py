"""Host side of the compression tables (table.py) on CPU: the cubic
re-interpolation used by the fused descriptor kernels against the quintic
table it is made from, its guard row and linear tail against the oracle's
tabulate beyond max, and the stride combinations it refuses. The tables are
built by the host builder on the water model's seeded weights with
statistics from the oracle."""

import importlib

import numpy as np
import pytest


@pytest.fixture(scope="module")
def tables(dpb):
    from oracle import model_ref, oracle

    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    tab = importlib.import_module("deepmd_kit_lr_pt_b200.table")
    cfg = wl.SeAConfig()
    p = wl.init_params(cfg, seed=1)
    coord, atype, box = wl.water_frame(4, seed=0)
    davg, dstd, mind = model_ref.env_stats(oracle.port(), cfg, coord, atype, box)
    return tab, tab.build_tables(p.emb, davg, dstd, cfg.sel, mind, cfg.rcut_smth, cfg.rcut)


def _quintic(T, info, first, xv):
    lower, upper, _, s0, s1 = info[:5]
    if xv >= upper:
        r = first + int((xv - upper) / s1)
        t = xv - (upper + (r - first) * s1)
    else:
        r = int((xv - lower) / s0)
        t = xv - (lower + r * s0)
    return sum(T[r, :, k] * t ** k for k in range(6))


def _cubic(C, ic, xv):
    K, h, lower = int(ic[5]), ic[3], ic[0]
    r = min(int((xv - lower) / h), K)
    t = xv - (lower + r * h)
    return C[r, 0] + t * (C[r, 1] + t * (C[r, 2] + t * C[r, 3]))


@pytest.mark.parametrize("m,tol", [(1, 1e-7), (2, 2e-6)])
def test_cubic_matches_quintic(tables, m, tol):
    """Within 1e-7 of |G| between the knots on the fine stride (2e-6 with
    knots every two fine strides), exact at the knots."""
    tab, tabs = tables
    rng = np.random.default_rng(m)
    for table, info in tabs:
        C, ic = tab.cubic_table(table, info, m)
        lower, upper, mx, s0, s1 = info[:5]
        M = table.shape[1] // 6
        T = table.reshape(-1, M, 6)
        first = int(round((upper - lower) / s0))
        K = int(ic[5])
        assert C.shape == (K + 1, 4, M) and ic[1] == mx and abs(ic[3] - s0 * m) < 1e-15
        assert K * m == first + int(round((mx - upper) / s1)) * int(round(s1 / s0))
        for xv in np.concatenate([rng.uniform(lower, upper, 200), rng.uniform(upper, mx, 200)]):
            q = _quintic(T, info, first, xv)
            assert np.abs(_cubic(C, ic, xv) - q).max() <= tol * max(1.0, np.abs(q).max()), xv
        # knots: the quintic's value and slope exactly
        for k in rng.integers(0, first // m, 20):
            np.testing.assert_array_equal(C[k, 0], T[k * m, :, 0])
            np.testing.assert_array_equal(C[k, 1], T[k * m, :, 1])


def test_cubic_guard_row_and_tail(tables, port):
    """The guard row holds the value and slope at max, and beyond max the
    cubic path's linear tail equals the quintic table's C1 tail as the
    oracle's tabulate evaluates it (one neighbor, em = (1, 0, 0, 0))."""
    tab, tabs = tables
    table, info = tabs[0]
    C, ic = tab.cubic_table(table, info, 1)
    K, mx = int(ic[5]), float(info[2])
    M = table.shape[1] // 6
    np.testing.assert_array_equal(C[K, 2:], 0.0)
    em = np.array([[[1.0, 0.0, 0.0, 0.0]]])
    for xv in (mx, mx + 0.37, mx + 3.0):
        q = port.tabulate(table, info, np.array([[xv]]), em, M).reshape(4, M)[0]
        c = C[K, 0] + C[K, 1] * (xv - mx)
        assert np.abs(c - q).max() <= 1e-9 * max(1.0, np.abs(q).max()), xv


def test_cubic_refuses_strides_that_do_not_nest(tables):
    tab, tabs = tables
    table, info = tabs[0]
    bad = info.copy()
    bad[4] = 0.15  # stride1 not a whole multiple of stride0
    assert tab.cubic_table(table, bad, 1) is None
    assert tab.cubic_table(table, info, 3) is None  # 3 divides neither 10 nor the fine count
    assert tab.cubic_table(table[:-1], info, 1) is None  # row count off the grid
