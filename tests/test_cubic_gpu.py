"""The cubic re-interpolation of the compression tables in the fused
descriptor kernels (table_degree=3) against the reference's quintic table
(table_degree=5) on the same frames: the descriptor, its gradient and the
energy / force / virial agree to FP32 resolution (the cubic Hermite
remainder is about 1e-8 of the embedding values; the bar is 1e-6 relative
for xyz / D / net_deriv, and the path's tolerances against FP64 for E/F/V)."""

import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(dpb):
    imp = importlib.import_module
    return (imp("deepmd_kit_lr_pt_b200.workload"), imp("deepmd_kit_lr_pt_b200.model"),
            imp("deepmd_kit_lr_pt_b200.table"), imp("deepmd_kit_lr_pt_b200.batch"))


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(1e-30, np.abs(b).max()))


@pytest.mark.parametrize("m,tol", [(1, 1e-7), (2, 2e-6)])
def test_cubic_table_matches_quintic_on_host(mods, m, tol):
    """table.cubic_table reproduces the quintic's value and slope at every
    knot exactly and stays within 1e-7 of |G| between knots on the fine
    stride (2e-6 with knots every two fine strides) (FP64, host)."""
    wl, mdl, tab, _ = mods
    coord, atype, box = wl.water_frame(4, seed=0)
    p = mdl.prepare(mdl.init_params(mdl.SeAConfig(), seed=1), coord, atype, box)
    rng = np.random.default_rng(0)
    for table, info in p.tables:
        C, ic = tab.cubic_table(table, info, m)
        lower, upper, mx, s0, s1 = info[:5]
        M = table.shape[1] // 6
        T = table.reshape(-1, M, 6)
        first = int(round((upper - lower) / s0))
        K = int(ic[5])
        h = s0 * m
        assert C.shape == (K + 1, 4, M) and ic[1] == mx and abs(ic[3] - h) < 1e-15
        x = np.concatenate([rng.uniform(lower, upper, 300), rng.uniform(upper, mx, 300)])
        for xv in x:
            r = first + int((xv - upper) / s1) if xv >= upper else int((xv - lower) / s0)
            t = xv - (upper + (r - first) * s1 if xv >= upper else lower + r * s0)
            q = sum(T[r, :, k] * t ** k for k in range(6))
            rc = min(int((xv - lower) / h), K)
            tc = xv - (lower + rc * h)
            c = C[rc, 0] + tc * (C[rc, 1] + tc * (C[rc, 2] + tc * C[rc, 3]))
            assert np.abs(c - q).max() <= tol * max(1.0, np.abs(q).max()), xv


def test_cubic_descriptor_matches_quintic(mods):
    wl, mdl, _, _ = mods
    coord, atype, box = wl.water_frame(6, seed=4)
    p = mdl.prepare(mdl.init_params(mdl.SeAConfig(), seed=1), coord, atype, box)
    ev5 = mdl.SeAEvaluator(p, atype, box, table_degree=5)
    ev3 = mdl.SeAEvaluator(p, atype, box, table_degree=3)
    e5, f5, v5 = ev5.compute(coord)
    e3, f3, v3 = ev3.compute(coord)
    ev3.check()
    assert _rel(ev3.xyz.cpu(), ev5.xyz.cpu()) < 1e-6
    assert _rel(ev3.D.cpu(), ev5.D.cpu()) < 1e-6
    assert _rel(ev3.net_deriv.cpu(), ev5.net_deriv.cpu()) < 1e-5
    n = atype.size
    assert abs(e3 - e5) / n < 1e-7
    assert float(np.sqrt(np.mean((f3 - f5) ** 2))) < 1e-7


def test_cubic_batched_and_extrapolation(mods):
    """Batched water / Cu frames, one atom pair squeezed below the table's
    minimum distance (the extrapolated region past max): degree 3 against
    degree 5."""
    wl, mdl, _, bt = mods
    rng = np.random.default_rng(3)
    frames = [wl.water_frame_density(200, rng), wl.cu_frame(256, rng)]
    cfg = mdl.SeAConfig(sel=(46, 92, 60))
    p = mdl.prepare_frames(mdl.init_params(cfg, seed=2), frames)
    c0 = frames[0][0].copy()
    c0[1] = c0[0] + (c0[1] - c0[0]) * 0.35  # an O-H at ~0.33 A
    frames[0] = (c0, frames[0][1], frames[0][2])
    out = {}
    for deg in (5, 3):
        ev = bt.BatchEvaluator(p, frames, table_degree=deg)
        out[deg] = ev.compute()
        ev.check()
    (E5, F5, V5), (E3, F3, V3) = out[5], out[3]
    np.testing.assert_allclose(E3, E5, rtol=1e-7, atol=1e-6)
    assert float(np.sqrt(np.mean((F3 - F5) ** 2))) < 1e-6
    np.testing.assert_allclose(V3, V5, rtol=1e-6, atol=1e-5)
