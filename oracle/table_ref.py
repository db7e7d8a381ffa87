"""Test infrastructure only: the reference compressor's table build in numpy.

A CPU restatement of DPTabulate for se_e2_a with type_one_side (the checker
side of the FP64 table build; the product builds its tables on the device):

* bounds: deepmd/utils/tabulate.py:468-486 (_get_env_mat_range: floor/ceil
  of the normalised first slot, taken per column of the statistics shaped
  [ntypes, nnei, 4]), then :94-96 (min/max over the trailing axes) and
  :115-125 (min/max over the neighbor types whose sel is non-zero);
* grid: :126-137 (stride0 on [lower, upper), stride1 on
  [upper, extrapolate * upper), the end point, nspline);
* embedding-net value and derivatives: deepmd/utils/tabulate_math.py:353-470
  (_make_data) with the chain-rule helpers :136-262 for tanh;
* Hermite quintic coefficients: deepmd/utils/tabulate.py:275-371
  (_build_lower);
* table_info: deepmd/pt/model/descriptor/se_a.py:722-734 with the bounds
  converted to int (tabulate.py:463-466).

Pinned by tests/golden/table_golden.npz (the reference compressor's own
output on the seeded model). Only tests and the reference arm of bench.py
use it.
"""

from __future__ import annotations

import numpy as np


def _switch(x: float, rmin: float, rmax: float) -> float:
    """deepmd/utils/tabulate.py:488-499 (_spline5_switch)."""
    if x < rmin:
        return 1.0
    if x < rmax:
        u = (x - rmin) / (rmax - rmin)
        return u * u * u * (-6 * u * u + 15 * u - 10) + 1
    return 0.0


def env_mat_range(davg, dstd, min_nbor_dist, rcut_smth, rcut):
    """Per-type (lower, upper) as ints of the table input range."""
    nt = davg.shape[0]
    a = np.asarray(davg, np.float64).reshape(nt, -1, 4)[:, 0]
    s = np.asarray(dstd, np.float64).reshape(nt, -1, 4)[:, 0]
    sw = _switch(min_nbor_dist, rcut_smth, rcut)
    lower = np.floor(-a / s).min(axis=1)
    upper = np.ceil(((1.0 / min_nbor_dist) * sw - a) / s).max(axis=1)
    return lower, upper


def net_values(layers, xx):
    """(y, dy/dx, d2y/dx2) of a tanh embedding net on the column xx, layer by
    layer as _make_data propagates them (first layer: scalar input)."""
    x = np.asarray(xx, np.float64).reshape(-1, 1)
    y = dy = d2 = None
    for k, (W, b) in enumerate(layers):
        W = np.asarray(W, np.float64)
        b = np.asarray(b, np.float64)
        n_in, n_out = W.shape
        if k == 0:
            t = np.tanh(x @ W + b)
            g = 1.0 - t * t                  # tanh'
            gg = -2.0 * t * g                # tanh''
            w = W.reshape(-1)[:n_out][None, :]
            ny, ndy, nd2 = t, g * w, gg * w * w
            if n_out == 1:
                ny, ndy = ny + x, ndy + 1.0
            elif n_out == 2:
                ny, ndy = ny + np.concatenate([x, x], 1), ndy + 1.0
        else:
            t = np.tanh(y @ W + b)
            g = 1.0 - t * t
            gg = -2.0 * t * g
            a1 = dy @ W
            ny, ndy, nd2 = t, g * a1, g * (d2 @ W) + gg * a1 * a1
            if n_out == n_in:
                ny, ndy, nd2 = ny + y, ndy + dy, nd2 + d2
            elif n_out == 2 * n_in:
                ny = ny + np.concatenate([y, y], 1)
                ndy = ndy + np.concatenate([dy, dy], 1)
                nd2 = nd2 + np.concatenate([d2, d2], 1)
        y, dy, d2 = ny, ndy, nd2
    return y, dy, d2


def build_tables(emb_layers, davg, dstd, sel, min_nbor_dist, rcut_smth, rcut,
                 extrapolate=5.0, stride0=0.01, stride1=0.1):
    """[(table [nspline, 6M] float64, table_info [6] float64)] per neighbor
    type's embedding net."""
    lower, upper = env_mat_range(davg, dstd, min_nbor_dist, rcut_smth, rcut)
    keep = np.array([s > 0 for s in sel])
    uu = float(np.max(upper[keep]))
    ll = float(np.min(lower[keep]))
    xx = np.arange(ll, uu, stride0, dtype=np.float64)
    xx = np.append(xx, np.arange(uu, extrapolate * uu, stride1, dtype=np.float64))
    xx = np.append(xx, np.array([extrapolate * uu]))
    nspline = int((uu - ll) / stride0 + (extrapolate * uu - uu) / stride1)
    out = []
    for layers in emb_layers:
        vv, dd, d2 = net_values(layers, xx)
        M = vv.shape[1]
        tt = np.full((nspline, M), stride1)
        tt[: int((uu - ll) / stride0), :] = stride0
        hh = vv[1:nspline + 1] - vv[:nspline]
        d0, d1 = dd[:nspline], dd[1:nspline + 1]
        c0, c1 = d2[:nspline], d2[1:nspline + 1]
        tab = np.zeros((nspline, 6 * M))
        tab[:, 0::6] = vv[:nspline]
        tab[:, 1::6] = d0
        tab[:, 2::6] = 0.5 * c0
        tab[:, 3::6] = (1 / (2 * tt ** 3)) * (20 * hh - (8 * d1 + 12 * d0) * tt
                                              - (3 * c0 - c1) * tt * tt)
        tab[:, 4::6] = (1 / (2 * tt ** 4)) * (-30 * hh + (14 * d1 + 16 * d0) * tt
                                              + (3 * c0 - 2 * c1) * tt * tt)
        tab[:, 5::6] = (1 / (2 * tt ** 5)) * (12 * hh - 6 * (d1 + d0) * tt
                                              + (c1 - c0) * tt * tt)
        info = np.array([int(ll), int(uu), int(uu) * extrapolate, stride0, stride1, -1.0])
        out.append((tab, info))
    return out
