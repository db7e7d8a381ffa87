"""FP64 construction of the compressed-embedding tables (model compression).

For each embedding net (one per neighbor type with type_one_side), the net
output G(x) in R^M and its first two derivatives are evaluated in FP64 on a
grid of x = normalized s(r)/r values, and each interval [x_r, x_r + h) is
replaced by the quintic Hermite polynomial that matches value, slope and
curvature at both ends. Row r of the table holds, for every channel m, the six
coefficients (ascending powers of t = x - x_r) at columns 6m..6m+5: the layout
the tabulate kernels read (source/lib/src/tabulate.cc:190-197).

Grid and bounds follow the reference compressor (deepmd/utils/tabulate.py:
67-152, 468-486): lower = floor(min_t(-davg_t / dstd_t)), upper =
ceil(max_t((s(r_min)/r_min - davg_t) / dstd_t)) over the radial column, stride0
on [lower, upper), stride1 on [upper, extrapolate * upper), and
table_info = [lower, upper, extrapolate * upper, stride0, stride1, -1]
(deepmd/pt/model/descriptor/se_a.py:725-734).
"""

from __future__ import annotations

import numpy as np


def spline5_switch(x: float, rmin: float, rmax: float) -> float:
    if x < rmin:
        return 1.0
    if x < rmax:
        u = (x - rmin) / (rmax - rmin)
        return u * u * u * (-6 * u * u + 15 * u - 10) + 1
    return 0.0


def embedding_derivatives(layers, x: np.ndarray):
    """Value, first and second x-derivatives of a tanh embedding net.

    ``layers`` is a list of (W [n_in, n_out], b [n_out]); a layer adds a
    residual when n_out == n_in (x) or n_out == 2 n_in ([x, x])
    (deepmd/dpmodel/utils/network.py:282-330). Forward-mode chain rule in FP64.
    """
    y = np.asarray(x, np.float64).reshape(-1, 1)
    dy = np.ones_like(y)
    d2y = np.zeros_like(y)
    for W, b in layers:
        W = np.asarray(W, np.float64)
        z = y @ W + b
        t = np.tanh(z)
        s = 1.0 - t * t  # tanh'
        dz = dy @ W
        d2z = d2y @ W
        ny = t
        ndy = s * dz
        nd2y = s * d2z - 2.0 * t * s * dz * dz
        n_in, n_out = W.shape
        if n_out == n_in:
            ny, ndy, nd2y = ny + y, ndy + dy, nd2y + d2y
        elif n_out == 2 * n_in:
            ny = ny + np.concatenate([y, y], 1)
            ndy = ndy + np.concatenate([dy, dy], 1)
            nd2y = nd2y + np.concatenate([d2y, d2y], 1)
        y, dy, d2y = ny, ndy, nd2y
    return y, dy, d2y


def hermite_quintic(xx: np.ndarray, vv, dd, d2, nspline: int, steps: np.ndarray) -> np.ndarray:
    """Coefficients [nspline, 6M] of the quintic matching (v, v', v'') at both
    ends of every interval; ``steps`` is the interval width per row."""
    M = vv.shape[1]
    h = steps[:, None]
    y0, y1 = vv[:nspline], vv[1:nspline + 1]
    g0, g1 = dd[:nspline], dd[1:nspline + 1]
    c0, c1 = d2[:nspline], d2[1:nspline + 1]
    dv = y1 - y0
    out = np.zeros((nspline, 6 * M))
    out[:, 0::6] = y0
    out[:, 1::6] = g0
    out[:, 2::6] = 0.5 * c0
    out[:, 3::6] = (20 * dv - (8 * g1 + 12 * g0) * h - (3 * c0 - c1) * h * h) / (2 * h**3)
    out[:, 4::6] = (-30 * dv + (14 * g1 + 16 * g0) * h + (3 * c0 - 2 * c1) * h * h) / (2 * h**4)
    out[:, 5::6] = (12 * dv - 6 * (g1 + g0) * h + (c1 - c0) * h * h) / (2 * h**5)
    return out


def env_range(davg: np.ndarray, dstd: np.ndarray, min_nbor_dist: float, rcut_smth: float,
              rcut: float):
    """Per center type (lower, upper) of the normalized radial input."""
    sw = spline5_switch(min_nbor_dist, rcut_smth, rcut)
    a0 = davg.reshape(davg.shape[0], -1, 4)[:, 0, 0]
    s0 = dstd.reshape(dstd.shape[0], -1, 4)[:, 0, 0]
    lower = np.floor(-a0 / s0)
    upper = np.ceil(((1.0 / min_nbor_dist) * sw - a0) / s0)
    return lower, upper


def build_tables(emb_layers, davg, dstd, sel, min_nbor_dist: float, rcut_smth: float,
                 rcut: float, extrapolate: float = 5.0, stride0: float = 0.01,
                 stride1: float = 0.1):
    """One FP64 table per neighbor type (type_one_side).

    Returns a list of (table [nspline, 6M] float64, info [6] float64)."""
    lower, upper = env_range(davg, dstd, min_nbor_dist, rcut_smth, rcut)
    ntypes = len(sel)
    valid = [t for t in range(ntypes) if sel[t] > 0]
    out = []
    for net in range(len(emb_layers)):
        uu = float(np.max(upper[valid]))
        ll = float(np.min(lower[valid]))
        xx = np.arange(ll, uu, stride0, dtype=np.float64)
        xx = np.append(xx, np.arange(uu, extrapolate * uu, stride1, dtype=np.float64))
        xx = np.append(xx, np.array([extrapolate * uu]))
        nspline = int((uu - ll) / stride0 + (extrapolate * uu - uu) / stride1)
        vv, dd, d2 = embedding_derivatives(emb_layers[net], xx)
        steps = np.full(nspline, stride1)
        steps[: int((uu - ll) / stride0)] = stride0
        table = hermite_quintic(xx, vv, dd, d2, nspline, steps)
        info = np.array([int(ll), int(uu), int(uu) * extrapolate, stride0, stride1, -1.0])
        out.append((table, info))
    return out
