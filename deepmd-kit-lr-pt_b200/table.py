"""FP64 construction of the compressed-embedding tables (model compression).

For each embedding net (one per neighbor type with type_one_side), the net
output G(x) in R^M and its first two derivatives are evaluated in FP64 on a
grid of x = normalized s(r)/r values, and each interval [x_r, x_r + h) is
replaced by the quintic Hermite polynomial that matches value, slope and
curvature at both ends. Row r of the table holds, for every channel m, the six
coefficients (ascending powers of t = x - x_r) at columns 6m..6m+5: the layout
the tabulate kernels read (source/lib/src/tabulate.cc:190-197).

Grid and bounds follow the reference compressor (deepmd/utils/tabulate.py:
67-152, 468-486): lower / upper from the four normalised columns of the
first slot (floor of -davg/dstd, ceil of (s(r_min)/r_min - davg)/dstd, min /
max over columns and types), stride0 on [lower, upper), stride1 on
[upper, extrapolate * upper), and
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
    """Per center type (lower, upper) of the normalized table input.

    As the reference compressor does for se_a (deepmd/utils/tabulate.py:
    468-486 with the descriptor's statistics shaped [ntypes, nnei, 4], then
    :94-96): the bounds are taken over the four columns of the first slot,
    (0 - davg) / dstd and (s(r_min)/r_min - davg) / dstd, floored / ceiled
    per column, then the minimum / maximum over the columns; the angular
    columns (davg 0, their own dstd) usually set the upper bound."""
    sw = spline5_switch(min_nbor_dist, rcut_smth, rcut)
    a0 = davg.reshape(davg.shape[0], -1, 4)[:, 0, :]
    s0 = dstd.reshape(dstd.shape[0], -1, 4)[:, 0, :]
    lower = np.floor(-a0 / s0).min(axis=1)
    upper = np.ceil(((1.0 / min_nbor_dist) * sw - a0) / s0).max(axis=1)
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
        xx, steps, nspline = _grid(ll, uu, extrapolate, stride0, stride1)
        vv, dd, d2 = embedding_derivatives(emb_layers[net], xx)
        table = hermite_quintic(xx, vv, dd, d2, nspline, steps)
        info = np.array([int(ll), int(uu), int(uu) * extrapolate, stride0, stride1, -1.0])
        out.append((table, info))
    return out


def _grid(ll: float, uu: float, extrapolate: float, stride0: float, stride1: float):
    """The compressor's x grid, interval widths and row count
    (deepmd/utils/tabulate.py:135-147)."""
    xx = np.arange(ll, uu, stride0, dtype=np.float64)
    xx = np.append(xx, np.arange(uu, extrapolate * uu, stride1, dtype=np.float64))
    xx = np.append(xx, np.array([extrapolate * uu]))
    nspline = int((uu - ll) / stride0 + (extrapolate * uu - uu) / stride1)
    steps = np.full(nspline, stride1)
    steps[: int((uu - ll) / stride0)] = stride0
    return xx, steps, nspline


def build_tables_device(emb_layers, davg, dstd, sel, min_nbor_dist: float, rcut_smth: float,
                        rcut: float, device="cuda:0", extrapolate: float = 5.0,
                        stride0: float = 0.01, stride1: float = 0.1):
    """build_tables on the GPU (dpb_se_a_build_table_f64): the same grid and
    table_info, the embedding-net derivatives and the Hermite coefficients in
    FP64 on the device. Returns a list of (table [nspline, 6M] FP64 device
    tensor, info [6] numpy) per neighbor type."""
    import ctypes

    import torch

    from . import _capi

    dev = torch.device(device)
    lower, upper = env_range(davg, dstd, min_nbor_dist, rcut_smth, rcut)
    valid = [t for t in range(len(sel)) if sel[t] > 0]
    uu = float(np.max(upper[valid]))
    ll = float(np.min(lower[valid]))
    xx, steps, nspline = _grid(ll, uu, extrapolate, stride0, stride1)
    x_d = torch.tensor(xx, dtype=torch.float64, device=dev)
    s_d = torch.tensor(steps, dtype=torch.float64, device=dev)
    info = np.array([int(ll), int(uu), int(uu) * extrapolate, stride0, stride1, -1.0])
    out = []
    for net in emb_layers:
        Ws = [torch.tensor(np.asarray(W, np.float64), device=dev).contiguous() for W, _ in net]
        bs = [torch.tensor(np.asarray(b, np.float64), device=dev).contiguous() for _, b in net]
        widths = np.array([1] + [int(W.shape[1]) for W, _ in net], np.int32)
        M = int(widths[-1])
        sbytes = int(_capi.lib().dpb_se_a_build_table_scratch_bytes(xx.size, M))
        scratch = torch.empty(sbytes, dtype=torch.uint8, device=dev)
        table = torch.empty((nspline, 6 * M), dtype=torch.float64, device=dev)
        wp = (ctypes.c_void_p * len(Ws))(*[w.data_ptr() for w in Ws])
        bp = (ctypes.c_void_p * len(bs))(*[b.data_ptr() for b in bs])
        _capi.call("dpb_se_a_build_table_f64", _capi.ptr(table), _capi.ptr(x_d), _capi.ptr(s_d),
                   xx.size, nspline, wp, bp, widths.ctypes.data, len(net), _capi.ptr(scratch),
                   sbytes, torch.cuda.current_stream(dev).cuda_stream)
        torch.cuda.synchronize(dev)
        out.append((table, info.copy()))
    return out



def cubic_table(table: np.ndarray, info: np.ndarray, stride_mult: int = 1):
    """The compressed embedding of one table re-interpolated by a cubic
    Hermite polynomial on the fine stride everywhere, for the fused
    descriptor kernels (dpb_se_a_descriptor_*_cubic_f32): the quintic rows
    give the value and slope at every knot x_k = lower + k stride0 (the
    knots of the stride1 rows at k / (stride1 / stride0) of their interval),
    and each interval [x_k, x_k + h) gets the cubic matching both ends,
        c0 = y0, c1 = d0, c2 = (3 (y1 - y0) / h - 2 d0 - d1) / h,
        c3 = (2 (y0 - y1) / h + d0 + d1) / h^2.
    The difference to the quintic is the cubic Hermite remainder
    h^4 / 384 |G''''| (about 1e-8 of |G| for the water model's nets, below
    FP32 resolution); loading 4 coefficients per channel instead of 6 cuts
    the table bytes every neighbor slot gathers by a third.

    With stride_mult m > 1 the knots are every m fine strides (h = m
    stride0; m must divide both the fine-region knot count and stride1 /
    stride0): half or fewer table rows, at an interpolation error m^4 times
    larger.

    Returns (coefficients [K + 1, 4, M] float64, coefficient-major rows with
    a last guard row [y(max), y'(max), 0, 0] for the linear extrapolation
    beyond max; info [lower, max, max, h, h, K]), or None when the strides do
    not nest (stride1 not a whole multiple of stride0, or not of h)."""
    lower, upper, mx, s0, s1 = (float(v) for v in info[:5])
    first = int(round((upper - lower) / s0))
    ratio = int(round(s1 / s0))
    n1 = int(round((mx - upper) / s1))
    M = table.shape[1] // 6
    m = int(stride_mult)
    if (ratio < 1 or abs(ratio * s0 - s1) > 1e-9 * s1 or abs(first * s0 - (upper - lower)) >
            1e-9 * max(1.0, abs(upper - lower)) or first + n1 != table.shape[0] or m < 1 or
            first % m or ratio % m):
        return None
    T = np.asarray(table, np.float64).reshape(-1, M, 6)
    K = first + n1 * ratio
    y = np.empty((K + 1, M))
    d = np.empty((K + 1, M))
    y[:first] = T[:first, :, 0]
    d[:first] = T[:first, :, 1]

    def poly(c, t):
        v = c[..., 5]
        g = 5.0 * c[..., 5]
        for p in range(4, -1, -1):
            v = v * t + c[..., p]
        for p in range(4, 0, -1):
            g = g * t + p * c[..., p]
        return v, g

    for j in range(ratio):
        v, g = poly(T[first:first + n1], j * s0)
        y[first + j:K:ratio] = v
        d[first + j:K:ratio] = g
    y[K], d[K] = poly(T[-1], s1)
    if m > 1:  # every m-th knot
        y, d, K = y[::m], d[::m], K // m
    h = s0 * m
    C = np.zeros((K + 1, 4, M))
    C[:K, 0] = y[:K]
    C[:K, 1] = d[:K]
    C[:K, 2] = (3.0 * (y[1:] - y[:K]) / h - 2.0 * d[:K] - d[1:]) / h
    C[:K, 3] = (2.0 * (y[:K] - y[1:]) / h + d[:K] + d[1:]) / (h * h)
    C[K, 0] = y[K]
    C[K, 1] = d[K]
    return C, np.array([lower, mx, mx, h, h, float(K)])
