"""Split-TF32 tensor-core GEMM (dpb_gemm_tf32x3_f32: 3 TF32 products per k
step by default, 4 with the fit_terms knob) and the fitting networks built
on it, against FP64 references. The split keeps FP32-level accuracy: relative
errors of a few 1e-6 on these sizes; the bar is 2e-5 relative to the output
scale (the FP32 bar of the reference tests is 1e-5 absolute on O(1) values)."""

import ctypes
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(scope="module")
def mdl(dpb):
    return importlib.import_module("deepmd_kit_lr_pt_b200.model")


def _ptrs(ts):
    return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


def _run(dpb, mdl, A, Bs, type_rows, mode, aux0=None, aux1=None, bias=None, idt=None, w=None,
         split_in_kernel=False):
    M, K = A.shape
    N = Bs[0].shape[0]
    if split_in_kernel:  # FP32 weights, b_lo = NULL: the kernel splits them
        th = [torch.tensor(np.ascontiguousarray(b, np.float32), device=DEV) for b in Bs]
        tl = None
    else:
        hi, lo = zip(*[mdl.tf32_split(b) for b in Bs])
        th = [torch.tensor(h, device=DEV) for h in hi]
        tl = [torch.tensor(l, device=DEV) for l in lo]
    out0 = torch.zeros((M, N), dtype=torch.float32, device=DEV)
    out1 = torch.zeros((M, N), dtype=torch.float32, device=DEV)
    e = torch.zeros(M, dtype=torch.float32, device=DEV)
    st = torch.zeros(1, dtype=torch.int32, device=DEV)
    tr = np.asarray(type_rows, np.int32)
    keep = []

    def vec(vs):
        if vs is None:
            return None
        ts = [torch.tensor(np.asarray(v, np.float32), device=DEV) for v in vs]
        keep.extend(ts)
        return _ptrs(ts)

    cap = dpb._capi
    ta = torch.tensor(A, device=DEV)
    x0 = None if aux0 is None else torch.tensor(aux0, device=DEV)
    x1 = None if aux1 is None else torch.tensor(aux1, device=DEV)
    cap.call("dpb_gemm_tf32x3_f32", cap.ptr(ta), M, K, _ptrs(th), None if tl is None else _ptrs(tl),
             N, tr.ctypes.data,
             len(Bs), mode, cap.ptr(out0), cap.ptr(out1), cap.ptr(x0), cap.ptr(x1), vec(bias),
             vec(idt), vec(w), cap.ptr(e), cap.ptr(st), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    cap.call("dpb_status_check", cap.ptr(st), torch.cuda.current_stream().cuda_stream)
    return out0.cpu().numpy(), out1.cpu().numpy(), e.cpu().numpy()


def _ref(A, Bs, type_rows):
    out, r = [], 0
    for B, n in zip(Bs, type_rows):
        out.append(A[r:r + n].astype(np.float64) @ B.astype(np.float64).T)
        r += n
    return np.concatenate(out)


def _rel(a, b):
    return float(np.abs(a - b).max() / max(1e-30, np.abs(b).max()))


@pytest.mark.parametrize("M,K,N,rows", [(256, 64, 80, [128, 128]), (300, 240, 240, [100, 200]),
                                        (777, 1600, 240, [259, 518]), (640, 240, 1600, [640])])
def test_gemm_store(dpb, mdl, M, K, N, rows):
    rng = np.random.default_rng(M + K + N)
    A = rng.normal(size=(M, K)).astype(np.float32)
    Bs = [rng.normal(size=(N, K)).astype(np.float32) / np.sqrt(K) for _ in rows]
    out0, _, _ = _run(dpb, mdl, A, Bs, rows, 0)
    ref = _ref(A, Bs, rows)
    err = _rel(out0, ref)
    print(f"M={M} K={K} N={N}: rel err {err:.2e}")
    assert err < 2e-5


@pytest.mark.parametrize("M,K,N,rows,mode", [(256, 64, 80, [128, 128], 0),
                                             (300, 240, 240, [100, 200], 1),
                                             (777, 1600, 240, [259, 518], 0),
                                             (640, 240, 1600, [640], 5)])
def test_gemm_weight_split_in_kernel_is_exact(dpb, mdl, M, K, N, rows, mode):
    """FP32 weights split into TF32 hi / lo in shared memory give bit-for-bit
    the result of the pre-split weights (same rounding, exact remainder)."""
    rng = np.random.default_rng(7 + M)
    A = rng.normal(size=(M, K)).astype(np.float32) * 0.5
    Bs = [rng.normal(size=(N, K)).astype(np.float32) / np.sqrt(K) for _ in rows]
    kw = dict(bias=[rng.normal(size=N) for _ in rows]) if mode == 1 else dict(
        aux0=rng.normal(size=(M, N)).astype(np.float32), aux1=rng.normal(size=(M, N)).astype(
            np.float32)) if mode == 5 else {}
    pre = _run(dpb, mdl, A, Bs, rows, mode, **kw)
    ker = _run(dpb, mdl, A, Bs, rows, mode, split_in_kernel=True, **kw)
    for a, b in zip(pre, ker):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("N", [240, 320, 400])  # tiles of 80, 160 and 80 columns
def test_gemm_epilogues(dpb, mdl, N):
    _check_epilogues(dpb, mdl, N)


def _check_epilogues(dpb, mdl, N):
    rng = np.random.default_rng(3 + N)
    rows, M, K = [96, 290], 386, 240
    A = rng.normal(size=(M, K)).astype(np.float32) * 0.5
    Bs = [rng.normal(size=(N, K)).astype(np.float32) / np.sqrt(K) for _ in rows]
    acc = _ref(A, Bs, rows)
    tid = np.repeat(np.arange(2), rows)
    bias = [rng.normal(size=N) for _ in rows]
    idt = [rng.normal(0.1, 0.01, size=N) for _ in rows]
    w = [rng.normal(size=N) for _ in rows]
    b = np.stack(bias)[tid]
    d = np.stack(idt)[tid]
    wv = np.stack(w)[tid]
    x0 = rng.normal(size=(M, N)).astype(np.float32) * 0.5
    x1 = rng.normal(size=(M, N)).astype(np.float32)
    tol = 2e-5
    o0, _, _ = _run(dpb, mdl, A, Bs, rows, 1, bias=bias)
    assert _rel(o0, np.tanh(acc + b)) < tol
    o0, o1, _ = _run(dpb, mdl, A, Bs, rows, 2, aux0=x0, bias=bias, idt=idt)
    y = np.tanh(acc + b)
    assert _rel(o0, y) < tol and _rel(o1, x0 + d * y) < tol
    o0, _, e = _run(dpb, mdl, A, Bs, rows, 3, aux0=x0, bias=bias, idt=idt, w=w)
    h = x0 + d * y
    assert _rel(e, (h * wv).sum(1)) < tol and _rel(o0, wv * d * (1 - y * y)) < tol
    o0, o1, _ = _run(dpb, mdl, A, Bs, rows, 4, aux0=x0, idt=idt, w=w)
    g = wv + acc
    assert _rel(o1, g) < tol and _rel(o0, g * d * (1 - x0 * x0)) < tol
    o0, _, _ = _run(dpb, mdl, A, Bs, rows, 5, aux0=x0, aux1=x1)
    assert _rel(o0, (x1 + acc) * (1 - x0 * x0)) < tol


def test_fitting_tc_matches_fp64(dpb, mdl):
    cfg = mdl.SeAConfig()
    p = mdl.init_params(cfg, seed=2)
    rows = [64, 200]
    n = sum(rows)
    rng = np.random.default_rng(0)
    D = (rng.normal(size=(n, 1600)) * 0.05).astype(np.float32)
    fit = mdl._FittingTC(p, rows, DEV)
    dD = torch.zeros((n, 1600), dtype=torch.float32, device=DEV)
    E = torch.zeros(1, dtype=torch.float64, device=DEV)
    fit.forward_backward(torch.tensor(D, device=DEV), dD, E)
    ref = mdl._Fitting(p, torch.float64, DEV)
    Dt = torch.tensor(D, dtype=torch.float64, device=DEV)
    e0, g0 = ref.forward_backward(0, Dt[:rows[0]])
    e1, g1 = ref.forward_backward(1, Dt[rows[0]:])
    Eref = float(e0.sum() + e1.sum())
    gref = torch.cat([g0, g1]).cpu().numpy()
    print(f"E {float(E):.8f} ref {Eref:.8f}; dD rel {_rel(dD.cpu().numpy(), gref):.2e}")
    assert abs(float(E) - Eref) / n < 1e-6
    assert _rel(dD.cpu().numpy(), gref) < 2e-5


@pytest.mark.parametrize("M,K,N,rows", [(300, 240, 240, [100, 200]), (386, 480, 240, [96, 290])])
def test_gemm_240_tile(dpb, mdl, M, K, N, rows):
    """The one-tile-per-128-rows configuration (fit_n_tile = 240, K <= 512):
    the plain product and every fused epilogue, as with the narrower tiles."""
    from deepmd_kit_lr_pt_b200 import autotune

    old = autotune.get("fit_n_tile")
    autotune.set_knob("fit_n_tile", 240)
    try:
        rng = np.random.default_rng(M + K)
        A = rng.normal(size=(M, K)).astype(np.float32) * 0.5
        Bs = [rng.normal(size=(N, K)).astype(np.float32) / np.sqrt(K) for _ in rows]
        acc = _ref(A, Bs, rows)
        o0, _, _ = _run(dpb, mdl, A, Bs, rows, 0)
        assert _rel(o0, acc) < 2e-5
        tid = np.repeat(np.arange(len(rows)), rows)
        bias = [rng.normal(size=N) for _ in rows]
        idt = [rng.normal(0.1, 0.01, size=N) for _ in rows]
        w = [rng.normal(size=N) for _ in rows]
        b, d, wv = np.stack(bias)[tid], np.stack(idt)[tid], np.stack(w)[tid]
        x0 = rng.normal(size=(M, N)).astype(np.float32) * 0.5
        o0, o1, _ = _run(dpb, mdl, A, Bs, rows, 2, aux0=x0, bias=bias, idt=idt)
        y = np.tanh(acc + b)
        assert _rel(o0, y) < 2e-5 and _rel(o1, x0 + d * y) < 2e-5
        o0, _, e = _run(dpb, mdl, A, Bs, rows, 3, aux0=x0, bias=bias, idt=idt, w=w)
        h = x0 + d * y
        assert _rel(e, (h * wv).sum(1)) < 2e-5 and _rel(o0, wv * d * (1 - y * y)) < 2e-5
    finally:
        autotune.set_knob("fit_n_tile", old)


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (77, 240, 1600), (300, 1600, 240), (129, 65, 33),
                                   (64, 64, 16), (5000, 240, 240)])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_gemm_f64_matches_fp64_reference(dpb, M, N, K, ta, tb):
    """dpb_gemm_f64 (FP64 plain path, FP64 training) against an FP64 matmul:
    every transpose combination, ragged edges, the bias and accumulate
    epilogues; the FP64 bar 1e-12 relative to the output scale."""
    from deepmd_kit_lr_pt_b200 import autotune

    for big in (1, 0):  # the 128 x 64 and the 64 x 64 tile forms
        autotune.set_knob("gemm_simt_big", big)
        try:
            _check_gemm_f64(dpb, M, N, K, ta, tb)
        finally:
            autotune.set_knob("gemm_simt_big", 1)


def _check_gemm_f64(dpb, M, N, K, ta, tb):
    rng = np.random.default_rng(M * 7 + N * 3 + K + 11 * ta + 5 * tb)
    A = rng.normal(size=(K, M) if ta else (M, K))
    B = rng.normal(size=(N, K) if tb else (K, N))
    bias = rng.normal(size=N)
    C0 = rng.normal(size=(M, N))
    At, Bt = torch.tensor(A, device=DEV), torch.tensor(B, device=DEV)
    C = torch.tensor(C0, device=DEV)
    cap = dpb._capi
    s = torch.cuda.current_stream().cuda_stream
    cap.call("dpb_gemm_f64", cap.ptr(C), cap.ptr(At), cap.ptr(Bt), cap.ptr(torch.tensor(bias, device=DEV)),
             M, N, K, A.shape[1], B.shape[1], N, ta, tb, 1, s)
    ref = (A.T if ta else A) @ (B.T if tb else B) + bias + C0
    got = C.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()) * max(1, K) ** 0.5
    # no bias, no accumulate: C is overwritten
    C.fill_(7.0)
    cap.call("dpb_gemm_f64", cap.ptr(C), cap.ptr(At), cap.ptr(Bt), None, M, N, K, A.shape[1],
             B.shape[1], N, ta, tb, 0, s)
    ref = (A.T if ta else A) @ (B.T if tb else B)
    assert np.abs(C.cpu().numpy() - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()) * max(1, K) ** 0.5


def test_fitting_f64_matches_torch_autograd(dpb, mdl):
    """The FP64 plain path's fitting networks (FP64 GEMM + fitting-layer
    kernels): atomic energies and dE/dD against FP64 torch autograd."""
    cfg = mdl.SeAConfig()
    p = mdl.init_params(cfg, seed=4)
    rows = [70, 190]
    n = sum(rows)
    rng = np.random.default_rng(1)
    D = rng.normal(size=(n, 1600)) * 0.05
    fit = mdl._FittingF64(p, rows, DEV)
    Dt = torch.tensor(D, device=DEV)
    dD = torch.zeros_like(Dt)
    e = torch.zeros(n, dtype=torch.float64, device=DEV)
    fit.forward_backward(Dt, dD, e, torch.cuda.current_stream().cuda_stream)
    ref = mdl._Fitting(p, torch.float64, DEV)
    e0, g0 = ref.forward_backward(0, Dt[:rows[0]])
    e1, g1 = ref.forward_backward(1, Dt[rows[0]:])
    np.testing.assert_allclose(e.cpu().numpy(), torch.cat([e0, e1]).cpu().numpy(), atol=1e-11,
                               rtol=0)
    np.testing.assert_allclose(dD.cpu().numpy(), torch.cat([g0, g1]).cpu().numpy(), atol=1e-12,
                               rtol=0)


@pytest.mark.parametrize("split_in_kernel", [False, True])
def test_gemm_alike_rows_fp32_resolution(dpb, mdl, split_in_kernel):
    """Rows that are all alike (the atoms of a crystal see nearly the same
    descriptor). The tensor cores' FP32 accumulation loses up to an ulp of
    the running sum per instruction, always in the same direction, so over
    K = 1600 the outputs drift (about 1.5e-5 of the output scale with one
    accumulator per tile). Chunked accumulation (a fresh accumulator every
    kchunk k-blocks, the chunk sums added on the CUDA cores) cuts that at
    least 3x with the default chunks; with the cross products first in
    chunks of 2 k-blocks the error is at FP32-GEMM level (below 1e-6)."""
    from deepmd_kit_lr_pt_b200 import autotune

    rng = np.random.default_rng(41)
    K, N = 1600, 240
    row = (rng.normal(size=K) * 0.05 + 0.3).astype(np.float32)
    A = np.tile(row, (256, 1)) + (rng.normal(size=(256, K)) * 1e-4).astype(np.float32)
    A = A.astype(np.float32)
    Bs = [(rng.normal(size=(N, K)) / np.sqrt(K)).astype(np.float32)]
    ref = _ref(A, Bs, [256])
    errs = {}
    names = ("fit_terms", "fit_kchunk", "fit_kchunk_cross_first")
    old = {k: autotune.get(k) for k in names}
    try:
        for terms in (3, 4):
            for kc, cf in ((0, 0), (8, 0), (4, 0), (4, 1), (2, 1)):
                autotune.set_knob("fit_terms", terms)
                autotune.set_knob("fit_kchunk", kc)
                autotune.set_knob("fit_kchunk_cross_first", cf)
                o0, _, _ = _run(dpb, mdl, A, Bs, [256], 0, split_in_kernel=split_in_kernel)
                errs[terms, kc, cf] = _rel(o0, ref)
    finally:
        for k, v in old.items():
            autotune.set_knob(k, v)
    print("alike rows, K=1600, max relative error by (products, kchunk, cross first):",
          {k: f"{v:.2e}" for k, v in errs.items()})
    d = (old["fit_terms"], old["fit_kchunk"], old["fit_kchunk_cross_first"])
    assert d[1] > 0
    assert errs[d] * 3 < errs[d[0], 0, 0]
    assert errs[d[0], 2, 1] < 1e-6


@pytest.mark.parametrize("kchunk,cross", [(0, 0), (1, 1), (2, 1), (4, 1), (4, 0), (8, 0)])
@pytest.mark.parametrize("M,K,N,rows,mode", [(300, 240, 240, [100, 200], 1),
                                             (777, 1600, 240, [259, 518], 0),
                                             (257, 96, 240, [257], 3)])
def test_gemm_chunked_accumulation_modes(dpb, mdl, kchunk, cross, M, K, N, rows, mode):
    """Every chunk size gives the GEMM to FP32 accuracy, including a K that
    is not a whole number of chunks and the energy-accumulating last layer."""
    from deepmd_kit_lr_pt_b200 import autotune

    rng = np.random.default_rng(M + kchunk)
    A = (rng.normal(size=(M, K)) * 0.5).astype(np.float32)
    Bs = [(rng.normal(size=(N, K)) / np.sqrt(K)).astype(np.float32) for _ in rows]
    bias = [rng.normal(size=N).astype(np.float32) for _ in rows]
    idt = [(rng.normal(size=N) * 0.1).astype(np.float32) for _ in rows]
    w = [(rng.normal(size=N) / np.sqrt(N)).astype(np.float32) for _ in rows]
    aux0 = rng.normal(size=(M, N)).astype(np.float32) * 0.5
    old = autotune.get("fit_kchunk"), autotune.get("fit_kchunk_cross_first")
    try:
        autotune.set_knob("fit_kchunk", kchunk)
        autotune.set_knob("fit_kchunk_cross_first", cross)
        o0, o1, e = _run(dpb, mdl, A, Bs, rows, mode, aux0=aux0, bias=bias, idt=idt, w=w)
    finally:
        autotune.set_knob("fit_kchunk", old[0])
        autotune.set_knob("fit_kchunk_cross_first", old[1])
    acc = _ref(A, Bs, rows)
    tb = np.concatenate([np.tile(b, (n, 1)) for b, n in zip(bias, rows)])
    if mode == 0:
        assert _rel(o0, acc) < 2e-5
    elif mode == 1:
        np.testing.assert_allclose(o0, np.tanh(acc + tb), atol=1e-5, rtol=0)
    else:  # EPI_LAST: y = tanh(acc + b); h = aux0 + idt y; e += h . w
        td = np.concatenate([np.tile(d, (n, 1)) for d, n in zip(idt, rows)])
        tw = np.concatenate([np.tile(x, (n, 1)) for x, n in zip(w, rows)])
        y = np.tanh(acc + tb)
        np.testing.assert_allclose(e, ((aux0 + td * y) * tw).sum(1), atol=5e-5, rtol=0)
        np.testing.assert_allclose(o0, tw * td * (1 - y * y), atol=1e-5, rtol=0)
