"""The allocation-free neighbor-list entry point (dpb_build_nlist_noalloc_f64).

It is meant for callers that cannot call cudaMalloc, such as an MD engine's
force callback running inside the engine's own device-memory pool. Its
results must equal those of dpb_build_nlist_f64 (which takes caller scratch)
on the same inputs, over two calls in a row (the built-in working array keeps
the previous call's contents, so the second call checks that everything that
must start at zero is reset), for two frames in one call (the frames' cell
grids are built one after the other in the same array) and at the largest
size the array accepts. This file is collected last on purpose.
"""

import ctypes
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
MEM = 512


def _frame(port, wl, n_side, seed):
    coord, atype, box = wl.water_frame(n_side, seed=seed)
    c, t, _ = port.copy_coord(coord, atype, 6.0, box)
    return c, t, atype.size


def _rows(nrows):
    rows = torch.full((nrows, MEM), -1, dtype=torch.int32, device=DEV)
    fn = rows.data_ptr() + torch.arange(nrows, dtype=torch.int64, device=DEV) * (MEM * 4)
    return rows, fn


def _run(dpb, name, c, t, nloc, nall, nframes):
    """One call of dpb_build_nlist_f64 (caller scratch) or of the
    allocation-free entry point on the same inputs."""
    cap = dpb._capi
    ct = torch.tensor(np.ascontiguousarray(c).reshape(-1), device=DEV)
    tt = torch.tensor(np.ascontiguousarray(t).reshape(-1), device=DEV)
    ilist = torch.empty(nframes * nloc, dtype=torch.int32, device=DEV)
    numneigh = torch.empty(nframes * nloc, dtype=torch.int32, device=DEV)
    rows, fn = _rows(nframes * nloc)
    mx = ctypes.c_int(0)
    s = torch.cuda.current_stream().cuda_stream
    if name == "noalloc":
        code = cap.lib().dpb_build_nlist_noalloc_f64(
            cap.ptr(ilist), cap.ptr(numneigh), cap.ptr(fn), ctypes.addressof(mx), cap.ptr(ct),
            nloc, nall, MEM, ctypes.c_float(6.0), nframes, cap.ptr(tt), s)
    else:
        nb = int(cap.lib().dpb_build_nlist_scratch_bytes(nloc, nall))
        scratch = torch.empty(nb, dtype=torch.uint8, device=DEV)
        code = cap.lib().dpb_build_nlist_f64(
            cap.ptr(ilist), cap.ptr(numneigh), cap.ptr(fn), ctypes.addressof(mx),
            cap.ptr(scratch), nb, cap.ptr(ct), nloc, nall, MEM, ctypes.c_float(6.0), nframes,
            cap.ptr(tt), s)
    cap.check(code, name)
    return ilist.cpu().numpy(), numneigh.cpu().numpy(), rows.cpu().numpy(), mx.value


def _assert_same(a, b):
    il0, nn0, r0, mx0 = a
    il1, nn1, r1, mx1 = b
    np.testing.assert_array_equal(il1, il0)
    np.testing.assert_array_equal(nn1, nn0)
    assert mx1 == mx0
    valid = np.arange(MEM)[None, :] < nn0[:, None]
    np.testing.assert_array_equal(np.where(valid, r1, -1), np.where(valid, r0, -1))


@pytest.mark.parametrize("frames", [[(4, 7), (5, 8)]])
def test_noalloc_equals_scratch_version_two_calls(dpb, port, frames):
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    for n_side, seed in frames:  # two calls in a row on the shared array
        c, t, nloc = _frame(port, wl, n_side, seed)
        want = _run(dpb, "scratch", c, t, nloc, c.shape[0], 1)
        got = _run(dpb, "noalloc", c, t, nloc, c.shape[0], 1)
        _assert_same(want, got)


def test_noalloc_two_frames_in_one_call(dpb, port):
    """nframes = 2: each frame's grid is rebuilt in the same array."""
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    c0, t0, nloc = _frame(port, wl, 5, 21)
    c1, t1, _ = _frame(port, wl, 5, 22)
    nall = min(c0.shape[0], c1.shape[0])  # the same extended size for both frames
    c = np.concatenate([c0[:nall], c1[:nall]])
    t = np.concatenate([t0[:nall], t1[:nall]])
    want = _run(dpb, "scratch", c, t, nloc, nall, 2)
    got = _run(dpb, "noalloc", c, t, nloc, nall, 2)
    _assert_same(want, got)
    # the second frame's rows differ from the first's (its own grid was used)
    assert not np.array_equal(got[1][:nloc], got[1][nloc:])


def test_noalloc_at_the_size_limit(dpb, port):
    """The largest accepted nall (dpb_cell_grid_bytes(nall) + 256 == 4 MiB)
    runs and matches; one more extended atom is rejected."""
    cap = dpb._capi
    lim = int(cap.lib().dpb_build_nlist_noalloc_max_bytes())
    nmax = 64
    while cap.lib().dpb_cell_grid_bytes(nmax * 2) + 256 <= lim:
        nmax *= 2
    lo, hi = nmax, nmax * 2
    while hi - lo > 1:
        mid = (lo + hi) // 2
        lo, hi = (mid, hi) if cap.lib().dpb_cell_grid_bytes(mid) + 256 <= lim else (lo, mid)
    nmax = lo
    assert nmax == 209_670
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    c, t, _ = _frame(port, wl, 38, 5)
    assert c.shape[0] > nmax
    c, t, nloc = c[:nmax], t[:nmax], 30_000  # the first 30,000 atoms as centers
    want = _run(dpb, "scratch", c, t, nloc, nmax, 1)
    got = _run(dpb, "noalloc", c, t, nloc, nmax, 1)
    _assert_same(want, got)
    code = cap.lib().dpb_build_nlist_noalloc_f64(None, None, None, None, None, nloc, nmax + 1,
                                                 MEM, ctypes.c_float(6.0), 1, None, None)
    assert code == 2 and "built-in array" in cap.last_error()


def test_noalloc_rejects_oversized_input(dpb):
    cap = dpb._capi
    limit = cap.lib().dpb_build_nlist_noalloc_max_bytes()
    assert limit == 4 << 20
    big = 10_000_000  # needs far more than the built-in array holds
    code = cap.lib().dpb_build_nlist_noalloc_f64(None, None, None, None, None, 16, big, 64,
                                                 ctypes.c_float(6.0), 1, None, None)
    assert code == 2
    assert "built-in array" in cap.last_error()
