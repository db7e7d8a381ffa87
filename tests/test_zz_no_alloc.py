"""The allocation-free neighbor-list entry point (dpb_build_nlist_noalloc_f64).

It is meant for callers that cannot call cudaMalloc, such as an MD engine's
force callback running inside the engine's own device-memory pool. Its
results must equal those of dpb_build_nlist_f64 (which takes caller scratch)
on the same inputs, over two calls in a row (the built-in working array keeps
the previous call's contents, so the second call checks that everything that
must start at zero is reset). This file is collected last on purpose.
"""

import ctypes
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _frame(port, wl, n_side, seed):
    coord, atype, box = wl.water_frame(n_side, seed=seed)
    c, t, _ = port.copy_coord(coord, atype, 6.0, box)
    return c, t, atype.size


def _noalloc(dpb, c, t, nloc, mem):
    cap = dpb._capi
    ct = torch.tensor(c, device=DEV)
    tt = torch.tensor(t, device=DEV)
    ilist = torch.empty(nloc, dtype=torch.int32, device=DEV)
    numneigh = torch.empty(nloc, dtype=torch.int32, device=DEV)
    rows = torch.full((nloc, mem), -1, dtype=torch.int32, device=DEV)
    fn = rows.data_ptr() + torch.arange(nloc, dtype=torch.int64, device=DEV) * (mem * 4)
    mx = ctypes.c_int(0)
    code = cap.lib().dpb_build_nlist_noalloc_f64(
        cap.ptr(ilist), cap.ptr(numneigh), cap.ptr(fn), ctypes.addressof(mx), cap.ptr(ct),
        nloc, c.shape[0], mem, ctypes.c_float(6.0), 1, cap.ptr(tt),
        torch.cuda.current_stream().cuda_stream)
    cap.check(code, "build_nlist_noalloc")
    return ilist.cpu().numpy(), numneigh.cpu().numpy(), rows.cpu().numpy(), mx.value


@pytest.mark.parametrize("frames", [[(4, 7), (5, 8)]])
def test_noalloc_equals_scratch_version_two_calls(dpb, port, frames):
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    for n_side, seed in frames:  # two calls in a row on the shared array
        c, t, nloc = _frame(port, wl, n_side, seed)
        il0, nn0, rows0, mx0 = dpb.ops.build_nlist(torch.tensor(c, device=DEV), nloc, 6.0,
                                                   atype=torch.tensor(t, device=DEV),
                                                   mem_size=512)
        il1, nn1, rows1, mx1 = _noalloc(dpb, c, t, nloc, 512)
        np.testing.assert_array_equal(il1, il0.cpu().numpy())
        np.testing.assert_array_equal(nn1, nn0.cpu().numpy())
        assert mx1 == mx0
        r0 = rows0.cpu().numpy()
        for i in range(nloc):
            np.testing.assert_array_equal(rows1[i, : nn1[i]], r0[i, : nn1[i]])


def test_noalloc_rejects_oversized_input(dpb):
    cap = dpb._capi
    limit = cap.lib().dpb_build_nlist_noalloc_max_bytes()
    assert limit == 4 << 20
    big = 10_000_000  # needs far more than the built-in array holds
    code = cap.lib().dpb_build_nlist_noalloc_f64(None, None, None, None, None, 16, big, 64,
                                                 ctypes.c_float(6.0), 1, None, None)
    assert code == 2
    assert "built-in array" in cap.last_error()
