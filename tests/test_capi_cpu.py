"""CPU-side checks of the C-ABI library: it loads without a GPU, exports every
entry point include/dpb200.h declares, the ctypes argument specs agree with
the header, and the product refuses CPU tensors instead of falling back."""

import os
import re
import subprocess

import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dpb200.h")


def _declared():
    text = open(HEADER).read()
    decls = {}
    for m in re.finditer(r"DPB_API\s+[\w\s\*]+?\b(dpb_\w+)\s*\(([^;]*?)\)\s*;", text, re.S):
        args = [a.strip() for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        decls[m.group(1)] = args
    return decls


def test_header_declares_entry_points():
    d = _declared()
    assert "dpb_tabulate_fusion_se_a_f32" in d and "dpb_prod_force_a_f64" in d
    assert len(d) >= 29


def test_library_exports_every_declared_symbol(dpb):
    lib = dpb._capi.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = sorted(set(_declared()) - exported)
    assert not missing, f"declared but not exported: {missing}"


def test_ctypes_specs_match_header(dpb):
    d = _declared()
    from deepmd_kit_lr_pt_b200 import _capi

    for name, spec in _capi._FUNCS.items():
        assert name in d, name
        assert len(spec) == len(d[name]), f"{name}: spec {len(spec)} args, header {len(d[name])}"
        for kind, arg in zip(spec, d[name]):
            if kind == "p":
                assert "*" in arg or "dpb_stream_t" in arg, (name, arg)
            elif kind == "i":
                assert arg.startswith("int ") and "*" not in arg, (name, arg)
            elif kind == "f":
                assert arg.startswith("float ") and "*" not in arg, (name, arg)
            elif kind == "L":
                assert arg.startswith("long long"), (name, arg)
            elif kind == "d":
                assert arg.startswith("double ") and "*" not in arg, (name, arg)


def test_library_loads_and_reports_version(dpb):
    lib = dpb._capi.lib()
    assert lib.dpb_abi_version() == 1
    # size queries run on the host without a device
    assert dpb._capi.lib().dpb_cell_grid_bytes(1000) > 1000 * 8


def test_cpu_tensors_are_refused(dpb):
    table = torch.zeros((4, 48), dtype=torch.float64)
    info = torch.tensor([0, 0.2, 0.4, 0.01, 0.1, -1], dtype=torch.float64)
    with pytest.raises(Exception, match="CPU"):
        torch.ops.deepmd.tabulate_fusion_se_a(table, info, torch.zeros((4, 4), dtype=torch.float64),
                                              torch.zeros((4, 4, 4), dtype=torch.float64), 8)
    with pytest.raises(dpb._capi.DPBInvalidArgument):
        dpb.ops.prod_force_a(torch.zeros((1, 4)), torch.zeros((1, 12)),
                             torch.zeros((1, 1), dtype=torch.int32), 1, 1)


def test_cxx_dropin_exports_reference_symbols(dpb):
    """libdpb200.so defines every deepmd:: GPU function on this path under the
    mangled name the reference headers produce (tests/golden/ref_abi_symbols.txt)."""
    want = open(os.path.join(ROOT, "tests", "golden", "ref_abi_symbols.txt")).read().split()
    out = subprocess.run(["nm", "-D", "--defined-only", dpb._capi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    have = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [s for s in want if s not in have]
    assert len(want) == 25 and not missing, missing


def test_tile_knob_registry(dpb):
    """The tile-shape knobs list their options, accept only those, and read
    back what was set (no device needed)."""
    from deepmd_kit_lr_pt_b200 import autotune

    names = autotune.names()
    assert {"desc_atoms_per_cta", "desc_coef_l1", "fit_n_tile", "fit_split_b",
            "batch_atoms_per_cta",
            "train_rows_per_group", "train_warps_per_cta", "geometry_fused",
            "pdl"} <= set(names)
    assert autotune.options("pdl") == [0, 1] and autotune.options("geometry_fused") == [0, 1]
    for n in names:
        opts = autotune.options(n)
        old = autotune.get(n)
        assert old in opts and len(opts) >= 2
        autotune.set_knob(n, opts[0])
        assert autotune.get(n) == opts[0]
        autotune.set_knob(n, old)
    with pytest.raises(dpb._capi.DPBInvalidArgument):
        autotune.set_knob("desc_atoms_per_cta", 3)
    with pytest.raises(dpb._capi.DPBInvalidArgument):
        autotune.get("no_such_knob")


def test_step_scratch_sizes(dpb):
    """Host-side sizes of the single-frame step's buffers (no device needed):
    the geometry pass's scratch also covers its separate-kernel fallback, and
    the energy-sum work buffer holds one partial per block plus the ticket."""
    import ctypes

    import numpy as np

    lib = dpb._capi.lib()
    box = np.diag([49.67, 49.67, 49.67]).reshape(9).astype(np.float64)
    rc = ctypes.c_float(6.0)
    geo = int(lib.dpb_geometry_scratch_bytes(12288, rc, box.ctypes.data))
    sep = int(lib.dpb_copy_coord_scratch_bytes(12288, rc, box.ctypes.data))
    assert geo >= sep > 0
    # three ints per local atom at least (cell, slot, order)
    assert geo >= 3 * 4 * 12288
    assert int(lib.dpb_fit_energy_sum_work_bytes()) >= 8 * 149


def test_noalloc_size_limit_host_side(dpb):
    """The allocation-free neighbor list accepts nall up to the figure its
    documentation gives (dpb_cell_grid_bytes(nall) + 256 <= its 4 MiB array:
    209,670 extended atoms) and rejects one more before touching a device."""
    import ctypes

    cap = dpb._capi
    lib = cap.lib()
    limit = int(lib.dpb_build_nlist_noalloc_max_bytes())
    assert limit == 4 << 20
    nmax = 209_670
    assert lib.dpb_cell_grid_bytes(nmax) + 256 <= limit
    assert lib.dpb_cell_grid_bytes(nmax + 1) + 256 > limit
    # the rejection happens on the host, before any CUDA call
    code = lib.dpb_build_nlist_noalloc_f64(None, None, None, None, None, 16, nmax + 1, 64,
                                           ctypes.c_float(6.0), 1, None, None)
    assert code == 2 and "built-in array" in cap.last_error()


def test_step_description_layout_matches_ctypes(dpb):
    """The ctypes mirrors of dpb_bt_step_desc / dpb_gemm_layer have the
    layout the library was compiled with."""
    import ctypes

    from deepmd_kit_lr_pt_b200 import batch

    lib = dpb._capi.lib()
    assert lib.dpb_bt_step_desc_layout(0) == ctypes.sizeof(batch.BtStepDesc)
    assert lib.dpb_bt_step_desc_layout(1) == batch.BtStepDesc.fit.offset
    assert lib.dpb_bt_step_desc_layout(2) == batch.BtStepDesc.status.offset
    assert lib.dpb_bt_step_desc_layout(3) == ctypes.sizeof(batch.GemmLayer)
    assert lib.dpb_bt_step_desc_layout(4) == batch.GemmLayer.w.offset
