"""ctypes binding of the C-ABI in include/dpb200.h (libdpb200.so).

The library is the only compute path: if it cannot be loaded, importing the
package fails (no CPU fallback).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libdpb200.so")


class DPBError(RuntimeError):
    """deepmd::deepmd_exception counterpart ("DeePMD-kit Error: ...")."""


class DPBCapacityError(DPBError):
    """Return code 1 of build_nlist_gpu / copy_coord_gpu: buffers too small."""


class DPBInvalidArgument(DPBError, ValueError):
    """std::invalid_argument / TORCH_CHECK failures of the reference ops."""


class DPBCudaError(DPBError):
    """DPErrcheck failure."""


class DPBOutOfMemory(DPBError, MemoryError):
    """deepmd::deepmd_exception_oom."""


class DPBNlistCapacityError(DPBError):
    """deepmd::deepmd_exception_nlist_capacity."""


class DPBOverflowError(DPBError):
    """Neighbor sort-key overflow (the reference traps on the device here)."""


_ERRORS = {
    1: DPBCapacityError,
    2: DPBInvalidArgument,
    3: DPBCudaError,
    4: DPBOutOfMemory,
    5: DPBNlistCapacityError,
    6: DPBOverflowError,
}

P, I, F, LL, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_longlong, ctypes.c_double
_SPEC = {"p": P, "i": I, "f": F, "L": LL, "d": D}

# name -> argument kinds (p pointer, i int, f float, L long long, d double)
_FUNCS = {
    "dpb_status_check": "pp",
    "dpb_zero_async": "pLp",
    "dpb_normalize_coord_f64": "pipp",
    "dpb_normalize_coord_f32": "pipp",
    # out_c, out_t, mapping, nall(host), scratch, scratch_bytes, in_c, in_t,
    # nloc, mem_nall, rcut, boxt(host), stream
    "dpb_copy_coord_f64": "pppppLppiifpp",
    "dpb_copy_coord_f32": "pppppLppiifpp",
    "dpb_cell_grid_build_f64": "pLpifp",
    "dpb_cell_grid_build_f32": "pLpifp",
    "dpb_build_nlist_f64": "pppppLpiiifipp",
    "dpb_build_nlist_f32": "pppppLpiiifipp",
    "dpb_prod_env_mat_a_f64": "pppppp" "ipppi" "ppiiiff" "pipp",
    "dpb_prod_env_mat_a_f32": "pppppp" "ipppi" "ppiiiff" "pipp",
    "dpb_prod_env_mat_a_mixed": "pppppp" "ipppi" "ppiiiff" "pipp",
    "dpb_ghost_shift_f64": "pppppip",
    "dpb_ghost_refresh_f64": "pppppip",
    "dpb_env_mat_a_cells_f64": "pppppp" "p" "ppiiff" "pipp",
    "dpb_env_mat_a_cells_f32": "pppppp" "p" "ppiiff" "pipp",
    "dpb_env_mat_a_cells_mixed": "pppppp" "p" "ppiiff" "pipp",
    "dpb_tabulate_fusion_se_a_f64": "pppppiiip",
    "dpb_tabulate_fusion_se_a_f32": "pppppiiip",
    "dpb_tabulate_fusion_se_a_grad_f64": "ppppppp" "iiip",
    "dpb_tabulate_fusion_se_a_grad_f32": "ppppppp" "iiip",
    "dpb_tabulate_fusion_se_a_grad_grad_f64": "ppppppp" "iiip",
    "dpb_tabulate_fusion_se_a_grad_grad_f32": "ppppppp" "iiip",
    "dpb_prod_force_a_f64": "ppppiiiip",
    "dpb_prod_force_grad_a_f64": "ppppiiip",
    "dpb_prod_force_grad_a_f32": "ppppiiip",
    "dpb_prod_virial_grad_a_f64": "pppppiip",
    "dpb_prod_virial_grad_a_f32": "pppppiip",
    "dpb_prod_force_a_f32": "ppppiiiip",
    "dpb_prod_virial_a_f64": "pppppp" "iiip",
    "dpb_prod_virial_a_f32": "pppppp" "iiip",
    "dpb_copy_coord_async_f64": "ppppp" "L" "ppiifpp",
    "dpb_cell_grid_build_async_f64": "pLpipfp",
    "dpb_geometry_cells_f64": "ppppp" "L" "p" "L" "ppiifppp",
    "dpb_fit_energy_sum_f32": "ppidpp",
    "dpb_se_a_pack_table_f32": "ppiip",
    "dpb_se_a_build_table_f64": "pppiipppipLp",
    "dpb_batch_env_mat_a_f32": "pppppppppp" "ppppp" "iiff" "pipp",
    "dpb_batch_force_virial_a": "ppppppp" "ppppp" "iiiiff" "p",
    "dpb_batch_energy": "pppppip",
    "dpb_batch_env_mat_a_f64": "pppppppppp" "ppppp" "iiff" "pipp",
    "dpb_batch_force_virial_a_f64": "ppppppp" "ppppp" "iiiiff" "p",
    "dpb_batch_energy_f64": "pppppip",
    "dpb_se_a_descriptor_fwd_f32": "pppp" "pp" "pi" "iiip",
    "dpb_se_a_descriptor_bwd_f32": "ppppp" "pp" "pi" "iiip",
    "dpb_se_a_descriptor_fwd_cubic_f32": "pppp" "pp" "pi" "iiip",
    "dpb_se_a_descriptor_bwd_cubic_f32": "ppppp" "pp" "pi" "iiip",
    "dpb_force_virial_a_f32": "pppppp" "pp" "iiiip",
    "dpb_force_virial_a_f64": "pppppp" "pp" "iiiip",
    "dpb_build_nlist_noalloc_f64": "ppppp" "iiif" "i" "pp",
    "dpb_force_virial_a_env_mixed": "pppppppp" "iiii" "ff" "p",
    "dpb_force_virial_a_env_mixed_acc": "pppppppp" "iiii" "ff" "p",
    "dpb_gemm_tf32x3_f32": "pii" "pp" "i" "pi" "i" "pppp" "ppp" "pp" "p",
    "dpb_force_virial_a_env_f64": "pppppppp" "iiii" "ff" "p",
    "dpb_copy_coord_cells_f64": "ppppp" "L" "pp" "ii" "pp" "p",
    "dpb_copy_coord_cells_f32": "ppppp" "L" "pp" "ii" "pp" "p",
    "dpb_use_nlist_map": "pp" "ii" "p",
    "dpb_nlist_rows_to_device": "pppp" "i" "ppp" "i" "p" "L" "p",
    "dpb_gemm_f64": "pppp" "iiiiii" "iii" "p",
    "dpb_gemm_f32": "pppp" "iiiiii" "iii" "p",
    "dpb_transpose_f32": "pp" "iiiii" "p",
}
_TRAIN = {
    "dpb_se_a_train_fwd": "pppppppppp" "iii" "pp",
    "dpb_se_a_train_bwd": "pppppppppppp" "iii" "p",
    "dpb_se_a_train_tan": "pppppppppppppp" "i" "pppp" "iii" "ff" "p",
    "dpb_se_a_train_rev": "pppppppppppppppppp" "i" "pppp" "iii" "p" "ff" "p",
    "dpb_fit_act": "pppp" "iii" "p",
    "dpb_fit_tan": "ppppp" "iii" "p",
    "dpb_fit_bwd": "pppp" "ii" "p",
    "dpb_fit_rev": "ppppppppp" "ii" "p",
    "dpb_fit_res_adj": "pp" "iii" "p",
    "dpb_fit_out": "pppp" "d" "ii" "p",
    "dpb_fit_out_adj": "pppppppp" "ii" "p",
    "dpb_train_lam": "pppp" "i" "p",
    "dpb_adam": "pppp" "L" "p" "ddd" "p",
}
for _name, _spec in _TRAIN.items():
    for _suf in ("f32", "f64"):
        _FUNCS[f"{_name}_{_suf}"] = _spec
_FUNCS.update({"dpb_tune_count": "", "dpb_tune_get": "p", "dpb_tune_options": "ppi",
               "dpb_tune_set": "pi"})
# the batched step as one launch (description struct: batch.BtStepDesc)
_FUNCS.update({"dpb_bt_step_create": "pp", "dpb_bt_step_launch": "pp",
               "dpb_bt_step_destroy": "p"})
_SIZE_QUERIES = {
    "dpb_copy_coord_scratch_bytes": ("ifp", LL),
    "dpb_cell_grid_bytes": ("i", LL),
    "dpb_cell_grid_bytes_packed": ("i", LL),
    "dpb_geometry_scratch_bytes": ("ifp", LL),
    "dpb_fit_energy_sum_work_bytes": ("", LL),
    "dpb_build_nlist_scratch_bytes": ("ii", LL),
    "dpb_build_nlist_noalloc_max_bytes": ("", LL),
    "dpb_se_a_build_table_scratch_bytes": ("ii", LL),
    "dpb_copy_coord_cells_scratch_bytes": ("ip", LL),
    "dpb_nlist_rows_scratch_bytes": ("pi", LL),
    "dpb_bt_step_desc_layout": ("i", LL),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load libdpb200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python deepmd-kit-lr-pt_b200/build.py` "
            "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    for name, spec in _FUNCS.items():
        f = getattr(L, name)
        f.argtypes = [_SPEC[c] for c in spec]
        f.restype = I
    for name, (spec, rt) in _SIZE_QUERIES.items():
        f = getattr(L, name)
        f.argtypes = [_SPEC[c] for c in spec]
        f.restype = rt
    L.dpb_last_error.restype = ctypes.c_char_p
    L.dpb_tune_name.argtypes = [I]
    L.dpb_tune_name.restype = ctypes.c_char_p
    L.dpb_abi_version.restype = I
    _lib = L
    return L


def last_error() -> str:
    return lib().dpb_last_error().decode(errors="replace")


def check(code: int, what: str = "") -> None:
    """Raise the exception class that mirrors the reference's error type."""
    if code == 0:
        return
    cls = _ERRORS.get(code, DPBError)
    msg = last_error()
    raise cls(f"DeePMD-kit Error: {what + ': ' if what else ''}{msg}")


def call(name: str, *args) -> int:
    """Call an entry point and raise on failure."""
    code = getattr(lib(), name)(*args)
    check(code, name)
    return code


def ptr(x) -> int | None:
    """Device/host address of a torch tensor or numpy array (None stays NULL)."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return x.data_ptr()


def exported_symbols() -> list[str]:
    return sorted(list(_FUNCS) + list(_SIZE_QUERIES) +
                  ["dpb_last_error", "dpb_abi_version", "dpb_tune_name"])
