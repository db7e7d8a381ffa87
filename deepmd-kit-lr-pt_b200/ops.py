"""Tensor-level operators over the C-ABI, mirroring the reference's operator
surface for the se_e2_a path.

* ``torch.ops.deepmd.tabulate_fusion_se_a`` (+ its grad / grad_grad ops) with
  the schema and autograd of source/op/pt/tabulate_multi_device.cc:
  914-996 (forward), 764-864 (grad, whose backward is grad_grad) and
  1669-1723 (registration). Device checks mirror CheckTabulateDevices
  (:61-86): ``table_info`` must be on the CPU, every other tensor on the
  table's device.
* Python functions with the argument meaning of the ``deepmd::*_gpu`` C++
  functions (source/lib/include): ``copy_coord``, ``normalize_coord``,
  ``build_nlist``, ``prod_env_mat_a``, ``prod_force_a``, ``prod_virial_a``,
  plus the fused ``env_mat_a_cells`` (neighbor search + format + env mat).

All kernels run on the current torch CUDA stream. Outputs are allocated here
(torch's caching allocator); the C-ABI itself never allocates. CPU tensors are
rejected: this package has no CPU implementation.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi
from ._capi import call, ptr

_ENV_CAP = 1024


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _need_cuda(*ts: torch.Tensor, what: str) -> None:
    for t in ts:
        if t is not None and not t.is_cuda:
            raise _capi.DPBInvalidArgument(
                f"DeePMD-kit Error: {what}: the B200 implementation needs CUDA tensors "
                f"(got a tensor on {t.device}); there is no CPU implementation")


def _suffix(dtype: torch.dtype) -> str:
    if dtype == torch.float64:
        return "f64"
    if dtype == torch.float32:
        return "f32"
    raise _capi.DPBInvalidArgument(f"DeePMD-kit Error: unsupported dtype {dtype}")


def _host_f64(x, n: int | None = None) -> np.ndarray:
    if isinstance(x, torch.Tensor):
        x = x.detach().cpu().numpy()
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    if n is not None and a.size != n:
        raise _capi.DPBInvalidArgument(f"DeePMD-kit Error: expected {n} values, got {a.size}")
    return a


def _host_i32(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32).reshape(-1))


# ------------------------------------------------------------ coordinates --

def normalize_coord(coord: torch.Tensor, box) -> torch.Tensor:
    """normalize_coord_gpu (coord.h:56-59): wrap into the box; returns a copy."""
    _need_cuda(coord, what="normalize_coord")
    out = coord.contiguous().clone()
    sfx = _suffix(out.dtype)
    b = _host_f64(box, 9)
    if sfx == "f32":
        b = b.astype(np.float32)
    call(f"dpb_normalize_coord_{sfx}", ptr(out), out.numel() // 3, b.ctypes.data, _stream())
    return out


def copy_coord(coord: torch.Tensor, atype: torch.Tensor, rcut: float, box,
               mem_nall: int | None = None):
    """copy_coord_gpu (coord.h:72-85) with the ghost order of copy_coord_cpu.

    Returns (coord_ext [nall,3], atype_ext [nall], mapping [nall]). Retries
    with a larger buffer on the capacity return code, as the reference's
    callers do (source/op/tf/prod_env_mat_multi_device.cc:2444-2470)."""
    _need_cuda(coord, atype, what="copy_coord")
    c = coord.contiguous().view(-1)
    t = atype.to(torch.int32).contiguous().view(-1)
    nloc = t.numel()
    sfx = _suffix(c.dtype)
    b = _host_f64(box, 9)
    bx = b if sfx == "f64" else b.astype(np.float32)
    lib = _capi.lib()
    sbytes = int(lib.dpb_copy_coord_scratch_bytes(nloc, ctypes.c_float(rcut), b.ctypes.data))
    scratch = torch.empty(sbytes, dtype=torch.uint8, device=c.device)
    mem = mem_nall if mem_nall is not None else max(64, nloc * 8)
    while True:
        out_c = torch.empty((mem, 3), dtype=c.dtype, device=c.device)
        out_t = torch.empty(mem, dtype=torch.int32, device=c.device)
        mapping = torch.empty(mem, dtype=torch.int32, device=c.device)
        nall = ctypes.c_int(0)
        code = getattr(lib, f"dpb_copy_coord_{sfx}")(
            ptr(out_c), ptr(out_t), ptr(mapping), ctypes.addressof(nall), ptr(scratch),
            sbytes, ptr(c), ptr(t), nloc, mem, ctypes.c_float(rcut), bx.ctypes.data, _stream())
        if code == 1 and mem_nall is None:
            # the capacity code reports the ghost count needed; always grow
            mem = max(nall.value, mem + 1)
            continue
        _capi.check(code, "copy_coord")
        n = nall.value
        return out_c[:n], out_t[:n], mapping[:n]


# ---------------------------------------------------------- neighbor list --

def build_nlist(c_cpy: torch.Tensor, nloc: int, rcut: float, atype: torch.Tensor | None = None,
                mem_size: int | None = None, nframes: int = 1):
    """build_nlist_gpu (neighbor_list.h:260-270), rows in ascending j.

    Returns (ilist [nf*nloc], numneigh [nf*nloc], rows [nf*nloc, mem_size],
    max_list_size). Retries with a doubled row size on the capacity code."""
    _need_cuda(c_cpy, atype, what="build_nlist")
    c = c_cpy.contiguous().view(-1)
    nall = c.numel() // 3 // nframes
    sfx = _suffix(c.dtype)
    t = None if atype is None else atype.to(torch.int32).contiguous().view(-1)
    rows_n = nframes * nloc
    lib = _capi.lib()
    sbytes = int(lib.dpb_build_nlist_scratch_bytes(nloc, nall))
    scratch = torch.empty(sbytes, dtype=torch.uint8, device=c.device)
    mem = mem_size if mem_size is not None else 256
    while True:
        ilist = torch.empty(rows_n, dtype=torch.int32, device=c.device)
        numneigh = torch.empty(rows_n, dtype=torch.int32, device=c.device)
        rows = torch.full((rows_n, max(mem, 1)), -1, dtype=torch.int32, device=c.device)
        firstneigh = _row_pointers(rows)
        mx = ctypes.c_int(0)
        code = getattr(lib, f"dpb_build_nlist_{sfx}")(
            ptr(ilist), ptr(numneigh), ptr(firstneigh), ctypes.addressof(mx), ptr(scratch),
            sbytes, ptr(c), nloc, nall, mem, ctypes.c_float(rcut), nframes, ptr(t), _stream())
        if code == 1 and mem_size is None:
            mem = max(2 * mem, mx.value)
            continue
        _capi.check(code, "build_nlist")
        return ilist, numneigh, rows, mx.value


def _row_pointers(rows: torch.Tensor) -> torch.Tensor:
    """Device array of row addresses (the firstneigh of a device InputNlist)."""
    n, w = rows.shape
    base = rows.data_ptr()
    addr = base + torch.arange(n, dtype=torch.int64, device=rows.device) * (w * 4)
    return addr


def prod_env_mat_a(coord: torch.Tensor, atype: torch.Tensor, ilist: torch.Tensor,
                   numneigh: torch.Tensor, rows: torch.Tensor, avg: torch.Tensor,
                   std: torch.Tensor, nloc: int, rcut: float, rcut_smth: float, sec,
                   nframes: int = 1):
    """prod_env_mat_a_gpu (prod_env_mat.h:97-116) from an input list.

    Returns (em [nf*nloc, nnei*4], em_deriv [nf*nloc, nnei*12],
    rij [nf*nloc, nnei*3], nlist [nf*nloc, nnei])."""
    _need_cuda(coord, atype, ilist, numneigh, rows, avg, std, what="prod_env_mat_a")
    c = coord.contiguous().view(-1)
    sfx = _suffix(c.dtype)
    t = atype.to(torch.int32).contiguous().view(-1)
    nall = t.numel() // nframes
    s = _host_i32(sec)
    nnei = int(s[-1])
    R = nframes * nloc
    dev = c.device
    em = torch.empty((R, nnei * 4), dtype=c.dtype, device=dev)
    emd = torch.empty((R, nnei * 12), dtype=c.dtype, device=dev)
    rij = torch.empty((R, nnei * 3), dtype=c.dtype, device=dev)
    nlist = torch.empty((R, nnei), dtype=torch.int32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    fn = _row_pointers(rows)
    call(f"dpb_prod_env_mat_a_{sfx}", ptr(em), ptr(emd), ptr(rij), ptr(nlist), ptr(c), ptr(t),
         R, ptr(ilist), ptr(numneigh), ptr(fn), rows.shape[1],
         ptr(avg.to(c.dtype).contiguous()), ptr(std.to(c.dtype).contiguous()),
         nloc, nall, nframes, ctypes.c_float(rcut), ctypes.c_float(rcut_smth),
         s.ctypes.data, s.size, ptr(status), _stream())
    call("dpb_status_check", ptr(status), _stream())
    return em, emd, rij, nlist


class CellGrid:
    """Device cell grid over nall points (see dpb_cell_grid_build_*)."""

    def __init__(self, nall: int, device):
        self.nall = nall
        self.nbytes = int(_capi.lib().dpb_cell_grid_bytes(nall))
        self.buf = torch.empty(self.nbytes, dtype=torch.uint8, device=device)

    def build(self, coord: torch.Tensor, rcut: float) -> "CellGrid":
        sfx = _suffix(coord.dtype)
        call(f"dpb_cell_grid_build_{sfx}", ptr(self.buf), self.nbytes, ptr(coord),
             self.nall, ctypes.c_float(rcut), _stream())
        return self


def env_mat_a_cells(coord_ext: torch.Tensor, atype_ext: torch.Tensor, nloc: int,
                    avg: torch.Tensor, std: torch.Tensor, rcut: float, rcut_smth: float,
                    sec, out_dtype: torch.dtype | None = None, with_deriv: bool = True,
                    grid: CellGrid | None = None, status: torch.Tensor | None = None,
                    check: bool = True):
    """Fused neighbor search + format + env mat over the extended system.

    out_dtype float32 with float64 coordinates selects the mixed-precision
    kernel (FP64 coordinate differences, FP32 outputs)."""
    _need_cuda(coord_ext, atype_ext, avg, std, what="env_mat_a_cells")
    c = coord_ext.contiguous()
    nall = c.shape[0]
    t = atype_ext.to(torch.int32).contiguous()
    odt = out_dtype or c.dtype
    if c.dtype == torch.float64 and odt == torch.float32:
        name = "dpb_env_mat_a_cells_mixed"
    elif c.dtype == odt:
        name = f"dpb_env_mat_a_cells_{_suffix(odt)}"
    else:
        raise _capi.DPBInvalidArgument("DeePMD-kit Error: unsupported precision combination")
    s = _host_i32(sec)
    nnei = int(s[-1])
    dev = c.device
    if grid is None:
        grid = CellGrid(nall, dev)
    grid.build(c, rcut)
    em = torch.empty((nloc, nnei * 4), dtype=odt, device=dev)
    emd = torch.empty((nloc, nnei * 12), dtype=odt, device=dev) if with_deriv else None
    rij = torch.empty((nloc, nnei * 3), dtype=odt, device=dev) if with_deriv else None
    nlist = torch.empty((nloc, nnei), dtype=torch.int32, device=dev)
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=dev)
    call(name, ptr(em), ptr(emd), ptr(rij), ptr(nlist), ptr(c), ptr(t), ptr(grid.buf),
         ptr(avg.to(odt).contiguous()), ptr(std.to(odt).contiguous()), nloc, nall,
         ctypes.c_float(rcut), ctypes.c_float(rcut_smth), s.ctypes.data, s.size,
         ptr(status), _stream())
    if check:
        call("dpb_status_check", ptr(status), _stream())
    return em, emd, rij, nlist


# -------------------------------------------------------- force / virial --

def prod_force_a(net_deriv: torch.Tensor, in_deriv: torch.Tensor, nlist: torch.Tensor,
                 nloc: int, nall: int, nframes: int = 1) -> torch.Tensor:
    """prod_force_a_gpu (prod_force.h:71-79): force [nframes, nall, 3]."""
    _need_cuda(net_deriv, in_deriv, nlist, what="prod_force_a")
    nd = net_deriv.contiguous()
    sfx = _suffix(nd.dtype)
    nnei = nlist.numel() // (nframes * nloc) if nloc > 0 else 0
    force = torch.empty((nframes, nall, 3), dtype=nd.dtype, device=nd.device)
    call(f"dpb_prod_force_a_{sfx}", ptr(force), ptr(nd), ptr(in_deriv.to(nd.dtype).contiguous()),
         ptr(nlist.to(torch.int32).contiguous()), nloc, nall, nnei, nframes, _stream())
    return force


def prod_virial_a(net_deriv: torch.Tensor, env_deriv: torch.Tensor, rij: torch.Tensor,
                  nlist: torch.Tensor, nloc: int, nall: int):
    """prod_virial_a_gpu (prod_virial.h:29-38): (virial [9], atom_virial [nall, 9])."""
    _need_cuda(net_deriv, env_deriv, rij, nlist, what="prod_virial_a")
    nd = net_deriv.contiguous()
    sfx = _suffix(nd.dtype)
    nnei = nlist.numel() // nloc if nloc > 0 else 0
    virial = torch.empty(9, dtype=nd.dtype, device=nd.device)
    av = torch.empty((nall, 9), dtype=nd.dtype, device=nd.device)
    call(f"dpb_prod_virial_a_{sfx}", ptr(virial), ptr(av), ptr(nd),
         ptr(env_deriv.to(nd.dtype).contiguous()), ptr(rij.to(nd.dtype).contiguous()),
         ptr(nlist.to(torch.int32).contiguous()), nloc, nall, nnei, _stream())
    return virial, av


def prod_force_grad_a(grad: torch.Tensor, env_deriv: torch.Tensor, nlist: torch.Tensor,
                      nloc: int, nframes: int = 1) -> torch.Tensor:
    """prod_force_grad_a_gpu (prod_force_grad.h:26-32): d(force . grad)/d(net_deriv),
    [nframes * nloc, nnei * 4]."""
    _need_cuda(grad, env_deriv, nlist, what="prod_force_grad_a")
    ed = env_deriv.contiguous()
    sfx = _suffix(ed.dtype)
    nnei = nlist.numel() // (nframes * nloc) if nloc > 0 else 0
    out = torch.empty((nframes * nloc, nnei * 4), dtype=ed.dtype, device=ed.device)
    call(f"dpb_prod_force_grad_a_{sfx}", ptr(out), ptr(grad.to(ed.dtype).contiguous()), ptr(ed),
         ptr(nlist.to(torch.int32).contiguous()), nloc, nnei, nframes, _stream())
    return out


def prod_virial_grad_a(grad: torch.Tensor, env_deriv: torch.Tensor, rij: torch.Tensor,
                       nlist: torch.Tensor, nloc: int) -> torch.Tensor:
    """prod_virial_grad_a_gpu (prod_virial_grad.h:26-32): d(virial . grad)/d(net_deriv),
    [nloc, nnei * 4]."""
    _need_cuda(grad, env_deriv, rij, nlist, what="prod_virial_grad_a")
    ed = env_deriv.contiguous()
    sfx = _suffix(ed.dtype)
    nnei = nlist.numel() // nloc if nloc > 0 else 0
    out = torch.empty((nloc, nnei * 4), dtype=ed.dtype, device=ed.device)
    call(f"dpb_prod_virial_grad_a_{sfx}", ptr(out), ptr(grad.to(ed.dtype).contiguous()),
         ptr(ed), ptr(rij.to(ed.dtype).contiguous()), ptr(nlist.to(torch.int32).contiguous()),
         nloc, nnei, _stream())
    return out


# ------------------------------------------------- torch.ops.deepmd.* ops --

def _check_tab(table, table_info, tensors, what):
    # CheckTabulateDevices (tabulate_multi_device.cc:61-86)
    if table_info.device.type != "cpu":
        raise _capi.DPBInvalidArgument("table_info must be on the CPU")
    for name, t in tensors:
        if t is not None and t.device != table.device:
            raise _capi.DPBInvalidArgument(
                f"{name} must be on the same device as table; table is on {table.device} "
                f"but {name} is on {t.device}")
    _need_cuda(table, what=what)


def _info_host(table_info: torch.Tensor, dtype) -> np.ndarray:
    a = table_info.detach().contiguous().view(-1).numpy()
    return np.ascontiguousarray(a.astype(np.float64 if dtype == torch.float64 else np.float32))


def table_rows_needed(info: np.ndarray) -> int:
    """Rows locate_xx can address (tabulate.cc:21-30,45-73): the kernels read up
    to row first + int((nextafter(max, lower) - upper) / stride1)."""
    lower, upper, mx, s0, s1 = (info[k] for k in range(5))
    first = int((upper - lower) / s0)
    if info.dtype == np.float32:
        bxx = np.nextafter(np.float32(mx), np.float32(lower))
    else:
        bxx = np.nextafter(mx, lower)
    return first + int((bxx - upper) / s1) + 1


def _check_table_size(table: torch.Tensor, info: np.ndarray, M: int) -> None:
    need = table_rows_needed(info) * 6 * M
    if table.numel() < need:
        raise _capi.DPBInvalidArgument(
            f"DeePMD-kit Error: the table holds {table.numel()} values but table_info "
            f"addresses {need} (= rows x 6 x last_layer_size)")


def _tab_fwd_impl(table, table_info, em_x, em, last_layer_size):
    _check_tab(table, table_info, [("em_x", em_x), ("em", em)], "tabulate_fusion_se_a")
    if table.dim() != 2:
        raise _capi.DPBInvalidArgument("Dim of table should be 2")
    if em_x.dim() != 2:
        raise _capi.DPBInvalidArgument("Dim of input should be 2")
    if em.dim() != 3:
        raise _capi.DPBInvalidArgument("Dim of input should be 3")
    if em.size(2) != 4:
        raise _capi.DPBInvalidArgument(
            f"The environment basis dimension must be 4 for se_a, got {em.size(2)}")
    M = int(last_layer_size)
    if not (0 < M <= 1024):
        raise _capi.DPBInvalidArgument(
            f"last_layer_size must be between 1 and 1024 for GPU tabulation, but got {M}")
    sfx = _suffix(table.dtype)
    nloc, nnei = em.size(0), em.size(1)
    out = torch.empty((nloc, 4, M), dtype=table.dtype, device=table.device)
    info = _info_host(table_info, table.dtype)
    if nnei > 0:
        _check_table_size(table, info, M)
    call(f"dpb_tabulate_fusion_se_a_{sfx}", ptr(out), ptr(table.contiguous()), info.ctypes.data,
         ptr(em_x.contiguous()), ptr(em.contiguous()), nloc, nnei, M, _stream())
    return [out]


def _tab_grad_impl(table, table_info, em_x, em, dy, descriptor):
    _check_tab(table, table_info, [("em_x", em_x), ("em", em), ("dy", dy)],
               "tabulate_fusion_se_a_grad")
    sfx = _suffix(table.dtype)
    nloc, nnei = em.size(0), em.size(1)
    M = descriptor.size(-1)
    dx = torch.zeros_like(em_x)
    de = torch.zeros_like(em)
    info = _info_host(table_info, table.dtype)
    if nnei > 0:
        _check_table_size(table, info, M)
    call(f"dpb_tabulate_fusion_se_a_grad_{sfx}", ptr(dx), ptr(de), ptr(table.contiguous()),
         info.ctypes.data, ptr(em_x.contiguous()), ptr(em.contiguous()), ptr(dy.contiguous()),
         nloc, nnei, M, _stream())
    return [dx, de]


def _tab_grad_grad_impl(table, table_info, em_x, em, dz_dy_dem_x, dz_dy_dem, descriptor,
                        is_sorted):
    _check_tab(table, table_info, [("em_x", em_x), ("em", em)],
               "tabulate_fusion_se_a_grad_grad")
    sfx = _suffix(table.dtype)
    nloc, nnei = em.size(0), em.size(1)
    M = descriptor.size(-1)
    out = torch.empty_like(descriptor)
    info = _info_host(table_info, table.dtype)
    if nnei > 0:
        _check_table_size(table, info, M)
    call(f"dpb_tabulate_fusion_se_a_grad_grad_{sfx}", ptr(out), ptr(table.contiguous()),
         info.ctypes.data, ptr(em_x.contiguous()), ptr(em.contiguous()),
         ptr(dz_dy_dem_x.contiguous()), ptr(dz_dy_dem.contiguous()), nloc, nnei, M, _stream())
    return [out]


_LIB = None


def register_torch_ops() -> None:
    """Define deepmd::tabulate_fusion_se_a{,_grad,_grad_grad} (idempotent)."""
    global _LIB
    if _LIB is not None:
        return
    try:
        torch.ops.deepmd.tabulate_fusion_se_a  # noqa: B018
        raise RuntimeError(
            "torch.ops.deepmd.tabulate_fusion_se_a is already registered by another "
            "library in this process; load only one implementation of the deepmd ops")
    except (AttributeError, RuntimeError) as e:
        if "already registered" in str(e):
            raise
    lib = torch.library.Library("deepmd", "FRAGMENT")
    lib.define("tabulate_fusion_se_a(Tensor table, Tensor table_info, Tensor em_x, "
               "Tensor em, int last_layer_size) -> Tensor[]")
    lib.define("tabulate_fusion_se_a_grad(Tensor table, Tensor table_info, Tensor em_x, "
               "Tensor em, Tensor dy, Tensor descriptor) -> Tensor[]")
    lib.define("tabulate_fusion_se_a_grad_grad(Tensor table, Tensor table_info, "
               "Tensor em_x, Tensor em, Tensor dz_dy_dem_x, Tensor dz_dy_dem, "
               "Tensor descriptor, bool is_sorted) -> Tensor[]")
    for name, fn in (("tabulate_fusion_se_a", _tab_fwd_impl),
                     ("tabulate_fusion_se_a_grad", _tab_grad_impl),
                     ("tabulate_fusion_se_a_grad_grad", _tab_grad_grad_impl)):
        lib.impl(name, fn, "CUDA")
        lib.impl(name, _cpu_refusal(name), "CPU")

    # autograd: forward -> grad (tabulate_multi_device.cc:961-995),
    # grad -> grad_grad w.r.t. dy only (:818-863)
    def fwd_setup(ctx, inputs, output):
        table, table_info, em_x, em, _ = inputs
        ctx.save_for_backward(table, table_info, em_x, em, output[0])

    def fwd_backward(ctx, grads):
        table, table_info, em_x, em, desc = ctx.saved_tensors
        dy = grads[0].contiguous()
        dx, de = torch.ops.deepmd.tabulate_fusion_se_a_grad(table, table_info, em_x, em, dy,
                                                           desc)
        return None, None, dx, de, None

    def grad_setup(ctx, inputs, output):
        table, table_info, em_x, em, dy, desc = inputs
        ctx.save_for_backward(table, table_info, em_x, em, desc)

    def grad_backward(ctx, grads):
        table, table_info, em_x, em, desc = ctx.saved_tensors
        gx = grads[0] if grads[0] is not None else torch.zeros_like(em_x)
        ge = grads[1] if grads[1] is not None else torch.zeros_like(em)
        dz = torch.ops.deepmd.tabulate_fusion_se_a_grad_grad(
            table, table_info, em_x, em, gx.contiguous(), ge.contiguous(), desc, True)[0]
        return None, None, None, None, dz, None

    torch.library.register_autograd("deepmd::tabulate_fusion_se_a", fwd_backward,
                                    setup_context=fwd_setup, lib=lib)
    torch.library.register_autograd("deepmd::tabulate_fusion_se_a_grad", grad_backward,
                                    setup_context=grad_setup, lib=lib)
    _LIB = lib


def _cpu_refusal(name):
    def f(*args, **kwargs):
        raise _capi.DPBInvalidArgument(
            f"DeePMD-kit Error: deepmd::{name}: this is the B200 (CUDA) implementation; "
            "CPU tensors are not supported")
    return f
