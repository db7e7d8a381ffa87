"""Test infrastructure only: numpy bindings of the CPU checkers.

Two libraries sit behind the same Python functions:

* ``port`` -- ``oracle/_build/libdporacle.so``, the plain-C restatement in
  ``oracle/dp_oracle.c`` (always built; travels with the repository);
* ``ref``  -- ``oracle/_ref/libdpref.so``, the reference DeePMD-kit CPU library
  compiled from its own sources (``source/lib/src/*.cc``) plus
  ``oracle/ref_shim.cc``; present only where the reference tree was available
  at build time.

``ref_gpu()`` loads ``oracle/_ref/libdpref_gpu.so``, the reference's own CUDA
kernels (``source/lib/src/gpu/*.cu``, built for sm_100a) behind
``oracle/ref_gpu_shim.cu``, for the GPU tests that compare them with this
package's drop-ins.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product never does.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "libdporacle.so")
REF_SO = os.path.join(HERE, "_ref", "libdpref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libdpref_gpu.so")
# the reference source tree, given by the environment (no built-in location)
REF_TREE = os.environ.get("DEEPMD_REFERENCE_TREE", "")

_i = ctypes.c_int
_f = ctypes.c_float
_p = ctypes.c_void_p


def _have_tree(tree: str) -> bool:
    return bool(tree) and os.path.isdir(os.path.join(tree, "source", "lib"))


def build(ref: bool | None = None, ref_gpu: bool | None = None,
          ref_tree: str | None = None) -> None:
    """Compile the checkers with ``make -C oracle`` (the reference libraries
    only when its source tree is given -- ``ref_tree`` or the environment
    variable DEEPMD_REFERENCE_TREE -- and exists; the GPU one also needs
    nvcc)."""
    tree = ref_tree if ref_tree is not None else REF_TREE
    targets = ["port"]
    have_tree = _have_tree(tree)
    if ref is None:
        ref = have_tree
    if ref_gpu is None:
        ref_gpu = have_tree and os.path.exists("/usr/local/cuda/bin/nvcc")
    if ref:
        targets.append("ref")
    if ref_gpu:
        targets.append("refgpu")
    extra = [f"REF={tree}"] if have_tree else []
    subprocess.run(["make", "-s", "-C", HERE, *targets, *extra], check=True)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_p)


class _Lib:
    """One checker library; `prefix` is "orc" (port) or "dpref" (reference)."""

    def __init__(self, path: str, prefix: str):
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        self.kind = "port" if prefix == "orc" else "reference"

    def fn(self, name: str):
        f = getattr(self.lib, f"{self.prefix}_{name}")
        f.restype = _i
        return f

    # ------------------------------------------------------------ geometry
    def normalize_coord(self, coord, boxt):
        c = np.ascontiguousarray(coord, dtype=np.float64).copy()
        b = np.ascontiguousarray(boxt, dtype=np.float64).reshape(9)
        name = "normalize_coord" if self.prefix == "orc" else "normalize_coord_f64"
        f = getattr(self.lib, f"{self.prefix}_{name}")
        f(_ptr(c), _i(c.size // 3), _ptr(b))
        return c

    def copy_coord(self, coord, atype, rcut, boxt, mem_nall=None):
        c = np.ascontiguousarray(coord, dtype=np.float64).reshape(-1)
        t = np.ascontiguousarray(atype, dtype=np.int32).reshape(-1)
        b = np.ascontiguousarray(boxt, dtype=np.float64).reshape(9)
        nloc = t.size
        mem = mem_nall if mem_nall is not None else max(64, nloc * 30)
        out_c = np.zeros(mem * 3, np.float64)
        out_t = np.zeros(mem, np.int32)
        mapping = np.zeros(mem, np.int32)
        nall = ctypes.c_int(0)
        name = "copy_coord" if self.prefix == "orc" else "copy_coord_f64"
        f = getattr(self.lib, f"{self.prefix}_{name}")
        f.restype = _i
        ret = f(_ptr(out_c), _ptr(out_t), _ptr(mapping), ctypes.byref(nall),
                _ptr(c), _ptr(t), _i(nloc), _i(mem), _f(rcut), _ptr(b))
        n = nall.value
        if ret == 1 and mem_nall is None:
            return self.copy_coord(coord, atype, rcut, boxt, mem_nall=n)
        if ret != 0:
            raise RuntimeError(f"copy_coord failed ({ret}); nall={n}")
        return out_c[: 3 * n].reshape(n, 3), out_t[:n].copy(), mapping[:n].copy()

    def cell_info(self, rcut, boxt):
        b = np.ascontiguousarray(boxt, dtype=np.float64).reshape(9)
        ci = np.zeros(23, np.int32)
        name = "compute_cell_info" if self.prefix == "orc" else "compute_cell_info_f64"
        f = getattr(self.lib, f"{self.prefix}_{name}")
        f.restype = _i
        if f(_ptr(ci), _f(rcut), _ptr(b)) != 0:
            raise RuntimeError("compute_cell_info failed")
        return ci

    def build_nlist(self, c_cpy, nloc, rcut, atype=None, mem_size=None, nframes=1):
        dt = c_cpy.dtype
        suf = "f64" if dt == np.float64 else "f32"
        c = np.ascontiguousarray(c_cpy).reshape(-1)
        nall = c.size // 3 // nframes
        mem = mem_size if mem_size is not None else nall
        rows = nframes * nloc
        ilist = np.zeros(rows, np.int32)
        numneigh = np.zeros(rows, np.int32)
        rowbuf = np.full(rows * max(mem, 1), -1, np.int32)
        mx = ctypes.c_int(0)
        t = None if atype is None else np.ascontiguousarray(atype, dtype=np.int32)
        ret = self.fn(f"build_nlist_{suf}")(
            _ptr(ilist), _ptr(numneigh), _ptr(rowbuf), ctypes.byref(mx), _ptr(c),
            _i(nloc), _i(nall), _i(mem), _f(rcut), _i(nframes), _ptr(t))
        return ret, ilist, numneigh, rowbuf.reshape(rows, max(mem, 1)), mx.value

    # ------------------------------------------------------------- env mat
    def prod_env_mat_a(self, coord, atype, ilist, numneigh, rowbuf, avg, std,
                       nloc, rcut, rcut_smth, sec, nframes=1):
        dt = np.float64 if coord.dtype == np.float64 else np.float32
        suf = "f64" if dt == np.float64 else "f32"
        c = np.ascontiguousarray(coord, dtype=dt).reshape(-1)
        t = np.ascontiguousarray(atype, dtype=np.int32).reshape(-1)
        nall = t.size // nframes
        nnei = int(sec[-1])
        rows = nframes * nloc
        em = np.zeros(rows * nnei * 4, dt)
        emd = np.zeros(rows * nnei * 12, dt)
        rij = np.zeros(rows * nnei * 3, dt)
        nlist = np.zeros(rows * nnei, np.int32)
        s = np.ascontiguousarray(sec, dtype=np.int32)
        rb = np.ascontiguousarray(rowbuf, dtype=np.int32)
        ret = self.fn(f"prod_env_mat_a_{suf}")(
            _ptr(em), _ptr(emd), _ptr(rij), _ptr(nlist), _ptr(c), _ptr(t),
            _i(rows), _ptr(np.ascontiguousarray(ilist, np.int32)),
            _ptr(np.ascontiguousarray(numneigh, np.int32)), _ptr(rb),
            _i(rb.shape[1]), _ptr(np.ascontiguousarray(avg, dt)),
            _ptr(np.ascontiguousarray(std, dt)), _i(nloc), _i(nall),
            _i(nframes), _f(rcut), _f(rcut_smth), _ptr(s), _i(s.size))
        if ret != 0:
            raise RuntimeError("prod_env_mat_a failed")
        return (em.reshape(rows, nnei * 4), emd.reshape(rows, nnei * 12),
                rij.reshape(rows, nnei * 3), nlist.reshape(rows, nnei))

    # ------------------------------------------------------------ tabulate
    def tabulate(self, table, info, em_x, em, M):
        dt = table.dtype
        suf = "f64" if dt == np.float64 else "f32"
        nloc, nnei = em.shape[0], em.shape[1]
        out = np.zeros(nloc * 4 * M, dt)
        self.fn(f"tabulate_fusion_se_a_{suf}")(
            _ptr(out), _ptr(np.ascontiguousarray(table)), _ptr(np.ascontiguousarray(info, dt)),
            _ptr(np.ascontiguousarray(em_x, dt)), _ptr(np.ascontiguousarray(em, dt)),
            _i(nloc), _i(nnei), _i(M))
        return out.reshape(nloc, 4, M)

    def tabulate_grad(self, table, info, em_x, em, dy, M):
        dt = table.dtype
        suf = "f64" if dt == np.float64 else "f32"
        nloc, nnei = em.shape[0], em.shape[1]
        dx = np.zeros(nloc * nnei, dt)
        de = np.zeros(nloc * nnei * 4, dt)
        self.fn(f"tabulate_fusion_se_a_grad_{suf}")(
            _ptr(dx), _ptr(de), _ptr(np.ascontiguousarray(table)),
            _ptr(np.ascontiguousarray(info, dt)), _ptr(np.ascontiguousarray(em_x, dt)),
            _ptr(np.ascontiguousarray(em, dt)), _ptr(np.ascontiguousarray(dy, dt)),
            _i(nloc), _i(nnei), _i(M))
        return dx.reshape(nloc, nnei), de.reshape(nloc, nnei, 4)

    def tabulate_grad_grad(self, table, info, em_x, em, dz_dem_x, dz_dem, M):
        dt = table.dtype
        suf = "f64" if dt == np.float64 else "f32"
        nloc, nnei = em.shape[0], em.shape[1]
        out = np.zeros(nloc * 4 * M, dt)
        self.fn(f"tabulate_fusion_se_a_grad_grad_{suf}")(
            _ptr(out), _ptr(np.ascontiguousarray(table)),
            _ptr(np.ascontiguousarray(info, dt)), _ptr(np.ascontiguousarray(em_x, dt)),
            _ptr(np.ascontiguousarray(em, dt)), _ptr(np.ascontiguousarray(dz_dem_x, dt)),
            _ptr(np.ascontiguousarray(dz_dem, dt)), _i(nloc), _i(nnei), _i(M))
        return out.reshape(nloc, 4, M)

    # ------------------------------------------------------- force / virial
    def prod_force_a(self, net_deriv, env_deriv, nlist, nloc, nall, nframes=1):
        dt = net_deriv.dtype
        suf = "f64" if dt == np.float64 else "f32"
        nnei = nlist.size // (nframes * nloc)
        force = np.zeros(nframes * nall * 3, dt)
        self.fn(f"prod_force_a_{suf}")(
            _ptr(force), _ptr(np.ascontiguousarray(net_deriv)),
            _ptr(np.ascontiguousarray(env_deriv, dt)),
            _ptr(np.ascontiguousarray(nlist, np.int32)), _i(nloc), _i(nall),
            _i(nnei), _i(nframes))
        return force.reshape(nframes, nall, 3)

    def prod_virial_a(self, net_deriv, env_deriv, rij, nlist, nloc, nall):
        dt = net_deriv.dtype
        suf = "f64" if dt == np.float64 else "f32"
        nnei = nlist.size // nloc
        virial = np.zeros(9, dt)
        av = np.zeros(nall * 9, dt)
        self.fn(f"prod_virial_a_{suf}")(
            _ptr(virial), _ptr(av), _ptr(np.ascontiguousarray(net_deriv)),
            _ptr(np.ascontiguousarray(env_deriv, dt)), _ptr(np.ascontiguousarray(rij, dt)),
            _ptr(np.ascontiguousarray(nlist, np.int32)), _i(nloc), _i(nall), _i(nnei))
        return virial, av.reshape(nall, 9)

    def prod_force_grad_a(self, grad, env_deriv, nlist, nloc, nframes=1):
        dt = env_deriv.dtype
        suf = "f64" if dt == np.float64 else "f32"
        nnei = nlist.size // (nframes * nloc)
        out = np.zeros(nframes * nloc * nnei * 4, dt)
        self.fn(f"prod_force_grad_a_{suf}")(
            _ptr(out), _ptr(np.ascontiguousarray(grad, dt)),
            _ptr(np.ascontiguousarray(env_deriv)),
            _ptr(np.ascontiguousarray(nlist, np.int32)), _i(nloc), _i(nnei), _i(nframes))
        return out.reshape(nframes * nloc, nnei * 4)

    def prod_virial_grad_a(self, grad, env_deriv, rij, nlist, nloc):
        dt = env_deriv.dtype
        suf = "f64" if dt == np.float64 else "f32"
        nnei = nlist.size // nloc
        out = np.zeros(nloc * nnei * 4, dt)
        self.fn(f"prod_virial_grad_a_{suf}")(
            _ptr(out), _ptr(np.ascontiguousarray(grad, dt)),
            _ptr(np.ascontiguousarray(env_deriv)), _ptr(np.ascontiguousarray(rij, dt)),
            _ptr(np.ascontiguousarray(nlist, np.int32)), _i(nloc), _i(nnei))
        return out.reshape(nloc, nnei * 4)


_cache: dict[str, _Lib] = {}


def port() -> _Lib:
    """The C restatement (builds it on first use if missing)."""
    if "port" not in _cache:
        if not os.path.exists(PORT_SO):
            build(ref=False)
        _cache["port"] = _Lib(PORT_SO, "orc")
    return _cache["port"]


def ref() -> _Lib | None:
    """The compiled reference CPU library, or None where it was not built."""
    if "ref" not in _cache:
        if not os.path.exists(REF_SO):
            if _have_tree(REF_TREE):
                build(ref=True)
            else:
                return None
        _cache["ref"] = _Lib(REF_SO, "dpref")
    return _cache["ref"]


def ref_gpu():
    """ctypes handle of the reference CUDA kernels (refgpu_* entry points, each
    returning 0 or 1 when the reference raised), or None where not built."""
    if "ref_gpu" not in _cache:
        if not os.path.exists(REF_GPU_SO):
            return None
        lib = ctypes.CDLL(REF_GPU_SO)
        for name in ("build_nlist_f64", "prod_env_mat_a_f64", "prod_env_mat_a_f32",
                     "tabulate_fusion_se_a_f64", "tabulate_fusion_se_a_f32",
                     "tabulate_fusion_se_a_grad_f64", "tabulate_fusion_se_a_grad_f32",
                     "prod_force_a_f64", "prod_force_a_f32", "prod_virial_a_f64",
                     "prod_virial_a_f32"):
            getattr(lib, "refgpu_" + name).restype = _i
        _cache["ref_gpu"] = lib
    return _cache["ref_gpu"]


def best() -> _Lib:
    """The reference library where available, else the restatement."""
    return ref() or port()


def format_nlist_i(posi, atype, i_idx, cand, rcut, sec):
    """Restated format_nlist_i_cpu for one atom (fmt_nlist.cc:98-143)."""
    lib = port().lib
    dt = posi.dtype
    suf = "f64" if dt == np.float64 else "f32"
    n = int(sec[-1])
    out = np.zeros(n, np.int32)
    c = np.ascontiguousarray(cand, np.int32)
    s = np.ascontiguousarray(sec, np.int32)
    f = getattr(lib, f"orc_format_nlist_i_{suf}")
    f.restype = _i
    r = f(_ptr(out), _ptr(np.ascontiguousarray(posi).reshape(-1)),
          _ptr(np.ascontiguousarray(atype, np.int32)), _i(i_idx), _ptr(c),
          _i(c.size), _f(rcut), _ptr(s), _i(s.size))
    return r, out


def rec_boxt(boxt):
    """Restated reciprocal box (SimulationRegion_Impl.h:455-480)."""
    lib = port().lib
    b = np.ascontiguousarray(boxt, np.float64).reshape(9)
    r = np.zeros(9, np.float64)
    v = ctypes.c_double(0)
    lib.orc_rec_boxt(_ptr(r), ctypes.byref(v), _ptr(b))
    return r, v.value
