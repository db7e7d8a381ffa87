"""Many frames of uneven size and species mix evaluated together, captured as
one CUDA graph. Two forms of the step:

* fused (default, knob batch_fused = 1): ONE persistent cooperative launch
  per step (dpb_bt_step_launch): cells, env rows + descriptor forward, the six
  fitting GEMMs on the tensor cores, descriptor backward + forces, energies,
  separated by grid barriers inside the kernel;
* staged: one launch per stage over all frames (geometry through per-frame
  cell lists with periodic images, dpb_batch_env_mat_a_f32; the descriptor
  and the tensor-core fitting over the concatenated rows;
  dpb_batch_force_virial_a and dpb_batch_energy per frame).

Frames must have orthorhombic boxes whose edges are all at least rcut.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi
from ._capi import call, ptr
from .model import DEFAULT_TABLE_DEGREE, PipelineTables, SeAParams, _FittingTC

CELL_MARGIN = 1.0001  # cell edge >= rcut * margin, as the single-frame grid

_P, _I, _F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float


class GemmLayer(ctypes.Structure):
    """dpb_gemm_layer of include/dpb200.h."""
    _fields_ = [("A", _P), ("K", _I), ("b_hi", _P), ("b_lo", _P), ("N", _I), ("mode", _I),
                ("out0", _P), ("out1", _P), ("aux0", _P), ("aux1", _P), ("bias", _P),
                ("idt", _P), ("w", _P)]


class BtStepDesc(ctypes.Structure):
    """dpb_bt_step_desc of include/dpb200.h."""
    _fields_ = [("nframes", _I), ("nrows", _I), ("atom_off", _P), ("cell_off", _P),
                ("box", _P), ("ncell", _P), ("row_frame", _P), ("coord", _P), ("type", _P),
                ("cw", _P), ("cell_of", _P), ("cell_start", _P), ("cell_atoms", _P),
                ("avg", _P), ("std_", _P), ("rcut", _F), ("rcut_smth", _F), ("sec", _P),
                ("nsec", _I), ("em", _P), ("nlist", _P), ("tables", _P), ("table_info", _P),
                ("table_degree", _I), ("M", _I), ("naxis", _I), ("drow", _P), ("xyz", _P),
                ("descrpt", _P), ("d_descrpt", _P), ("net_deriv", _P), ("type_rows", _P),
                ("ntypes", _I), ("fit", GemmLayer * 6), ("e_rows", _P), ("e_const", _P),
                ("energy", _P), ("force", _P), ("virial", _P), ("sync", _P), ("status", _P),
                ("pass_ns", _P)]


class FrameTable:
    """Device frame table of F frames whose atoms are concatenated in frame
    order: atom_off [F + 1], cell_off [F + 1], box [F, 3], ncell [F, 3],
    row_frame [N], type [N], drow [N] (the atom's row when rows are grouped
    by type, stable) and the geometry scratch (cw, cell_of, cell_atoms,
    cell_start). Frames need orthorhombic boxes with every edge >= rcut."""

    def __init__(self, cfg, frames, device):
        self.dev = dev = torch.device(device)
        self.nframes = F = len(frames)
        if F == 0:
            raise _capi.DPBInvalidArgument("no frames")
        counts, boxes, ncell, types = [], [], [], []
        for f, (_, atype, box) in enumerate(frames):
            b = np.asarray(box, np.float64).reshape(3, 3)
            if np.any(b - np.diag(np.diag(b))):
                raise _capi.DPBInvalidArgument(f"frame {f}: the batched path needs an "
                                               "orthorhombic box")
            L = np.diag(b)
            nc = np.floor(L / (cfg.rcut * CELL_MARGIN)).astype(np.int64)
            if np.any(nc < 1):
                raise _capi.DPBInvalidArgument(
                    f"frame {f}: box edges {L} must be at least rcut ({cfg.rcut})")
            if int(np.prod(nc)) > 4096 or atype.size > 600000:
                raise _capi.DPBInvalidArgument(f"frame {f}: more than 4096 cells or 600,000 "
                                               "atoms")
            if atype.size and (atype.min() < 0 or atype.max() >= cfg.ntypes):
                raise _capi.DPBInvalidArgument(f"frame {f}: atom types outside "
                                               f"[0, {cfg.ntypes})")
            counts.append(int(atype.size))
            boxes.append(L)
            ncell.append(nc)
            types.append(np.asarray(atype, np.int32))
        self.counts = np.array(counts)
        self.N = N = int(self.counts.sum())
        atom_off = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int32)
        cells = np.array([int(np.prod(c)) + 1 for c in ncell])
        cell_off = np.concatenate([[0], np.cumsum(cells)]).astype(np.int32)
        row_frame = np.repeat(np.arange(F, dtype=np.int32), self.counts)
        self.atype = atype_all = np.concatenate(types)
        self.types = types
        i32 = lambda a: torch.tensor(np.ascontiguousarray(a, np.int32), device=dev)  # noqa: E731
        self.atom_off_h = atom_off
        self.atom_off, self.cell_off = i32(atom_off), i32(cell_off)
        self.box = torch.tensor(np.array(boxes), dtype=torch.float64, device=dev)
        self.ncell = i32(np.array(ncell))
        self.row_frame_h = row_frame
        self.row_frame = i32(row_frame)
        self.type = i32(atype_all)
        self.cw = torch.zeros((N, 3), dtype=torch.float64, device=dev)
        self.cell_of = torch.zeros(N, dtype=torch.int32, device=dev)
        self.cell_atoms = torch.zeros(N, dtype=torch.int32, device=dev)
        self.cell_start = torch.zeros(int(cell_off[-1]), dtype=torch.int32, device=dev)
        order = np.argsort(atype_all, kind="stable")
        drow = np.empty(N, np.int32)
        drow[order] = np.arange(N, dtype=np.int32)
        self.drow_h = drow
        self.drow = i32(drow)
        self.tcount = np.bincount(atype_all, minlength=cfg.ntypes)

    def frame_slice(self, f: int) -> slice:
        return slice(int(self.atom_off_h[f]), int(self.atom_off_h[f + 1]))


class BatchEvaluator:
    """Energy [F], force [N, 3] and virial [F, 9] of F frames whose atoms are
    concatenated in frame order (compressed FP32 path, FP64 sums)."""

    def __init__(self, params: SeAParams, frames, device="cuda:0",
                 table_degree: int = DEFAULT_TABLE_DEGREE, fused: bool | None = None):
        cfg = params.cfg
        self.cfg, self.params = cfg, params
        self.dev = dev = torch.device(device)
        self.ft = ft = FrameTable(cfg, frames, dev)
        self.nframes = F = ft.nframes
        self.counts, self.N, N = ft.counts, ft.N, ft.N
        self.atom_off_h = ft.atom_off_h
        self.atom_off, self.cell_off, self.box, self.ncell = (ft.atom_off, ft.cell_off, ft.box,
                                                              ft.ncell)
        self.row_frame, self.type, self.drow = ft.row_frame, ft.type, ft.drow
        self.cw, self.cell_of, self.cell_atoms, self.cell_start = (ft.cw, ft.cell_of,
                                                                   ft.cell_atoms, ft.cell_start)
        nnei, M, ax = cfg.nnei, cfg.neuron[-1], cfg.axis_neuron
        f64, f32 = torch.float64, torch.float32
        z = lambda shape, dt: torch.zeros(shape, dtype=dt, device=dev)  # noqa: E731
        self.coord = z((N, 3), f64)
        self.em = z((N, nnei * 4), f32)
        self.nlist = z((N, nnei), torch.int32)
        self.xyz = z((N, 4, M), f32)
        self.D = z((N, M * ax), f32)
        self.dD = z((N, M * ax), f32)
        self.net_deriv = z((N, nnei * 4), f32)
        self.force = z((N, 3), f64)
        self.virial = z((F, 9), f64)
        self.energy = z(F, f64)
        self.status = z(1, torch.int32)
        self.avg = torch.tensor(params.davg, dtype=f32, device=dev)
        self.std = torch.tensor(params.dstd, dtype=f32, device=dev)
        self.fit = _FittingTC(params, ft.tcount, dev)
        const_t = np.array([float(params.fit[t]["out"][1][0]) + float(params.bias_atom_e[t])
                            for t in range(cfg.ntypes)])
        per_frame = np.array([np.bincount(t, minlength=cfg.ntypes) @ const_t for t in ft.types])
        self.e_const = torch.tensor(per_frame, dtype=f64, device=dev)
        self.ptab = PipelineTables(params, dev, table_degree)
        self.graph = None
        self.plan = None
        if fused is None:
            fused = _capi.lib().dpb_tune_get(b"batch_fused") != 0
        if fused:
            self._make_plan()
        self.set_coords([fr[0] for fr in frames])

    def _make_plan(self):
        """The description of the one-launch step (dpb_bt_step_create)."""
        cfg, ft, fit = self.cfg, self.ft, self.fit
        M, ax = cfg.neuron[-1], cfg.axis_neuron
        w, din = fit.width, fit.din
        self.sync = torch.zeros(8, dtype=torch.int32, device=self.dev)
        # global timer at the start and after each pass of the launch (ns)
        self.pass_ns = torch.zeros(12, dtype=torch.int64, device=self.dev)
        d = BtStepDesc()
        d.nframes, d.nrows = self.nframes, self.N
        for name, t in (("atom_off", self.atom_off), ("cell_off", self.cell_off),
                        ("box", self.box), ("ncell", self.ncell), ("row_frame", self.row_frame),
                        ("coord", self.coord), ("type", self.type), ("cw", self.cw),
                        ("cell_of", self.cell_of), ("cell_start", self.cell_start),
                        ("cell_atoms", self.cell_atoms), ("avg", self.avg), ("std_", self.std),
                        ("em", self.em), ("nlist", self.nlist), ("drow", self.drow),
                        ("xyz", self.xyz), ("descrpt", self.D), ("d_descrpt", self.dD),
                        ("net_deriv", self.net_deriv), ("e_rows", fit.e),
                        ("e_const", self.e_const), ("energy", self.energy),
                        ("force", self.force), ("virial", self.virial), ("sync", self.sync),
                        ("status", self.status), ("pass_ns", self.pass_ns)):
            setattr(d, name, t.data_ptr())
        d.rcut, d.rcut_smth = cfg.rcut, cfg.rcut_smth
        self._sec = np.ascontiguousarray(cfg.sec, dtype=np.int32)
        d.sec, d.nsec = self._sec.ctypes.data, self._sec.size
        pt = self.ptab
        d.tables = ctypes.cast(pt.ptrs, _P)
        d.table_info = pt.info.ctypes.data
        d.table_degree, d.M, d.naxis = pt.degree, M, ax
        d.type_rows, d.ntypes = fit.type_rows.ctypes.data, fit.ntypes
        E = fit

        def layer(A, K, B, N, mode, out0, out1=None, aux0=None, aux1=None, bias=None,
                  idt=None, wv=None):
            g = GemmLayer()
            g.A, g.K, g.N, g.mode = A.data_ptr(), K, N, mode
            g.b_hi, g.b_lo = ctypes.cast(B[0], _P), ctypes.cast(B[1], _P)
            for name, t in (("out0", out0), ("out1", out1), ("aux0", aux0), ("aux1", aux1)):
                setattr(g, name, None if t is None else t.data_ptr())
            for name, v in (("bias", bias), ("idt", idt), ("w", wv)):
                setattr(g, name, None if v is None else ctypes.cast(v, _P))
            return g

        layers = [
            layer(self.D, din, E.B1f, w, E.EPI_TANH, E.H1, bias=E.b1),
            layer(E.H1, w, E.B2f, w, E.EPI_RES_DT, E.Y2, E.H2, aux0=E.H1, bias=E.b2, idt=E.d2),
            layer(E.H2, w, E.B3f, w, E.EPI_LAST, E.G3, aux0=E.H2, bias=E.b3, idt=E.d3,
                  wv=E.w4),
            layer(E.G3, w, E.B3b, w, E.EPI_BWD_DT, E.G2, E.g2, aux0=E.Y2, idt=E.d2, wv=E.w4),
            layer(E.G2, w, E.B2b, w, E.EPI_BWD_RES, E.G1, aux0=E.H1, aux1=E.g2),
            layer(E.G1, w, E.B1b, din, E.EPI_STORE, self.dD)]
        for k, g in enumerate(layers):
            d.fit[k] = g
        self._desc = d
        handle = ctypes.c_void_p()
        call("dpb_bt_step_create", ctypes.byref(handle), ctypes.byref(d))
        self._split = _capi.lib().dpb_tune_get(b"batch_fused_split") != 0
        self.plan = handle

    def pass_times_us(self) -> dict | None:
        """Durations (us) of the passes of the last one-launch step, from the
        global timer read by the first CTA after each grid barrier."""
        if self.plan is None:
            return None
        t = self.pass_ns.cpu().numpy().astype(np.float64)
        fit = ["fit_layer1", "fit_layer2", "fit_layer3", "fit_layer3_bwd", "fit_layer2_bwd",
               "fit_layer1_bwd"]
        if self._split:
            names = ["cells", "env", "descriptor_fwd"] + fit + ["energy_descriptor_bwd",
                                                                 "force_virial"]
        else:
            names = ["cells", "env_descriptor_fwd"] + fit + ["energy_descriptor_bwd_force"]
        return {n: (t[k + 1] - t[k]) / 1e3 for k, n in enumerate(names)}

    def __del__(self):
        if getattr(self, "plan", None) is not None and _capi is not None:
            try:
                _capi.lib().dpb_bt_step_destroy(self.plan)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self.plan = None

    def set_coords(self, coords):
        """Host coordinates of every frame (a list, or one [N, 3] array)."""
        c = np.concatenate([np.asarray(x, np.float64).reshape(-1, 3) for x in coords]) \
            if isinstance(coords, (list, tuple)) else np.asarray(coords, np.float64)
        self.coord.copy_(torch.as_tensor(c.reshape(self.N, 3)))

    # ---- one step over all frames, no host synchronisation
    def step(self):
        cfg, s = self.cfg, torch.cuda.current_stream().cuda_stream
        if self.plan is not None:
            call("dpb_bt_step_launch", self.plan, s)
            return
        M, ax, F, N = cfg.neuron[-1], cfg.axis_neuron, self.nframes, self.N
        call("dpb_batch_env_mat_a_f32", ptr(self.em), ptr(self.nlist), ptr(self.cw),
             ptr(self.cell_of), ptr(self.cell_start), ptr(self.cell_atoms), ptr(self.coord),
             ptr(self.type), ptr(self.avg), ptr(self.std), ptr(self.atom_off),
             ptr(self.cell_off), ptr(self.box), ptr(self.ncell), ptr(self.row_frame), F, N,
             ctypes.c_float(cfg.rcut), ctypes.c_float(cfg.rcut_smth), cfg.sec.ctypes.data,
             cfg.sec.size, ptr(self.status), s)
        pt = self.ptab
        call(pt.fwd, ptr(self.xyz), ptr(self.D), ptr(self.drow), ptr(self.em), pt.ptrs,
             pt.info.ctypes.data, cfg.sec.ctypes.data, cfg.sec.size, N, M, ax, s)
        self.fit.layers(self.D, self.dD)
        call(pt.bwd, ptr(self.net_deriv), ptr(self.dD), ptr(self.drow), ptr(self.xyz),
             ptr(self.em), pt.ptrs, pt.info.ctypes.data, cfg.sec.ctypes.data, cfg.sec.size, N,
             M, ax, s)
        call("dpb_batch_force_virial_a", ptr(self.force), ptr(self.virial),
             ptr(self.net_deriv), ptr(self.cw), ptr(self.type), ptr(self.std),
             ptr(self.nlist), ptr(self.atom_off), ptr(self.cell_off), ptr(self.box),
             ptr(self.ncell), ptr(self.row_frame), F, N, cfg.nnei, cfg.ntypes,
             ctypes.c_float(cfg.rcut), ctypes.c_float(cfg.rcut_smth), s)
        call("dpb_batch_energy", ptr(self.energy), ptr(self.fit.e), ptr(self.drow),
             ptr(self.e_const), ptr(self.atom_off), F, s)

    def capture(self, warmup: int = 2):
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self.step()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.step()
        torch.cuda.synchronize()
        return self

    def replay(self):
        if self.graph is None:
            self.step()
        else:
            self.graph.replay()

    def check(self):
        """Raise if a step overflowed a capacity (reads the status words)."""
        s = torch.cuda.current_stream().cuda_stream
        call("dpb_status_check", ptr(self.status), s)
        call("dpb_status_check", ptr(self.fit.status), s)

    def compute(self, coords=None):
        """(energy [F], force [N, 3], virial [F, 9]) as host arrays."""
        if coords is not None:
            self.set_coords(coords)
        self.replay()
        torch.cuda.synchronize()
        return (self.energy.cpu().numpy(), self.force.cpu().numpy(),
                self.virial.cpu().numpy())

    def frame_slice(self, f: int) -> slice:
        return slice(int(self.atom_off_h[f]), int(self.atom_off_h[f + 1]))

    def tune(self, reps: int = 10, use_cache: bool = True) -> dict:
        """Autotune the tile shapes of this step (atoms per CTA of the env /
        force and descriptor kernels, fitting GEMM N tile) on its own frames;
        leaves the step captured with the fastest shapes."""
        from . import autotune

        if self.plan is not None:  # the one-launch step has its shapes fixed
            self.capture()
            return {}
        cfg = self.cfg
        sig = (f"batch:{self.nframes}f:{self.N}a:deg{self.ptab.degree}:"
               f"sel{'-'.join(map(str, cfg.sel))}:"
               f"M{cfg.neuron[-1]}:fit{'-'.join(map(str, cfg.fitting))}")
        return autotune.tune(self.replay, lambda: self.capture(),
                             ["batch_atoms_per_cta", "desc_atoms_per_cta", "desc_coef_l1",
                              "fit_n_tile", "fit_split_b", "pdl"],
                             signature=sig, reps=reps, device=self.dev, use_cache=use_cache)
