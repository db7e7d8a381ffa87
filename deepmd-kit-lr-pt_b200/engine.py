"""The MD-engine entry point of the compressed se_e2_a path: forward_lower.

An engine such as LAMMPS keeps its own extended system (local atoms first,
then the ghosts its domain decomposition made) and its own neighbor list of
the local atoms, built with a skin and reused for several steps. The
reference serves it through the model's ``forward_lower`` (DeepPotPT.cc:
171-378 calls deepmd/pt/model/model/make_model.py:528-646 with the extended
coordinates, types, the padded neighbor list and the ghost-to-owner mapping)
and gets back the energy, the forces on every EXTENDED atom (the engine sums
ghost forces onto their owners in its reverse communication) and the
virial. ``ForwardLower`` does the same on this package's kernels:

  the engine's list (any order, within rcut + skin) is formatted against
  rcut into the sel slots and the env matrix (dpb_prod_env_mat_a_mixed),
  then the fused compressed descriptor, the tensor-core fitting, the
  descriptor backward, and the force / virial pass with an identity mapping
  (so forces stay on the extended atoms; virial = sum over pairs of
  f_ij (x) r_ij, prod_virial.cc:55-63).

Types of the local atoms fix the grouping of fitting rows by center type; it
is recomputed when ``rebuilt=True`` is passed (the engine re-neighbored).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi, ops
from ._capi import call, ptr
from .model import DEFAULT_TABLE_DEGREE, PipelineTables, SeAParams, _FittingTC


class ForwardLower:
    """forward_lower of a compressed se_e2_a model for an engine's system of
    at most ``nloc_max`` local and ``nall_max`` extended atoms whose neighbor
    rows hold at most ``max_nbor`` entries."""

    def __init__(self, params: SeAParams, nloc_max: int, nall_max: int, max_nbor: int = 512,
                 device="cuda:0", table_degree: int = DEFAULT_TABLE_DEGREE):
        cfg = params.cfg
        if not params.tables:
            raise _capi.DPBInvalidArgument("forward_lower needs the compressed model's tables")
        self.cfg, self.params = cfg, params
        self.dev = dev = torch.device(device)
        self.nloc_max, self.nall_max, self.max_nbor = int(nloc_max), int(nall_max), int(max_nbor)
        nnei, M, ax = cfg.nnei, cfg.neuron[-1], cfg.axis_neuron
        f32, f64 = torch.float32, torch.float64
        z = lambda shape, dt: torch.zeros(shape, dtype=dt, device=dev)  # noqa: E731
        n = self.nloc_max
        self.em = z((n, nnei * 4), f32)
        self.nlist = z((n, nnei), torch.int32)
        self.net_deriv = z((n, nnei * 4), f32)
        self.xyz = z((n, 4, M), f32)
        self.D = z((n, M * ax), f32)
        self.dD = z((n, M * ax), f32)
        # energy, extended force and virial side by side
        self.results = z(1 + 3 * self.nall_max + 9, f64)
        self.identity = torch.arange(self.nall_max, dtype=torch.int32, device=dev)
        self.status = z(1, torch.int32)
        self.avg = torch.tensor(params.davg, dtype=f32, device=dev)
        self.std = torch.tensor(params.dstd, dtype=f32, device=dev)
        self.ptab = PipelineTables(params, dev, table_degree)
        self.fit = None
        self.nloc = -1

    def _group(self, atype_loc: np.ndarray):
        """Fitting rows grouped by center type for the current local types."""
        cfg = self.cfg
        order = np.argsort(atype_loc, kind="stable")
        row = np.empty(atype_loc.size, np.int32)
        row[order] = np.arange(atype_loc.size, dtype=np.int32)
        self.drow = torch.tensor(row, device=self.dev)
        counts = np.bincount(atype_loc, minlength=cfg.ntypes)
        self.fit = _FittingTC(self.params, counts, self.dev)

    def __call__(self, ext_coord: torch.Tensor, ext_atype: torch.Tensor, nloc: int,
                 numneigh: torch.Tensor, firstneigh: torch.Tensor, ilist: torch.Tensor | None = None,
                 rebuilt: bool = False):
        """(energy [1] FP64, extended force [nall, 3] FP64, virial [9] FP64)
        as device tensors (views of one result buffer, valid until the next
        call). ext_coord [nall, 3] FP64 and ext_atype [nall] int32 on the
        device, local atoms first; numneigh [nloc] and firstneigh [nloc]
        (device row pointers, int64) the engine's list of the local atoms,
        rows of at most max_nbor extended-atom indices within rcut + skin in
        any order; ilist [nloc] (default 0..nloc-1)."""
        cfg, s = self.cfg, torch.cuda.current_stream(self.dev).cuda_stream
        nall = int(ext_coord.shape[0])
        if nloc > self.nloc_max or nall > self.nall_max or nloc > nall:
            raise _capi.DPBInvalidArgument(
                f"forward_lower: nloc={nloc}, nall={nall} exceed the capacity "
                f"({self.nloc_max}, {self.nall_max})")
        ops._need_cuda(ext_coord, ext_atype, numneigh, firstneigh, what="forward_lower")
        c = ext_coord.to(torch.float64).contiguous()
        t = ext_atype.to(torch.int32).contiguous()
        if rebuilt or self.fit is None or nloc != self.nloc:
            self._group(t[:nloc].cpu().numpy())
            self.nloc = nloc
            self._ilist = torch.arange(nloc, dtype=torch.int32, device=self.dev)
        il = self._ilist if ilist is None else ilist.to(torch.int32).contiguous()
        M, ax = cfg.neuron[-1], cfg.axis_neuron
        sec = cfg.sec
        call("dpb_zero_async", ptr(self.results), 8 * self.results.numel(), s)
        energy = self.results[0:1]
        force = self.results[1:1 + 3 * nall].view(nall, 3)
        virial = self.results[1 + 3 * self.nall_max:]
        call("dpb_prod_env_mat_a_mixed", ptr(self.em), None, None, ptr(self.nlist), ptr(c),
             ptr(t), nloc, ptr(il), ptr(numneigh.to(torch.int32).contiguous()),
             ptr(firstneigh), self.max_nbor, ptr(self.avg), ptr(self.std), nloc, nall, 1,
             ctypes.c_float(cfg.rcut), ctypes.c_float(cfg.rcut_smth), sec.ctypes.data, sec.size,
             ptr(self.status), s)
        pt = self.ptab
        call(pt.fwd, ptr(self.xyz), ptr(self.D), ptr(self.drow), ptr(self.em), pt.ptrs,
             pt.info.ctypes.data, sec.ctypes.data, sec.size, nloc, M, ax, s)
        self.fit.forward_backward(self.D[:nloc], self.dD[:nloc], energy)
        call(pt.bwd, ptr(self.net_deriv), ptr(self.dD), ptr(self.drow), ptr(self.xyz),
             ptr(self.em), pt.ptrs, pt.info.ctypes.data, sec.ctypes.data, sec.size, nloc, M,
             ax, s)
        call("dpb_force_virial_a_env_mixed_acc", ptr(force), ptr(virial), ptr(self.net_deriv),
             ptr(c), ptr(t), ptr(self.std), ptr(self.nlist), ptr(self.identity), nloc, nall,
             cfg.nnei, cfg.ntypes, ctypes.c_float(cfg.rcut), ctypes.c_float(cfg.rcut_smth), s)
        return energy, force, virial

    def check(self):
        """Raise if the last call overflowed a capacity (reads device words)."""
        s = torch.cuda.current_stream(self.dev).cuda_stream
        call("dpb_status_check", ptr(self.status), s)
        if self.fit is not None:
            call("dpb_status_check", ptr(self.fit.status), s)
