"""Training step of the uncompressed se_e2_a energy model with an energy,
force and virial loss: hand-written forward, force backward and the second
derivative the loss gradient needs, behind torch.autograd.Function.

The reference trains this model with PyTorch autograd: the force is
-dE/dr from ``torch.autograd.grad(..., create_graph=True)``
(deepmd/pt/model/model/transform_output.py:70-101) and the loss
(deepmd/pt/loss/ener.py:219-340) is differentiated through it. Here:

* forward  (SeATrainer._forward): geometry (dpb_batch_env_mat_a_*), the
  embedding and descriptor (dpb_se_a_train_fwd_*), the fitting net (the
  project's GEMMs: 3xTF32 tensor cores in FP32, dpb_gemm_f64 in FP64; layer
  kernels dpb_fit_*), E per frame; the force backward through the
  fitting (dpb_fit_bwd_*) and the embedding (dpb_se_a_train_bwd_*) to
  g = dE/d(em); force and virial (dpb_batch_force_virial_a*);
* backward (SeATrainer._backward), given dL/dE, dL/dF, dL/dV: the force
  depends on the weights only through g, so
  dL/dtheta = sum_f Ebar_f dE_f/dtheta + d/dtheta <u, g>, u = dL/dg
  recomputed from the coordinates; the second term is a tangent pass along u
  (dpb_se_a_train_tan_*, dpb_fit_tan_*) followed by one reverse pass over
  primal and tangent (dpb_fit_rev_*, dpb_se_a_train_rev_*). The environment
  derivative is recomputed, never stored.

Parameters live in one flat tensor (``SeATrainer.flat``) whose named views
carry the reference state_dict names (deepmd/pt/model/network/mlp.py layers
``matrix``, ``bias``, ``idt``). Only one forward may be outstanding: its
buffers feed the following backward.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _capi
from ._capi import call, ptr
from .batch import FrameTable
from .model import SeAParams

# epilogues of dpb_gemm_tf32x3_f32 (include/dpb200.h)
EPI_STORE, EPI_TANH, EPI_RES_DT = 0, 1, 2

EMB_PREFIX = "atomic_model.descriptor.sea.filter_layers.networks"
FIT_PREFIX = "atomic_model.fitting_net.filter_layers.networks"


def param_specs(params: SeAParams):
    """[(name, array)] of every trainable tensor, in the flat layout order."""
    specs = []
    for t, net in enumerate(params.emb):
        for l, (W, b) in enumerate(net):
            specs.append((f"{EMB_PREFIX}.{t}.layers.{l}.matrix", np.asarray(W)))
            specs.append((f"{EMB_PREFIX}.{t}.layers.{l}.bias", np.asarray(b)))
    for t, f in enumerate(params.fit):
        for l, (W, b, d) in enumerate(f["layers"]):
            specs.append((f"{FIT_PREFIX}.{t}.layers.{l}.matrix", np.asarray(W)))
            specs.append((f"{FIT_PREFIX}.{t}.layers.{l}.bias", np.asarray(b)))
            if d is not None:
                specs.append((f"{FIT_PREFIX}.{t}.layers.{l}.idt", np.asarray(d)))
        Wo, bo = f["out"]
        L = len(f["layers"])
        specs.append((f"{FIT_PREFIX}.{t}.layers.{L}.matrix", np.asarray(Wo).reshape(-1, 1)))
        specs.append((f"{FIT_PREFIX}.{t}.layers.{L}.bias", np.asarray(bo).reshape(1)))
    return specs


def fold_flags(params: SeAParams) -> np.ndarray:
    """[ntypes * ntypes] flags: 1 when the padded slots of section t of a
    type-ti center all have the same avg/std (one env row for all of them)."""
    cfg = params.cfg
    nt, sec = cfg.ntypes, cfg.sec
    avg = np.asarray(params.davg).reshape(nt, cfg.nnei, 4)
    std = np.asarray(params.dstd).reshape(nt, cfg.nnei, 4)
    out = np.zeros(nt * nt, np.uint8)
    for ti in range(nt):
        for t in range(nt):
            a, s = avg[ti, sec[t]:sec[t + 1]], std[ti, sec[t]:sec[t + 1]]
            if a.size and np.all(a == a[:1]) and np.all(s == s[:1]):
                out[ti * nt + t] = 1
    return out


def _res(w_out: int, w_in: int) -> int:
    return 1 if w_out == w_in else (2 if w_out == 2 * w_in else 0)


class EnergyStdLoss:
    """The reference energy/force/virial loss (deepmd/pt/loss/ener.py:48-340)
    in its MSE, per-atom-mask form (the mask is all ones for real atoms, so a
    batch of frames of uneven size reduces as the reference's padded batch
    does): with prefactors p = limit + (start - limit) * lr / starter_lr,
        L = p_e mean_f((E_f - Ehat_f)^2 / n_f)
          + p_f sum (F - Fhat)^2 / (3 N)
          + p_v mean_f(mean_9((V_f - Vhat_f)^2) / n_f),
    n_f the atoms of frame f and N all atoms. A term is on when both its
    start and limit prefactors are nonzero (ener.py:163-165)."""

    def __init__(self, starter_learning_rate: float = 1.0, start_pref_e: float = 0.0,
                 limit_pref_e: float = 0.0, start_pref_f: float = 0.0, limit_pref_f: float = 0.0,
                 start_pref_v: float = 0.0, limit_pref_v: float = 0.0):
        self.starter_learning_rate = starter_learning_rate
        self.start_pref_e, self.limit_pref_e = start_pref_e, limit_pref_e
        self.start_pref_f, self.limit_pref_f = start_pref_f, limit_pref_f
        self.start_pref_v, self.limit_pref_v = start_pref_v, limit_pref_v
        self.has_e = start_pref_e != 0.0 and limit_pref_e != 0.0
        self.has_f = start_pref_f != 0.0 and limit_pref_f != 0.0
        self.has_v = start_pref_v != 0.0 and limit_pref_v != 0.0

    def prefactors(self, learning_rate: float) -> np.ndarray:
        coef = learning_rate / self.starter_learning_rate
        pe = self.limit_pref_e + (self.start_pref_e - self.limit_pref_e) * coef
        pf = self.limit_pref_f + (self.start_pref_f - self.limit_pref_f) * coef
        pv = self.limit_pref_v + (self.start_pref_v - self.limit_pref_v) * coef
        return np.array([pe if self.has_e else 0.0, pf if self.has_f else 0.0,
                         pv if self.has_v else 0.0])

    def forward(self, model_pred: dict, label: dict, natoms, learning_rate: float):
        """(loss, more_loss); model_pred / label hold "energy" [F], "force"
        [N, 3] (frames concatenated) and "virial" [F, 9]; natoms [F] atoms per
        frame. Differentiable w.r.t. the predictions."""
        p = self.prefactors(learning_rate)
        E, Fp, V = model_pred["energy"], model_pred["force"], model_pred["virial"]
        inv = 1.0 / torch.as_tensor(natoms, dtype=E.dtype, device=E.device)
        loss = torch.zeros((), dtype=torch.float64, device=E.device)
        more = {}
        if self.has_e:
            se = torch.square(E.reshape(-1) - label["energy"].reshape(-1))
            loss = loss + p[0] * torch.mean(se * inv)
            more["rmse_e"] = torch.sqrt(torch.mean(se * inv ** 2)).detach()
        if self.has_f:
            d = (label["force"] - Fp).reshape(-1)
            l2 = torch.sum(torch.square(d)) / d.numel()
            loss = loss + p[1] * l2
            more["rmse_f"] = torch.sqrt(l2).detach()
        if self.has_v:
            pv = torch.mean(torch.square(label["virial"].reshape(-1, 9) - V.reshape(-1, 9)), -1)
            loss = loss + p[2] * torch.mean(pv * inv)
            more["rmse_v"] = torch.sqrt(torch.mean(pv * inv ** 2)).detach()
        more["loss"] = loss.detach()
        return loss, more

    __call__ = forward


def loss_grads(E, F, V, Eh, Fh, Vh, inv, pref):
    """(loss, dL/dE, dL/dF, dL/dV) of EnergyStdLoss in closed form, with the
    atom-count reciprocals inv [F] and the prefactors pref [3] as device
    tensors (so a captured step reads their current values)."""
    nf = E.shape[0]
    dE = E - Eh
    dF = F - Fh
    dV = V - Vh
    nfc = dF.numel()
    loss = (pref[0] * torch.mean(dE * dE * inv) + pref[1] * torch.sum(dF * dF) / nfc +
            pref[2] * torch.mean(torch.mean(dV * dV, -1) * inv))
    gE = pref[0] * 2.0 / nf * dE * inv
    gF = pref[1] * 2.0 / nfc * dF
    gV = pref[2] * 2.0 / (9 * nf) * dV * inv[:, None]
    return loss, gE, gF, gV


class _SeAEnergyForceVirial(torch.autograd.Function):
    """(E [F], F [N, 3], V [F, 9]) of the trainer's frames as a function of
    its flat parameters; backward is the hand-written second derivative."""

    @staticmethod
    def forward(ctx, trainer, flat):
        E, F, V = trainer._forward()
        ctx.trainer = trainer
        ctx.version = trainer._version
        return E.clone(), F.clone(), V.clone()

    @staticmethod
    def backward(ctx, gE, gF, gV):
        tr = ctx.trainer
        if tr._version != ctx.version:
            raise RuntimeError("se_a training: another forward ran since this output was made; "
                               "call backward before the next forward")
        z = lambda shape: torch.zeros(shape, dtype=torch.float64, device=tr.dev)  # noqa: E731
        gE = z(tr.ft.nframes) if gE is None else gE
        gF = z((tr.ft.N, 3)) if gF is None else gF
        gV = z((tr.ft.nframes, 9)) if gV is None else gV
        return None, tr._backward(gE, gF, gV).clone()


class SeATrainer:
    """Frames, flat parameters and the device buffers of one training batch.

    frames: [(coord [n, 3], atype [n], box [3, 3])], orthorhombic boxes with
    edges >= rcut; dtype: torch.float32 (training) or torch.float64 (checks).
    """

    def __init__(self, params: SeAParams, frames, dtype=torch.float32, device="cuda:0",
                 loss: EnergyStdLoss | None = None):
        if dtype not in (torch.float32, torch.float64):
            raise _capi.DPBInvalidArgument("dtype must be torch.float32 or torch.float64")
        cfg = params.cfg
        if len(cfg.neuron) != 3:
            raise _capi.DPBInvalidArgument("the training kernels take a 3-layer embedding net")
        self.cfg, self.params, self.dtype = cfg, params, dtype
        self.dev = dev = torch.device(device)
        self.suf = "f32" if dtype == torch.float32 else "f64"
        self.ft = ft = FrameTable(cfg, frames, dev)
        N, F = ft.N, ft.nframes
        nnei, M, ax = cfg.nnei, cfg.neuron[-1], cfg.axis_neuron
        self.M, self.ax = M, ax
        specs = param_specs(params)
        self.names = [n for n, _ in specs]
        self.shapes = [a.shape for _, a in specs]
        # every tensor starts on a 16-byte boundary of the flat vector (the
        # tensor-core GEMM reads biases and writes weight gradients in place);
        # the gaps stay zero and get zero gradients
        self.sizes = [int(a.size) for _, a in specs]
        padded = [(n + 3) // 4 * 4 for n in self.sizes]
        self.offsets = np.concatenate([[0], np.cumsum(padded)]).astype(np.int64)
        flat = np.zeros(int(self.offsets[-1]))
        for k, (_, a) in enumerate(specs):
            flat[int(self.offsets[k]):int(self.offsets[k]) + self.sizes[k]] = np.ravel(a)
        self.flat = torch.tensor(flat, dtype=dtype, device=dev).requires_grad_(True)
        self.grad = torch.zeros(self.flat.numel(), dtype=dtype, device=dev)
        self.adam_m = torch.zeros_like(self.grad)
        self.adam_v = torch.zeros_like(self.grad)
        self.adam_step = 0
        self._hp = torch.zeros(3, dtype=torch.float64, device=dev)
        self._pv = self._views(self.flat.detach())
        self._gv = self._views(self.grad)
        nt = cfg.ntypes
        # embedding pointer tables [type * 3 + layer]
        self.widths = np.array([1, *cfg.neuron], np.int32)
        vp = lambda xs: (ctypes.c_void_p * len(xs))(*[x.data_ptr() for x in xs])  # noqa: E731
        ew = [self._pv[f"{EMB_PREFIX}.{t}.layers.{l}.matrix"] for t in range(nt) for l in range(3)]
        eb = [self._pv[f"{EMB_PREFIX}.{t}.layers.{l}.bias"] for t in range(nt) for l in range(3)]
        gw = [self._gv[f"{EMB_PREFIX}.{t}.layers.{l}.matrix"] for t in range(nt) for l in range(3)]
        gb = [self._gv[f"{EMB_PREFIX}.{t}.layers.{l}.bias"] for t in range(nt) for l in range(3)]
        self.Wp, self.bp, self.gWp, self.gbp = vp(ew), vp(eb), vp(gw), vp(gb)
        self.sec = cfg.sec
        self.fold = fold_flags(params)
        f64 = torch.float64
        z = lambda shape, dt=dtype: torch.zeros(shape, dtype=dt, device=dev)  # noqa: E731
        self.coord = z((N, 3), f64)
        self.em = z((N, nnei * 4))
        self.nlist = z((N, nnei), torch.int32)
        self.status = z(1, torch.int32)
        self.avg = torch.tensor(params.davg, dtype=dtype, device=dev).contiguous()
        self.std = torch.tensor(params.dstd, dtype=dtype, device=dev).contiguous()
        self.xyz = z((N, 4, M))
        self.D = z((N, M * ax))
        self.Dbar = z((N, M * ax))
        self.net_deriv = z((N, nnei * 4))
        self.xyz_t = z((N, 4, M))
        self.xbar = z((2, N, 4, M))  # adjoints of xyz and xyz' (kernel scratch)
        self.Dt = z((N, M * ax))
        self.DbarJ = z((N, M * ax))
        self.Ddbar = z((N, M * ax))
        self.e_rows = z(N)
        self.lam = z(N)
        self.e_const = z(F, f64)
        self.energy = z(F, f64)
        self.force = z((N, 3), f64)
        self.virial = z((F, 9), f64)
        # fitting: per center type, rows [o, o + n) of the type-grouped order
        self.fit_rows = []
        o = 0
        for t in range(nt):
            n = int(ft.tcount[t])
            self.fit_rows.append((o, n))
            o += n
        self.fit_layers = []  # per type: [(W, b, d, gW, gb, gd, w_in, w_out)], out
        widths_in = M * ax
        self.fbuf = []
        for t in range(nt):
            f = params.fit[t]
            L = len(f["layers"])
            layers = []
            w_in = widths_in
            for l in range(L):
                key = f"{FIT_PREFIX}.{t}.layers.{l}"
                W = self._pv[key + ".matrix"]
                has_d = (key + ".idt") in self._pv
                layers.append(dict(W=W, b=self._pv[key + ".bias"],
                                   d=self._pv[key + ".idt"] if has_d else None,
                                   gW=self._gv[key + ".matrix"], gb=self._gv[key + ".bias"],
                                   gd=self._gv[key + ".idt"] if has_d else None,
                                   w_in=w_in, w_out=W.shape[1]))
                w_in = W.shape[1]
            key = f"{FIT_PREFIX}.{t}.layers.{L}"
            out = dict(W=self._pv[key + ".matrix"], b=self._pv[key + ".bias"],
                       gW=self._gv[key + ".matrix"], gb=self._gv[key + ".bias"], w=w_in,
                       ebias=float(params.bias_atom_e[t]))
            self.fit_layers.append((layers, out))
            n = self.fit_rows[t][1]
            bufs = [{k: z((n, ly["w_out"])) for k in ("Y", "H", "G", "Zb", "Zd", "Hd", "A",
                                                       "Ad", "Zbd")} for ly in layers]
            for ly, bf in zip(layers, bufs):
                self._tc_setup(ly, bf, n, z)
            self.fbuf.append(bufs)
        self._e_dummy = z(1)
        self._rows_cache = {}
        self._streams = [torch.cuda.Stream(device=dev) for _ in range(nt)]
        self.loss = loss
        self._natoms_inv = torch.tensor(1.0 / np.maximum(ft.counts, 1), dtype=f64, device=dev)
        self._pref = torch.zeros(3, dtype=f64, device=dev)
        self.labels = None
        self._version = 0
        self.graph = None
        self.set_coords([fr[0] for fr in frames])

    def _tc_setup(self, ly, bf, n, z):
        """Tensor-core buffers of one FP32 fitting layer: W^T for x W (and
        the tangent), and the transposed operands of the weight gradient."""
        w_in, w_out = ly["w_in"], ly["w_out"]
        res = _res(w_out, w_in)
        ly["WT"] = None
        ly["d_or_one"] = ly["d"]
        if self._tc_ok(w_out, w_in) and (res == 1 or (res == 0 and ly["d"] is None)):
            ly["WT"] = z((w_out, w_in))
            if res == 1 and ly["d"] is None:
                ly["d_or_one"] = torch.ones(w_out, dtype=self.dtype, device=self.dev)
            if res == 0:
                bf["H"] = bf["Y"]  # tanh(x W + b) is the layer's output
        bf["At"] = bf["Bt"] = None
        kp = (2 * n + 3) // 4 * 4
        if self._tc_ok(w_out, kp) and n > 0:
            bf["At"] = z((w_in, kp))
            bf["Bt"] = z((w_out, kp))

    # ---------------------------------------------------------- parameters
    def _views(self, base: torch.Tensor) -> dict:
        return {n: base[int(self.offsets[k]):int(self.offsets[k]) + self.sizes[k]]
                .view(self.shapes[k]) for k, n in enumerate(self.names)}

    def named_parameters(self) -> dict:
        """{reference state_dict name: view of the flat parameters}."""
        return self._views(self.flat.detach())

    def named_grads(self, grad: torch.Tensor | None = None) -> dict:
        return self._views(self.grad if grad is None else grad)

    def set_coords(self, coords):
        c = np.concatenate([np.asarray(x, np.float64).reshape(-1, 3) for x in coords]) \
            if isinstance(coords, (list, tuple)) else np.asarray(coords, np.float64)
        self.coord.copy_(torch.as_tensor(c.reshape(self.ft.N, 3)))

    def set_labels(self, energy, force, virial):
        """Labels of the loss: energy [F], force [N, 3], virial [F, 9]."""
        f64 = torch.float64
        t = lambda a, shape: torch.as_tensor(np.asarray(a, np.float64).reshape(shape),  # noqa: E731
                                             dtype=f64).to(self.dev)
        lab = (t(energy, (self.ft.nframes,)), t(force, (self.ft.N, 3)),
               t(virial, (self.ft.nframes, 9)))
        if self.labels is None:
            self.labels = lab
        else:
            for dst, src in zip(self.labels, lab):
                dst.copy_(src)

    # ------------------------------------------------------------ forward
    # ------------------------------------------------------------- GEMMs
    # The fitting layers' products on this package's GEMMs: in FP32 the
    # 3xTF32 tensor-core GEMM (dpb_gemm_tf32x3_f32, weights split into TF32
    # hi / lo in the kernel) wherever its output width is a multiple of 80,
    # else the FP32 SIMT GEMM; in FP64 dpb_gemm_f64.
    def _mm(self, C, A, B, bias, M, N, K, ta, tb, acc, s):
        """C = op(A) op(B) (+ bias) (+ C), row-major operands."""
        call(f"dpb_gemm_{self.suf}", ptr(C), ptr(A), ptr(B), ptr(bias), M, N, K,
             int(A.shape[-1]), int(B.shape[-1]), int(C.shape[-1]), ta, tb, acc, s)

    def _tc_ok(self, N: int, K: int) -> bool:
        return self.suf == "f32" and N % 80 == 0 and K % 4 == 0

    def _tc(self, A, M, K, B, N, mode, out0, s, out1=None, aux0=None, bias=None, idt=None):
        """out0 (, out1) = epilogue(A [M, K] B^T) with B [N, K] FP32 (split in
        the kernel), one row group."""
        vp = lambda t: None if t is None else (ctypes.c_void_p * 1)(t.data_ptr())  # noqa: E731
        call("dpb_gemm_tf32x3_f32", ptr(A), M, K, vp(B), None, N, self._rows1(M), 1, mode,
             ptr(out0), ptr(out1), ptr(aux0), None, vp(bias), vp(idt), None, ptr(self._e_dummy),
             ptr(self.status), s)

    def _rows1(self, M):
        a = self._rows_cache.get(M)
        if a is None:
            a = self._rows_cache[M] = np.array([M], np.int32)
        return a.ctypes.data

    def _adj_in(self, out, Zb, W, G, w_out, w_in, s):
        """out = Zb W^T + (adjoint of the layer's residual, from G)."""
        n = out.shape[0]
        if self._tc_ok(w_in, w_out):
            self._tc(Zb, n, w_out, W, w_in, EPI_STORE, out, s)
        else:
            self._mm(out, Zb, W, None, n, w_in, w_out, 0, 1, 0, s)
        if _res(w_out, w_in):
            call(f"dpb_fit_res_adj_{self.suf}", ptr(out), ptr(G), n, w_out, w_in, s)

    def _weights_t(self, s):
        """W^T of every fitting layer whose forward runs on the tensor cores
        (the weights change every step)."""
        for layers, _ in self.fit_layers:
            for ly in layers:
                if ly.get("WT") is not None:
                    call("dpb_transpose_f32", ptr(ly["WT"]), ptr(ly["W"]), ly["w_in"],
                         ly["w_out"], ly["w_out"], ly["w_in"], ly["w_in"], s)

    def _forward(self):
        cfg, ft, suf = self.cfg, self.ft, self.suf
        s = torch.cuda.current_stream(self.dev).cuda_stream
        N, F = ft.N, ft.nframes
        sec = self.sec
        rc, rs = ctypes.c_float(cfg.rcut), ctypes.c_float(cfg.rcut_smth)
        self._version += 1
        self._weights_t(s)
        call(f"dpb_batch_env_mat_a_{suf}", ptr(self.em), ptr(self.nlist), ptr(ft.cw),
             ptr(ft.cell_of), ptr(ft.cell_start), ptr(ft.cell_atoms), ptr(self.coord),
             ptr(ft.type), ptr(self.avg), ptr(self.std), ptr(ft.atom_off), ptr(ft.cell_off),
             ptr(ft.box), ptr(ft.ncell), ptr(ft.row_frame), F, N, rc, rs, sec.ctypes.data,
             sec.size, ptr(self.status), s)
        call(f"dpb_se_a_train_fwd_{suf}", ptr(self.xyz), ptr(self.D), ptr(self.em),
             ptr(self.nlist), ptr(ft.type), ptr(ft.drow), self.Wp, self.bp,
             self.widths.ctypes.data, sec.ctypes.data, sec.size, N, self.ax,
             self.fold.ctypes.data, s)
        self._each_type(self._fit_forward_type)
        e_fn = "dpb_batch_energy" if suf == "f32" else "dpb_batch_energy_f64"
        call(e_fn, ptr(self.energy), ptr(self.e_rows), ptr(ft.drow), ptr(self.e_const),
             ptr(ft.atom_off), F, s)
        call(f"dpb_se_a_train_bwd_{suf}", ptr(self.net_deriv), ptr(self.xbar), ptr(self.em),
             ptr(self.xyz),
             ptr(self.Dbar), ptr(self.nlist), ptr(ft.type), ptr(ft.drow), self.Wp, self.bp,
             self.widths.ctypes.data, sec.ctypes.data, sec.size, N, self.ax, s)
        f_fn = "dpb_batch_force_virial_a" if suf == "f32" else "dpb_batch_force_virial_a_f64"
        call(f_fn, ptr(self.force), ptr(self.virial), ptr(self.net_deriv), ptr(ft.cw),
             ptr(ft.type), ptr(self.std), ptr(self.nlist), ptr(ft.atom_off), ptr(ft.cell_off),
             ptr(ft.box), ptr(ft.ncell), ptr(ft.row_frame), F, N, cfg.nnei, cfg.ntypes, rc, rs, s)
        return self.energy, self.force, self.virial

    def _each_type(self, fn):
        """fn(t, stream handle) for every center type with rows; the types'
        fitting chains are independent and run on side streams forked from
        (and joined back into) the current stream."""
        cur = torch.cuda.current_stream(self.dev)
        active = [t for t in range(self.cfg.ntypes) if self.fit_rows[t][1] > 0]
        if len(active) <= 1:
            for t in active:
                fn(t, cur.cuda_stream)
            return
        for t in active:
            st = self._streams[t]
            st.wait_stream(cur)
            with torch.cuda.stream(st):
                fn(t, st.cuda_stream)
        for t in active:
            cur.wait_stream(self._streams[t])

    def _fit_forward_type(self, t, s):
        """Fitting net of center type t: atomic energies and dE/dD."""
        suf = self.suf
        (layers, out), bufs = self.fit_layers[t], self.fbuf[t]
        o, n = self.fit_rows[t]
        H = self.D[o:o + n]
        for ly, bf in zip(layers, bufs):
            if ly.get("WT") is not None:  # bias, tanh and residual in the epilogue
                if _res(ly["w_out"], ly["w_in"]):
                    self._tc(H, n, ly["w_in"], ly["WT"], ly["w_out"], EPI_RES_DT, bf["Y"], s,
                             out1=bf["H"], aux0=H, bias=ly["b"], idt=ly["d_or_one"])
                else:  # H aliases Y
                    self._tc(H, n, ly["w_in"], ly["WT"], ly["w_out"], EPI_TANH, bf["Y"], s,
                             bias=ly["b"])
            else:
                self._mm(bf["Y"], H, ly["W"], ly["b"], n, ly["w_out"], ly["w_in"], 0, 0, 0, s)
                call(f"dpb_fit_act_{suf}", ptr(bf["Y"]), ptr(bf["H"]), ptr(H), ptr(ly["d"]), n,
                     ly["w_out"], ly["w_in"], s)
            H = bf["H"]
        call(f"dpb_fit_out_{suf}", ptr(self.e_rows[o:o + n]), ptr(H), ptr(out["W"]),
             ptr(out["b"]), ctypes.c_double(out["ebias"]), n, out["w"], s)
        # dE/dD through the fitting
        G = bufs[-1]["G"]
        call(f"dpb_fit_out_adj_{suf}", ptr(G), None, None, None, ptr(H), None, ptr(out["W"]),
             None, n, out["w"], s)
        for l in range(len(layers) - 1, -1, -1):
            ly, bf = layers[l], bufs[l]
            call(f"dpb_fit_bwd_{suf}", ptr(bf["Zb"]), ptr(bf["G"]), ptr(bf["Y"]),
                 ptr(ly["d"]), n, ly["w_out"], s)
            dst = self.Dbar[o:o + n] if l == 0 else bufs[l - 1]["G"]
            self._adj_in(dst, bf["Zb"], ly["W"], bf["G"], ly["w_out"], ly["w_in"], s)

    def _fit_backward_type(self, t, s):
        """Tangent and reverse-over-tangent of the fitting net of center type
        t: its weight gradients and the adjoints of D and D'."""
        suf = self.suf
        (layers, out), bufs = self.fit_layers[t], self.fbuf[t]
        o, n = self.fit_rows[t]
        Hd = self.Dt[o:o + n]
        for ly, bf in zip(layers, bufs):
            if ly.get("WT") is not None:
                self._tc(Hd, n, ly["w_in"], ly["WT"], ly["w_out"], EPI_STORE, bf["Zd"], s)
            else:
                self._mm(bf["Zd"], Hd, ly["W"], None, n, ly["w_out"], ly["w_in"], 0, 0, 0, s)
            call(f"dpb_fit_tan_{suf}", ptr(bf["Hd"]), ptr(bf["Zd"]), ptr(Hd), ptr(bf["Y"]),
                 ptr(ly["d"]), n, ly["w_out"], ly["w_in"], s)
            Hd = bf["Hd"]
        call(f"dpb_fit_out_adj_{suf}", ptr(bufs[-1]["A"]), ptr(bufs[-1]["Ad"]),
             ptr(out["gW"]), ptr(out["gb"]), ptr(bufs[-1]["H"]), ptr(Hd), ptr(out["W"]),
             ptr(self.lam[o:o + n]), n, out["w"], s)
        for l in range(len(layers) - 1, -1, -1):
            ly, bf = layers[l], bufs[l]
            call(f"dpb_fit_rev_{suf}", ptr(bf["Zb"]), ptr(bf["Zbd"]), ptr(ly["gb"]),
                 ptr(ly["gd"]), ptr(bf["A"]), ptr(bf["Ad"]), ptr(bf["Y"]), ptr(bf["Zd"]),
                 ptr(ly["d"]), n, ly["w_out"], s)
            Hin = self.D[o:o + n] if l == 0 else bufs[l - 1]["H"]
            Hdin = self.Dt[o:o + n] if l == 0 else bufs[l - 1]["Hd"]
            self._weight_grad(ly, bf, Hin, Hdin, n, s)
            dA = self.DbarJ[o:o + n] if l == 0 else bufs[l - 1]["A"]
            dAd = self.Ddbar[o:o + n] if l == 0 else bufs[l - 1]["Ad"]
            self._adj_in(dA, bf["Zb"], ly["W"], bf["A"], ly["w_out"], ly["w_in"], s)
            self._adj_in(dAd, bf["Zbd"], ly["W"], bf["Ad"], ly["w_out"], ly["w_in"], s)

    def _weight_grad(self, ly, bf, Hin, Hdin, n, s):
        """gW = Hin^T Zb + Hdin^T Zbd (the gradient buffer was zeroed): on the
        tensor cores as one product along K = 2 n of the transposed operands
        [Hin | Hdin]^T and [Zb | Zbd]^T, else two SIMT products."""
        w_in, w_out = ly["w_in"], ly["w_out"]
        At, Bt = bf.get("At"), bf.get("Bt")
        if At is not None:
            kp = At.shape[1]
            call("dpb_transpose_f32", ptr(At), ptr(Hin), n, w_in, w_in, kp, n, s)
            call("dpb_transpose_f32", ptr(At[:, n:]), ptr(Hdin), n, w_in, w_in, kp, kp - n, s)
            call("dpb_transpose_f32", ptr(Bt), ptr(bf["Zb"]), n, w_out, w_out, kp, n, s)
            call("dpb_transpose_f32", ptr(Bt[:, n:]), ptr(bf["Zbd"]), n, w_out, w_out, kp,
                 kp - n, s)
            self._tc(At, w_in, kp, Bt, w_out, EPI_STORE, ly["gW"], s)
        else:
            self._mm(ly["gW"], Hin, bf["Zb"], None, w_in, w_out, n, 1, 0, 1, s)
            self._mm(ly["gW"], Hdin, bf["Zbd"], None, w_in, w_out, n, 1, 0, 1, s)

    # ----------------------------------------------------------- backward
    def _backward(self, gE, gF, gV):
        """Flat gradient of L given dL/dE [F], dL/dF [N, 3], dL/dV [F, 9]."""
        cfg, ft, suf = self.cfg, self.ft, self.suf
        s = torch.cuda.current_stream(self.dev).cuda_stream
        N, F = ft.N, ft.nframes
        sec = self.sec
        rc, rs = ctypes.c_float(cfg.rcut), ctypes.c_float(cfg.rcut_smth)
        f64 = torch.float64
        gE = gE.detach().to(f64).reshape(F).contiguous()
        gF = gF.detach().to(f64).reshape(N, 3).contiguous()
        gV = gV.detach().to(f64).reshape(F, 9).contiguous()
        self._gbufs = (gE, gF, gV)  # alive until the kernels have read them
        self.grad.zero_()
        call(f"dpb_train_lam_{suf}", ptr(self.lam), ptr(gE), ptr(ft.drow), ptr(ft.row_frame), N,
             s)
        call(f"dpb_se_a_train_tan_{suf}", ptr(self.xyz_t), ptr(self.Dt), ptr(self.xyz),
             ptr(self.avg), ptr(self.std), ptr(gF), ptr(gV), ptr(ft.cw), ptr(self.nlist),
             ptr(ft.type), ptr(ft.drow), ptr(ft.atom_off), ptr(ft.box), ptr(ft.row_frame), F,
             self.Wp, self.bp, self.widths.ctypes.data, sec.ctypes.data, sec.size, N, self.ax,
             rc, rs, s)
        self._each_type(self._fit_backward_type)
        call(f"dpb_se_a_train_rev_{suf}", self.gWp, self.gbp, ptr(self.xbar), ptr(self.xyz),
             ptr(self.xyz_t),
             ptr(self.DbarJ), ptr(self.Ddbar), ptr(self.avg), ptr(self.std), ptr(gF), ptr(gV),
             ptr(ft.cw), ptr(self.nlist), ptr(ft.type), ptr(ft.drow), ptr(ft.atom_off),
             ptr(ft.box), ptr(ft.row_frame), F, self.Wp, self.bp, self.widths.ctypes.data,
             sec.ctypes.data, sec.size, N, self.ax, self.fold.ctypes.data, rc, rs, s)
        return self.grad

    # ------------------------------------------------------------- public
    def energy_force_virial(self):
        """(E [F], F [N, 3], V [F, 9]) in FP64, differentiable w.r.t. ``flat``."""
        return _SeAEnergyForceVirial.apply(self, self.flat)

    def check(self):
        call("dpb_status_check", ptr(self.status), torch.cuda.current_stream(self.dev).cuda_stream)

    def compute(self, coords=None):
        """(E, F, V) as host arrays (no gradient)."""
        if coords is not None:
            self.set_coords(coords)
        with torch.no_grad():
            E, F, V = self._forward()
        torch.cuda.synchronize(self.dev)
        return E.cpu().numpy(), F.cpu().numpy(), V.cpu().numpy()

    # ---------------------------------------------------- fused train step
    def _set_step_scalars(self, lr, beta1, beta2):
        self.adam_step += 1
        t = self.adam_step
        hp = torch.tensor([lr, 1.0 - beta1 ** t, math.sqrt(1.0 - beta2 ** t)],
                          dtype=torch.float64)
        pref = torch.tensor(self.loss.prefactors(lr), dtype=torch.float64)
        self._hp.copy_(hp, non_blocking=False)
        self._pref.copy_(pref, non_blocking=False)

    def _step_body(self, beta1, beta2, eps):
        E, F, V = self._forward()
        Eh, Fh, Vh = self.labels
        loss, gE, gF, gV = loss_grads(E, F, V, Eh, Fh, Vh, self._natoms_inv, self._pref)
        self._loss = loss.reshape(1)
        self._backward(gE, gF, gV)
        call(f"dpb_adam_{self.suf}", ptr(self.flat.detach()), ptr(self.grad), ptr(self.adam_m),
             ptr(self.adam_v), self.grad.numel(), ptr(self._hp), ctypes.c_double(beta1),
             ctypes.c_double(beta2), ctypes.c_double(eps),
             torch.cuda.current_stream(self.dev).cuda_stream)
        return self._loss

    def train_step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999,
                   eps: float = 1e-8) -> torch.Tensor:
        """One step: forward, EnergyStdLoss, its gradient, Adam. Returns the
        loss (device tensor [1]); labels from set_labels, loss from the
        constructor."""
        if self.loss is None or self.labels is None:
            raise _capi.DPBInvalidArgument("train_step needs a loss and labels")
        self._set_step_scalars(lr, beta1, beta2)
        if self.graph is not None:
            if self._graph_adam != (beta1, beta2, eps):
                raise _capi.DPBInvalidArgument("the captured step used other Adam betas/eps")
            self.graph.replay()
            return self._loss
        with torch.no_grad():
            return self._step_body(beta1, beta2, eps)

    def capture(self, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        """Capture train_step into a CUDA graph (the learning rate, prefactors
        and Adam bias corrections are read from device memory each replay).
        Warm-up runs are full steps: they move the parameters."""
        if self.loss is None or self.labels is None:
            raise _capi.DPBInvalidArgument("capture needs a loss and labels")
        # warm-up step (library handles, workspaces) with lr 0 and the Adam
        # moments restored afterwards, so capturing leaves the state as it was
        saved = (self.adam_m.clone(), self.adam_v.clone(), self._hp.clone())
        self._hp.copy_(torch.tensor([0.0, 1.0, 1.0], dtype=torch.float64))
        self._pref.copy_(torch.tensor(self.loss.prefactors(self.loss.starter_learning_rate),
                                      dtype=torch.float64))
        st = torch.cuda.Stream(device=self.dev)
        st.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(st), torch.no_grad():
            self._step_body(beta1, beta2, eps)
        torch.cuda.current_stream(self.dev).wait_stream(st)
        torch.cuda.synchronize(self.dev)
        self.adam_m.copy_(saved[0])
        self.adam_v.copy_(saved[1])
        self._hp.copy_(saved[2])
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph), torch.no_grad():
            self._step_body(beta1, beta2, eps)
        torch.cuda.synchronize(self.dev)
        self._graph_adam = (beta1, beta2, eps)
        return self

    def tune(self, reps: int = 10, use_cache: bool = True) -> dict:
        """Autotune the training kernels' tile shapes (rows per group, warps
        per CTA, atoms per CTA of the batched geometry) on this batch with
        the learning rate held at zero; parameters and Adam moments are
        restored afterwards and the step is left captured."""
        from . import autotune

        if self.loss is None or self.labels is None:
            raise _capi.DPBInvalidArgument("tune needs a loss and labels")
        saved = (self.flat.detach().clone(), self.adam_m.clone(), self.adam_v.clone(),
                 self.adam_step)
        zero = torch.tensor([0.0, 1.0, 1.0], dtype=torch.float64)

        def step():
            self._hp.copy_(zero)
            self.graph.replay()

        cfg = self.cfg
        sig = (f"train:{self.ft.nframes}f:{self.ft.N}a:{self.suf}:"
               f"sel{'-'.join(map(str, cfg.sel))}:emb{'-'.join(map(str, cfg.neuron))}")
        res = autotune.tune(step, lambda: self.capture(),
                            ["train_rows_per_group", "train_warps_per_cta",
                             "batch_atoms_per_cta", "pdl"],
                            signature=sig, reps=reps, device=self.dev, use_cache=use_cache)
        self.flat.detach().copy_(saved[0])
        self.adam_m.copy_(saved[1])
        self.adam_v.copy_(saved[2])
        self.adam_step = saved[3]
        return res
