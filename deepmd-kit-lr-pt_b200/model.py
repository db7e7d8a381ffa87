"""se_e2_a energy model: parameters and the GPU energy/force/virial step.

Model (deepmd/pt/model/descriptor/se_a.py, deepmd/pt/model/task/ener.py):
  embedding  per neighbor type t (type_one_side): 1 -> n1 -> n2 -> M tanh,
             residual when a layer doubles its width (no timestep);
  descriptor xyz = sum_t R_t^T G_t(R_t[:, 0]) / nnei, D = xyz^T xyz[:, :axis];
  fitting    per center type: D -> f1 -> f2 -> f3 tanh with timestep residual
             (y = x + idt * tanh(xW + b) when widths match), then a linear
             output plus the per-type energy bias;
  E = sum_i e_i, F = -dE/dr (ghost contributions folded onto owners),
  virial = sum over pairs of f_ij (x) r_ij (prod_virial.cc:55-63).

Two evaluation paths share the geometry kernels:
  compressed (FP32): FP64 coordinate differences, FP32 env matrix, the FP32
     quintic table fused with the contraction and D, FP32 fitting, FP64
     energy/force/virial accumulation;
  plain (FP64): FP64 env matrix, the embedding MLP and fitting in FP64.
Both are stream-ordered without host synchronisation inside a step, so a step
is captured once into a CUDA graph and replayed.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi, ops, table as table_mod
from ._capi import call, ptr
from .workload import SeAConfig, SeAParams, init_params  # noqa: F401  (model definition)


# ------------------------------------------------------------ statistics --

def env_stats(params: SeAParams, coord: np.ndarray, atype: np.ndarray, box: np.ndarray,
              device="cuda:0", protection: float = 1e-2):
    """davg/dstd from the frame's own raw environment matrix
    (deepmd/dpmodel/utils/env_mat_stat.py:296-425, utils/env_mat_stat.py:24-101):
    per center type, the radial column's mean and std and the angular columns'
    std over all slots including padding; davg = [r_avg, 0, 0, 0],
    dstd = [r_std, a_std, a_std, a_std], tiled over the slots.
    Also returns the minimum neighbor distance of the frame."""
    cfg = params.cfg
    dev = torch.device(device)
    ce, te, _ = ops.copy_coord(torch.tensor(coord, device=dev), torch.tensor(atype, device=dev),
                               cfg.rcut, box)
    nloc = atype.size
    zeros = torch.zeros((cfg.ntypes, cfg.nnei * 4), dtype=torch.float64, device=dev)
    ones = torch.ones_like(zeros)
    em, _, rij, nlist = ops.env_mat_a_cells(ce, te, nloc, zeros, ones, cfg.rcut, cfg.rcut_smth,
                                            cfg.sec)
    em = em.view(nloc, cfg.nnei, 4).cpu().numpy()
    davg = np.zeros((cfg.ntypes, cfg.nnei, 4))
    dstd = np.ones((cfg.ntypes, cfg.nnei, 4))
    for t in range(cfg.ntypes):
        sel = em[atype == t]
        if sel.size == 0:
            dstd[t] *= 0.1
            continue
        r = sel[:, :, 0].reshape(-1)
        a = sel[:, :, 1:].reshape(-1)

        def std(v):
            s = np.sqrt(max(np.mean(v * v) - np.mean(v) ** 2, 0.0))
            return protection if abs(s) < protection else s

        davg[t, :, 0] = np.mean(r)
        dstd[t, :, 0] = std(r)
        dstd[t, :, 1:] = std(a)
    rr = rij.view(nloc, cfg.nnei, 3).cpu().numpy()
    valid = nlist.cpu().numpy() >= 0
    dist = np.linalg.norm(rr, axis=-1)[valid]
    min_dist = float(dist.min()) if dist.size else cfg.rcut
    return davg.reshape(cfg.ntypes, -1), dstd.reshape(cfg.ntypes, -1), min_dist


def env_stats_frames(params: SeAParams, frames, device="cuda:0", protection: float = 1e-2):
    """env_stats over several frames: the per-center-type moments of the raw
    environment matrix summed over all frames (a type absent from every frame
    keeps davg 0, dstd 1)."""
    cfg = params.cfg
    dev = torch.device(device)
    nt = cfg.ntypes
    s_r, s_r2, n_r = np.zeros(nt), np.zeros(nt), np.zeros(nt)
    s_a, s_a2, n_a = np.zeros(nt), np.zeros(nt), np.zeros(nt)
    min_dist = cfg.rcut
    zeros = torch.zeros((nt, cfg.nnei * 4), dtype=torch.float64, device=dev)
    ones = torch.ones_like(zeros)
    for coord, atype, box in frames:
        ce, te, _ = ops.copy_coord(torch.tensor(coord, device=dev),
                                   torch.tensor(atype, device=dev), cfg.rcut, box)
        nloc = atype.size
        em, _, rij, nlist = ops.env_mat_a_cells(ce, te, nloc, zeros, ones, cfg.rcut,
                                                cfg.rcut_smth, cfg.sec)
        em = em.view(nloc, cfg.nnei, 4).cpu().numpy()
        for t in range(nt):
            sel = em[atype == t]
            if sel.size == 0:
                continue
            r, a = sel[:, :, 0], sel[:, :, 1:]
            s_r[t] += r.sum()
            s_r2[t] += (r * r).sum()
            n_r[t] += r.size
            s_a[t] += a.sum()
            s_a2[t] += (a * a).sum()
            n_a[t] += a.size
        rr = rij.view(nloc, cfg.nnei, 3).cpu().numpy()
        valid = nlist.cpu().numpy() >= 0
        d = np.linalg.norm(rr, axis=-1)[valid]
        if d.size:
            min_dist = min(min_dist, float(d.min()))

    def std(s1, s2, n):
        v = np.sqrt(max(s2 / n - (s1 / n) ** 2, 0.0))
        return protection if abs(v) < protection else v

    davg = np.zeros((nt, cfg.nnei, 4))
    dstd = np.ones((nt, cfg.nnei, 4))
    for t in range(nt):
        if n_r[t] == 0:
            continue
        davg[t, :, 0] = s_r[t] / n_r[t]
        dstd[t, :, 0] = std(s_r[t], s_r2[t], n_r[t])
        dstd[t, :, 1:] = std(s_a[t], s_a2[t], n_a[t])
    return davg.reshape(nt, -1), dstd.reshape(nt, -1), min_dist


def prepare_frames(params: SeAParams, frames, device="cuda:0"):
    """prepare() for a set of frames (statistics over all of them)."""
    davg, dstd, min_dist = env_stats_frames(params, frames, device)
    params.davg, params.dstd = davg, dstd
    dev_tables = table_mod.build_tables_device(params.emb, davg, dstd, params.cfg.sel, min_dist,
                                               params.cfg.rcut_smth, params.cfg.rcut,
                                               device=device)
    params.tables = [(t.cpu().numpy(), info) for t, info in dev_tables]
    return params


def prepare(params: SeAParams, coord, atype, box, device="cuda:0", with_tables=True):
    """Statistics from the frame and (optionally) the FP64 compression tables
    (built on the device, dpb_se_a_build_table_f64)."""
    davg, dstd, min_dist = env_stats(params, coord, atype, box, device)
    params.davg, params.dstd = davg, dstd
    if with_tables:
        # FP64 tables built on the device, kept on the host as the model's
        # compressed data (the evaluators upload them in their own layout)
        dev_tables = table_mod.build_tables_device(params.emb, davg, dstd, params.cfg.sel,
                                                   min_dist, params.cfg.rcut_smth,
                                                   params.cfg.rcut, device=device)
        params.tables = [(t.cpu().numpy(), info) for t, info in dev_tables]
    return params


# --------------------------------------------------------------- fitting --

class _Fitting:
    """Per-type fitting networks on the device in one precision."""

    def __init__(self, params: SeAParams, dtype, device):
        self.layers = []
        self.out = []
        for f in params.fit:
            ls = []
            for W, b, d in f["layers"]:
                ls.append((torch.tensor(W, dtype=dtype, device=device),
                           torch.tensor(b, dtype=dtype, device=device),
                           None if d is None else torch.tensor(d, dtype=dtype, device=device)))
            self.layers.append(ls)
            Wo, bo = f["out"]
            self.out.append((torch.tensor(Wo, dtype=dtype, device=device),
                             torch.tensor(bo, dtype=dtype, device=device)))
        self.bias = torch.tensor(params.bias_atom_e, dtype=dtype, device=device)

    def forward_backward(self, t: int, x: torch.Tensor):
        """Atomic energies of type-t rows and their gradient w.r.t. the rows."""
        acts = []
        h = x
        for W, b, d in self.layers[t]:
            y = torch.tanh(torch.addmm(b, h, W))
            acts.append((h, y, W, d))
            h = h + d * y if d is not None else y
        Wo, bo = self.out[t]
        e = torch.addmm(bo, h, Wo).view(-1) + self.bias[t]
        g = Wo.view(1, -1).expand(h.shape[0], -1)
        for hin, y, W, d in reversed(acts):
            gz = g * (1.0 - y * y)
            if d is not None:
                gz = gz * d
                g = g + gz @ W.t()
            else:
                g = gz @ W.t()
        return e, g

    def forward(self, t: int, x: torch.Tensor):
        h = x
        for W, b, d in self.layers[t]:
            y = torch.tanh(torch.addmm(b, h, W))
            h = h + d * y if d is not None else y
        Wo, bo = self.out[t]
        return torch.addmm(bo, h, Wo).view(-1) + self.bias[t]


# Table representation of the fused descriptor kernels unless a caller picks
# one: the cubic re-interpolation (measured 0.852 -> 0.753 ms on the
# 12,288-atom water step; within the path's tolerances of the FP64 oracle)
DEFAULT_TABLE_DEGREE = 3


class PipelineTables:
    """The compression tables in the layout of the fused descriptor kernels:
    the reference's quintic rows, coefficient-major per row
    (dpb_se_a_pack_table_f32; degree 5), or their cubic re-interpolation on
    the fine stride (table.cubic_table; degree 3), in FP32 on the device."""

    def __init__(self, params: SeAParams, device, degree: int = DEFAULT_TABLE_DEGREE):
        if degree not in (3, 5):
            raise _capi.DPBInvalidArgument("table_degree must be 5 (the reference's quintic "
                                           "table) or 3 (its cubic re-interpolation)")
        dev = torch.device(device)
        M = params.cfg.neuron[-1]
        self.degree = degree
        self.tabs, infos = [], []
        s = torch.cuda.current_stream(dev).cuda_stream
        for t, info in params.tables:
            if degree == 3:
                # knots every table_cubic_stride fine strides (knob; 1: the
                # reference's fine stride)
                m = int(_capi.lib().dpb_tune_get(b"table_cubic_stride"))
                cub = table_mod.cubic_table(t, info, m)
                if cub is None and m > 1:
                    cub = table_mod.cubic_table(t, info)
                if cub is None:
                    raise _capi.DPBInvalidArgument(
                        "table_degree 3 needs stride1 to be a whole multiple of stride0")
                coef, ic = cub
                self.tabs.append(torch.tensor(coef.astype(np.float32).reshape(-1), device=dev))
                infos.append(ic)
            else:
                ref_layout = torch.tensor(t, dtype=torch.float32, device=dev)
                packed = torch.empty_like(ref_layout)
                call("dpb_se_a_pack_table_f32", ptr(packed), ptr(ref_layout), t.shape[0], M, s)
                self.tabs.append(packed)
                if packed.numel() < ops.table_rows_needed(info.astype(np.float32)) * 6 * M:
                    raise _capi.DPBInvalidArgument("table smaller than its table_info addresses")
                infos.append(info)
        torch.cuda.synchronize(dev)
        self.ptrs = (ctypes.c_void_p * len(self.tabs))(*[x.data_ptr() for x in self.tabs])
        self.info = np.ascontiguousarray(np.concatenate(infos).astype(np.float32))
        sfx = "_cubic_f32" if degree == 3 else "_f32"
        self.fwd = "dpb_se_a_descriptor_fwd" + sfx
        self.bwd = "dpb_se_a_descriptor_bwd" + sfx


class _FittingF64:
    """Per-type fitting networks of the FP64 plain path: the layers' GEMMs on
    the project's FP64 GEMM (dpb_gemm_f64), the activations, residuals, the
    atomic energies and the input gradient dE/dD on the fitting-layer kernels
    (dpb_fit_*_f64). Rows of D are grouped by center type; ``type_rows`` gives
    the group sizes (deepmd/pt/model/task/ener.py, layers as
    deepmd/dpmodel/utils/network.py:282-330)."""

    def __init__(self, params: SeAParams, type_rows, device):
        dev = torch.device(device)
        f64 = lambda a: torch.tensor(np.asarray(a, np.float64), device=dev).contiguous()  # noqa: E731
        self.groups = []
        o = 0
        widths_in = params.cfg.neuron[-1] * params.cfg.axis_neuron
        for t, f in enumerate(params.fit):
            n = int(type_rows[t])
            layers, w_in = [], widths_in
            for W, b, d in f["layers"]:
                w_out = int(np.asarray(W).shape[1])
                layers.append(dict(W=f64(W), b=f64(b), d=None if d is None else f64(d),
                                   w_in=w_in, w_out=w_out,
                                   Y=torch.empty((n, w_out), dtype=torch.float64, device=dev),
                                   H=torch.empty((n, w_out), dtype=torch.float64, device=dev),
                                   G=torch.empty((n, w_out), dtype=torch.float64, device=dev)))
                w_in = w_out
            Wo, bo = f["out"]
            out = dict(W=f64(np.asarray(Wo).reshape(-1)), b=f64(np.asarray(bo).reshape(1)),
                       ebias=float(params.bias_atom_e[t]), w=w_in)
            zb = torch.empty((n, max([ly["w_out"] for ly in layers] + [1])),
                             dtype=torch.float64, device=dev)
            self.groups.append((o, n, layers, out, zb))
            o += n
        self.n = o

    @staticmethod
    def _gemm(C, A, B, bias, M, N, K, lda, ldb, ldc, trans_b, acc, s):
        call("dpb_gemm_f64", ptr(C), ptr(A), ptr(B), ptr(bias), M, N, K, lda, ldb, ldc, 0,
             trans_b, acc, s)

    def forward_backward(self, D: torch.Tensor, dD: torch.Tensor, e_rows: torch.Tensor, s):
        """e_rows[r] = atomic energy of fitting row r (with the output and
        atomic energy biases); dD = dE/dD."""
        for o, n, layers, out, zb in self.groups:
            if n == 0:
                continue
            H, w_in = D[o:o + n], D.shape[1]
            for ly in layers:
                self._gemm(ly["Y"], H, ly["W"], ly["b"], n, ly["w_out"], w_in, w_in, ly["w_out"],
                           ly["w_out"], 0, 0, s)
                call("dpb_fit_act_f64", ptr(ly["Y"]), ptr(ly["H"]), ptr(H), ptr(ly["d"]), n,
                     ly["w_out"], w_in, s)
                H, w_in = ly["H"], ly["w_out"]
            call("dpb_fit_out_f64", ptr(e_rows[o:o + n]), ptr(H), ptr(out["W"]), ptr(out["b"]),
                 ctypes.c_double(out["ebias"]), n, out["w"], s)
            # dE/dH of the last hidden layer = Wo on every row, then back
            call("dpb_fit_out_adj_f64", ptr(layers[-1]["G"]), None, None, None, ptr(H), None,
                 ptr(out["W"]), None, n, out["w"], s)
            for k in range(len(layers) - 1, -1, -1):
                ly = layers[k]
                call("dpb_fit_bwd_f64", ptr(zb), ptr(ly["G"]), ptr(ly["Y"]), ptr(ly["d"]), n,
                     ly["w_out"], s)
                dst = dD[o:o + n] if k == 0 else layers[k - 1]["G"]
                # dst = Zb W^T, plus the residual's share of G
                self._gemm(dst, zb, ly["W"], None, n, ly["w_in"], ly["w_out"], ly["w_out"],
                           ly["w_out"], ly["w_in"], 1, 0, s)
                call("dpb_fit_res_adj_f64", ptr(dst), ptr(ly["G"]), n, ly["w_out"], ly["w_in"],
                     s)


def _tf32_rna(w: np.ndarray) -> np.ndarray:
    """Round-to-nearest (ties away) TF32 value of FP32 w, as
    cvt.rna.tf32.f32 computes it (finite inputs)."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x1000) & 0xFFFFE000).astype(np.uint32).view(np.float32)


def tf32_split(w: np.ndarray):
    """(hi, lo) FP32 arrays holding TF32 values: hi the TF32 rounding of w,
    lo the TF32 rounding of w - hi (hi + lo = w to 2^-24 relative)."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    hi = _tf32_rna(w)
    lo = _tf32_rna((w - hi).astype(np.float32))
    return hi, lo


class _FittingTC:
    """Per-type fitting networks, forward and input-gradient, as six fused
    split-TF32 tensor-core GEMMs (dpb_gemm_tf32x3_f32, FP32 accumulation in
    chunks). Rows of the descriptor are grouped by center type;
    ``type_rows`` gives the group sizes."""

    EPI_STORE, EPI_TANH, EPI_RES_DT, EPI_LAST, EPI_BWD_DT, EPI_BWD_RES = range(6)

    def __init__(self, params: SeAParams, type_rows, device):
        dev = torch.device(device)
        self.dev = dev
        cfg = params.cfg
        if len(cfg.fitting) != 3 or len(set(cfg.fitting)) != 1:
            raise _capi.DPBInvalidArgument(
                "the tensor-core fitting path handles three equal-width hidden layers")
        self.type_rows = np.ascontiguousarray(type_rows, dtype=np.int32)
        self.n = int(self.type_rows.sum())
        self.ntypes = cfg.ntypes
        self.width = cfg.fitting[0]
        self.din = cfg.neuron[-1] * cfg.axis_neuron
        f32 = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev)  # noqa: E731
        keep = []

        def split(mats):
            # (hi, lo, fp32): pre-split TF32 parts, and the FP32 weights for
            # the kernel's own split (fit_split_b knob)
            hs, ls, fs = [], [], []
            for m in mats:
                h, l = tf32_split(m)
                hs.append(f32(h))
                ls.append(f32(l))
                fs.append(f32(np.ascontiguousarray(m)))
            keep.extend(hs + ls + fs)
            arr = lambda ts: (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])  # noqa: E731
            return arr(hs), arr(ls), arr(fs)

        def vecs(vs):
            ts = [f32(v) for v in vs]
            keep.extend(ts)
            return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])

        L = [f["layers"] for f in params.fit]
        # B operands are [N, K] row-major: forward uses W^T, backward uses W
        self.B1f = split([l[0][0].T for l in L])
        self.B2f = split([l[1][0].T for l in L])
        self.B3f = split([l[2][0].T for l in L])
        self.B3b = split([l[2][0] for l in L])
        self.B2b = split([l[1][0] for l in L])
        self.B1b = split([l[0][0] for l in L])
        self.b1 = vecs([l[0][1] for l in L])
        self.b2 = vecs([l[1][1] for l in L])
        self.b3 = vecs([l[2][1] for l in L])
        self.d2 = vecs([l[1][2] for l in L])
        self.d3 = vecs([l[2][2] for l in L])
        self.w4 = vecs([f["out"][0][:, 0] for f in params.fit])
        self._keep = keep
        # per-type constant of the energy: output bias + atomic energy bias
        self.e_const = float(sum(int(self.type_rows[t]) * (float(params.fit[t]["out"][1][0])
                                                           + float(params.bias_atom_e[t]))
                                 for t in range(self.ntypes)))
        n, w = self.n, self.width
        z = lambda *shape: torch.zeros(shape, dtype=torch.float32, device=dev)  # noqa: E731
        self.H1, self.Y2, self.H2, self.G3 = z(n, w), z(n, w), z(n, w), z(n, w)
        self.g2, self.G2, self.G1 = z(n, w), z(n, w), z(n, w)
        self.e = z(n)
        self.esum_work = torch.zeros(int(_capi.lib().dpb_fit_energy_sum_work_bytes()),
                                     dtype=torch.uint8, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)

    def _gemm(self, A, K, B, N, mode, out0, out1=None, aux0=None, aux1=None, bias=None,
              idt=None, w=None, s=None):
        split_in_kernel = _capi.lib().dpb_tune_get(b"fit_split_b") == 1
        bh, bl = (B[2], None) if split_in_kernel else (B[0], B[1])
        call("dpb_gemm_tf32x3_f32", ptr(A), self.n, K, bh, bl, N, self.type_rows.ctypes.data,
             self.ntypes, mode, ptr(out0), ptr(out1), ptr(aux0), ptr(aux1), bias, idt, w,
             ptr(self.e), ptr(self.status), s)

    def forward_backward(self, D: torch.Tensor, dD: torch.Tensor, energy: torch.Tensor):
        """energy[0] = sum of atomic energies (FP64); dD = dE/dD (FP32)."""
        self.layers(D, dD, zero_e=False)
        # FP64 total, and self.e left zeroed for the next step's accumulation
        call("dpb_fit_energy_sum_f32", ptr(energy), ptr(self.e), self.n, self.e_const,
             ptr(self.esum_work), torch.cuda.current_stream().cuda_stream)

    def layers(self, D: torch.Tensor, dD: torch.Tensor, zero_e: bool = True):
        """The six GEMMs: self.e[r] = atomic energy of fitting row r without
        its constant (output bias + atomic energy bias); dD = dE/dD. With
        ``zero_e`` False, self.e must hold zeros already (forward_backward's
        energy sum leaves it so)."""
        s = torch.cuda.current_stream().cuda_stream
        w, din = self.width, self.din
        if zero_e:
            self.e.zero_()
        self._gemm(D, din, self.B1f, w, self.EPI_TANH, self.H1, bias=self.b1, s=s)
        self._gemm(self.H1, w, self.B2f, w, self.EPI_RES_DT, self.Y2, self.H2, aux0=self.H1,
                   bias=self.b2, idt=self.d2, s=s)
        self._gemm(self.H2, w, self.B3f, w, self.EPI_LAST, self.G3, aux0=self.H2, bias=self.b3,
                   idt=self.d3, w=self.w4, s=s)
        self._gemm(self.G3, w, self.B3b, w, self.EPI_BWD_DT, self.G2, self.g2, aux0=self.Y2,
                   idt=self.d2, w=self.w4, s=s)
        self._gemm(self.G2, w, self.B2b, w, self.EPI_BWD_RES, self.G1, aux0=self.H1,
                   aux1=self.g2, s=s)
        self._gemm(self.G1, w, self.B1b, din, self.EPI_STORE, dD, s=s)


# ------------------------------------------------------------ evaluators --

class _Stages:
    """Context manager factory recording CUDA events around named stages."""

    def __init__(self, timers):
        self.timers = timers

    def __call__(self, name):
        return _Stage(self.timers, name)


class _Stage:
    def __init__(self, timers, name):
        self.timers, self.name = timers, name

    def __enter__(self):
        if self.timers is not None:
            self.a = torch.cuda.Event(enable_timing=True)
            self.a.record()

    def __exit__(self, *exc):
        if self.timers is not None:
            b = torch.cuda.Event(enable_timing=True)
            b.record()
            self.timers.setdefault(self.name, []).append((self.a, b))
        return False


class SeAEvaluator:
    """Energy/force/virial of one frame of fixed size, types and box.

    mode "compressed": FP32 table path (needs params.tables);
    mode "plain": FP64 embedding-MLP path (the embedding net, descriptor and
    its backward on the se_a training kernels in FP64, the fitting on the
    FP64 GEMM; 3-layer embedding nets of widths <= 32 / 64 / 128).
    Device buffers are allocated once; ``step()`` runs one evaluation on the
    current coordinates in ``self.coord``; ``capture()`` records the step into
    a CUDA graph that ``replay()`` re-runs.

    ``skin > 0`` switches to an MD engine's pattern: ``rebuild()`` makes the
    ghosts and a neighbor list within rcut + skin (host synchronisation
    allowed there); each step only moves the ghosts with their owners
    (``dpb_ghost_refresh_f64``) and formats the kept list against rcut
    (``dpb_prod_env_mat_a_mixed``), as prod_env_mat_a_gpu does with the list
    LAMMPS passes."""

    def __init__(self, params: SeAParams, atype: np.ndarray, box: np.ndarray,
                 mode: str = "compressed", device="cuda:0", nall_capacity: int | None = None,
                 tensor_core_fitting: bool = True, skin: float = 0.0,
                 table_degree: int = DEFAULT_TABLE_DEGREE):
        cfg = params.cfg
        if mode not in ("compressed", "plain"):
            raise _capi.DPBInvalidArgument(f"mode must be 'compressed' or 'plain', not {mode!r}")
        self.cfg, self.params, self.mode = cfg, params, mode
        self.skin = float(skin)
        self.rc_list = float(cfg.rcut) + self.skin
        self.dev = torch.device(device)
        self.nloc = int(atype.size)
        self.box = np.ascontiguousarray(np.asarray(box, np.float64).reshape(9))
        self.atype = torch.tensor(atype, dtype=torch.int32, device=self.dev)
        self.sec = cfg.sec
        nloc, nnei = self.nloc, cfg.nnei
        lib = _capi.lib()
        self.copy_bytes = int(lib.dpb_copy_coord_scratch_bytes(
            nloc, ctypes.c_float(self.rc_list), self.box.ctypes.data))
        if nall_capacity is None:
            # ghosts are at most the ghost cells' share of the atoms; +25% slack
            nall_capacity = int(self._estimate_nall() * 1.25) + 64
        self.mem_nall = nall_capacity
        # with room for the cell-ordered candidate records of the env kernel
        self.grid_bytes = int(lib.dpb_cell_grid_bytes_packed(self.mem_nall))
        dev = self.dev
        fdt = torch.float32 if mode == "compressed" else torch.float64
        self.fdt = fdt
        self.coord = torch.zeros((nloc, 3), dtype=torch.float64, device=dev)
        self.coord_n = torch.zeros_like(self.coord)
        self.cext = torch.zeros((self.mem_nall, 3), dtype=torch.float64, device=dev)
        self.text = torch.zeros(self.mem_nall, dtype=torch.int32, device=dev)
        self.mapping = torch.zeros(self.mem_nall, dtype=torch.int32, device=dev)
        self.nall_dev = torch.zeros(1, dtype=torch.int32, device=dev)
        self.copy_scratch = torch.empty(self.copy_bytes, dtype=torch.uint8, device=dev)
        self.geo_bytes = int(lib.dpb_geometry_scratch_bytes(
            nloc, ctypes.c_float(cfg.rcut), self.box.ctypes.data))
        self.geo_scratch = torch.empty(self.geo_bytes, dtype=torch.uint8, device=dev)
        self.grid = torch.empty(self.grid_bytes, dtype=torch.uint8, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.avg = torch.tensor(params.davg, dtype=fdt, device=dev)
        self.std = torch.tensor(params.dstd, dtype=fdt, device=dev)
        self.em = torch.empty((nloc, nnei * 4), dtype=fdt, device=dev)
        self.nlist = torch.empty((nloc, nnei), dtype=torch.int32, device=dev)
        self.net_deriv = torch.empty((nloc, nnei * 4), dtype=fdt, device=dev)
        # energy, force and virial side by side: one device-to-host copy
        self.results = torch.zeros(1 + 3 * nloc + 9, dtype=torch.float64, device=dev)
        self.energy = self.results[0:1]
        self.force = self.results[1:1 + 3 * nloc].view(nloc, 3)
        self.virial = self.results[1 + 3 * nloc:]
        M, ax = cfg.neuron[-1], cfg.axis_neuron
        # atoms grouped by type for the per-type fitting networks
        order = np.argsort(atype, kind="stable")
        row = np.empty(nloc, np.int32)
        row[order] = np.arange(nloc, dtype=np.int32)
        self.drow = torch.tensor(row, device=dev)
        self.order = torch.tensor(order.astype(np.int64), device=dev)
        counts = np.bincount(atype, minlength=cfg.ntypes)
        self.type_ranges = [(int(s), int(s + c)) for s, c in
                            zip(np.concatenate([[0], np.cumsum(counts)[:-1]]), counts)]
        # the FP32 fitting must not silently drop to TF32 tensor-core math
        torch.backends.cuda.matmul.allow_tf32 = False
        if mode == "compressed":
            self.fitting = _Fitting(params, fdt, dev)
            self.xyz = torch.empty((nloc, 4, M), dtype=torch.float32, device=dev)
            self.D = torch.empty((nloc, M * ax), dtype=torch.float32, device=dev)
            self.dD = torch.empty_like(self.D)
            self.fit_tc = _FittingTC(params, counts, dev) if tensor_core_fitting else None
            self.ptab = PipelineTables(params, dev, table_degree)
        else:
            self._plain_setup(params, counts)
        if self.skin > 0:
            self.shift = torch.zeros_like(self.cext)
            self.ilist = torch.arange(nloc, dtype=torch.int32, device=dev)
            self.numneigh = torch.zeros(nloc, dtype=torch.int32, device=dev)
            self.nl_width = 0
            self.rows = None
            self.firstneigh = None
            self.nl_bytes = int(lib.dpb_build_nlist_scratch_bytes(nloc, self.mem_nall))
            self.nl_scratch = torch.empty(self.nl_bytes, dtype=torch.uint8, device=dev)
            self.built = False
        self.graph = None

    def _estimate_nall(self) -> int:
        # extended cells over local cells, times nloc (the reference's own
        # estimate in neighbor_list.cc:774-778), for the ghost cutoff in use
        b = self.box
        rc = self.rc_list
        L = np.array([np.linalg.norm(b[0:3]), np.linalg.norm(b[3:6]), np.linalg.norm(b[6:9])])
        nc = np.maximum(1, np.floor(L / rc))
        ng = np.floor(rc / (L / nc)) + 1
        return int(np.prod(nc + 2 * ng) / np.prod(nc) * self.nloc)

    def _plain_setup(self, params: SeAParams, counts):
        """Device buffers and weights of the FP64 plain path."""
        from .train import fold_flags

        cfg, dev, n = self.cfg, self.dev, self.nloc
        if len(cfg.neuron) != 3 or not (3 <= cfg.neuron[0] <= 32 and cfg.neuron[1] <= 64 and
                                        cfg.neuron[2] <= 128) or cfg.axis_neuron > 32:
            raise _capi.DPBInvalidArgument(
                "the FP64 plain path takes 3-layer embedding nets of widths <= 32 / 64 / 128 "
                "and axis_neuron <= 32")
        M, ax = cfg.neuron[-1], cfg.axis_neuron
        f64 = lambda a: torch.tensor(np.asarray(a, np.float64), device=dev).contiguous()  # noqa: E731
        self.emb_W = [f64(W) for net in params.emb for W, _ in net]
        self.emb_b = [f64(b) for net in params.emb for _, b in net]
        vp = lambda xs: (ctypes.c_void_p * len(xs))(*[x.data_ptr() for x in xs])  # noqa: E731
        self.Wp, self.bp = vp(self.emb_W), vp(self.emb_b)
        self.widths = np.array([1, *cfg.neuron], np.int32)
        self.fold = fold_flags(params)
        z = lambda *shape: torch.zeros(shape, dtype=torch.float64, device=dev)  # noqa: E731
        self.xyz = z(n, 4, M)
        self.D = z(n, M * ax)
        self.dD = z(n, M * ax)
        self.xbar = z(n, 4, M)
        self.e_rows = z(n)
        self.fit64 = _FittingF64(params, counts, dev)
        self.one_frame = torch.tensor([0, n], dtype=torch.int32, device=dev)
        self.zero_const = z(1)

    # ---- neighbor list with a skin, rebuilt on request (host syncs allowed)
    def rebuild(self):
        """Ghosts and the rcut + skin neighbor list from the current
        ``self.coord``; later steps reuse them until the next rebuild."""
        if self.skin <= 0:
            raise _capi.DPBInvalidArgument("rebuild() needs an evaluator made with skin > 0")
        cfg, nloc = self.cfg, self.nloc
        s = torch.cuda.current_stream().cuda_stream
        self.coord_n.copy_(self.coord)
        call("dpb_normalize_coord_f64", ptr(self.coord_n), nloc, self.box.ctypes.data, s)
        call("dpb_copy_coord_async_f64", ptr(self.cext), ptr(self.text), ptr(self.mapping),
             ptr(self.nall_dev), ptr(self.copy_scratch), self.copy_bytes, ptr(self.coord_n),
             ptr(self.atype), nloc, self.mem_nall, ctypes.c_float(self.rc_list),
             self.box.ctypes.data, s)
        nall = int(self.nall_dev.item())
        if nall > self.mem_nall:
            raise _capi.DPBCapacityError(
                f"DeePMD-kit Error: nall={nall} exceeds the capacity {self.mem_nall}")
        # ghost images relative to the raw (unwrapped) coordinates the steps move
        call("dpb_ghost_shift_f64", ptr(self.shift), ptr(self.cext), ptr(self.coord),
             ptr(self.mapping), ptr(self.nall_dev), self.mem_nall, s)
        width = max(self.nl_width, 256)
        while True:
            if self.rows is None or width != self.nl_width:
                self.rows = torch.full((nloc, width), -1, dtype=torch.int32, device=self.dev)
                fn = ops._row_pointers(self.rows)
                if self.firstneigh is None:
                    self.firstneigh = fn
                else:
                    self.firstneigh.copy_(fn)
                if width != self.nl_width and self.graph is not None:
                    self.graph = None  # the list width is a launch argument
                    self._recapture = True
                self.nl_width = width
            mx = ctypes.c_int(0)
            code = _capi.lib().dpb_build_nlist_f64(
                ptr(self.ilist), ptr(self.numneigh), ptr(self.firstneigh),
                ctypes.addressof(mx), ptr(self.nl_scratch), self.nl_bytes, ptr(self.cext),
                nloc, nall, width, ctypes.c_float(self.rc_list), 1, ptr(self.text), s)
            if code == 1 and mx.value > width:
                width = (mx.value * 5 // 4 + 31) // 32 * 32
                continue
            _capi.check(code, "build_nlist")
            break
        self.built = True
        return nall

    # ---- one step, no host synchronisation
    def step(self, timers: dict | None = None):
        """One evaluation. ``timers`` (eager runs only) collects a pair of CUDA
        events around every stage, keyed by stage name."""
        cfg, s = self.cfg, torch.cuda.current_stream().cuda_stream
        nloc, nnei = self.nloc, cfg.nnei
        tm = _Stages(timers)
        if self.mode == "compressed":
            # force / virial accumulators, zeroed here where no kernel boundary
            # of the step is delayed by it
            call("dpb_zero_async", ptr(self.results) + 8, 8 * (self.results.numel() - 1), s)
        if self.skin > 0:
            if not self.built:
                raise _capi.DPBInvalidArgument("call rebuild() before the first step")
            with tm("coord"):
                call("dpb_ghost_refresh_f64", ptr(self.cext), ptr(self.shift), ptr(self.coord),
                     ptr(self.mapping), ptr(self.nall_dev), self.mem_nall, s)
            env = "dpb_prod_env_mat_a_mixed" if self.mode == "compressed" else \
                "dpb_prod_env_mat_a_f64"
            with tm("env_mat"):
                call(env, ptr(self.em), None, None, ptr(self.nlist), ptr(self.cext),
                     ptr(self.text), nloc, ptr(self.ilist), ptr(self.numneigh),
                     ptr(self.firstneigh), self.nl_width, ptr(self.avg), ptr(self.std), nloc,
                     self.mem_nall, 1, ctypes.c_float(cfg.rcut), ctypes.c_float(cfg.rcut_smth),
                     self.sec.ctypes.data, self.sec.size, ptr(self.status), s)
        else:
            with tm("geometry"):
                # wrap into the box, ghosts, cell grid: one cooperative launch
                call("dpb_geometry_cells_f64", ptr(self.cext), ptr(self.text),
                     ptr(self.mapping), ptr(self.nall_dev), ptr(self.grid), self.grid_bytes,
                     ptr(self.geo_scratch), self.geo_bytes, ptr(self.coord), ptr(self.atype),
                     nloc, self.mem_nall, ctypes.c_float(cfg.rcut), self.box.ctypes.data,
                     ptr(self.status), s)
            env = "dpb_env_mat_a_cells_mixed" if self.mode == "compressed" else \
                "dpb_env_mat_a_cells_f64"
            with tm("env_mat"):
                # only em and nlist are stored: em_deriv and rij are recomputed
                # by the force/virial kernel
                call(env, ptr(self.em), None, None, ptr(self.nlist),
                     ptr(self.cext), ptr(self.text), ptr(self.grid), ptr(self.avg),
                     ptr(self.std), nloc, self.mem_nall, ctypes.c_float(cfg.rcut),
                     ctypes.c_float(cfg.rcut_smth), self.sec.ctypes.data, self.sec.size,
                     ptr(self.status), s)
        if self.mode == "compressed":
            self._descriptor_compressed(s, tm)
        else:
            self._descriptor_plain(s, tm)
        # the compressed path zeroed force / virial at the start of the step
        fv = "dpb_force_virial_a_env_mixed_acc" if self.mode == "compressed" else \
            "dpb_force_virial_a_env_f64"
        with tm("force_virial"):
            call(fv, ptr(self.force), ptr(self.virial), ptr(self.net_deriv), ptr(self.cext),
                 ptr(self.text), ptr(self.std), ptr(self.nlist), ptr(self.mapping), nloc, nloc,
                 nnei, cfg.ntypes, ctypes.c_float(cfg.rcut), ctypes.c_float(cfg.rcut_smth), s)

    def _descriptor_compressed(self, s, tm):
        cfg = self.cfg
        M, ax = cfg.neuron[-1], cfg.axis_neuron
        pt = self.ptab
        with tm("descriptor_fwd"):
            call(pt.fwd, ptr(self.xyz), ptr(self.D), ptr(self.drow), ptr(self.em), pt.ptrs,
                 pt.info.ctypes.data, self.sec.ctypes.data, self.sec.size, self.nloc, M, ax, s)
        with tm("fitting"):
            if self.fit_tc is not None:
                self.fit_tc.forward_backward(self.D, self.dD, self.energy)
            else:
                etot = torch.zeros((), dtype=torch.float64, device=self.dev)
                for t, (a, b) in enumerate(self.type_ranges):
                    if b == a:
                        continue
                    e, g = self.fitting.forward_backward(t, self.D[a:b])
                    self.dD[a:b].copy_(g)
                    etot = etot + e.to(torch.float64).sum()
                self.energy.copy_(etot.view(1))
        with tm("descriptor_bwd"):
            call(pt.bwd, ptr(self.net_deriv), ptr(self.dD), ptr(self.drow), ptr(self.xyz),
                 ptr(self.em), pt.ptrs, pt.info.ctypes.data, self.sec.ctypes.data,
                 self.sec.size, self.nloc, M, ax, s)

    def _descriptor_plain(self, s, tm):
        """Embedding net, descriptor, fitting and their backward in FP64:
        net_deriv = dE/d(em) and the energy, all in kernels of this package
        (deepmd/pt/model/descriptor/se_a.py:826-851 and the fitting net)."""
        cfg, n = self.cfg, self.nloc
        sec = self.sec
        with tm("embedding_fwd_fp64"):
            call("dpb_se_a_train_fwd_f64", ptr(self.xyz), ptr(self.D), ptr(self.em),
                 ptr(self.nlist), ptr(self.atype), ptr(self.drow), self.Wp, self.bp,
                 self.widths.ctypes.data, sec.ctypes.data, sec.size, n, cfg.axis_neuron,
                 self.fold.ctypes.data, s)
        with tm("fitting_fp64"):
            self.fit64.forward_backward(self.D, self.dD, self.e_rows, s)
            call("dpb_batch_energy_f64", ptr(self.energy), ptr(self.e_rows), ptr(self.drow),
                 ptr(self.zero_const), ptr(self.one_frame), 1, s)
        with tm("embedding_bwd_fp64"):
            call("dpb_se_a_train_bwd_f64", ptr(self.net_deriv), ptr(self.xbar), ptr(self.em),
                 ptr(self.xyz), ptr(self.dD), ptr(self.nlist), ptr(self.atype),
                 ptr(self.drow), self.Wp, self.bp, self.widths.ctypes.data, sec.ctypes.data,
                 sec.size, n, cfg.axis_neuron, s)

    # ---- graph capture / replay
    def capture(self, warmup: int = 2):
        if self.skin > 0 and not self.built:
            self.rebuild()
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
        self.io_graph = None  # recaptured by the next run_pinned()
        return self

    # ---- one graph from pinned host input to pinned host output
    def io_buffers(self):
        """(coord [nloc, 3], results [1 + 3 nloc + 9]): pinned host buffers
        of run_pinned(). Write the coordinates into ``coord``; after
        run_pinned() ``results`` holds the energy, the forces (row-major) and
        the virial, all FP64."""
        if getattr(self, "h_coord", None) is None:
            self.h_coord = torch.zeros((self.nloc, 3), dtype=torch.float64, pin_memory=True)
            self.h_results = torch.zeros(1 + 3 * self.nloc + 9, dtype=torch.float64,
                                         pin_memory=True)
            self.io_graph = None
        return self.h_coord, self.h_results

    def run_pinned(self):
        """One evaluation of the coordinates in io_buffers()[0] into
        io_buffers()[1]: the host-to-device copy, the step and the
        device-to-host copy of the results replayed as ONE CUDA graph, then
        one synchronisation. (energy, force [nloc, 3], virial [9]) are
        returned as views of the result buffer, valid until the next call.
        For evaluators without a skin list (with one, use compute())."""
        if self.skin > 0:
            raise _capi.DPBInvalidArgument("run_pinned: evaluators with a skin list use compute()")
        hc, hr = self.io_buffers()
        if self.io_graph is None or getattr(self, "_recapture", False):
            self._recapture = False
            s = torch.cuda.Stream(device=self.dev)
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                for _ in range(2):
                    self.coord.copy_(hc, non_blocking=True)
                    self.step()
                    hr.copy_(self.results, non_blocking=True)
            torch.cuda.current_stream().wait_stream(s)
            torch.cuda.synchronize()
            self.io_graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.io_graph):
                self.coord.copy_(hc, non_blocking=True)
                self.step()
                hr.copy_(self.results, non_blocking=True)
            torch.cuda.synchronize()
        self.io_graph.replay()
        torch.cuda.current_stream().synchronize()
        n = self.nloc
        return hr[0:1], hr[1:1 + 3 * n].view(n, 3), hr[1 + 3 * n:]

    def tune(self, reps: int = 10, use_cache: bool = True) -> dict:
        """Autotune the launch shapes of this step (atoms per CTA of the fused
        descriptor kernels, table-load cache policy, fitting GEMM N tile and
        weight split, programmatic dependent launch on or off); leaves it
        captured with the fastest."""
        from . import autotune

        cfg = self.cfg
        sig = (f"frame:{self.nloc}a:{self.mode}:skin{self.skin:g}:deg{self.ptab.degree}:"
               f"sel{'-'.join(map(str, cfg.sel))}:"
               f"M{cfg.neuron[-1]}:fit{'-'.join(map(str, cfg.fitting))}")
        return autotune.tune(self.replay, lambda: self.capture(),
                             ["desc_atoms_per_cta", "desc_coef_l1", "fit_n_tile", "fit_split_b",
                              "pdl"],
                             signature=sig, reps=reps,
                             device=self.dev, use_cache=use_cache)

    def replay(self):
        if getattr(self, "_recapture", False):
            self._recapture = False
            self.capture()
        if self.graph is None:
            self.step()
        else:
            self.graph.replay()

    def check(self):
        """Raise if the last step overflowed a capacity (reads device words)."""
        h = torch.stack([self.nall_dev[0], self.status[0]]).cpu().numpy()
        if h[0] > self.mem_nall:
            raise _capi.DPBCapacityError(
                f"DeePMD-kit Error: nall={h[0]} exceeds the capacity {self.mem_nall}")
        call("dpb_status_check", ptr(self.status), torch.cuda.current_stream().cuda_stream)
        if getattr(self, "fit_tc", None) is not None:
            call("dpb_status_check", ptr(self.fit_tc.status),
                 torch.cuda.current_stream().cuda_stream)
        return int(h[0])

    # ---- public call: host in, host out
    def compute(self, coord, out: torch.Tensor | None = None, rebuild: bool = False):
        """Energy (float), force [nloc, 3] and virial [9] of host coordinates.

        ``coord`` is a host array/tensor (pinned for an asynchronous copy);
        ``out`` an optional pinned host buffer of 1 + 3 nloc + 9 doubles;
        ``rebuild`` (skin > 0 only) remakes the ghosts and the list first (it
        is also done on the first call)."""
        if isinstance(coord, torch.Tensor):
            self.coord.copy_(coord.view(-1, 3), non_blocking=True)
        else:
            self.coord.copy_(torch.as_tensor(np.asarray(coord, np.float64).reshape(-1, 3)))
        if self.skin > 0 and (rebuild or not self.built):
            self.rebuild()
        self.replay()
        n = self.nloc
        if out is None:
            out = torch.empty(1 + 3 * n + 9, dtype=torch.float64, pin_memory=True)
        out.copy_(self.results, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        o = out.numpy()
        return float(o[0]), o[1:1 + 3 * n].reshape(-1, 3).copy(), o[1 + 3 * n:].copy()
