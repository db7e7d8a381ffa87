"""Test infrastructure only: FP64 CPU energy/force/virial of the se_e2_a model.

Geometry (ghost copy, neighbor list, env matrix, force/virial assembly) comes
from the C checkers in oracle.py (restatement or compiled reference); the
network part is FP64 torch on the CPU with autograd for dE/d(em):

* plain:      the embedding MLP (deepmd/pt/model/descriptor/se_a.py:834-837);
* compressed: the table op from the checker library, with its gradient from
              the checker's tabulate_fusion_se_a_grad (tabulate.cc:234-341).

Descriptor and fitting follow se_a.py:839-851 and the fitting network of
deepmd/dpmodel/utils/network.py:282-330 (timestep residual when widths match).
This oracle is pinned against the reference's own PyTorch model by
tests/golden/model_golden.npz (see tests/golden/make_model_golden.py).
"""

from __future__ import annotations

import numpy as np
import torch


def env_stats(lib, cfg, coord, atype, box, protection=1e-2):
    """davg/dstd and the minimum neighbor distance (env_mat_stat.py:296-425)."""
    nloc = atype.size
    c, t, m = lib.copy_coord(coord, atype, cfg.rcut, box)
    ret, il, nn, rb, _ = lib.build_nlist(c, nloc, cfg.rcut, atype=t, mem_size=c.shape[0])
    assert ret == 0
    z = np.zeros((cfg.ntypes, cfg.nnei * 4))
    o = np.ones_like(z)
    em, _, rij, nlist = lib.prod_env_mat_a(c, t, il, nn, rb, z, o, nloc, cfg.rcut,
                                           cfg.rcut_smth, cfg.sec)
    em = em.reshape(nloc, cfg.nnei, 4)
    davg = np.zeros((cfg.ntypes, cfg.nnei, 4))
    dstd = np.ones((cfg.ntypes, cfg.nnei, 4))
    for ty in range(cfg.ntypes):
        s = em[atype == ty]
        if s.size == 0:
            dstd[ty] *= 0.1
            continue
        r = s[:, :, 0].reshape(-1)
        a = s[:, :, 1:].reshape(-1)

        def std(v):
            x = np.sqrt(max(np.mean(v * v) - np.mean(v) ** 2, 0.0))
            return protection if abs(x) < protection else x

        davg[ty, :, 0] = np.mean(r)
        dstd[ty, :, 0] = std(r)
        dstd[ty, :, 1:] = std(a)
    d = np.linalg.norm(rij.reshape(nloc, cfg.nnei, 3), axis=-1)[nlist >= 0]
    return davg.reshape(cfg.ntypes, -1), dstd.reshape(cfg.ntypes, -1), float(d.min())


class _Tab(torch.autograd.Function):
    """Table op of the checker library with its first gradient."""

    @staticmethod
    def forward(ctx, em, lib, table, info, M):
        e = em.detach().numpy()
        out = lib.tabulate(table, info, e[:, :, 0].copy(), e, M)
        ctx.lib, ctx.table, ctx.info, ctx.M = lib, table, info, M
        ctx.save_for_backward(em)
        return torch.from_numpy(out)

    @staticmethod
    def backward(ctx, dy):
        (em,) = ctx.saved_tensors
        e = em.detach().numpy()
        dx, de = ctx.lib.tabulate_grad(ctx.table, ctx.info, e[:, :, 0].copy(), e,
                                       dy.detach().numpy().copy(), ctx.M)
        de = de.copy()
        de[:, :, 0] += dx
        return torch.from_numpy(de), None, None, None, None


def _embed(net, x):
    h = x
    for W, b in net:
        Wt = torch.from_numpy(np.asarray(W))
        y = torch.tanh(h @ Wt + torch.from_numpy(np.asarray(b)))
        if Wt.shape[1] == Wt.shape[0]:
            y = y + h
        elif Wt.shape[1] == 2 * Wt.shape[0]:
            y = y + torch.cat([h, h], -1)
        h = y
    return h


def _fit(f, x):
    h = x
    for W, b, d in f["layers"]:
        y = torch.tanh(h @ torch.from_numpy(W) + torch.from_numpy(b))
        if d is not None:
            h = h + torch.from_numpy(d) * y
        elif W.shape[0] == W.shape[1]:
            h = h + y
        else:
            h = y
    Wo, bo = f["out"]
    return (h @ torch.from_numpy(Wo) + torch.from_numpy(bo)).view(-1)


def evaluate(lib, params, coord, atype, box, mode="plain"):
    """(energy, force [nloc, 3], virial [9]) in FP64; mode plain|compressed."""
    cfg = params.cfg
    nloc = atype.size
    cn = lib.normalize_coord(np.asarray(coord, np.float64).reshape(-1), box).reshape(-1, 3)
    c, t, mapping = lib.copy_coord(cn, atype, cfg.rcut, box)
    nall = c.shape[0]
    ret, il, nn, rb, _ = lib.build_nlist(c, nloc, cfg.rcut, atype=t, mem_size=nall)
    assert ret == 0
    em, emd, rij, nlist = lib.prod_env_mat_a(c, t, il, nn, rb, params.davg, params.dstd, nloc,
                                             cfg.rcut, cfg.rcut_smth, cfg.sec)
    nnei = cfg.nnei
    emt = torch.from_numpy(em.reshape(nloc, nnei, 4).copy()).requires_grad_(True)
    xyz = torch.zeros((nloc, 4, cfg.neuron[-1]), dtype=torch.float64)
    sec = cfg.sec
    for ty in range(cfg.ntypes):
        a, b = int(sec[ty]), int(sec[ty + 1])
        if b == a:
            continue
        rr = emt[:, a:b, :]
        if mode == "plain":
            g = _embed(params.emb[ty], rr[:, :, :1])
            xyz = xyz + rr.transpose(1, 2) @ g
        else:
            table, info = params.tables[ty]
            xyz = xyz + _Tab.apply(rr, lib, np.ascontiguousarray(table), info, cfg.neuron[-1])
    xyz = xyz / nnei
    D = (xyz.transpose(1, 2) @ xyz[:, :, :cfg.axis_neuron]).reshape(nloc, -1)
    E = torch.zeros((), dtype=torch.float64)
    for ty in range(cfg.ntypes):
        sel = np.nonzero(atype == ty)[0]
        if sel.size:
            E = E + (_fit(params.fit[ty], D[torch.from_numpy(sel)]) + params.bias_atom_e[ty]).sum()
    (g,) = torch.autograd.grad(E, emt)
    nd = g.reshape(nloc, nnei * 4).numpy()
    fext = lib.prod_force_a(nd, emd, nlist, nloc, nall)[0]
    force = np.zeros((nloc, 3))
    np.add.at(force, mapping, fext)
    virial, _ = lib.prod_virial_a(nd, emd, rij, nlist, nloc, nall)
    return float(E.detach()), force, virial
