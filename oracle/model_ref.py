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


def _network_rows(lib, params, em_rows, atype_rows, mode):
    """Energy of a block of centers and its gradient w.r.t. their env rows."""
    cfg = params.cfg
    n, nnei = atype_rows.size, cfg.nnei
    emt = torch.from_numpy(em_rows.reshape(n, nnei, 4).copy()).requires_grad_(True)
    xyz = torch.zeros((n, 4, cfg.neuron[-1]), dtype=torch.float64)
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
    D = (xyz.transpose(1, 2) @ xyz[:, :, :cfg.axis_neuron]).reshape(n, -1)
    E = torch.zeros((), dtype=torch.float64)
    for ty in range(cfg.ntypes):
        sel = np.nonzero(atype_rows == ty)[0]
        if sel.size:
            E = E + (_fit(params.fit[ty], D[torch.from_numpy(sel)]) + params.bias_atom_e[ty]).sum()
    (g,) = torch.autograd.grad(E, emt)
    return float(E.detach()), g.reshape(n, nnei * 4).numpy()


def evaluate(lib, params, coord, atype, box, mode="plain", chunk=None):
    """(energy, force [nloc, 3], virial [9]) in FP64; mode plain|compressed.

    ``chunk`` evaluates the network over blocks of that many centers (the
    atomic energies are independent, so the result is the same; only the
    host memory of the autograd graph is bounded)."""
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
    em = em.reshape(nloc, nnei * 4)
    step = nloc if not chunk else int(chunk)
    E = 0.0
    nd = np.zeros((nloc, nnei * 4))
    for a in range(0, nloc, step):
        b = min(nloc, a + step)
        e, g = _network_rows(lib, params, em[a:b], np.asarray(atype)[a:b], mode)
        E += e
        nd[a:b] = g
    fext = lib.prod_force_a(nd, emd, nlist, nloc, nall)[0]
    force = np.zeros((nloc, 3))
    np.add.at(force, mapping, fext)
    virial, _ = lib.prod_virial_a(nd, emd, rij, nlist, nloc, nall)
    return E, force, virial


# ----------------------------------------------------------------- training --

EMB_PREFIX = "atomic_model.descriptor.sea.filter_layers.networks"
FIT_PREFIX = "atomic_model.fitting_net.filter_layers.networks"


def trainable(params):
    """{reference state_dict name: FP64 leaf tensor} of every trainable weight
    (embedding matrix/bias, fitting matrix/bias/idt, output layer)."""
    out = {}
    for t, net in enumerate(params.emb):
        for l, (W, b) in enumerate(net):
            out[f"{EMB_PREFIX}.{t}.layers.{l}.matrix"] = np.asarray(W)
            out[f"{EMB_PREFIX}.{t}.layers.{l}.bias"] = np.asarray(b)
    for t, f in enumerate(params.fit):
        for l, (W, b, d) in enumerate(f["layers"]):
            out[f"{FIT_PREFIX}.{t}.layers.{l}.matrix"] = np.asarray(W)
            out[f"{FIT_PREFIX}.{t}.layers.{l}.bias"] = np.asarray(b)
            if d is not None:
                out[f"{FIT_PREFIX}.{t}.layers.{l}.idt"] = np.asarray(d)
        L = len(f["layers"])
        out[f"{FIT_PREFIX}.{t}.layers.{L}.matrix"] = np.asarray(f["out"][0]).reshape(-1, 1)
        out[f"{FIT_PREFIX}.{t}.layers.{L}.bias"] = np.asarray(f["out"][1]).reshape(1)
    return {k: torch.tensor(v, dtype=torch.float64, requires_grad=True) for k, v in out.items()}


def _geometry(lib, params, coord, atype, box):
    cfg = params.cfg
    nloc = atype.size
    cn = lib.normalize_coord(np.asarray(coord, np.float64).reshape(-1), box).reshape(-1, 3)
    c, t, mapping = lib.copy_coord(cn, atype, cfg.rcut, box)
    nall = c.shape[0]
    ret, il, nn, rb, _ = lib.build_nlist(c, nloc, cfg.rcut, atype=t, mem_size=nall)
    assert ret == 0
    em, emd, rij, nlist = lib.prod_env_mat_a(c, t, il, nn, rb, params.davg, params.dstd, nloc,
                                             cfg.rcut, cfg.rcut_smth, cfg.sec)
    return em, emd, rij, nlist, mapping, nall


def _energy_force_virial(params, P, geo, atype, create_graph):
    """FP64 torch E, force [nloc, 3], virial [9] of one frame as functions of
    the weights P (create_graph keeps the force differentiable)."""
    cfg = params.cfg
    em, emd, rij, nlist, mapping, nall = geo
    nloc, nnei = atype.size, cfg.nnei
    emt = torch.from_numpy(em.reshape(nloc, nnei, 4).copy()).requires_grad_(True)
    xyz = torch.zeros((nloc, 4, cfg.neuron[-1]), dtype=torch.float64)
    sec = cfg.sec
    for ty in range(cfg.ntypes):
        a, b = int(sec[ty]), int(sec[ty + 1])
        if b == a:
            continue
        rr = emt[:, a:b, :]
        h = rr[:, :, :1]
        for l in range(len(cfg.neuron)):
            W = P[f"{EMB_PREFIX}.{ty}.layers.{l}.matrix"]
            y = torch.tanh(h @ W + P[f"{EMB_PREFIX}.{ty}.layers.{l}.bias"])
            if W.shape[1] == W.shape[0]:
                y = y + h
            elif W.shape[1] == 2 * W.shape[0]:
                y = y + torch.cat([h, h], -1)
            h = y
        xyz = xyz + rr.transpose(1, 2) @ h
    xyz = xyz / nnei
    D = (xyz.transpose(1, 2) @ xyz[:, :, :cfg.axis_neuron]).reshape(nloc, -1)
    E = torch.zeros((), dtype=torch.float64)
    for ty in range(cfg.ntypes):
        idx = np.nonzero(atype == ty)[0]
        if idx.size == 0:
            continue
        h = D[torch.from_numpy(idx)]
        L = len(params.fit[ty]["layers"])
        for l in range(L):
            key = f"{FIT_PREFIX}.{ty}.layers.{l}"
            W = P[key + ".matrix"]
            y = torch.tanh(h @ W + P[key + ".bias"])
            if key + ".idt" in P:
                y = y * P[key + ".idt"]
            h = h + y if W.shape[0] == W.shape[1] else y
        key = f"{FIT_PREFIX}.{ty}.layers.{L}"
        e = (h @ P[key + ".matrix"] + P[key + ".bias"]).view(-1) + float(params.bias_atom_e[ty])
        E = E + e.sum()
    (g,) = torch.autograd.grad(E, emt, create_graph=create_graph)
    # prod_force / prod_virial (prod_force.cc:23-72, prod_virial.cc:22-69) in torch
    ed = torch.from_numpy(emd.reshape(nloc, nnei, 4, 3).copy())
    q = torch.einsum("ina,inad->ind", g, ed)  # per slot
    nl = torch.from_numpy(nlist.reshape(nloc, nnei).astype(np.int64))
    mask = (nl >= 0).to(torch.float64).unsqueeze(-1)
    q = q * mask
    fext = torch.zeros((nall, 3), dtype=torch.float64)
    fext = fext.index_add(0, nl.clamp(min=0).reshape(-1), q.reshape(-1, 3))
    fext = fext.index_add(0, torch.arange(nloc), -q.sum(1))
    force = torch.zeros((nloc, 3), dtype=torch.float64).index_add(
        0, torch.from_numpy(np.asarray(mapping, np.int64)), fext)
    r = torch.from_numpy(rij.reshape(nloc, nnei, 3).copy())
    virial = torch.einsum("ind,ine->de", q, r).reshape(9)
    return E, force, virial


def train_loss_grads(lib, params, frames, labels, prefs, P=None):
    """EnergyStdLoss of a batch of frames and its gradient w.r.t. every
    trainable weight, by FP64 torch autograd through the force
    (create_graph), the way the reference trains (transform_output.py:70-101,
    ener.py:219-340). frames: [(coord, atype, box)]; labels: (E [F], F [N, 3],
    V [F, 9]); prefs: (p_e, p_f, p_v). Returns (loss, E, F, V, {name: grad})."""
    P = trainable(params) if P is None else P
    Es, Fs, Vs, nat = [], [], [], []
    for coord, atype, box in frames:
        geo = _geometry(lib, params, coord, atype, box)
        E, F, V = _energy_force_virial(params, P, geo, atype, create_graph=True)
        Es.append(E)
        Fs.append(F)
        Vs.append(V)
        nat.append(atype.size)
    E = torch.stack(Es)
    F = torch.cat(Fs)
    V = torch.stack(Vs)
    Eh, Fh, Vh = (torch.as_tensor(np.asarray(x, np.float64)) for x in labels)
    inv = 1.0 / torch.tensor(nat, dtype=torch.float64)
    pe, pf, pv = prefs
    loss = (pe * torch.mean((E - Eh.reshape(-1)) ** 2 * inv) +
            pf * torch.sum((Fh.reshape(-1, 3) - F) ** 2) / F.numel() +
            pv * torch.mean(torch.mean((Vh.reshape(-1, 9) - V) ** 2, -1) * inv))
    names = list(P)
    grads = torch.autograd.grad(loss, [P[k] for k in names])
    return (float(loss.detach()), E.detach().numpy(), F.detach().numpy(), V.detach().numpy(),
            {k: g.numpy() for k, g in zip(names, grads)})
