"""Reading (and writing) the reference's serialized se_e2_a energy model.

The reference stores a model as a PyTorch state dict: a training checkpoint
({"model": state_dict, ...}, deepmd/pt/train/training.py:1934-1960, keys
prefixed by the wrapper, e.g. "model.Default."), or a frozen / compressed
TorchScript file whose module has the same state dict
(deepmd/pt/entrypoints/compress.py:69-110). The entries this path reads are
the se_a descriptor's and the energy fitting's
(deepmd/pt/model/descriptor/se_a.py:537-576, task/fitting.py):

  atomic_model.descriptor.sea.mean / stddev           [ntypes, nnei, 4]
  atomic_model.descriptor.sea.filter_layers.networks.{t}.layers.{l}.matrix / bias
  atomic_model.descriptor.sea.compress_data.{t}       [nspline, 6 M] (compressed)
  atomic_model.descriptor.sea.compress_info.{t}       [6]            (compressed)
  atomic_model.fitting_net.filter_layers.networks.{t}.layers.{l}.matrix / bias / idt
  atomic_model.out_bias                               [1, ntypes, 1] (optional)

``params_from_state_dict`` turns them into SeAParams, the compression tables
included when the model was compressed (so the compressed path can run a
reference model without rebuilding its tables); ``params_to_state_dict``
writes the same entries back.
"""

from __future__ import annotations

import re

import numpy as np

from .workload import SeAConfig, SeAParams

DESC = "atomic_model.descriptor.sea."
FIT = "atomic_model.fitting_net.filter_layers."


def _np(x) -> np.ndarray:
    if hasattr(x, "detach"):
        x = x.detach().cpu().numpy()
    return np.asarray(x, np.float64)


def _strip(state: dict) -> dict:
    """Keys from "atomic_model." on (drops the wrapper / task prefixes)."""
    out = {}
    for k, v in state.items():
        i = k.find("atomic_model.")
        if i >= 0:
            out[k[i:]] = v
    return out


def load(path_or_state, sel=None, rcut: float | None = None,
         rcut_smth: float | None = None, trusted: bool = False) -> SeAParams:
    """SeAParams of a reference model: a state dict, a training checkpoint
    ({"model": state dict}) or the path of a checkpoint / TorchScript file.
    sel, rcut and rcut_smth are not part of the state dict (they are in the
    model's input script): a TorchScript model reports sel and rcut itself
    (get_sel / get_rcut of the reference model); otherwise give them (rcut
    and rcut_smth default to the reference's se_e2_a input defaults, 6.0 and
    0.5). A checkpoint file is read with torch.load(weights_only=True):
    tensors and plain containers only, which is all a reference checkpoint
    holds; trusted=True unpickles arbitrary objects, for files of a trusted
    origin only."""
    state = path_or_state
    if isinstance(state, str):
        import torch

        try:
            mod = torch.jit.load(state, map_location="cpu")
            sel = sel if sel is not None else tuple(int(x) for x in mod.get_sel())
            rcut = rcut if rcut is not None else float(mod.get_rcut())
            state = mod.state_dict()
        except RuntimeError:
            state = torch.load(state, map_location="cpu", weights_only=not trusted)
    if isinstance(state, dict) and "model" in state and isinstance(state["model"], dict):
        state = state["model"]
    return params_from_state_dict(state, sel=sel, rcut=6.0 if rcut is None else rcut,
                                  rcut_smth=0.5 if rcut_smth is None else rcut_smth)


def params_from_state_dict(state: dict, sel, rcut: float = 6.0,
                           rcut_smth: float = 0.5) -> SeAParams:
    """SeAParams from the state dict entries; sel [ntypes] must add up to
    the statistics' slot count."""
    sd = _strip(state)
    if DESC + "mean" not in sd:
        raise ValueError("not an se_e2_a model: no descriptor.sea.mean in the state dict")
    mean, std = _np(sd[DESC + "mean"]), _np(sd[DESC + "stddev"])
    ntypes, nnei = mean.shape[0], mean.shape[1]
    coll = "networks" if any(k.startswith(DESC + "filter_layers.networks.") for k in sd) \
        else "_networks"

    def layers(prefix):
        out = {}
        pat = re.compile(re.escape(prefix) + r"(\d+)\.layers\.(\d+)\.(matrix|bias|idt)$")
        for k, v in sd.items():
            m = pat.match(k)
            if m:
                out.setdefault(int(m.group(1)), {}).setdefault(int(m.group(2)), {})[m.group(3)] = \
                    _np(v)
        return out

    emb_l = layers(f"{DESC}filter_layers.{coll}.")
    fit_l = layers(f"{FIT}{coll}.")
    if sorted(emb_l) != list(range(ntypes)):
        raise ValueError("type_one_side se_e2_a expected: one embedding net per neighbor type")
    emb = []
    for t in range(ntypes):
        net = emb_l[t]
        emb.append([(net[l]["matrix"], net[l]["bias"]) for l in sorted(net)])
    neuron = tuple(int(W.shape[1]) for W, _ in emb[0])
    fit = []
    for t in range(ntypes):
        net = fit_l[t]
        ls = sorted(net)
        hidden = [(net[l]["matrix"], net[l]["bias"], net[l].get("idt")) for l in ls[:-1]]
        Wo, bo = net[ls[-1]]["matrix"], net[ls[-1]]["bias"]
        fit.append({"layers": hidden, "out": (Wo.reshape(-1, 1), bo.reshape(1))})
    fitting = tuple(int(W.shape[1]) for W, _, _ in fit[0]["layers"])
    axis = int(fit[0]["layers"][0][0].shape[0]) // neuron[-1]
    if sel is None or len(sel) != ntypes or int(sum(sel)) != nnei:
        raise ValueError(f"sel {sel} must give {ntypes} section lengths adding up to {nnei} "
                         "(the slots of the stored statistics)")
    cfg = SeAConfig(rcut=rcut, rcut_smth=rcut_smth, sel=tuple(int(x) for x in sel),
                    neuron=neuron, axis_neuron=axis, fitting=fitting)
    bias = np.zeros(ntypes)
    if "atomic_model.out_bias" in sd:
        bias = _np(sd["atomic_model.out_bias"]).reshape(-1)[:ntypes].copy()
    p = SeAParams(cfg=cfg, emb=emb, fit=fit, bias_atom_e=bias,
                  davg=mean.reshape(ntypes, -1), dstd=std.reshape(ntypes, -1))
    tabs = []
    for t in range(ntypes):
        d = sd.get(f"{DESC}compress_data.{t}")
        i = sd.get(f"{DESC}compress_info.{t}")
        if d is None or i is None or _np(d).size == 0:
            tabs = []
            break
        tabs.append((_np(d), _np(i)))
    p.tables = tabs
    return p


def params_to_state_dict(params: SeAParams) -> dict:
    """The entries above (torch FP64 tensors) for SeAParams."""
    import torch

    cfg = params.cfg
    t64 = lambda a: torch.tensor(np.asarray(a, np.float64))  # noqa: E731
    sd = {DESC + "mean": t64(np.asarray(params.davg).reshape(cfg.ntypes, cfg.nnei, 4)),
          DESC + "stddev": t64(np.asarray(params.dstd).reshape(cfg.ntypes, cfg.nnei, 4))}
    for t, net in enumerate(params.emb):
        for l, (W, b) in enumerate(net):
            sd[f"{DESC}filter_layers.networks.{t}.layers.{l}.matrix"] = t64(W)
            sd[f"{DESC}filter_layers.networks.{t}.layers.{l}.bias"] = t64(b)
    for t, f in enumerate(params.fit):
        for l, (W, b, d) in enumerate(f["layers"]):
            sd[f"{FIT}networks.{t}.layers.{l}.matrix"] = t64(W)
            sd[f"{FIT}networks.{t}.layers.{l}.bias"] = t64(b)
            if d is not None:
                sd[f"{FIT}networks.{t}.layers.{l}.idt"] = t64(d)
        L = len(f["layers"])
        sd[f"{FIT}networks.{t}.layers.{L}.matrix"] = t64(np.asarray(f["out"][0]).reshape(-1, 1))
        sd[f"{FIT}networks.{t}.layers.{L}.bias"] = t64(np.asarray(f["out"][1]).reshape(1))
    for t, (tab, info) in enumerate(params.tables):
        sd[f"{DESC}compress_data.{t}"] = t64(tab)
        sd[f"{DESC}compress_info.{t}"] = t64(info)
    sd["atomic_model.out_bias"] = t64(np.asarray(params.bias_atom_e).reshape(1, -1, 1))
    return sd
