"""Regenerate tests/golden/model_golden.npz: energy/force/virial of the
reference's own PyTorch se_e2_a model on seeded synthetic water frames.

The frames and weights come from the product's seeded generators
(workload.water_frame, model.init_params), the statistics from the oracle;
the reference model (deepmd.pt.model.model.get_model, imported from the
reference tree through ref_import_shim) is loaded with those weights and run
in FP64 on the CPU. Stored: the frame, the statistics, a weight checksum and
the reference E/F/V, plus the FP64 oracle's compressed-model E/F/V.

    python tests/golden/make_model_golden.py [REFERENCE_TREE]  (or DEEPMD_REFERENCE_TREE in the environment)
"""

from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _ref_tree() -> str:
    """The reference source tree: the first argument, else the environment
    variable DEEPMD_REFERENCE_TREE (checked when a fixture is made)."""
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DEEPMD_REFERENCE_TREE", "")
    if not tree or not os.path.isdir(tree):
        raise SystemExit("give the reference source tree as the first argument or in "
                         "DEEPMD_REFERENCE_TREE")
    return tree


OUT = os.path.join(HERE, "model_golden.npz")
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)


def weight_checksum(params) -> float:
    s = 0.0
    for net in params.emb:
        for W, b in net:
            s += float(np.sum(W)) + float(np.sum(b))
    for f in params.fit:
        for W, b, d in f["layers"]:
            s += float(np.sum(W)) + float(np.sum(b)) + (0.0 if d is None else float(np.sum(d)))
        s += float(np.sum(f["out"][0])) + float(np.sum(f["out"][1]))
    return s


def reference_model(params):
    import ref_import_shim

    ref_import_shim.install(_ref_tree())
    from deepmd.pt.model.model import get_model

    cfg = params.cfg
    spec = {
        "type_map": ["O", "H"],
        "descriptor": {"type": "se_e2_a", "sel": list(cfg.sel), "rcut_smth": cfg.rcut_smth,
                       "rcut": cfg.rcut, "neuron": list(cfg.neuron), "resnet_dt": False,
                       "axis_neuron": cfg.axis_neuron, "type_one_side": True,
                       "precision": "float64", "seed": 1, "activation_function": "tanh",
                       "exclude_types": [], "env_protection": 0.0, "set_davg_zero": False,
                       "trainable": True},
        "fitting_net": {"neuron": list(cfg.fitting), "resnet_dt": True, "seed": 1,
                        "precision": "float64", "activation_function": "tanh"},
    }
    m = get_model(spec)
    sd = m.state_dict()
    pre = "atomic_model.descriptor.sea."
    sd[pre + "mean"] = torch.tensor(params.davg.reshape(cfg.ntypes, cfg.nnei, 4))
    sd[pre + "stddev"] = torch.tensor(params.dstd.reshape(cfg.ntypes, cfg.nnei, 4))
    for coll in ("networks", "_networks"):
        for t, net in enumerate(params.emb):
            for l, (W, b) in enumerate(net):
                sd[f"{pre}filter_layers.{coll}.{t}.layers.{l}.matrix"] = torch.tensor(W)
                sd[f"{pre}filter_layers.{coll}.{t}.layers.{l}.bias"] = torch.tensor(b)
        fp = "atomic_model.fitting_net.filter_layers."
        for t, f in enumerate(params.fit):
            for l, (W, b, d) in enumerate(f["layers"]):
                sd[f"{fp}{coll}.{t}.layers.{l}.matrix"] = torch.tensor(W)
                sd[f"{fp}{coll}.{t}.layers.{l}.bias"] = torch.tensor(b)
                if d is not None:
                    sd[f"{fp}{coll}.{t}.layers.{l}.idt"] = torch.tensor(d)
            Wo, bo = f["out"]
            L = len(f["layers"])
            sd[f"{fp}{coll}.{t}.layers.{L}.matrix"] = torch.tensor(Wo)
            sd[f"{fp}{coll}.{t}.layers.{L}.bias"] = torch.tensor(bo)
    m.load_state_dict(sd)
    return m.eval()


def main() -> None:
    import __graft_entry__
    from oracle import model_ref, oracle

    pkg = __graft_entry__.load_package()
    import importlib

    mdl = importlib.import_module("deepmd_kit_lr_pt_b200.model")
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    tab = importlib.import_module("deepmd_kit_lr_pt_b200.table")
    del pkg
    lib = oracle.ref() or oracle.port()
    out = {}
    cases = {"w192": (4, 0), "w24": (2, 5)}
    cfg = mdl.SeAConfig()
    params = mdl.init_params(cfg, seed=1)
    out["weight_checksum"] = np.array(weight_checksum(params))
    out["param_seed"] = np.array(1)
    for name, (n_side, seed) in cases.items():
        coord, atype, box = wl.water_frame(n_side, seed=seed)
        davg, dstd, mind = model_ref.env_stats(lib, cfg, coord, atype, box)
        params.davg, params.dstd = davg, dstd
        params.tables = tab.build_tables(params.emb, davg, dstd, cfg.sel, mind, cfg.rcut_smth,
                                         cfg.rcut)
        m = reference_model(params)
        res = m(torch.tensor(coord).view(1, -1, 3), torch.tensor(atype.astype(np.int64)).view(1, -1),
                box=torch.tensor(box).view(1, 9))
        E = float(res["energy"].detach().reshape(-1)[0])
        F = res["force"].detach().numpy().reshape(-1, 3)
        V = res["virial"].detach().numpy().reshape(9)
        E0, F0, V0 = model_ref.evaluate(lib, params, coord, atype, box, mode="plain")
        Ec, Fc, Vc = model_ref.evaluate(lib, params, coord, atype, box, mode="compressed")
        print(f"{name}: E ref {E:.10f} oracle {E0:.10f} compressed {Ec:.10f}")
        print(f"   |dF| {np.abs(F - F0).max():.3e}  |dV| {np.abs(V - V0).max():.3e}  "
              f"compressed |dF| {np.abs(F - Fc).max():.3e}")
        for k, v in dict(coord=coord, atype=atype, box=box, davg=davg, dstd=dstd,
                         min_nbor_dist=np.array(mind), energy=np.array(E), force=F, virial=V,
                         energy_c=np.array(Ec), force_c=Fc, virial_c=Vc).items():
            out[f"{name}:{k}"] = v
    np.savez_compressed(OUT, **out)


if __name__ == "__main__":
    main()
