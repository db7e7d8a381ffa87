"""Regenerate tests/golden/train_golden.npz: the training loss of the
reference's own PyTorch se_e2_a model and its gradient w.r.t. every weight.

Two seeded 192-atom water frames (workload.water_frame), seeded weights
(model.init_params) and statistics from the oracle; labels are the oracle's
FP64 E/F/V plus seeded noise. The reference model (deepmd.pt.model.model.
get_model, in train mode so the force keeps its graph) and the reference
loss (deepmd.pt.loss.EnergyStdLoss with prefactors e 0.02, f 1000, v 0.02)
run in FP64 on the CPU; loss.backward() gives the reference's autograd
gradient. Stored per weight tensor: its full gradient when it has at most
4096 entries, else its row sums, column sums, Frobenius norm and 16
projections on seeded Gaussian directions (numpy default_rng(1000 + k) for
the k-th tensor in name order).

    python tests/golden/make_train_golden.py [REFERENCE_TREE]  (or DEEPMD_REFERENCE_TREE in the environment)
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


OUT = os.path.join(HERE, "train_golden.npz")
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

PREFS = (0.02, 1000.0, 0.02)
SEEDS = (0, 1)
FULL_MAX = 4096
NPROJ = 16


def summarize(name_order, grads):
    """{key: array} summary of a {name: gradient} dict (see module doc)."""
    out = {}
    for k, name in enumerate(name_order):
        g = np.asarray(grads[name], np.float64)
        if g.size <= FULL_MAX:
            out[f"full:{name}"] = g
        else:
            g2 = g.reshape(g.shape[0], -1)
            rng = np.random.default_rng(1000 + k)
            V = rng.standard_normal((NPROJ, g.size))
            out[f"rows:{name}"] = g2.sum(1)
            out[f"cols:{name}"] = g2.sum(0)
            out[f"norm:{name}"] = np.array(np.linalg.norm(g))
            out[f"proj:{name}"] = V @ g.reshape(-1)
    return out


def main() -> None:
    import __graft_entry__
    import make_model_golden
    from oracle import model_ref, oracle

    pkg = __graft_entry__.load_package()
    import importlib

    mdl = importlib.import_module("deepmd_kit_lr_pt_b200.model")
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    del pkg
    lib = oracle.ref() or oracle.port()
    cfg = mdl.SeAConfig()
    params = mdl.init_params(cfg, seed=3)
    frames = [wl.water_frame(4, seed=s) for s in SEEDS]
    davg, dstd, _ = model_ref.env_stats(lib, cfg, *frames[0])
    params.davg, params.dstd = davg, dstd
    # labels: oracle E/F/V + seeded noise
    rng = np.random.default_rng(7)
    E0, F0, V0 = [], [], []
    for c, a, b in frames:
        e, f, v = model_ref.evaluate(lib, params, c, a, b, mode="plain")
        E0.append(e)
        F0.append(f)
        V0.append(v)
    Eh = np.array(E0) + rng.normal(0.0, 2.0, len(frames))
    Fh = np.concatenate(F0) + rng.normal(0.0, 0.5, (sum(a.size for _, a, _ in frames), 3))
    Vh = np.array(V0) + rng.normal(0.0, 5.0, (len(frames), 9))

    # reference model + reference loss
    m = make_model_golden.reference_model(params)
    from deepmd.pt.loss import EnergyStdLoss

    m.train()
    loss_fn = EnergyStdLoss(starter_learning_rate=1.0, start_pref_e=PREFS[0],
                            limit_pref_e=PREFS[0], start_pref_f=PREFS[1], limit_pref_f=PREFS[1],
                            start_pref_v=PREFS[2], limit_pref_v=PREFS[2])
    nloc = frames[0][1].size
    nf = len(frames)
    inp = {"coord": torch.tensor(np.stack([c.reshape(-1, 3) for c, _, _ in frames])),
           "atype": torch.tensor(np.stack([a for _, a, _ in frames]).astype(np.int64)),
           "box": torch.tensor(np.stack([b.reshape(9) for _, _, b in frames]))}
    label = {"energy": torch.tensor(Eh).view(nf, 1), "force": torch.tensor(Fh).view(nf, nloc, 3),
             "virial": torch.tensor(Vh).view(nf, 9), "find_energy": 1.0, "find_force": 1.0,
             "find_virial": 1.0}
    m.zero_grad()
    pred, loss, more = loss_fn(inp, m, label, nloc, 1.0)
    loss.backward()
    ref_grads = {}
    for name, p in m.named_parameters():
        if p.grad is None:
            continue
        key = name.replace("._networks.", ".networks.")
        ref_grads[key] = p.grad.detach().numpy().copy()
    # the oracle's restatement of the same gradient, for the record
    oloss, oE, oF, oV, ograds = model_ref.train_loss_grads(lib, params, frames, (Eh, Fh, Vh),
                                                          PREFS)
    names = list(ograds)
    missing = sorted(set(names) - set(ref_grads))
    extra = sorted(set(ref_grads) - set(names))
    print("reference loss", float(loss), "oracle", oloss)
    print("names missing in the reference:", missing, "extra:", extra)
    worst = max(np.abs(ograds[n] - ref_grads[n]).max() / (np.abs(ref_grads[n]).max() + 1e-300)
                for n in names)
    print(f"oracle vs reference autograd: max relative gradient difference {worst:.3e}")
    print("E", pred["energy"].detach().numpy().reshape(-1), oE)
    out = {"names": np.array(names), "param_seed": np.array(3), "seeds": np.array(SEEDS),
           "prefs": np.array(PREFS), "davg": davg, "dstd": dstd,
           "label_energy": Eh, "label_force": Fh, "label_virial": Vh,
           "loss": np.array(float(loss)), "energy": pred["energy"].detach().numpy().reshape(-1),
           "force": pred["force"].detach().numpy().reshape(-1, 3),
           "virial": pred["virial"].detach().numpy().reshape(-1, 9)}
    out.update(summarize(names, ref_grads))
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
