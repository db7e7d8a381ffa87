"""Regenerate tests/golden/state_dict_golden.npz: the layout of the
reference's compressed se_e2_a model as a state dict.

The reference model is built as in make_model_golden.py (seeded weights of
model.init_params, seed 1; statistics of the 192-atom water frame), its
descriptor is compressed by the reference's own enable_compression, and for
every state-dict entry the name, the shape and two checksums (sum and sum of
absolute values) are stored, with the model's sel and rcut. The reader in
deepmd-kit-lr-pt_b200/checkpoint.py is checked against this layout.

    python tests/golden/make_state_dict_golden.py [REFERENCE_TREE]  (or DEEPMD_REFERENCE_TREE in the environment)
"""

from __future__ import annotations

import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
OUT = os.path.join(HERE, "state_dict_golden.npz")


def main() -> None:
    import __graft_entry__
    import make_model_golden as mmg
    from oracle import model_ref, oracle

    __graft_entry__.load_package()
    mdl = importlib.import_module("deepmd_kit_lr_pt_b200.model")
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    lib = oracle.ref() or oracle.port()
    cfg = mdl.SeAConfig()
    params = mdl.init_params(cfg, seed=1)
    coord, atype, box = wl.water_frame(4, seed=0)
    params.davg, params.dstd, mind = model_ref.env_stats(lib, cfg, coord, atype, box)
    m = mmg.reference_model(params)
    m.atomic_model.descriptor.enable_compression(mind)
    sd = {k: v for k, v in m.state_dict().items() if "atomic_model." in k}
    keys = sorted(sd)
    shapes = [np.array(sd[k].shape, np.int64) for k in keys]
    vals = [sd[k].detach().double().numpy() for k in keys]
    np.savez_compressed(
        OUT, keys=np.array(keys), ndim=np.array([s.size for s in shapes]),
        dims=np.concatenate(shapes) if shapes else np.zeros(0, np.int64),
        sums=np.array([float(v.sum()) for v in vals]),
        abssums=np.array([float(np.abs(v).sum()) for v in vals]),
        sel=np.array(m.get_sel()), rcut=np.array(m.get_rcut()),
        min_nbor_dist=np.array(mind))
    for k, s in zip(keys, shapes):
        print(k, tuple(s))


if __name__ == "__main__":
    main()
