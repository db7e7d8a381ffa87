"""Regenerate tests/golden/table_golden.npz: the compression tables of the
reference's own compressor for the seeded se_e2_a model.

The model weights come from the product's seeded generator (model.init_params,
seed 1), the statistics and the minimum neighbor distance from the oracle on
the 192-atom water frame (workload.water_frame(4, seed=0)); the reference
model is built and loaded as in make_model_golden.py and its descriptor's
enable_compression (deepmd/pt/model/descriptor/se_a.py:269-314, DPTabulate of
deepmd/utils/tabulate.py) makes the tables. Stored per embedding net: the
table_info, the table shape and every 32nd row (plus the last) of the
[nspline, 6M] FP64 table.

    python tests/golden/make_table_golden.py [REFERENCE_TREE]  (or DEEPMD_REFERENCE_TREE in the environment)
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
OUT = os.path.join(HERE, "table_golden.npz")
ROW_STEP = 32


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
    davg, dstd, mind = model_ref.env_stats(lib, cfg, coord, atype, box)
    params.davg, params.dstd = davg, dstd
    m = mmg.reference_model(params)
    d = m.atomic_model.descriptor
    d.enable_compression(mind)
    out = {"davg": davg, "dstd": dstd, "min_nbor_dist": np.array(mind),
           "weight_checksum": np.array(mmg.weight_checksum(params)),
           "row_step": np.array(ROW_STEP)}
    for t in range(cfg.ntypes):
        table = d.sea.compress_data[t].detach().numpy()
        info = d.sea.compress_info[t].detach().numpy()
        rows = np.unique(np.append(np.arange(0, table.shape[0], ROW_STEP), table.shape[0] - 1))
        out[f"net{t}:info"] = info
        out[f"net{t}:shape"] = np.array(table.shape)
        out[f"net{t}:rows"] = rows
        out[f"net{t}:table_rows"] = table[rows]
        print(f"net {t}: table {table.shape}, info {info}")
    np.savez_compressed(OUT, **out)


if __name__ == "__main__":
    main()
