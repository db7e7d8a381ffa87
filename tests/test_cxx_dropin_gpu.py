"""The deepmd:: C++ drop-ins run through the reference's own headers.

tests/cxx/dropin_harness (built against source/lib/include of the reference
and linked with libdpb200.so and the reference CPU library) runs
normalize_coord_gpu -> copy_coord_gpu -> build_nlist_gpu ->
prod_env_mat_a_gpu -> tabulate_fusion_se_a_gpu -> prod_force_a_gpu /
prod_virial_a_gpu, plus convert_nlist_gpu_device / free_nlist_gpu_device and
use_nlist_map, on a 192-atom water frame and compares each result with the
reference CPU function on the same inputs (as source/lib/tests/
test_env_mat_a.cc:960-1029 does). Bars: ghost arrays and neighbor lists
bit-exact; FP64 within 1e-10, FP32 within 1e-5 of the value scale.
"""

import json
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "tests", "cxx", "_build", "dropin_harness")


def _write_input(path):
    import importlib.util

    from oracle import model_ref, oracle, table_ref

    import sys

    name = "dpb_workload_standalone"
    wl = sys.modules.get(name)
    if wl is None:
        spec = importlib.util.spec_from_file_location(
            name, os.path.join(ROOT, "deepmd-kit-lr-pt_b200", "workload.py"))
        wl = importlib.util.module_from_spec(spec)
        sys.modules[name] = wl
        spec.loader.exec_module(wl)
    cfg = wl.SeAConfig()
    coord, atype, box = wl.water_frame(4, seed=31)
    coord = coord + 0.5 * box[0]  # outside the box: normalize_coord has work to do
    params = wl.init_params(cfg, seed=1)
    lib = oracle.ref() or oracle.port()
    davg, dstd, mind = model_ref.env_stats(lib, cfg, coord % box[0], atype, box)
    (table, info), _ = table_ref.build_tables(params.emb, davg, dstd, cfg.sel, mind,
                                              cfg.rcut_smth, cfg.rcut)
    M = cfg.neuron[-1]
    with open(path, "wb") as f:
        np.array([atype.size, cfg.ntypes, M, table.shape[0]], np.int32).tofile(f)
        np.array([cfg.rcut, cfg.rcut_smth], np.float32).tofile(f)
        cfg.sec.astype(np.int32).tofile(f)
        np.asarray(box, np.float64).tofile(f)
        np.asarray(coord, np.float64).reshape(-1).tofile(f)
        atype.astype(np.int32).tofile(f)
        davg.astype(np.float64).tofile(f)
        dstd.astype(np.float64).tofile(f)
        info.astype(np.float64).tofile(f)
        table.astype(np.float64).reshape(-1).tofile(f)


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    if not os.path.exists(HARNESS):
        pytest.skip("the C++ harness was not built (it needs the reference headers at build time)")
    path = str(tmp_path_factory.mktemp("cxx") / "in.bin")
    _write_input(path)
    out = subprocess.run([HARNESS, path], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    return {ln["precision"]: ln for ln in lines}


@pytest.mark.parametrize("precision", ["double", "float"])
def test_cxx_dropins_match_reference_cpu(results, precision):
    r = results[precision]
    print(json.dumps(r))
    tol = 1e-10 if precision == "double" else 1e-5
    assert r["build_ret"] == 0 and r["max_list"][0] == r["max_list"][1]
    assert r["nlist_equal"] and r["converted_equal"] and r["map_equal"]
    assert r["capacity_thrown"]
    if precision == "double":
        assert r["ghost_equal"] and r["normalize_err"] == 0.0
    assert r["normalize_err"] <= tol * 20.0  # coordinates up to ~19 A
    for k in ("em_err", "em_deriv_err", "rij_err", "tabulate_err"):
        assert r[k] <= tol * (1.0 if precision == "double" else 10.0), (k, r[k])
    assert r["force_err"] <= tol * max(1.0, r["force_scale"])
    assert r["virial_err"] <= tol * max(1.0, r["virial_scale"])
    assert r["atom_virial_err"] <= tol * max(1.0, r["virial_scale"])
