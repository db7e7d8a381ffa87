"""Regenerate tests/golden/ref_abi_symbols.txt: the mangled names of the
reference's deepmd:: GPU functions on the se_e2_a path, as the reference's own
headers declare them (source/lib/include, compiled with GOOGLE_CUDA=1).

A translation unit that takes the address of every float/double
instantiation is compiled against the reference headers; its undefined
symbols are the names a binary linked against the reference expects.

    python tests/golden/make_abi_golden.py [REFERENCE_TREE]  (or DEEPMD_REFERENCE_TREE in the environment)
"""

import os
import subprocess
import sys
import tempfile



def _ref_tree() -> str:
    """The reference source tree: the first argument, else the environment
    variable DEEPMD_REFERENCE_TREE (checked when a fixture is made)."""
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DEEPMD_REFERENCE_TREE", "")
    if not tree or not os.path.isdir(tree):
        raise SystemExit("give the reference source tree as the first argument or in "
                         "DEEPMD_REFERENCE_TREE")
    return tree


OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_abi_symbols.txt")

FUNCS = ["build_nlist_gpu", "prod_env_mat_a_gpu", "tabulate_fusion_se_a_gpu",
         "tabulate_fusion_se_a_grad_gpu", "tabulate_fusion_se_a_grad_grad_gpu",
         "prod_force_a_gpu", "prod_virial_a_gpu", "prod_force_grad_a_gpu",
         "prod_virial_grad_a_gpu", "normalize_coord_gpu", "copy_coord_gpu"]
PLAIN = ["convert_nlist_gpu_device", "free_nlist_gpu_device", "use_nlist_map"]

SRC = """#include "coord.h"
#include "neighbor_list.h"
#include "prod_env_mat.h"
#include "tabulate.h"
#include "prod_force.h"
#include "prod_virial.h"
#include "prod_force_grad.h"
#include "prod_virial_grad.h"
#include <vector>
""" + "".join(
    f"void* p_{f}_{t} = (void*)static_cast<decltype(&deepmd::{f}<{t}>)>(&deepmd::{f}<{t}>);\n"
    for f in FUNCS if f != "prod_env_mat_a_gpu" for t in ("float", "double")) + "".join(
    # prod_env_mat_a_gpu is overloaded (prod_env_mat.h:97-139): select the
    # nframes form by its full type
    f"void (*p_env_{t})({t}*, {t}*, {t}*, int*, const {t}*, const int*, "
    f"const deepmd::InputNlist&, int*, unsigned long long*, const int, const {t}*, "
    f"const {t}*, const int, const int, const int, const float, const float, "
    f"const std::vector<int>, const int*) = &deepmd::prod_env_mat_a_gpu<{t}>;\n"
    for t in ("float", "double")) + "".join(
    f"void* p_{f} = (void*)&deepmd::{f};\n" for f in PLAIN)


def main():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "abi.cc")
        obj = os.path.join(d, "abi.o")
        open(src, "w").write(SRC)
        subprocess.run(["g++", "-std=c++17", "-DGOOGLE_CUDA=1", "-c", src, "-o", obj,
                        "-I" + os.path.join(_ref_tree(), "source", "lib", "include"),
                        "-I/usr/local/cuda/include"], check=True)
        out = subprocess.run(["nm", "-u", obj], capture_output=True, text=True, check=True).stdout
    syms = sorted({ln.split()[-1] for ln in out.splitlines() if "6deepmd" in ln})
    open(OUT, "w").write("\n".join(syms) + "\n")
    print("\n".join(syms))


if __name__ == "__main__":
    main()
