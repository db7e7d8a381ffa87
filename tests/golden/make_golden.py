"""Regenerate tests/golden/ref_fixtures.npz from the reference's own tests.

Reads (as text) the golden vectors that the reference DeePMD-kit unit tests
hold for the se_e2_a path and stores them as numpy arrays, keyed
``<file>:<Class>:<name>``:

* source/lib/tests/test_env_mat_a.cc       (6-atom water fixture, expected_env)
* source/lib/tests/test_prod_force_a.cc    (expected_force)
* source/lib/tests/test_prod_virial_a.cc   (expected_virial, expected_atom_virial)
* source/lib/tests/test_coord.cc           (normalize / copy_coord fixtures)
* source/lib/tests/test_tabulate_se_a.cc   (table, em_x, em, expected outputs)
* source/lib/tests/test_prod_{force,virial}_grad_a.cc (expected_grad_net)
* source/lib/tests/test_fmt_nlist.cc       (expect_nlist_cpy of the formatted lists)
* source/lib/tests/test_neighbor_list.cc   (expect_nlist_cpy rows of build_nlist_cpu,
  stored flattened with their lengths)
* source/lib/tests/test_tabulate_extrapolate.cc (the file-scope table, table
  infos and constants of the extrapolation tests)
* source/tests/pt/test_tabulate_fusion_se_a.py (op goldens, set up in setUp)

Run in a container that holds the reference tree:

    python tests/golden/make_golden.py [REFERENCE_TREE]  (or DEEPMD_REFERENCE_TREE in the environment)

The output is committed; nothing at test time reads the reference tree.
"""

from __future__ import annotations

import ast
import os
import re
import sys

import numpy as np



def _ref_tree() -> str:
    """The reference source tree: the first argument, else the environment
    variable DEEPMD_REFERENCE_TREE (checked when a fixture is made)."""
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DEEPMD_REFERENCE_TREE", "")
    if not tree or not os.path.isdir(tree):
        raise SystemExit("give the reference source tree as the first argument or in "
                         "DEEPMD_REFERENCE_TREE")
    return tree


OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_fixtures.npz")

CC_FILES = [
    "source/lib/tests/test_env_mat_a.cc",
    "source/lib/tests/test_prod_force_a.cc",
    "source/lib/tests/test_prod_virial_a.cc",
    "source/lib/tests/test_coord.cc",
    "source/lib/tests/test_tabulate_se_a.cc",
    "source/lib/tests/test_prod_force_grad_a.cc",
    "source/lib/tests/test_prod_virial_grad_a.cc",
    "source/lib/tests/test_fmt_nlist.cc",
    "source/lib/tests/test_neighbor_list.cc",
]
NS_FILES = ["source/lib/tests/test_tabulate_extrapolate.cc"]
PY_FILE = "source/tests/pt/test_tabulate_fusion_se_a.py"

VEC_RE = re.compile(
    r"std::vector<(double|int)>\s+(\w+)\s*=\s*\{([^}]*)\};", re.S)
CLASS_RE = re.compile(r"^class\s+(\w+)", re.M)
NESTED_RE = re.compile(
    r"std::vector<std::vector<int>>\s+(\w+)\s*=\s*\{(.*?)\};", re.S)
ROW_RE = re.compile(r"std::vector<int>\(\{([^}]*)\}\)")
NS_VEC_RE = re.compile(r"const\s+std::vector<double>\s+(k\w+)\s*=\s*\{([^}]*)\};", re.S)
NS_SCALAR_RE = re.compile(r"constexpr\s+(double|int)\s+(k\w+)\s*=\s*(-?[\w.+-]+)\s*;")
SCALAR_RE = re.compile(r"^\s*(?:const\s+)?(double|int)\s+(\w+)\s*=\s*([-+0-9.eE]+)\s*;",
                       re.M)


def parse_cc(path: str, tag: str, out: dict) -> None:
    text = open(path).read()
    starts = [(m.start(), m.group(1)) for m in CLASS_RE.finditer(text)]
    starts.append((len(text), None))
    for (s, cls), (e, _) in zip(starts[:-1], starts[1:]):
        body = text[s:e]
        # stop at the first TEST_F so only the fixture members are read
        cut = body.find("TEST_F(")
        fixture = body if cut < 0 else body[:cut]
        for m in VEC_RE.finditer(fixture):
            kind, name, vals = m.groups()
            nums = [v.strip() for v in vals.replace("\n", " ").split(",") if v.strip()]
            dt = np.float64 if kind == "double" else np.int32
            try:
                vals_f = [float(v) for v in nums]
            except ValueError:  # an expression (e.g. 1 << 24): not a golden vector
                continue
            out[f"{tag}:{cls}:{name}"] = np.array(vals_f).astype(dt)
        for m in SCALAR_RE.finditer(fixture):
            kind, name, val = m.groups()
            out[f"{tag}:{cls}:{name}"] = np.array(float(val))
        # the tabulate fixture declares its sizes after the vectors
        for m in re.finditer(r"const int (\w+) = (\d+);", fixture):
            out[f"{tag}:{cls}:{m.group(1)}"] = np.array(int(m.group(2)))
        # rows of unequal length: flattened values and the row lengths
        for m in NESTED_RE.finditer(fixture):
            rows = [[int(v) for v in r.replace("\n", " ").split(",") if v.strip()]
                    for r in ROW_RE.findall(m.group(2))]
            out[f"{tag}:{cls}:{m.group(1)}"] = np.array([v for r in rows for v in r], np.int32)
            out[f"{tag}:{cls}:{m.group(1)}_len"] = np.array([len(r) for r in rows], np.int32)


def parse_ns(path: str, tag: str, out: dict) -> None:
    """File-scope constants (constexpr scalars and const vectors named k...,
    whose entries may name those scalars) of a test file without fixture
    classes."""
    text = open(path).read()
    scal: dict[str, float] = {}
    for kind, name, val in NS_SCALAR_RE.findall(text):
        v = scal[val.lstrip("-")] * (-1 if val.startswith("-") else 1) if val.lstrip(
            "-") in scal else float(val)
        scal[name] = v
        out[f"{tag}:{name}"] = np.array(int(v) if kind == "int" else v)
    for name, vals in NS_VEC_RE.findall(text):
        nums = []
        try:
            for v in vals.replace("//", " ").replace("\n", " ").split(","):
                v = v.strip()
                if v:
                    nums.append(scal[v] if v in scal else float(v))
        except ValueError:  # a function-local vector of variables, not a constant
            continue
        out[f"{tag}:{name}"] = np.array(nums, np.float64)


def parse_py(path: str, tag: str, out: dict) -> None:
    tree = ast.parse(open(path).read())
    for node in ast.walk(tree):
        if not (isinstance(node, ast.FunctionDef) and node.name == "setUp"):
            continue
        for st in node.body:
            if not isinstance(st, ast.Assign) or len(st.targets) != 1:
                continue
            tgt = st.targets[0]
            if not (isinstance(tgt, ast.Attribute) and isinstance(tgt.value, ast.Name)):
                continue
            name = tgt.attr
            call = st.value
            shape = None
            # torch.tensor([...], ...).reshape(a, b, ...)
            if (isinstance(call, ast.Call) and isinstance(call.func, ast.Attribute)
                    and call.func.attr == "reshape"):
                shape = tuple(ast.literal_eval(a) for a in call.args)
                call = call.func.value
            if (isinstance(call, ast.Call) and isinstance(call.func, ast.Attribute)
                    and call.func.attr == "tensor" and call.args):
                try:
                    vals = ast.literal_eval(call.args[0])
                except ValueError:
                    continue
                arr = np.array(vals, dtype=np.float64)
                if shape is not None:
                    arr = arr.reshape(shape)
                out[f"{tag}:{name}"] = arr
            elif isinstance(call, ast.Constant) and isinstance(call.value, (int, float)):
                out[f"{tag}:{name}"] = np.array(call.value)


def main() -> None:
    out: dict[str, np.ndarray] = {}
    for rel in CC_FILES:
        parse_cc(os.path.join(_ref_tree(), rel), os.path.basename(rel), out)
    for rel in NS_FILES:
        parse_ns(os.path.join(_ref_tree(), rel), os.path.basename(rel), out)
    parse_py(os.path.join(_ref_tree(), PY_FILE), os.path.basename(PY_FILE), out)
    np.savez_compressed(OUT, **out)
    for k in sorted(out):
        print(f"{k:70s} {out[k].shape}")


if __name__ == "__main__":
    main()
