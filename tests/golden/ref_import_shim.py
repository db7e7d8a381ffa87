"""Test-only import shim that makes the reference's Python package importable
in this container for generating golden vectors (never used at test time).

The reference package expects build-generated files and several optional
third-party modules. This shim (1) registers an in-memory ``deepmd.lib``
package whose directory holds a minimal ``run_config.ini``, (2) aliases
``array_api_compat`` to the copy vendored inside scipy, and (3) installs
permissive stub modules for optional dependencies that the se_e2_a model code
path does not use.
"""

from __future__ import annotations

import os
import sys
import tempfile
import types


class _Stub(types.ModuleType):
    def __getattr__(self, name):  # permissive: any attribute is a stub
        if name.startswith("__"):
            raise AttributeError(name)
        return _Stub(f"{self.__name__}.{name}")

    def __call__(self, *a, **k):
        return _Stub(self.__name__ + "()")


def reference_tree(argv_index: int = 1) -> str:
    """The reference source tree: the script's argument, else the
    environment variable DEEPMD_REFERENCE_TREE."""
    tree = sys.argv[argv_index] if len(sys.argv) > argv_index else \
        os.environ.get("DEEPMD_REFERENCE_TREE", "")
    if not tree or not os.path.isdir(tree):
        raise SystemExit("give the reference source tree as the first argument or in "
                         "DEEPMD_REFERENCE_TREE")
    return tree


def install(ref_root: str | None = None) -> None:
    ref_root = ref_root or reference_tree()
    if ref_root not in sys.path:
        sys.path.insert(0, ref_root)
    import torch

    tmp = tempfile.mkdtemp(prefix="dplib_")
    with open(os.path.join(tmp, "run_config.ini"), "w") as f:
        f.write("[CONFIG]\nenable_tensorflow = 0\nenable_pytorch = 1\n"
                f"pt_version = {torch.__version__.split('+')[0]}\npt_cxx11_abi_flag = 1\n"
                "tf_version = 0\ntf_cxx11_abi_flag = 1\nmodel_version = 1.1\n"
                "dp_variant = cpu\n")
    lib = types.ModuleType("deepmd.lib")
    lib.__path__ = [tmp]
    lib.__file__ = os.path.join(tmp, "__init__.py")
    sys.modules["deepmd.lib"] = lib
    import scipy._external.array_api_compat as aac  # noqa: F401
    import importlib

    sys.modules["array_api_compat"] = importlib.import_module("scipy._external.array_api_compat")
    for sub in ("numpy", "common", "torch"):
        try:
            sys.modules[f"array_api_compat.{sub}"] = importlib.import_module(
                f"scipy._external.array_api_compat.{sub}")
        except ImportError:
            pass
    for name in ("h5py", "wcmatch", "dpdata", "lmdb", "msgpack_numpy", "mendeleev",
                 "dargs", "dargs.json_schema"):
        if name not in sys.modules:
            sys.modules[name] = _Stub(name)
    wg = _Stub("wcmatch.glob")
    for k in ("GLOBSTAR", "BRACE", "NEGATE", "EXTGLOB", "DOTGLOB"):
        setattr(wg, k, 0)
    sys.modules["wcmatch.glob"] = wg
    import deepmd  # noqa: F401

    deepmd.lib = lib
