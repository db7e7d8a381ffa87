"""Build recipe for the sm_100a kernel library ``libdpb200.so`` (in-tree).

    python deepmd-kit-lr-pt_b200/build.py [--verbose] [--ptxas-info]

Every ``csrc/*.cu`` / ``csrc/*.cc`` file is compiled once per change (object
files are cached next to the sources under ``_build/``) and linked into
``deepmd-kit-lr-pt_b200/lib/libdpb200.so``. nvcc cross-compiles for sm_100a
without a GPU; the library travels with the repository to the GPU host.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import hashlib
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib", "libdpb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                  "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
                  "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _digest(path: str, extra: list[str]) -> str:
    h = hashlib.sha1()
    h.update(" ".join(extra).encode())
    with open(path, "rb") as f:
        h.update(f.read())
    # headers the sources include
    for hdr in sorted(glob.glob(os.path.join(CSRC, "*.cuh")) +
                      glob.glob(os.path.join(CSRC, "*.h")) +
                      glob.glob(os.path.join(ROOT, "include", "*.h")) +
                      glob.glob(os.path.join(ROOT, "include", "*", "*.h"))):
        with open(hdr, "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def _compile(src: str, ptxas_info: bool, verbose: bool) -> str:
    flags = list(NVFLAGS)
    if ptxas_info:
        flags += ["-Xptxas", "-v"]
    name = os.path.basename(src)
    obj = os.path.join(BUILD, f"{name}.{_digest(src, flags)}.o")
    if os.path.exists(obj) and not ptxas_info:
        return obj
    cmd = [NVCC, *flags, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed on {name}")
    if ptxas_info or verbose:
        sys.stderr.write(r.stdout + r.stderr)
    return obj


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile and link the library; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cc")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, ptxas_info, verbose), srcs))
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(LIB + ".tmp", LIB)
    # drop the objects of earlier source versions: the cache holds one object
    # per source file
    keep = set(objs)
    for old in glob.glob(os.path.join(BUILD, "*.o")):
        if old not in keep:
            os.remove(old)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, ptxas_info=a.ptxas_info))
