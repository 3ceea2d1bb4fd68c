"""Ahead-of-time build of the CUDA library (sm_100a) that the package loads.

Compiles csrc/*.cu with nvcc into sbg/libsbg_geneig.so, in-tree, so the built
library travels with the source tree.  Rebuilds only when a source or header is
newer than the library.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
INCLUDE = os.path.join(REPO, "include")
LIB = os.path.join(PKG_DIR, "sbg", "libsbg_geneig.so")
BUILD_DIR = os.path.join(PKG_DIR, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "sbg", "*.h")) + [__file__]
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, obj: str, verbose: bool) -> None:
    flags = [f for f in NVCC_FLAGS if f != "-shared"]
    cmd = [nvcc(), *flags, f"-I{INCLUDE}", f"-I{CSRC}", "-c", src, "-o", obj + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(obj + ".tmp", obj)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles each source to an object in _build/ (in parallel), then links the library."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = [os.path.join(BUILD_DIR, os.path.basename(s)[:-3] + ".o") for s in sources()]
    workers = max(1, min(len(objs), os.cpu_count() or 1))
    with ThreadPoolExecutor(workers) as ex:
        for f in [ex.submit(_compile, s, o, verbose) for s, o in zip(sources(), objs)]:
            f.result()
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
