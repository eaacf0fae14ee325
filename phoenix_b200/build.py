"""Build the sm_100a shared library phoenix_b200/libphx.so with nvcc.

The library is built in-tree (not installed) so that it ships with the
repository to the GPU host.  ``python -m phoenix_b200.build`` rebuilds it;
``build(force=False)`` skips the compile when the library is newer than
every source.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libphx.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-DPHX_NVCC_VERSION=\"12.9\""]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + \
        sorted(glob.glob(os.path.join(CSRC, "*.hpp"))) + [os.path.join(ROOT, "include", "phx.h")]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


UNITS = ["phx_runtime.cu", "phx_noalloc.cu", "phx_batch.cu"]
OBJ_DIR = os.path.join(PKG, "_build")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + proc.stdout[-8000:] + proc.stderr[-8000:])
    return proc


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every translation unit (in parallel) and link libphx.so."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(OBJ_DIR, exist_ok=True)
    extra = ["-Xptxas=-v"] if ptxas_info else []
    objs = [os.path.join(OBJ_DIR, u.replace(".cu", ".o")) for u in UNITS]
    cmds = [[NVCC] + extra + ARCH_FLAGS + CFLAGS + ["-c", "-o", o, os.path.join(CSRC, u)] for u, o in zip(UNITS, objs)]
    with ThreadPoolExecutor(len(cmds)) as ex:
        procs = list(ex.map(lambda c: _run(c, verbose), cmds))
    if ptxas_info or verbose:
        for p in procs:
            sys.stderr.write(p.stderr)
    _run([NVCC] + ARCH_FLAGS + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcufft"], verbose)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
