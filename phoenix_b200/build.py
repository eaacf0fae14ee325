"""Build the sm_100a shared library phoenix_b200/libphx.so with nvcc, and the
command line phoenix_b200/bin/phoenix_b200 with its file-format library
phoenix_b200/libphx_io.so (host C++).

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


# The command line (host C++ over the C ABI) and its file-format library
CLI_DIR = os.path.join(PKG, "cli")
IO_LIB = os.path.join(PKG, "libphx_io.so")
CLI_BIN = os.path.join(PKG, "bin", "phoenix_b200")
CXX = os.environ.get("CXX_HOST", "g++")
# no -march: no FMA contraction, so host envelope arithmetic rounds as the
# reference's build does
HOST_FLAGS = ["-O2", "-std=c++20", "-ffp-contract=off", "-fno-fast-math", "-Wall"]


def _host_sources():
    return sorted(glob.glob(os.path.join(CLI_DIR, "*.hpp")) + glob.glob(os.path.join(CLI_DIR, "*.cpp"))) + \
        [os.path.join(ROOT, "include", "phx.h")]


def build_host(force: bool = False, verbose: bool = False) -> None:
    """Compile libphx_io.so and the command line bin/phoenix_b200 (links libphx.so)."""
    def stale(target):
        return force or not os.path.exists(target) or \
            any(os.path.getmtime(s) > os.path.getmtime(target) for s in _host_sources())

    if stale(IO_LIB):
        _run([CXX] + HOST_FLAGS + ["-fPIC", "-shared", "-fvisibility=hidden", "-o", IO_LIB + ".tmp",
                                   os.path.join(CLI_DIR, "phx_io_capi.cpp")], verbose)
        os.replace(IO_LIB + ".tmp", IO_LIB)
    if stale(CLI_BIN) or os.path.getmtime(LIB) > os.path.getmtime(CLI_BIN):
        os.makedirs(os.path.dirname(CLI_BIN), exist_ok=True)
        _run([CXX] + HOST_FLAGS + ["-o", CLI_BIN + ".tmp", os.path.join(CLI_DIR, "phx_cli.cpp"), "-L" + PKG, "-lphx",
                                   "-Wl,-rpath,$ORIGIN/.."], verbose)
        os.replace(CLI_BIN + ".tmp", CLI_BIN)
    # the names pyphoenix looks for (PHOENIX_gpu_fp32*, PHOENIX_gpu_fp64*); the
    # executable takes its precision from its name
    for prec in ("fp32", "fp64"):
        link = os.path.join(os.path.dirname(CLI_BIN), f"PHOENIX_gpu_{prec}")
        if not os.path.islink(link):
            if os.path.exists(link):
                os.remove(link)
            os.symlink(os.path.basename(CLI_BIN), link)


UNITS = ["phx_runtime.cu", "phx_noalloc.cu", "phx_batch.cu"]
OBJ_DIR = os.path.join(PKG, "_build")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"{cmd[0]} failed:\n" + proc.stdout[-8000:] + proc.stderr[-8000:])
    return proc


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every translation unit (in parallel) and link libphx.so."""
    if not force and up_to_date():
        build_host(False, verbose)
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
    build_host(force, verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
