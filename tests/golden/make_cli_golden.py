"""Generate the command-line fixtures of tests/golden/cli/ by running the
reference executable (the PHOENIX CPU build, oracle/_ref/phoenix_cpu_{fp64,fp32},
``make -C oracle ref``) on small command lines.

Every case is a directory holding the seeded input files the command line
loads, ``case.json`` (the argument list, the precision and which outputs are
compared exactly) and ``ref/``, the files the reference wrote into its
``--path`` (``times.txt``, wall-clock timings, is left out).  The command-line
tests run phoenix_b200's executable on the same arguments and compare.

Run from the repository root:  python tests/golden/make_cli_golden.py
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "cli")
REF_BIN = {"fp64": os.path.join(ROOT, "oracle", "_ref", "phoenix_cpu_fp64"),
           "fp32": os.path.join(ROOT, "oracle", "_ref", "phoenix_cpu_fp32")}

STRONG = ["--hbarscaled", "0.6582", "--meff", "0.5", "--gammaC", "0.2", "--gammaR", "0.3", "--gc", "0.05",
          "--gr", "0.08", "--R", "0.04", "--gpm", "-0.01", "--deltaLT", "0.3"]


def write_txt(path, arr, L_x, L_y):
    arr = np.asarray(arr)
    n_r, n_c = arr.shape
    with open(path, "w") as f:
        f.write(f"# SIZE {n_c} {n_r} {L_x} {L_y} {L_x / (n_c - 1)} {L_y / (n_r - 1)} :: PHOENIX_ MATRIX\n")
        for blk in (np.real(arr), np.imag(arr)):
            for row in blk:
                f.write(" ".join(f"{v:.17g}" for v in row) + "\n")


def cases():
    c = {}
    # RK4, zero boundaries, random start, positional and named envelopes with a
    # cos temporal group, every output key, history matrices, 17 digits
    c["rk4_txt_fp64"] = dict(prec="fp64", exact=True, inputs={}, args=[
        "--N", "16", "12", "--L", "20", "15", "--tmax", "0.1", "--dt", "0.01", "--outEvery", "0.03", *STRONG,
        "--pump", "2.0", "add", "3.0", "3.0", "0", "0", "both", "1", "none", "gauss",
        "--potential", "0.5", "add", "width", "4", "4", "pos", "1", "1", "pol", "plus", "exponent", "2", "charge", "1",
        "time", "cos", "0.05", "0.1", "3.0",
        "--initRandom", "0.1", "42", "--output", "all", "--fileoutPrecision", "17",
        "--historyMatrix", "2", "14", "1", "11", "1", "--historyTime", "0", "2"])
    # DP45 adaptive, periodic, loaded start and reservoir, k-space mask (fft
    # output), npy
    c["dp45_npy_fp64"] = dict(prec="fp64", exact=False, inputs={"psi": (16, 16, 1.0, 11), "n": (16, 16, 0.5, 12)}, args=[
        "--N", "16", "16", "--L", "20", "20", "--tmax", "0.12", "--dt", "0.01", "--outEvery", "0.05", *STRONG,
        "--boundary", "periodic", "periodic", "--iterator", "DP45", "-adaptive", "--tol", "1e-6", "--rkvdt", "1e-5", "0.05",
        "--initState", "load", "psi.txt", "1", "add", "plus",
        "--initReservoir", "load", "n.txt", "1", "add", "plus",
        "--pump", "2.5", "add", "width", "3", "3", "type", "gauss",
        "--fftMask", "1", "add", "0.6", "0.6", "0", "0", "both", "4", "none", "gauss+noDivide+local",
        "--fftEvery", "0.04", "--of", "npy", "--output", "wavefunction,reservoir,fft,scalar,pump"])
    # FP32 RK4 TE/TM, pulse with an iexp group, MATLAB files
    c["tetm_mat_fp32"] = dict(prec="fp32", exact=True, inputs={}, args=[
        "--N", "12", "12", "--L", "15", "15", "--tmax", "0.05", "--dt", "0.005", "--outEvery", "0.02", *STRONG, "-tetm",
        "--boundary", "periodic", "zero",
        "--pump", "2.0", "add", "3.0", "3.0", "0", "0", "both", "1", "none", "gauss",
        "--pulse", "1.0", "add", "2.0", "2.0", "0", "0", "plus", "1", "none", "gauss", "momenta", "0.3", "0",
        "time", "iexp", "0.02", "0.01", "5.0",
        "--initRandom", "0.2", "7", "--of", "mat", "--output", "all"])
    # Heun3 with a loaded temporal table, PHOENIX binary (.ash) files, a name prefix
    c["heun3_ash_fp64"] = dict(prec="fp64", exact=True, inputs={"table": None}, args=[
        "--N", "14", "10", "--L", "18", "12", "--tmax", "0.06", "--dt", "0.005", "--outEvery", "0.02", *STRONG,
        "--iterator", "Heun3", "--boundary", "zero", "periodic",
        "--pump", "1.5", "add", "3.0", "3.0", "0", "0", "both", "1", "none", "gauss", "time", "load", "table.txt",
        "--potential", "0.3", "add", "2.5", "2.5", "1", "0", "both", "1", "none", "ring",
        "--initRandom", "0.3", "5", "--of", "ash", "--name", "run", "--output", "all"])
    return c


def make_inputs(case, d):
    for name, spec in case["inputs"].items():
        if name == "table":
            t = np.linspace(0.0, 0.08, 9)
            with open(os.path.join(d, "table.txt"), "w") as f:
                f.write("# t re im\n")
                for tt in t:
                    f.write(f"{tt:.17g} {1.0 + 0.5 * np.sin(40 * tt):.17g} 0\n")
            continue
        n_c, n_r, amp, seed = spec
        rng = np.random.default_rng(seed)
        if name == "psi":
            a = amp * (rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c)))
        else:
            a = amp * rng.random((n_r, n_c)) + 0j
        write_txt(os.path.join(d, f"{name}.txt"), a, 20.0, 20.0)


def main(argv):
    todo = cases()
    for name in argv[1:] or list(todo):
        case = todo[name]
        d = os.path.join(OUT, name)
        if os.path.isdir(d):
            shutil.rmtree(d)
        os.makedirs(d)
        make_inputs(case, d)
        with tempfile.TemporaryDirectory() as tmp:
            for f in os.listdir(d):
                shutil.copy(os.path.join(d, f), tmp)
            cmd = [REF_BIN[case["prec"]], *case["args"], "--path", "ref", "--threads", "1", "--subgrids", "1", "1"]
            proc = subprocess.run(cmd, cwd=tmp, capture_output=True, text=True, timeout=600)
            if proc.returncode != 0:
                raise RuntimeError(f"{name}: reference failed\n{proc.stdout[-3000:]}\n{proc.stderr[-2000:]}")
            os.makedirs(os.path.join(d, "ref"))
            for root, _, files in os.walk(os.path.join(tmp, "ref")):
                for f in files:
                    if f == "times.txt" or f.endswith("_times.txt"):
                        continue
                    rel = os.path.relpath(os.path.join(root, f), os.path.join(tmp, "ref"))
                    os.makedirs(os.path.dirname(os.path.join(d, "ref", rel)), exist_ok=True)
                    shutil.copy(os.path.join(root, f), os.path.join(d, "ref", rel))
        with open(os.path.join(d, "case.json"), "w") as f:
            json.dump({"args": case["args"], "precision": case["prec"], "exact": case["exact"]}, f, indent=1)
        print(name, sorted(os.listdir(os.path.join(d, "ref"))))


if __name__ == "__main__":
    main(sys.argv)
