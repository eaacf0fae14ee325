"""Run the reference binary on the benchmark-size parity cases of
tests/golden/config_cases.py and store digests of its outputs in
tests/golden/config_digests.json.

The PHOENIX CPU build (``make -C oracle ref`` -> oracle/_ref/phoenix_cpu_*,
compiled from the reference sources without -march, so without FMA
contraction) reads the seeded inputs as 17-digit PHOENIX text matrices and
writes its final wavefunction and reservoir as .npy.  Digested per output:
SHA-256 of the values with signed zeros made positive (x + 0.0), the L2 norm
and a strided sample.  Fixed-step cases without a k-space filter run on
subgrids of 128 x 128 points with every host core (the reference's RK4
results do not depend on the subgrid split); the filter and adaptive cases
run on one subgrid, whose halo enters the reference's Dormand-Prince norm.

Run from the repository root:  python tests/golden/make_config_golden.py [case ...]
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import config_cases as CC  # noqa: E402
import make_golden as MG  # noqa: E402

OUT = os.path.join(HERE, "config_digests.json")


def _write(path, arr):
    arr = np.asarray(arr)
    n_r, n_c = arr.shape
    with open(path, "w") as f:
        f.write(f"# SIZE {n_c} {n_r} {CC.L} {CC.L} {CC.L / (n_c - 1)} {CC.L / (n_r - 1)} :: PHOENIX_ MATRIX\n")
        np.savetxt(f, np.real(arr).astype(np.float64), fmt="%.17g")
        np.savetxt(f, np.imag(arr).astype(np.float64), fmt="%.17g")


def describe(a):
    a = np.asarray(a) + 0.0  # -0.0 -> +0.0
    s = CC.sample(a)
    return {"sha256": CC.digest(a), "dtype": str(a.dtype), "l2": float(np.linalg.norm(a)),
            "sample_re": np.real(s).astype(np.float64).tolist(), "sample_im": np.imag(s).astype(np.float64).tolist()}


def run(name):
    case = CC.cases()[name]
    fields = CC.inputs(name)
    n = case["N_c"]
    binary = MG.REF_BIN[case["dtype"]]
    single = bool(case.get("adaptive") or case.get("mask_cut"))
    sub = "1" if single else str(max(1, n // 128))
    cores = str(os.cpu_count() or 1)
    with tempfile.TemporaryDirectory() as tmp:
        args = [binary, "--N", str(n), str(n), "--L", repr(CC.L), repr(CC.L), "--dt", repr(case["dt"]),
                "--tmax", repr(case["t_max"]), "--outEvery", "1e9", "--output", "wavefunction,reservoir",
                "--of", "npy", "--path", os.path.join(tmp, "out"), "--threads", cores, "--subgrids", sub, sub,
                "--fftEvery", repr(case.get("fft_every", 1e9)), "--hbarscaled", repr(case["h_bar_s"]),
                "--meff", repr(case["m_eff"]), "--gammaC", repr(case["gamma_c"]), "--gammaR", repr(case["gamma_r"]),
                "--gc", repr(case["g_c"]), "--gr", repr(case["g_r"]), "--R", repr(case["R"]),
                "--gpm", repr(case["g_pm"]), "--deltaLT", repr(case["delta_LT"]), "--iterator", case["iterator"],
                "--boundary", "periodic", "periodic"]
        if case.get("adaptive"):
            args += ["-adaptive", "--tol", repr(case["tol"]), "--rkvdt", repr(case["dt_min"]), repr(case["dt_max"])]
        comps = ["plus", "minus"] if case.get("tetm") else ["plus"]
        if case.get("tetm"):
            args += ["-tetm"]
        for comp in comps:
            f = os.path.join(tmp, f"psi_{comp}.txt")
            _write(f, fields[f"psi_{comp}"])
            args += ["--initState", "load", f, "1", "add", comp]
        for key, flag in (("pump_0", "--pump"), ("potential_0", "--potential"), ("fft_mask", "--fftMask")):
            if key in fields:
                f = os.path.join(tmp, key + ".txt")
                _write(f, fields[key])
                args += [flag, "load", f, "1", "add", "both"]
        t0 = time.time()
        proc = subprocess.run(args, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"{name}: reference failed\n{proc.stdout[-3000:]}\n{proc.stderr[-3000:]}")
        rec = {"case": case, "inputs_sha256": CC.input_digest(fields), "cmdline": [os.path.basename(binary)] + args[1:],
               "reference_seconds": round(time.time() - t0, 1), "outputs": {}}
        for comp in comps:
            psi = np.load(os.path.join(tmp, "out", f"wavefunction_{comp}.npy"))
            rv = np.load(os.path.join(tmp, "out", f"reservoir_{comp}.npy"))
            rec["outputs"][f"psi_{comp}"] = describe(psi)
            # the reservoir is stored complex by the reference; its imaginary
            # part stays exactly zero with real pump envelopes
            assert not np.any(np.imag(rv)), f"{name}: complex reservoir"
            rec["outputs"][f"n_{comp}"] = describe(np.real(rv))
    # strip run-specific temporary paths from the record
    rec["cmdline"] = [a if not a.startswith(tempfile.gettempdir()) else os.path.basename(a) for a in rec["cmdline"]]
    return rec


def main(argv):
    names = argv[1:] or list(CC.cases())
    db = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for name in names:
        rec = run(name)
        db[name] = rec
        with open(OUT, "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)
        print(f"{name}: {rec['reference_seconds']} s", flush=True)


if __name__ == "__main__":
    main(sys.argv)
