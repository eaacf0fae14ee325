"""Generate tests/golden/noise_stats.json: statistics of the reference's
stochastic (--dw) runs.

The reference draws its noise from a per-point mt19937 on the CPU (cuRAND on
the GPU), a stream nobody else can reproduce, so parity with noise is
statistical: this script runs the PHOENIX CPU build (oracle/_ref, compiled
from the reference sources by ``make -C oracle ref``) on one small case with
four seeds and records ensemble statistics of the final fields; the test
(tests/test_noise.py) runs the oracle, whose counter-based noise the GPU
reproduces bit for bit, on the same case and compares.

Case: 64 x 64 periodic box of 20 um, uniform psi0 = 1 and n0 = 1, no pump,
g_c = 0.05 (so the stochastic drift -(1/hbar) g_c (-i psi)/dV turns the
phase), R = 0.04 (so R n/dV drives n), dw = 0.05, dt = 0.01, 50 RK4 steps.
Statistics over the grid: mean psi (deterministic part), variance of psi
about its mean (noise power), mean n, nearest-neighbour correlation of the
fluctuations.

Run from the repository root:  python tests/golden/make_noise_stats.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import REF_BIN, write_txt  # noqa: E402

CASE = dict(N_c=64, N_r=64, L_x=20.0, L_y=20.0, h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.05,
            g_r=0.08, R=0.04, g_pm=0.0, delta_LT=0.0, dtype="f64", iterator="RK4", dt=0.01,
            t_max=50 * 0.01 * (1 - 1e-9), periodic_x=1, periodic_y=1, n0_amp=1.0, dw=0.05)
# the reference seeds point i with seed + i (kernel_random_numbers.cu:7-10), so
# independent realisations need seeds further apart than the 72 x 72 padded grid
SEEDS = (10000, 20000, 30000, 40000, 50000, 60000, 70000, 80000)


def statistics(psi, n):
    """Grid statistics of one final state (shared with tests/test_noise.py)."""
    m = psi.mean()
    f = psi - m
    var = float(np.mean(np.abs(f) ** 2))
    corr = float(np.real(np.mean(f * np.conj(np.roll(f, 1, axis=1)))) / var)
    return {"mean_re": float(m.real), "mean_im": float(m.imag), "var": var, "var_re": float(np.mean(f.real ** 2)),
            "var_im": float(np.mean(f.imag ** 2)), "mean_n": float(np.real(n).mean()), "corr_x": corr}


def run_reference(seed):
    c = CASE
    with tempfile.TemporaryDirectory() as tmp:
        ones = np.ones((c["N_r"], c["N_c"]), dtype=np.complex128)
        fpsi, fn = os.path.join(tmp, "psi.txt"), os.path.join(tmp, "n.txt")
        write_txt(fpsi, ones, c["L_x"], c["L_y"])
        write_txt(fn, ones, c["L_x"], c["L_y"])
        args = [REF_BIN[c["dtype"]], "--N", str(c["N_c"]), str(c["N_r"]), "--L", repr(c["L_x"]), repr(c["L_y"]),
                "--dt", repr(c["dt"]), "--tmax", repr(c["t_max"]), "--outEvery", "1e9",
                "--output", "wavefunction,reservoir", "--of", "npy", "--path", os.path.join(tmp, "out"),
                "--threads", "1", "--subgrids", "1", "1", "--hbarscaled", repr(c["h_bar_s"]), "--meff",
                repr(c["m_eff"]), "--gammaC", repr(c["gamma_c"]), "--gammaR", repr(c["gamma_r"]), "--gc",
                repr(c["g_c"]), "--gr", repr(c["g_r"]), "--R", repr(c["R"]), "--gpm", repr(c["g_pm"]),
                "--deltaLT", repr(c["delta_LT"]), "--iterator", c["iterator"], "--boundary", "periodic", "periodic",
                "--initState", "load", fpsi, "1", "add", "plus", "--initReservoir", "load", fn, "1", "add", "plus",
                "--dw", repr(c["dw"]), "--initRandom", "0", str(seed)]
        proc = subprocess.run(args, capture_output=True, text=True, timeout=600)
        if proc.returncode != 0:
            raise RuntimeError(proc.stdout[-3000:] + proc.stderr[-3000:])
        psi = np.load(os.path.join(tmp, "out", "wavefunction_plus.npy"))
        n = np.load(os.path.join(tmp, "out", "reservoir_plus.npy"))
    return statistics(psi, n)


def main():
    out = {"case": CASE, "seeds": list(SEEDS), "reference": [run_reference(s) for s in SEEDS],
           "cmd": "python tests/golden/make_noise_stats.py"}
    with open(os.path.join(HERE, "noise_stats.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out["reference"], indent=1))


if __name__ == "__main__":
    main()
