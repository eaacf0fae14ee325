"""Generate the golden fixtures of tests/golden/ by running the reference.

The PHOENIX CPU build is compiled from the reference sources by
``make -C oracle ref`` into ``oracle/_ref/phoenix_cpu_{fp64,fp32}`` (no
-march, so no FMA contraction).  For every case below this script draws
seeded inputs with numpy, writes them as PHOENIX text matrices
(``# SIZE Nc Nr ...`` header, real block then imaginary block, 17 significant
digits, read back by FileHandler::loadMatrixFromFile,
source/system/filehandler.cpp:160-198), runs the binary with the case's
flags and stores inputs, parameters and the binary's final matrices
(``--of npy``) in ``tests/golden/<case>.npz``.

Run from the repository root:  python tests/golden/make_golden.py
The fixtures are committed; tests never need the reference at run time.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_BIN = {
    "f64": os.path.join(ROOT, "oracle", "_ref", "phoenix_cpu_fp64"),
    "f32": os.path.join(ROOT, "oracle", "_ref", "phoenix_cpu_fp32"),
}

# Physics of the polariton configs in meV / ps / um: hbar = 0.6582 meV ps,
# m_eff = 5.6e-4 m_e = 3.1840 meV ps^2 / um^2.
BASE = dict(h_bar_s=0.6582, m_eff=3.1840, gamma_c=0.15, gamma_r=0.225, g_c=6e-6, g_r=1.2e-5, R=0.01,
            g_pm=-1.2e-6, delta_LT=0.05)
# A parameter set that makes every term of the right-hand side significant
# on a small grid within a few dozen steps.
STRONG = dict(h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.05, g_r=0.08, R=0.04,
              g_pm=-0.01, delta_LT=0.3)


def write_txt(path, arr, L_x, L_y):
    """PHOENIX text matrix: header, N_r lines of real parts, N_r lines of imaginary parts."""
    arr = np.asarray(arr)
    n_r, n_c = arr.shape
    re = np.real(arr).astype(np.float64)
    im = np.imag(arr).astype(np.float64)
    with open(path, "w") as f:
        f.write(f"# SIZE {n_c} {n_r} {L_x} {L_y} {L_x / (n_c - 1)} {L_y / (n_r - 1)} :: PHOENIX_ MATRIX\n")
        for blk in (re, im):
            for row in blk:
                f.write(" ".join(f"{v:.17g}" for v in row) + "\n")


def coords(n_c, n_r, L_x, L_y):
    """Envelope coordinates x = -L/2 + dx*col (envelope.cpp:346-347)."""
    dx, dy = L_x / (n_c - 1), L_y / (n_r - 1)
    x = -L_x / 2.0 + dx * np.arange(n_c)
    y = -L_y / 2.0 + dy * np.arange(n_r)
    return np.meshgrid(x, y)


def make_inputs(case, rng):
    n_c, n_r, L_x, L_y = case["N_c"], case["N_r"], case["L_x"], case["L_y"]
    X, Y = coords(n_c, n_r, L_x, L_y)
    amp = case.get("psi_amp", 1e-2)
    out = {}
    comps = ["plus", "minus"] if case.get("tetm") else ["plus"]
    for comp in comps:
        out[f"psi_{comp}"] = amp * (rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c)))
        if case.get("n0_amp", 0.0):
            out[f"n_{comp}"] = case["n0_amp"] * rng.random((n_r, n_c)) + 0j
    for g, (peak, width, x0) in enumerate(case.get("pumps", [])):
        out[f"pump_{g}"] = peak * np.exp(-((X - x0) ** 2 + Y ** 2) / (2 * width ** 2)) + 0j
    for g, rms in enumerate(case.get("potentials", [])):
        out[f"potential_{g}"] = rms * rng.standard_normal((n_r, n_c)) + 0j
    for g, (peak, width) in enumerate(case.get("pulses", [])):
        out[f"pulse_{g}"] = peak * np.exp(-(X ** 2 + Y ** 2) / (2 * width ** 2)) * np.exp(1j * 0.3 * X)
    if case.get("mask_cut"):
        # super-Gaussian low-pass in the reference's real-space coordinate convention
        # (the reference fft-shifts the mask, solver_initialization.cu:152-168)
        kx = (2.0 * np.arange(n_c) / (n_c - 1) - 1.0)
        ky = (2.0 * np.arange(n_r) / (n_r - 1) - 1.0)
        KX, KY = np.meshgrid(kx, ky)
        c = case["mask_cut"]
        out["fft_mask"] = np.exp(-(((KX / c) ** 2 + (KY / c) ** 2) / 2.0) ** 4) + 0j
    return out


def temporal_flags(spec):
    if spec is None or spec[0] == "constant":
        return []
    kind, t0, sigma, freq = spec
    return ["time", kind, repr(t0), repr(sigma), repr(freq)]


def run_case(name, case):
    rng = np.random.default_rng(case["seed"])
    inputs = make_inputs(case, rng)
    prec = case["dtype"]
    L_x, L_y = case["L_x"], case["L_y"]
    with tempfile.TemporaryDirectory() as tmp:
        args = [REF_BIN[prec], "--N", str(case["N_c"]), str(case["N_r"]), "--L", repr(L_x), repr(L_y),
                "--dt", repr(case["dt"]), "--tmax", repr(case["t_max"]), "--outEvery", "1e9",
                "--output", "wavefunction,reservoir", "--of", "npy", "--path", os.path.join(tmp, "out"),
                "--threads", "1", "--subgrids", "1", "1",
                "--fftEvery", repr(case.get("fft_every", 1e9)),
                "--hbarscaled", repr(case["h_bar_s"]), "--meff", repr(case["m_eff"]),
                "--gammaC", repr(case["gamma_c"]), "--gammaR", repr(case["gamma_r"]),
                "--gc", repr(case["g_c"]), "--gr", repr(case["g_r"]), "--R", repr(case["R"]),
                "--gpm", repr(case["g_pm"]), "--deltaLT", repr(case["delta_LT"]),
                "--iterator", case["iterator"]]
        bx = "periodic" if case["periodic_x"] else "zero"
        by = "periodic" if case["periodic_y"] else "zero"
        args += ["--boundary", bx, by]
        if case.get("adaptive"):
            args += ["-adaptive", "--tol", repr(case["tol"]), "--rkvdt", repr(case["dt_min"]), repr(case["dt_max"])]
        if case.get("tetm"):
            args += ["-tetm"]
        if case.get("imag_time"):
            args += ["--imagTime", repr(case["imag_time"])]
        comps = ["plus", "minus"] if case.get("tetm") else ["plus"]
        for comp in comps:
            f = os.path.join(tmp, f"psi_{comp}.txt")
            write_txt(f, inputs[f"psi_{comp}"], L_x, L_y)
            args += ["--initState", "load", f, "1", "add", comp]
            if f"n_{comp}" in inputs:
                f = os.path.join(tmp, f"n_{comp}.txt")
                write_txt(f, inputs[f"n_{comp}"], L_x, L_y)
                args += ["--initReservoir", "load", f, "1", "add", comp]
        for g, _ in enumerate(case.get("pumps", [])):
            f = os.path.join(tmp, f"pump_{g}.txt")
            write_txt(f, inputs[f"pump_{g}"], L_x, L_y)
            args += ["--pump", "load", f, "1", "add", "both"] + temporal_flags(case.get("pump_t", [None] * 8)[g])
        for g, _ in enumerate(case.get("potentials", [])):
            f = os.path.join(tmp, f"potential_{g}.txt")
            write_txt(f, inputs[f"potential_{g}"], L_x, L_y)
            args += ["--potential", "load", f, "1", "add", "both"] + temporal_flags(case.get("potential_t", [None] * 8)[g])
        for g, _ in enumerate(case.get("pulses", [])):
            f = os.path.join(tmp, f"pulse_{g}.txt")
            write_txt(f, inputs[f"pulse_{g}"], L_x, L_y)
            args += ["--pulse", "load", f, "1", "add", "both"] + temporal_flags(case.get("pulse_t", [None] * 8)[g])
        if "fft_mask" in inputs:
            f = os.path.join(tmp, "fft_mask.txt")
            write_txt(f, inputs["fft_mask"], L_x, L_y)
            args += ["--fftMask", "load", f, "1", "add", "both"]
        proc = subprocess.run(args, capture_output=True, text=True, timeout=600)
        if proc.returncode != 0:
            raise RuntimeError(f"{name}: reference failed\n{proc.stdout[-3000:]}\n{proc.stderr[-3000:]}")
        outs = {}
        for comp in comps:
            outs[f"out_psi_{comp}"] = np.load(os.path.join(tmp, "out", f"wavefunction_{comp}.npy"))
            rv = os.path.join(tmp, "out", f"reservoir_{comp}.npy")
            if os.path.exists(rv):
                outs[f"out_n_{comp}"] = np.load(rv)
        # round inputs exactly as the reference read them (17 digits round-trips double)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), params=json.dumps(case), cmdline=json.dumps(args[1:]),
                            **{f"in_{k}": v for k, v in inputs.items()}, **outs)
        print(f"{name}: ok ({len(args)} args)")


def cases():
    c = {}
    grid = dict(N_c=32, N_r=32, L_x=20.0, L_y=20.0)
    c["rk4_f64_periodic"] = dict(grid, **STRONG, dtype="f64", iterator="RK4", dt=0.01, t_max=0.4 * (1 - 1e-9),
                                 periodic_x=1, periodic_y=1, seed=11, psi_amp=1.0, pumps=[(4.0, 3.0, 0.0)],
                                 potentials=[0.2])
    c["rk4_f64_zero"] = dict(grid, **STRONG, dtype="f64", iterator="RK4", dt=0.01, t_max=0.3 * (1 - 1e-9),
                             periodic_x=0, periodic_y=0, seed=12, psi_amp=1.0, n0_amp=0.5,
                             pumps=[(4.0, 3.0, 1.0)], potentials=[0.2])
    c["rk4_f64_mixed_rect"] = dict(N_c=48, N_r=32, L_x=30.0, L_y=20.0, **STRONG, dtype="f64", iterator="RK4",
                                   dt=0.01, t_max=0.3 * (1 - 1e-9), periodic_x=1, periodic_y=0, seed=13,
                                   psi_amp=1.0, pumps=[(4.0, 3.0, -2.0)])
    c["rk4_f64_nores"] = dict(grid, **STRONG, dtype="f64", iterator="RK4", dt=0.01, t_max=0.3 * (1 - 1e-9),
                              periodic_x=1, periodic_y=1, seed=14, psi_amp=1.0, potentials=[0.3])
    c["rk4_f64_temporal"] = dict(grid, **STRONG, dtype="f64", iterator="RK4", dt=0.01, t_max=0.3 * (1 - 1e-9),
                                 periodic_x=1, periodic_y=1, seed=15, psi_amp=0.5,
                                 pumps=[(4.0, 3.0, 0.0), (2.0, 2.0, 3.0)],
                                 pump_t=[("gauss", 0.1, 0.2, 1.0), ("cos", 0.05, 0.3, 20.0)],
                                 potentials=[0.2], potential_t=[("cos", 0.0, 0.5, 10.0)],
                                 pulses=[(1.0, 3.0)], pulse_t=[("iexp", 0.15, 0.1, 5.0)])
    c["rk4_f32_periodic"] = dict(grid, **STRONG, dtype="f32", iterator="RK4", dt=0.01, t_max=0.4 * (1 - 1e-9),
                                 periodic_x=1, periodic_y=1, seed=16, psi_amp=1.0, pumps=[(4.0, 3.0, 0.0)],
                                 potentials=[0.2])
    c["rk4_f64_mask"] = dict(grid, **STRONG, dtype="f64", iterator="RK4", dt=0.01, t_max=0.4 * (1 - 1e-9),
                             periodic_x=1, periodic_y=1, seed=17, psi_amp=1.0, pumps=[(4.0, 3.0, 0.0)],
                             mask_cut=0.6, fft_every=0.05)
    c["rk4_f64_baseline_phys"] = dict(N_c=64, N_r=64, L_x=100.0, L_y=100.0, **BASE, dtype="f64", iterator="RK4",
                                      dt=0.04, t_max=4.0 * (1 - 1e-9), periodic_x=1, periodic_y=1, seed=1,
                                      psi_amp=1e-2, pumps=[(5.0625, 10.0, 0.0)])
    c["dp45_f64_adaptive"] = dict(grid, **STRONG, dtype="f64", iterator="DP45", adaptive=1, tol=1e-6, dt_min=1e-5,
                                  dt_max=0.05, dt=0.01, t_max=0.3, periodic_x=1, periodic_y=1, seed=18,
                                  psi_amp=1.0, pumps=[(4.0, 3.0, 0.0)], potentials=[0.2])
    c["dp45_f64_fixed"] = dict(grid, **STRONG, dtype="f64", iterator="DP45", dt=0.01, t_max=0.2 * (1 - 1e-9),
                               periodic_x=0, periodic_y=0, seed=19, psi_amp=1.0, pumps=[(4.0, 3.0, 0.0)])
    c["tetm_f64_periodic"] = dict(grid, **STRONG, dtype="f64", iterator="RK4", tetm=1, dt=0.01,
                                  t_max=0.3 * (1 - 1e-9), periodic_x=1, periodic_y=1, seed=20, psi_amp=1.0,
                                  pumps=[(4.0, 3.0, 0.0)], potentials=[0.2])
    c["tetm_f64_zero"] = dict(grid, **STRONG, dtype="f64", iterator="RK4", tetm=1, dt=0.01,
                              t_max=0.2 * (1 - 1e-9), periodic_x=0, periodic_y=0, seed=21, psi_amp=1.0,
                              pumps=[(4.0, 3.0, 0.0)])
    # the fixed-step tableaux of the reference's other registered iterators:
    # mixed boundaries (periodic x, zero y) so the extended stage regions of
    # the zero axis are exercised, pump + potential, 20 steps
    # (RK3 and Ralston4 are left out: the reference's RK3 final sum lists a
    # fourth weight and reads a k plane past its three-plane stack, and its
    # Ralston4 declares k_max 3 for four stages and writes past the stack;
    # neither output is defined)
    for k, (it, seed) in enumerate([("SSPRK3", 32), ("MP", 33), ("Heun2", 34), ("Heun3", 35),
                                    ("HW", 36), ("Newton", 37), ("Nystroem", 38), ("Ralston", 39),
                                    ("Ralston3", 40), ("Rule38", 42)]):
        c[f"tab_{it.lower()}_f64_mixed"] = dict(N_c=40, N_r=32, L_x=25.0, L_y=20.0, **STRONG, dtype="f64",
                                                 iterator=it, dt=0.005, t_max=20 * 0.005 * (1 - 1e-9),
                                                 periodic_x=1, periodic_y=0, seed=seed, psi_amp=1.0,
                                                 n0_amp=0.5, pumps=[(4.0, 3.0, 0.0)], potentials=[0.2])
    # adaptive tableaux (DP45 has its own cases above)
    ad = dict(**STRONG, dtype="f64", adaptive=1, tol=1e-6, dt_min=1e-5, dt_max=0.05, dt=0.01, t_max=0.2,
              psi_amp=1.0, pumps=[(4.0, 3.0, 0.0)], potentials=[0.2])
    for it, (px, py), seed in [("BoSha", (1, 1), 51), ("CashKarp", (1, 0), 52), ("Fehlberg2", (0, 0), 53),
                               ("Fehlberg5", (1, 1), 54), ("DP85", (1, 0), 55), ("NSRK78", (0, 0), 56)]:
        c[f"tab_{it.lower()}_f64_adaptive"] = dict(grid, **ad, iterator=it, periodic_x=px, periodic_y=py, seed=seed)
    c["tab_dp85_f64_fixed"] = dict(grid, **STRONG, dtype="f64", iterator="DP85", dt=0.01, t_max=10 * 0.01 * (1 - 1e-9),
                                   periodic_x=0, periodic_y=0, seed=57, psi_amp=1.0, n0_amp=0.5,
                                   pumps=[(4.0, 3.0, 0.0)])
    c["tab_nsrk78_f64_fixed"] = dict(grid, **STRONG, dtype="f64", iterator="NSRK78", dt=0.01,
                                     t_max=10 * 0.01 * (1 - 1e-9), periodic_x=1, periodic_y=0, seed=58, psi_amp=1.0,
                                     pumps=[(4.0, 3.0, 0.0)], potentials=[0.2])
    c["tab_bosha_f32_fixed"] = dict(grid, **STRONG, dtype="f32", iterator="BoSha", dt=0.005,
                                    t_max=20 * 0.005 * (1 - 1e-9), periodic_x=1, periodic_y=1, seed=59, psi_amp=1.0,
                                    pumps=[(4.0, 3.0, 0.0)], potentials=[0.2])
    # (no SSFM case: the reference CPU build ends its first SSFM step with a
    # segmentation fault, with or without a k-space mask)
    c["tab_ssprk3_f32_periodic"] = dict(grid, **STRONG, dtype="f32", iterator="SSPRK3", dt=0.005,
                                        t_max=20 * 0.005 * (1 - 1e-9), periodic_x=1, periodic_y=1, seed=43,
                                        psi_amp=1.0, pumps=[(4.0, 3.0, 0.0)], potentials=[0.2])
    # imaginary-time propagation (--imagTime): complex step (0, -dt) in every
    # stage sum, then every field scaled to sum |f|^2 dV = A over its padded
    # buffer.  Without a reservoir (no pump, no initial reservoir) except the
    # last case, where the complex step makes the reservoir complex.
    im = dict(**STRONG, imag_time=2.5, psi_amp=1.0, potentials=[0.2])
    c["imag_rk4_f64_periodic"] = dict(grid, **im, dtype="f64", iterator="RK4", dt=0.01,
                                      t_max=20 * 0.01 * (1 - 1e-9), periodic_x=1, periodic_y=1, seed=61)
    c["imag_rk4_f64_zero"] = dict(grid, **im, dtype="f64", iterator="RK4", dt=0.01, t_max=20 * 0.01 * (1 - 1e-9),
                                  periodic_x=0, periodic_y=0, seed=62)
    c["imag_rk4_f32_mixed"] = dict(N_c=40, N_r=32, L_x=25.0, L_y=20.0, **im, dtype="f32", iterator="RK4", dt=0.01,
                                   t_max=20 * 0.01 * (1 - 1e-9), periodic_x=1, periodic_y=0, seed=63)
    c["imag_heun3_f64_mixed"] = dict(N_c=40, N_r=32, L_x=25.0, L_y=20.0, **im, dtype="f64", iterator="Heun3",
                                     dt=0.005, t_max=20 * 0.005 * (1 - 1e-9), periodic_x=0, periodic_y=1, seed=64)
    c["imag_nsrk78_f64_zero"] = dict(grid, **im, dtype="f64", iterator="NSRK78", dt=0.01,
                                     t_max=10 * 0.01 * (1 - 1e-9), periodic_x=0, periodic_y=0, seed=65)
    c["imag_dp45_f64_adaptive"] = dict(grid, **im, dtype="f64", iterator="DP45", adaptive=1, tol=1e-6, dt_min=1e-5,
                                       dt_max=0.05, dt=0.01, t_max=0.2, periodic_x=1, periodic_y=1, seed=66)
    c["imag_rk4_f64_reservoir"] = dict(grid, **im, dtype="f64", iterator="RK4", dt=0.01,
                                       t_max=10 * 0.01 * (1 - 1e-9), periodic_x=1, periodic_y=1, seed=67,
                                       pumps=[(4.0, 3.0, 0.0)])
    return c


def main(argv):
    todo = cases()
    names = argv[1:] or list(todo)
    for n in names:
        run_case(n, todo[n])


if __name__ == "__main__":
    main(sys.argv)
