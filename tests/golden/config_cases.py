"""Parity cases at the benchmark configurations' own sizes.

The small golden fixtures (tests/golden/*.npz) pin every code path on 32^2 to
64^2 grids.  The cases here run the workloads the benchmark times, at their
own sizes: the 1024^2 polariton with disorder and k-space mask (RK4 FP64 with
the mask every 100 iterations, RK4 FP32, Dormand-Prince 5(4) adaptive at tol
1e-6) and the TE/TM spinor with a ring pump (1024^2 FP64 and FP32, 4096^2
FP32, deterministic).  Their outputs are 16 MB to 256 MB, too large to
commit, so tests/golden/make_config_golden.py runs the reference binary on
them once and stores a digest of each output (config_digests.json): the
SHA-256 of the array bytes as the reference wrote them (--of npy), its L2
norm and a strided sample of values.  Inputs are regenerated from seeds by
``inputs(name)``; their own SHA-256 is stored too, so a platform whose numpy
draws differently fails loudly instead of comparing different runs.

Physics (meV, ps, um): hbar 0.6582, m_eff = 5.6e-4 m_e = 3.1840, gamma_c
0.15, gamma_r 0.225, g_c 6e-6, g_r 1.2e-5, R 0.01, 100 um periodic box,
pump at 1.5x threshold (P_th = gamma_c gamma_r / R).
"""
from __future__ import annotations

import hashlib

import numpy as np

L = 100.0
PHYS = dict(h_bar_s=0.6582, m_eff=3.1840, gamma_c=0.15, gamma_r=0.225, g_c=6e-6, g_r=1.2e-5, R=0.01)
P_TH = 0.15 * 0.225 / 0.01
DT_1024 = 0.02


def _grid(n):
    x = -L / 2 + L / (n - 1) * np.arange(n)
    return np.meshgrid(x, x)


def disorder(n, rms, seed, corr=1.0):
    """Gaussian random potential: white noise smoothed by a Gaussian kernel of
    correlation length `corr` um, scaled to `rms` meV."""
    noise = np.random.default_rng(seed).standard_normal((n, n))
    k = 2 * np.pi * np.fft.fftfreq(n, d=L / (n - 1))
    KX, KY = np.meshgrid(k, k)
    pot = np.real(np.fft.ifft2(np.fft.fft2(noise) * np.exp(-(KX ** 2 + KY ** 2) * corr ** 2 / 2)))
    return pot * (rms / np.sqrt(np.mean(pot ** 2)))


def super_gauss_mask(n, cut=0.8, order=4):
    """k-space low-pass in the reference's local [-1, 1] coordinates (the
    reference fft-shifts it once): exp(-((x^2 + y^2) / (2 cut^2))^order)."""
    loc = -1.0 + 2.0 * np.arange(n) / (n - 1)
    LX, LY = np.meshgrid(loc, loc)
    return np.exp(-((0.5 * ((LX / cut) ** 2 + (LY / cut) ** 2)) ** order))


def _case(n, dtype, iterator="RK4", **kw):
    c = dict(N_c=n, N_r=n, L_x=L, L_y=L, **PHYS, g_pm=0.0, delta_LT=0.0, dtype=dtype, iterator=iterator,
             periodic_x=1, periodic_y=1)
    c.update(kw)
    return c


def cases():
    """name -> case dictionary (the keys of tests/golden/make_golden.py)."""
    dt = DT_1024
    c = {}
    # config 2: 1024^2, disorder 0.1 meV rms, mask every 100 iterations
    scalar = dict(pumps=[(1.5 * P_TH, 10.0, 0.0)], potentials=[0.1], seed=2)
    c["cfg2_rk4_f64_mask_1024"] = _case(1024, "f64", dt=dt, t_max=200 * dt * (1 - 1e-9), mask_cut=0.8,
                                        fft_every=100 * dt * (1 - 1e-6), **scalar)
    c["cfg2_rk4_f32_1024"] = _case(1024, "f32", dt=dt, t_max=200 * dt * (1 - 1e-9), **scalar)
    c["cfg2_dp45_f64_mask_1024"] = _case(1024, "f64", iterator="DP45", adaptive=1, tol=1e-6, dt_min=1e-4,
                                         dt_max=3.0, dt=dt, t_max=1.0, mask_cut=0.8, fft_every=0.5, **scalar)
    # config 3: TE/TM spinor, ring pump (radius 20 um, width 3 um), deterministic
    tetm = dict(tetm=1, g_pm=-1.2e-6, delta_LT=0.05, ring_pump=(1.5 * P_TH, 20.0, 3.0), seed=4)
    c["cfg3_tetm_f64_1024"] = _case(1024, "f64", dt=dt, t_max=100 * dt * (1 - 1e-9), **tetm)
    c["cfg3_tetm_f32_1024"] = _case(1024, "f32", dt=dt, t_max=100 * dt * (1 - 1e-9), **tetm)
    dt4 = DT_1024 / 16
    c["cfg3_tetm_f32_4096"] = _case(4096, "f32", dt=dt4, t_max=50 * dt4 * (1 - 1e-9), **tetm)
    return c


def inputs(name):
    """The seeded input fields of a case (full-grid numpy arrays, float64 /
    complex128, the values the reference reads back from 17-digit text)."""
    case = cases()[name]
    n = case["N_c"]
    rng = np.random.default_rng(case["seed"])
    X, Y = _grid(n)
    out = {}
    comps = ["plus", "minus"] if case.get("tetm") else ["plus"]
    for comp in comps:
        out[f"psi_{comp}"] = 1e-2 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    if "ring_pump" in case:
        peak, radius, width = case["ring_pump"]
        out["pump_0"] = peak * np.exp(-(np.sqrt(X ** 2 + Y ** 2) - radius) ** 2 / (2 * width ** 2)) + 0j
    else:
        peak, width, _ = case["pumps"][0]
        out["pump_0"] = peak * np.exp(-(X ** 2 + Y ** 2) / (2 * width ** 2)) + 0j
    if case.get("potentials"):
        out["potential_0"] = disorder(n, case["potentials"][0], case["seed"] + 1) + 0j
    if case.get("mask_cut"):
        out["fft_mask"] = super_gauss_mask(n, case["mask_cut"]) + 0j
    return out


def oracle_case(name):
    """The case dictionary in the form oracle.phx_oracle.run takes (a ring
    pump is a loaded matrix like any other pump)."""
    case = dict(cases()[name])
    if "ring_pump" in case:
        case["pumps"] = [(case.pop("ring_pump")[0], 0.0, 0.0)]
    return case


def digest(a):
    """SHA-256 of an array's bytes in C order."""
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def input_digest(fields):
    h = hashlib.sha256()
    for k in sorted(fields):
        h.update(k.encode())
        h.update(np.ascontiguousarray(fields[k]).tobytes())
    return h.hexdigest()


SAMPLE_STRIDE = 61


def sample(a):
    """A strided sample of a field (rows and columns every 61 points)."""
    return np.asarray(a)[::SAMPLE_STRIDE, ::SAMPLE_STRIDE]
