"""Stochastic noise (--dw).

The reference's noise stream (cuRAND XORWOW on the GPU, a per-point
mt19937 on the CPU) cannot be reproduced, so parity is established in two
steps:
  * statistics: the oracle (same distribution and placement as the
    reference, drawn from Philox4x32-10 + Box-Muller) against ensemble
    statistics of the reference's own CPU build on the same case
    (tests/golden/noise_stats.json, written by make_noise_stats.py);
  * bits: the GPU kernels against the oracle, which draw the same numbers.
The generator itself is checked against the published Philox4x32-10
known-answer vectors and for normality.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle import phx_oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _olib():
    lib = O.lib()
    lib.phx_oracle_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32]
    lib.phx_oracle_noise_normal2.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(C.c_float),
                                             C.POINTER(C.c_float)]
    return lib


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors of Salmon et al. (Random123 kat_vectors)."""
    lib = _olib()
    kats = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
            ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
            ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
             (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, want in kats:
        a = (C.c_uint32 * 4)(*ctr)
        lib.phx_oracle_philox4x32_10(a, key[0], key[1])
        assert tuple(a) == want


def test_normal_pairs_are_standard_normal():
    lib = _olib()
    n = 100_000
    z = np.empty((n, 2), np.float32)
    z0, z1 = C.c_float(), C.c_float()
    for i in range(n):
        lib.phx_oracle_noise_normal2(12345, i // 1000, i % 1000, C.byref(z0), C.byref(z1))
        z[i] = z0.value, z1.value
    x = z.ravel().astype(np.float64)
    assert abs(x.mean()) < 0.01
    assert abs(x.var() - 1.0) < 0.015
    k = np.mean((x - x.mean()) ** 4) / x.var() ** 2
    assert abs(k - 3.0) < 0.06
    assert abs(np.corrcoef(z[:, 0], z[:, 1])[0, 1]) < 0.01
    assert abs(np.mean(np.abs(x) > 3.0) - 0.0027) < 0.0006
    from scipy import stats
    assert stats.kstest(x, "norm").pvalue > 1e-4


def _stats(psi, n):
    m = psi.mean()
    f = psi - m
    var = float(np.mean(np.abs(f) ** 2))
    corr = float(np.real(np.mean(f * np.conj(np.roll(f, 1, axis=1)))) / var)
    return {"mean_re": float(m.real), "mean_im": float(m.imag), "var": var, "var_re": float(np.mean(f.real ** 2)),
            "var_im": float(np.mean(f.imag ** 2)), "mean_n": float(np.real(n).mean()), "corr_x": corr}


def noise_case_fields(case):
    ones = np.ones((case["N_r"], case["N_c"]), np.complex128)
    return {"psi_plus": ones, "n_plus": ones}


def test_oracle_noise_statistics_match_the_reference():
    """Ensemble statistics of the oracle's noisy runs equal those of the
    reference CPU build on the same case (8 independent seeds each): every
    statistic within 5 combined standard errors of the ensemble means."""
    with open(os.path.join(GOLDEN, "noise_stats.json")) as f:
        g = json.load(f)
    case = dict(g["case"])
    fields = noise_case_fields(case)
    ours = []
    for seed in range(1, 9):
        case["seed"] = seed
        out, rec = O.run(case, fields)
        assert rec["steps"] == 50
        ours.append(_stats(out["psi_plus"], out["n_plus"]))
    ref = g["reference"]
    assert len(ref) == 8
    for k in ("mean_re", "mean_im", "var", "var_re", "var_im", "mean_n", "corr_x"):
        a = np.array([r[k] for r in ours])
        b = np.array([r[k] for r in ref])
        se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
        assert abs(a.mean() - b.mean()) < 5 * se, (k, a.mean(), b.mean(), se)
    # the stochastic drift turns the phase of the mean field: far from the noiseless run
    quiet, _ = O.run(dict(case, dw=0.0), fields)
    assert abs(np.angle(quiet["psi_plus"].mean()) - np.angle(complex(np.mean([r["mean_re"] for r in ref]),
                                                                        np.mean([r["mean_im"] for r in ref])))) > 0.3


def test_noise_off_for_non_positive_amplitude():
    """The reference applies noise only for dw > 0 (system_initialization.cpp:244)."""
    with open(os.path.join(GOLDEN, "noise_stats.json")) as f:
        case = dict(json.load(f)["case"])
    fields = noise_case_fields(case)
    case["t_max"] = 5 * case["dt"] * (1 - 1e-9)
    a, _ = O.run(dict(case, dw=0.0), fields)
    b, _ = O.run(dict(case, dw=-0.05, seed=9), fields)
    np.testing.assert_array_equal(a["psi_plus"], b["psi_plus"])
