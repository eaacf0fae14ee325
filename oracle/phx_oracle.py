"""ctypes binding of the C restatement oracle/phx_oracle.c.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the CPU-baseline leg of bench.py, always as the checker.  The product
(phoenix_b200) never imports it.

``run(params, fields, max_steps)`` takes the same case dictionaries as
tests/golden/make_golden.py and full-grid numpy fields, and returns the final
fields plus the iteration record.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libphx_oracle.so")
MAX_GROUPS = 8
TEMPORAL = {"constant": 0, "iexp": 1, "osc": 1, "cos": 2, "gauss": 3}
# REGISTER_SOLVER keys of the reference, numbered as in include/phx.h
ITERATORS = {"RK4": 0, "DP45": 1, "RK3": 2, "SSPRK3": 3, "MP": 4, "HEUN2": 5, "HEUN3": 6, "HW": 7, "NEWTON": 8,
             "NYSTROEM": 9, "RALSTON": 10, "RALSTON3": 11, "RALSTON4": 12, "RULE38": 13, "BOSHA": 14,
             "CASHKARP": 15, "FEHLBERG2": 16, "FEHLBERG5": 17, "DP85": 18, "NSRK78": 19, "SSFM": 20}


class Temporal(C.Structure):
    _fields_ = [("kind", C.c_int), ("t0", C.c_double), ("sigma", C.c_double), ("freq", C.c_double)]


class Params(C.Structure):
    _fields_ = [
        ("N_c", C.c_int32), ("N_r", C.c_int32), ("L_x", C.c_double), ("L_y", C.c_double),
        ("h_bar_s", C.c_double), ("m_eff", C.c_double), ("gamma_c", C.c_double), ("gamma_r", C.c_double),
        ("g_c", C.c_double), ("g_r", C.c_double), ("R", C.c_double), ("g_pm", C.c_double), ("delta_LT", C.c_double),
        ("periodic_x", C.c_int32), ("periodic_y", C.c_int32), ("tetm", C.c_int32), ("use_reservoir", C.c_int32),
        ("iterator", C.c_int32), ("adaptive", C.c_int32), ("dt", C.c_double), ("t0", C.c_double),
        ("t_max", C.c_double), ("tol", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double),
        ("fft_every", C.c_double), ("use_fft_mask", C.c_int32), ("n_pump", C.c_int32), ("n_potential", C.c_int32),
        ("n_pulse", C.c_int32), ("pump_t", Temporal * MAX_GROUPS), ("potential_t", Temporal * MAX_GROUPS),
        ("pulse_t", Temporal * MAX_GROUPS), ("stochastic_amplitude", C.c_double), ("seed", C.c_uint64),
        ("imag_time_amplitude", C.c_double),
    ]


class Derived(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("dx", "dy", "dV", "one_over_dx2", "one_over_dy2", "m2_over_dx2_p_dy2",
                                           "m_eff_scaled", "one_over_h_bar_s")]


class Result(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("steps", C.c_int64), ("accepted", C.c_int64),
                ("rejected", C.c_int64), ("fft_applied", C.c_int64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
        _lib = C.CDLL(LIB_PATH)
        for sfx in ("f64", "f32"):
            fn = getattr(_lib, f"phx_oracle_run_{sfx}")
            fn.restype = C.c_int
            fn.argtypes = [C.POINTER(Params)] + [C.c_void_p] * 12 + [C.c_int64, C.POINTER(Result)]
            d = getattr(_lib, f"phx_oracle_derive_{sfx}")
            d.restype = None
            d.argtypes = [C.POINTER(Params), C.POINTER(Derived)]
    return _lib


def _temporal(spec):
    t = Temporal()
    if spec is None or spec[0] == "constant":
        t.kind = 0
    else:
        t.kind, t.t0, t.sigma, t.freq = TEMPORAL[spec[0]], float(spec[1]), float(spec[2]), float(spec[3])
    return t


def make_params(case):
    p = Params()
    for k in ("N_c", "N_r"):
        setattr(p, k, int(case[k]))
    for k in ("L_x", "L_y", "h_bar_s", "m_eff", "gamma_c", "gamma_r", "g_c", "g_r", "R", "g_pm", "delta_LT", "dt",
              "t_max"):
        setattr(p, k, float(case[k]))
    p.t0 = float(case.get("t0", 0.0))
    p.tol = float(case.get("tol", 0.1))
    p.dt_min = float(case.get("dt_min", 1e-4))
    p.dt_max = float(case.get("dt_max", 3.0))
    p.fft_every = float(case.get("fft_every", 1e9))
    p.periodic_x, p.periodic_y = int(case["periodic_x"]), int(case["periodic_y"])
    p.tetm = int(case.get("tetm", 0))
    npump = len(case.get("pumps", []))
    p.use_reservoir = int(npump > 0 or bool(case.get("n0_amp", 0.0)))
    p.iterator = ITERATORS[case["iterator"].upper()]
    p.adaptive = int(case.get("adaptive", 0))
    p.use_fft_mask = int(bool(case.get("mask_cut")))
    p.stochastic_amplitude = float(case.get("dw", 0.0))
    p.seed = int(case.get("seed", 0))
    p.imag_time_amplitude = float(case.get("imag_time", 0.0))
    p.n_pump, p.n_potential, p.n_pulse = npump, len(case.get("potentials", [])), len(case.get("pulses", []))
    for fam, n in (("pump", p.n_pump), ("potential", p.n_potential), ("pulse", p.n_pulse)):
        specs = case.get(f"{fam}_t", [None] * n)
        arr = getattr(p, f"{fam}_t")
        for g in range(n):
            arr[g] = _temporal(specs[g] if g < len(specs) else None)
    return p


def derive(case, dtype="f64"):
    p = make_params(case)
    d = Derived()
    getattr(lib(), f"phx_oracle_derive_{dtype}")(C.byref(p), C.byref(d))
    return {n: getattr(d, n) for n, _ in Derived._fields_}


def _cplx(a, real_t):
    a = np.asarray(a, dtype=np.complex128)
    out = np.empty(a.shape + (2,), dtype=real_t)
    out[..., 0] = a.real
    out[..., 1] = a.imag
    return np.ascontiguousarray(out)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def run(case, fields, max_steps=1 << 62):
    """fields: dict with psi_plus[, psi_minus, n_plus, n_minus, pump_g, potential_g, pulse_g, fft_mask]."""
    dtype = case["dtype"]
    real_t = np.float64 if dtype == "f64" else np.float32
    p = make_params(case)
    shape = (int(case["N_r"]), int(case["N_c"]))
    zeros = np.zeros(shape, dtype=np.complex128)
    psi_p = _cplx(fields["psi_plus"], real_t)
    n_p = _cplx(fields.get("n_plus", zeros), real_t)
    psi_m = n_m = None
    if p.tetm:
        psi_m = _cplx(fields["psi_minus"], real_t)
        n_m = _cplx(fields.get("n_minus", zeros), real_t)

    def stack(prefix, n, cplx):
        if n == 0:
            return None
        arrs = [np.asarray(fields[f"{prefix}_{g}"]) for g in range(n)]
        if cplx:
            return np.ascontiguousarray(np.stack([_cplx(a, real_t) for a in arrs]))
        return np.ascontiguousarray(np.stack([np.real(a).astype(real_t) for a in arrs]))

    pump = stack("pump", p.n_pump, False)
    pot = stack("potential", p.n_potential, False)
    pulse = stack("pulse", p.n_pulse, True)
    mask = None
    if p.use_fft_mask:
        mask = np.ascontiguousarray(np.real(fields["fft_mask"]).astype(real_t))
    res = Result()
    fn = getattr(lib(), f"phx_oracle_run_{dtype}")
    rc = fn(C.byref(p), _ptr(psi_p), _ptr(n_p), _ptr(psi_m), _ptr(n_m), _ptr(pump), None, _ptr(pot), None,
            _ptr(pulse), None, _ptr(mask), None, C.c_int64(max_steps), C.byref(res))
    if rc != 0:
        raise RuntimeError(f"oracle returned {rc}")
    out = {"psi_plus": psi_p[..., 0] + 1j * psi_p[..., 1], "n_plus": n_p[..., 0] + 1j * n_p[..., 1]}
    if p.tetm:
        out["psi_minus"] = psi_m[..., 0] + 1j * psi_m[..., 1]
        out["n_minus"] = n_m[..., 0] + 1j * n_m[..., 1]
    rec = {n: getattr(res, n) for n, _ in Result._fields_}
    return out, rec


def fields_from_golden(z):
    """Input fields of a tests/golden/*.npz fixture."""
    f = {}
    for k in z.files:
        if k.startswith("in_"):
            f[k[3:]] = z[k]
    return f
