"""SSFM on the GPU against the oracle (tests/test_ssfm.py pins the oracle's
split step to the closed-form linear solution; the reference's own SSFM
build crashes).  cuFFT and CUDA's exp / sin / cos against the oracle's
radix-2 DFT and glibc: agreement to rounding."""
import numpy as np
import pytest

import phoenix_b200 as pb
from oracle import phx_oracle as O

pytestmark = pytest.mark.gpu

STRONG = dict(h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.05, g_r=0.08, R=0.04, g_pm=-0.01,
              delta_LT=0.3)


def case_fields(dtype, n_c=32, n_r=32, tetm=False, seed=0, **extra):
    rng = np.random.default_rng(seed)
    L_x, L_y = 20.0, 20.0 * n_r / n_c
    case = dict(N_c=n_c, N_r=n_r, L_x=L_x, L_y=L_y, **STRONG, dtype=dtype, iterator="SSFM", dt=0.005,
                t_max=20 * 0.005 * (1 - 1e-9), periodic_x=1, periodic_y=1, n0_amp=0.5, tetm=int(tetm),
                pumps=[(4.0, 3.0, 0.0)], potentials=[0.2], pulses=[(1.0, 3.0)],
                pulse_t=[("iexp", 0.05, 0.1, 5.0)], **extra)
    comps = ["plus", "minus"] if tetm else ["plus"]
    f = {"pump_0": 4.0 * rng.random((n_r, n_c)), "potential_0": 0.2 * rng.standard_normal((n_r, n_c)),
         "pulse_0": rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c))}
    for c in comps:
        f[f"psi_{c}"] = rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c))
        f[f"n_{c}"] = 0.5 * rng.random((n_r, n_c))
    return case, f


def compare(case, fields, tol):
    sp = pb.system_from_case(case)
    with pb.SolverFactory.create(sp) as s:
        pb.load_case_fields(s, case, fields)
        info = s.run()
        out = {k: s.get_field(k) for k in (["psi_plus", "n_plus"] + (["psi_minus", "n_minus"] if sp.use_twin_mode else []))}
    ref, rec = O.run(case, fields)
    assert info.iterations == rec["steps"] >= 20
    assert info.kernel_launches > 0
    for k, v in out.items():
        want = ref[k] if k.startswith("psi") else np.real(ref[k])
        err = np.linalg.norm(v - want) / np.linalg.norm(want)
        assert err <= tol, (k, err)


@pytest.mark.parametrize("shape", [(32, 32), (40, 24)])
def test_ssfm_fp64_matches_oracle(require_gpu, shape):
    compare(*case_fields("f64", *shape, seed=1), tol=1e-11)


def test_ssfm_fp64_noise_matches_oracle(require_gpu):
    compare(*case_fields("f64", seed=2, dw=0.05), tol=1e-11)


def test_ssfm_tetm_fp64_matches_oracle(require_gpu):
    compare(*case_fields("f64", tetm=True, seed=3, dw=0.02), tol=1e-11)


def test_ssfm_fp32_matches_oracle(require_gpu):
    compare(*case_fields("f32", seed=4), tol=2e-5)
