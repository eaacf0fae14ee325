"""Imaginary-time propagation (--imagTime) on the GPU.

The reference golden fixtures (imag_*.npz) run through tests/test_gpu_parity.py;
here:
* larger grids against the oracle (RK4 and a fixed tableau, both norm modes);
* the interior norm mode keeps sum |psi|^2 dV = A after every iteration;
* a non-interacting condensate in a harmonic trap relaxes to the Gaussian
  ground state exp(-r^2 / (2 a^2)), a^2 = hbar / (m omega);
* SSFM with a reservoir: both fields normalised, against the oracle.
"""
import numpy as np
import pytest

import phoenix_b200 as pb
from oracle import phx_oracle as O

pytestmark = pytest.mark.gpu

STRONG = dict(h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.05, g_r=0.08, R=0.04, g_pm=-0.01,
              delta_LT=0.3)


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def case_of(n, iterator, dtype, steps, dt, px, py, **kw):
    c = dict(N_c=n, N_r=n, L_x=40.0, L_y=40.0, **STRONG, dtype=dtype, iterator=iterator, dt=dt,
             t_max=steps * dt * (1 - 1e-9), periodic_x=px, periodic_y=py, seed=7, imag_time=2.5,
             potentials=[0.2])
    c.update(kw)
    return c


def fields_of(case, rng):
    n_r, n_c = case["N_r"], case["N_c"]
    f = {"psi_plus": rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c)),
         "potential_0": 0.2 * rng.standard_normal((n_r, n_c)) + 0j}
    if case.get("pumps"):
        f["pump_0"] = np.full((n_r, n_c), 0.5) + 0j
        f["n_plus"] = rng.random((n_r, n_c)) + 0j
    return f


def run_gpu(case, fields, **over):
    sp = pb.system_from_case(case, **over)
    with pb.SolverFactory.create(sp) as s:
        pb.load_case_fields(s, case, fields)
        info = s.run()
        out = {"psi_plus": s.get_field("psi_plus")}
        if sp.use_reservoir:
            out["n_plus"] = s.get_field("n_plus")
        return out, info


@pytest.mark.parametrize("iterator,px,py", [("RK4", 1, 1), ("RK4", 0, 1), ("Heun3", 0, 0), ("NSRK78", 1, 0)])
def test_imaginary_time_matches_oracle_fp64(require_gpu, iterator, px, py):
    case = case_of(128, iterator, "f64", 40, 0.005, px, py)
    fields = fields_of(case, np.random.default_rng(1))
    out, info = run_gpu(case, fields)
    ref, rec = O.run(case, fields)
    assert info.iterations == rec["steps"] == 40
    assert rel_l2(out["psi_plus"], ref["psi_plus"]) < 1e-12


def test_interior_norm_mode_keeps_the_norm(require_gpu):
    case = case_of(96, "RK4", "f64", 25, 0.005, 0, 0)
    fields = fields_of(case, np.random.default_rng(2))
    out, _ = run_gpu(case, fields, norm_mode="interior")
    dV = (40.0 / 95) ** 2
    assert abs(np.sum(np.abs(out["psi_plus"]) ** 2) * dV - 2.5) < 1e-12 * 2.5
    # the reference mode counts the halo rings as well: a smaller interior norm
    out_ref, _ = run_gpu(case, fields)
    assert np.sum(np.abs(out_ref["psi_plus"]) ** 2) * dV < 2.5


def test_harmonic_trap_relaxes_to_gaussian_ground_state(require_gpu):
    hbar, m, a = 0.6582, 3.184, 2.0
    omega = hbar / (m * a * a)
    n, L = 128, 30.0
    x = -L / 2 + L / (n - 1) * np.arange(n)
    X, Y = np.meshgrid(x, x)
    V = 0.5 * m * omega ** 2 * (X ** 2 + Y ** 2)
    sp = pb.SystemParameters(N_c=n, N_r=n, L_x=L, L_y=L, h_bar_s=hbar, m_eff=m, gamma_c=0.0, gamma_r=0.0, g_c=0.0,
                             g_r=0.0, R=0.0, g_pm=0.0, delta_LT=0.0, use_reservoir=False, dtype="f64",
                             iterator="RK4", dt=0.1, t_max=1e9, fft_every=1e12, imag_time_amplitude=1.0,
                             potential_temporal=[pb.Temporal()], norm_mode="interior")
    rng = np.random.default_rng(3)
    with pb.Solver(sp) as s:
        s.set_field("psi_plus", np.exp(-((X - 1.0) ** 2 + Y ** 2) / 20.0) * (1 + 0.2 * rng.random((n, n))))
        s.set_field("potential_plus", V, 0)
        s.run(4000)
        psi = s.get_field("psi_plus")
    g = np.exp(-(X ** 2 + Y ** 2) / (2 * a * a))
    overlap = abs(np.vdot(g, psi)) / (np.linalg.norm(g) * np.linalg.norm(psi))
    print("ground-state overlap", overlap)
    assert overlap > 1 - 1e-4
    dV = (L / (n - 1)) ** 2
    assert abs(np.sum(np.abs(psi) ** 2) * dV - 1.0) < 1e-12


def test_ssfm_imaginary_time_normalises_both_fields(require_gpu):
    case = case_of(64, "SSFM", "f64", 20, 0.01, 1, 1, pumps=[(0.5, 1.0, 0.0)])
    fields = fields_of(case, np.random.default_rng(4))
    out, _ = run_gpu(case, fields)
    dV = (40.0 / 63) ** 2
    assert abs(np.sum(np.abs(out["psi_plus"]) ** 2) * dV - 2.5) < 1e-12 * 2.5
    assert abs(np.sum(out["n_plus"] ** 2) * dV - 2.5) < 1e-12 * 2.5
    ref, _ = O.run(case, fields)
    assert rel_l2(out["psi_plus"], ref["psi_plus"]) < 1e-11
    assert rel_l2(out["n_plus"], np.real(ref["n_plus"])) < 1e-11
