"""The one-kernel RK4 iterations of the TE/TM spinor (rk4_tetm_fused_kernel) and
of the scalar model beyond the TMA iteration (rk4_scalar_general_kernel), the defaults,
against the per-stage kernels (PHX_TETM_FUSED=0, PHX_GENERAL_FUSED=0), which the
reference fixtures also pin (tests/test_gpu_parity.py): bit-identical fields on grids that are not
multiples of the tile, for both boundary kinds, several pump / potential /
pulse groups with time dependence, and stochastic noise."""
import numpy as np
import pytest

import phoenix_b200 as pb

pytestmark = pytest.mark.gpu

STRONG = dict(h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.05, g_r=0.08, R=0.04, g_pm=-0.01,
              delta_LT=0.3)


def make(n_c, n_r, dtype, px, py, dw):
    case = dict(N_c=n_c, N_r=n_r, L_x=30.0, L_y=30.0 * n_r / n_c, **STRONG, dtype=dtype, iterator="RK4", tetm=1,
                dt=0.005, t_max=1e9, periodic_x=px, periodic_y=py, seed=5, dw=dw,
                pumps=[(4.0, 3.0, 0.0), (2.0, 2.0, 1.0)], pump_t=[None, ("cos", 0.05, 0.3, 20.0)],
                potentials=[0.2, 0.1], potential_t=[("gauss", 0.02, 0.1, 1.0), None],
                pulses=[(1.0, 3.0)], pulse_t=[("iexp", 0.03, 0.05, 5.0)])
    rng = np.random.default_rng(11)
    f = {}
    for c in ("plus", "minus"):
        f[f"psi_{c}"] = rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c))
        f[f"n_{c}"] = rng.random((n_r, n_c))
    for g in range(2):
        f[f"pump_{g}"] = 3.0 * rng.random((n_r, n_c))
        f[f"potential_{g}"] = 0.2 * rng.standard_normal((n_r, n_c))
    f["pulse_0"] = 0.5 * (rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c)))
    return case, f


def run(case, fields, iters):
    sp = pb.system_from_case(case)
    with pb.Solver(sp) as s:
        pb.load_case_fields(s, case, fields)
        info = s.run(iters)
        return {k: s.get_field(k) for k in ("psi_plus", "psi_minus", "n_plus", "n_minus")}, info


@pytest.mark.parametrize("dtype,px,py,dw", [("f32", 1, 1, 0.0), ("f32", 0, 1, 0.02), ("f64", 1, 0, 0.0),
                                            ("f64", 0, 0, 0.02)])
def test_fused_tetm_iteration_matches_stage_kernels(require_gpu, monkeypatch, dtype, px, py, dw):
    case, fields = make(70, 46, dtype, px, py, dw)
    monkeypatch.setenv("PHX_TETM_FUSED", "1")
    fused, info = run(case, fields, 12)
    # one kernel per iteration, plus the ring refills of zero axes after each
    assert info.iterations == 12 and info.kernel_launches <= 12 * 5
    monkeypatch.setenv("PHX_TETM_FUSED", "0")
    staged, _ = run(case, fields, 12)
    for k in fused:
        np.testing.assert_array_equal(fused[k], staged[k], err_msg=k)


def make_scalar(n_c, n_r, dtype, px, py, dw, reservoir):
    case, f = make(n_c, n_r, dtype, px, py, dw)
    case.pop("tetm")
    case["potential_t"] = [("iexp", 0.02, 0.1, 4.0), None]  # a complex potential coefficient
    if not reservoir:
        case["pumps"], case["pump_t"] = [], []
        f.pop("n_plus")
    return case, f


def run_scalar(case, fields, iters):
    sp = pb.system_from_case(case)
    with pb.Solver(sp) as s:
        pb.load_case_fields(s, case, fields)
        info = s.run(iters)
        out = {"psi_plus": s.get_field("psi_plus")}
        if sp.use_reservoir:
            out["n_plus"] = s.get_field("n_plus")
        return out, info


@pytest.mark.parametrize("dtype,px,py,dw,res", [("f32", 1, 1, 0.02, True), ("f32", 0, 1, 0.0, False),
                                                ("f64", 1, 0, 0.02, True), ("f64", 0, 0, 0.02, False)])
def test_general_scalar_iteration_matches_stage_kernels(require_gpu, monkeypatch, dtype, px, py, dw, res):
    """Scalar runs the TMA iteration does not take (noise, pulses, two pump and
    potential groups, a complex temporal coefficient) run one kernel per
    iteration (rk4_scalar_general_kernel): the same bits as the stage kernels."""
    case, fields = make_scalar(70, 46, dtype, px, py, dw, res)
    monkeypatch.setenv("PHX_GENERAL_FUSED", "1")
    fused, info = run_scalar(case, fields, 12)
    assert info.iterations == 12 and info.kernel_launches <= 12 * 3
    monkeypatch.setenv("PHX_GENERAL_FUSED", "0")
    staged, info2 = run_scalar(case, fields, 12)
    assert info2.kernel_launches >= 12 * 4
    for k in fused:
        np.testing.assert_array_equal(fused[k], staged[k], err_msg=k)
