"""The Dormand-Prince 5(4) attempt in one launch (dp45_fused_kernel) against
the k-stack stage kernels (PHX_DP45_FUSED=0) and the oracle.

The one-kernel attempt evaluates every point with the stage kernels'
operations in their order, so after an accepted step the state is
bit-identical; the FP64 error and norm sums are added in another order, so
later step sizes agree to rounding.  Grids that are not multiples of the
32 x 16 tile, zero / periodic / mixed boundaries (the zero axes exercise the
extended stage regions and the reference-norm rings that edge tiles add),
FP32 and FP64, both norm modes.
"""
import ctypes as C

import numpy as np
import pytest

import phoenix_b200 as pb
from phoenix_b200 import _lib as L
from oracle import phx_oracle as O

pytestmark = pytest.mark.gpu

STRONG = dict(h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.05, g_r=0.08, R=0.04, g_pm=0.0,
              delta_LT=0.0)


def case(n_c, n_r, px, py, dtype, t_max, seed):
    return dict(N_c=n_c, N_r=n_r, L_x=0.25 * n_c, L_y=0.25 * n_r, **STRONG, dtype=dtype, iterator="DP45", adaptive=1,
                tol=1e-6, dt_min=1e-5, dt_max=0.05, dt=0.01, t_max=t_max, periodic_x=px, periodic_y=py, seed=seed,
                pumps=[(4.0, 3.0, 0.0)], potentials=[0.2])


def fields(c):
    rng = np.random.default_rng(c["seed"])
    n_r, n_c = c["N_r"], c["N_c"]
    x = -c["L_x"] / 2 + c["L_x"] / (n_c - 1) * np.arange(n_c)
    y = -c["L_y"] / 2 + c["L_y"] / (n_r - 1) * np.arange(n_r)
    X, Y = np.meshgrid(x, y)
    return {"psi_plus": rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c)),
            "pump_0": 4.0 * np.exp(-(X ** 2 + Y ** 2) / 18.0),
            "potential_0": 0.2 * rng.standard_normal((n_r, n_c))}


def run(c, f, monkeypatch, fused, iterations=None, norm="reference"):
    monkeypatch.setenv("PHX_DP45_FUSED", "1" if fused else "0")
    sp = pb.system_from_case(c, norm_mode=norm)
    with pb.SolverFactory.create(sp) as s:
        pb.load_case_fields(s, c, f)
        s.profile(True)
        info = s.run(iterations) if iterations else s.run()
        prof = s.profile_read()
        return s.get_field("psi_plus"), s.get_field("n_plus"), info, prof


BCS = [(1, 1), (0, 0), (1, 0), (0, 1)]


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("bc", BCS, ids=["periodic", "zero", "px_zy", "zx_py"])
def test_first_accepted_step_bit_identical_to_stage_kernels(require_gpu, monkeypatch, dtype, bc):
    c = case(70, 50, bc[0], bc[1], dtype, 1e9, 31)
    f = fields(c)
    a = run(c, f, monkeypatch, True, 1)
    b = run(c, f, monkeypatch, False, 1)
    assert "dp45_fused" in a[3] and "dp45_fused" not in b[3]
    assert (a[2].accepted, a[2].rejected) == (b[2].accepted, b[2].rejected)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2].dt == pytest.approx(b[2].dt, rel=1e-12 if dtype == "f64" else 1e-5)


@pytest.mark.parametrize("bc", BCS, ids=["periodic", "zero", "px_zy", "zx_py"])
def test_adaptive_run_matches_oracle(require_gpu, monkeypatch, bc):
    c = case(100, 68, bc[0], bc[1], "f64", 0.3, 32)
    f = fields(c)
    psi, nres, info, prof = run(c, f, monkeypatch, True)
    assert prof["dp45_fused"]["launches"] == info.accepted + info.rejected
    ref, rec = O.run(c, f)
    assert (info.iterations, info.accepted, info.rejected) == (rec["steps"], rec["accepted"], rec["rejected"])
    for got, want in ((psi, ref["psi_plus"]), (nres, np.real(ref["n_plus"]))):
        assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)


def test_interior_norm_mode_matches_stage_kernels(require_gpu, monkeypatch):
    c = case(64, 48, 0, 1, "f64", 0.2, 33)
    f = fields(c)
    a = run(c, f, monkeypatch, True, norm="interior")
    b = run(c, f, monkeypatch, False, norm="interior")
    assert (a[2].accepted, a[2].rejected) == (b[2].accepted, b[2].rejected)
    assert np.linalg.norm(a[0] - b[0]) <= 1e-12 * np.linalg.norm(b[0])


def test_complex_potential_envelope_falls_back_to_stage_kernels(require_gpu, monkeypatch):
    """An iexp potential envelope makes the temporal coefficient complex: those
    attempts run on the stage kernels (same results as with the switch off)."""
    c = case(64, 32, 1, 1, "f64", 0.1, 34)
    c["potential_t"] = [("iexp", 0.0, 0.5, 10.0)]
    f = fields(c)
    a = run(c, f, monkeypatch, True)
    b = run(c, f, monkeypatch, False)
    assert "dp45_fused" not in a[3]
    np.testing.assert_array_equal(a[0], b[0])


@pytest.mark.parametrize("bc", [(1, 1), (0, 0)], ids=["periodic", "zero"])
def test_forced_fixed_steps_between_fused_attempts(require_gpu, monkeypatch, bc):
    """phx_iterate(force_fixed_time_step) runs a fixed DP45 step on the stage
    kernels (the main loop's step onto an output time), which write the state's
    periodic images four deep; the next one-kernel attempt reads seven.  Mixed
    sequences agree with the stage kernels alone to the rounding of the FP64
    norm sums (which set later step sizes); images left stale three rings deep
    would differ by about dt times the right-hand side."""
    c = case(66, 40, bc[0], bc[1], "f64", 1e9, 35)
    f = fields(c)
    outs = []
    for fused in (True, False):
        monkeypatch.setenv("PHX_DP45_FUSED", "1" if fused else "0")
        sp = pb.system_from_case(c)
        with pb.SolverFactory.create(sp) as s:
            pb.load_case_fields(s, c, f)
            for k in range(9):
                info = L.StepInfo()
                L.check(s._lib.phx_iterate(s._h, 1 if k % 3 == 2 else 0, C.byref(info)), s._h)
            outs.append((s.get_field("psi_plus"), s.get_field("n_plus"), s.t, s.dt))
    for a, b in ((outs[0][0], outs[1][0]), (outs[0][1], outs[1][1])):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-10 * np.abs(b).max())
    assert outs[0][2] == pytest.approx(outs[1][2], rel=1e-12)
    assert outs[0][3] == pytest.approx(outs[1][3], rel=1e-10)
