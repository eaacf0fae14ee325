"""The other registered iterators on the GPU (generic k-stack stage kernels)
against the oracle, bit for bit: every tableau on a zero/periodic mixed grid
in FP64 and FP32, TE/TM and noise through a tableau, and every stage launch
shape.  The reference's own outputs for ten of them are the golden fixtures
tests/golden/tab_*.npz (replayed by test_gpu_parity.py)."""
import numpy as np
import pytest

import phoenix_b200 as pb
from oracle import phx_oracle as O

pytestmark = pytest.mark.gpu

ITERS = ["RK3", "SSPRK3", "MP", "Heun2", "Heun3", "HW", "Newton", "Nystroem", "Ralston", "Ralston3", "Ralston4",
         "Rule38"]
STRONG = dict(h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.05, g_r=0.08, R=0.04, g_pm=-0.01,
              delta_LT=0.3)


def case_fields(it, dtype, tetm=False, px=1, py=0, seed=0, **extra):
    n_c, n_r, L_x, L_y = 40, 32, 25.0, 20.0
    rng = np.random.default_rng(seed)
    x = -L_x / 2 + L_x / (n_c - 1) * np.arange(n_c)
    y = -L_y / 2 + L_y / (n_r - 1) * np.arange(n_r)
    X, Y = np.meshgrid(x, y)
    case = dict(N_c=n_c, N_r=n_r, L_x=L_x, L_y=L_y, **STRONG, dtype=dtype, iterator=it, dt=0.005,
                t_max=15 * 0.005 * (1 - 1e-9), periodic_x=px, periodic_y=py, n0_amp=0.5, tetm=int(tetm),
                pumps=[(4.0, 3.0, 0.0)], potentials=[0.2], **extra)
    comps = ["plus", "minus"] if tetm else ["plus"]
    f = {"pump_0": 4.0 * np.exp(-(X ** 2 + Y ** 2) / 18.0), "potential_0": 0.2 * rng.standard_normal((n_r, n_c))}
    for c in comps:
        f[f"psi_{c}"] = rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c))
        f[f"n_{c}"] = 0.5 * rng.random((n_r, n_c))
    return case, f


def run_gpu(case, fields):
    sp = pb.system_from_case(case)
    with pb.SolverFactory.create(sp) as s:
        pb.load_case_fields(s, case, fields)
        info = s.run()
        comps = ["plus", "minus"] if sp.use_twin_mode else ["plus"]
        out = {}
        for c in comps:
            out[f"psi_{c}"] = s.get_field(f"psi_{c}")
            out[f"n_{c}"] = s.get_field(f"n_{c}")
        return out, info


def check(case, fields):
    out, info = run_gpu(case, fields)
    ref, rec = O.run(case, fields)
    # 15 steps of dt (FP32 accumulates t in float and may take a 16th, as the reference does)
    assert info.iterations == rec["steps"] >= 15
    for k, v in out.items():
        np.testing.assert_array_equal(v, ref[k] if k.startswith("psi") else np.real(ref[k]), err_msg=k)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("it", ITERS)
def test_tableau_matches_oracle(require_gpu, it, dtype):
    check(*case_fields(it, dtype, seed=hash(it) % 1000))


@pytest.mark.parametrize("it", ["Heun3", "Nystroem", "RK3"])
def test_tableau_tetm_matches_oracle(require_gpu, it):
    check(*case_fields(it, "f64", tetm=True, px=0, py=0, seed=5))


@pytest.mark.parametrize("it", ["SSPRK3", "Rule38"])
def test_tableau_noise_matches_oracle(require_gpu, it):
    check(*case_fields(it, "f64", px=1, py=1, seed=6, dw=0.05))


@pytest.mark.parametrize("shape", [0, 1, 2, 3])
def test_tableau_every_launch_shape(require_gpu, shape, monkeypatch):
    monkeypatch.setenv("PHX_STAGE_SHAPE", str(shape))
    check(*case_fields("Nystroem", "f32", px=0, py=1, seed=7))


ADAPTIVE = ["DP45", "BoSha", "CashKarp", "Fehlberg2", "Fehlberg5", "DP85", "NSRK78"]


def check_adaptive(case, fields, tol=1e-12):
    out, info = run_gpu(case, fields)
    ref, rec = O.run(case, fields)
    assert info.iterations == rec["steps"]
    assert (info.accepted, info.rejected) == (rec["accepted"], rec["rejected"])
    for k, v in out.items():
        want = ref[k] if k.startswith("psi") else np.real(ref[k])
        err = float(np.linalg.norm(v - want) / np.linalg.norm(want))
        assert err <= tol, (k, err)


@pytest.mark.parametrize("it", ADAPTIVE)
@pytest.mark.parametrize("bc", [(0, 0), (1, 0)])
def test_adaptive_tableau_matches_oracle(require_gpu, it, bc):
    """Adaptive stepping through the halo-padded reference norm (rings up to
    H = 13 for NSRK78 on zero boundaries); the norms are summed in FP64 here
    and in the build precision by the reference, so results agree to 1e-12."""
    case, f = case_fields(it, "f64", px=bc[0], py=bc[1], seed=11, adaptive=1, tol=1e-6, dt_min=1e-5, dt_max=0.05)
    case["t_max"] = 0.1
    check_adaptive(case, f)


@pytest.mark.parametrize("it", ["DP85", "NSRK78", "CashKarp"])
def test_adaptive_tableau_fixed_dt_matches_oracle(require_gpu, it):
    check(*case_fields(it, "f64", px=0, py=0, seed=12))


@pytest.mark.parametrize("it", ["BoSha", "Fehlberg5"])
def test_adaptive_tableau_tetm_and_noise(require_gpu, it):
    case, f = case_fields(it, "f64", tetm=True, px=1, py=1, seed=13, adaptive=1, tol=1e-6, dt_min=1e-5, dt_max=0.05,
                          dw=0.02)
    case["t_max"] = 0.08
    check_adaptive(case, f)
