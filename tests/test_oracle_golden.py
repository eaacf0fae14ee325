"""The C restatement oracle (oracle/phx_oracle.c) against the reference's own
outputs (tests/golden/*.npz, produced by tests/golden/make_golden.py from the
PHOENIX CPU build).  FP64 and FP32 must agree bit for bit: the oracle keeps
the reference's operand order and is compiled without FMA contraction, like
the reference binary."""
import glob
import json
import os

import numpy as np
import pytest

from oracle import phx_oracle as O

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
OUT_KEYS = ("psi_plus", "n_plus", "psi_minus", "n_minus")


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_bitwise(path):
    z = np.load(path)
    case = json.loads(str(z["params"]))
    out, rec = O.run(case, O.fields_from_golden(z))
    checked = 0
    for k in OUT_KEYS:
        gk = "out_" + k
        if gk in z.files and k in out:
            np.testing.assert_array_equal(out[k], z[gk], err_msg=f"{k} differs from the reference")
            checked += 1
    assert checked >= 1
    assert rec["steps"] > 0


def test_oracle_derived_constants_match_calculate_auto():
    case = dict(N_c=64, N_r=32, L_x=100.0, L_y=50.0, h_bar_s=0.6582, m_eff=3.184, gamma_c=0.15, gamma_r=0.225,
                g_c=6e-6, g_r=1.2e-5, R=0.01, g_pm=0.0, delta_LT=0.0, dt=0.01, t_max=1.0, periodic_x=1,
                periodic_y=1, iterator="RK4", dtype="f64")
    d = O.derive(case, "f64")
    dx = 100.0 / 63
    dy = 50.0 / 31
    assert d["dx"] == dx and d["dy"] == dy
    assert d["one_over_dx2"] == 1.0 / (dx * dx)
    assert d["m2_over_dx2_p_dy2"] == -2.0 * (1.0 / (dx * dx) + 1.0 / (dy * dy))
    assert d["m_eff_scaled"] == -0.5 * 0.6582 * 0.6582 / 3.184
    assert d["one_over_h_bar_s"] == 1.0 / 0.6582
    f = O.derive(case, "f32")
    assert f["dx"] == float(np.float32(np.float32(100.0) / np.float32(63)))


def test_oracle_rk4_is_deterministic_and_subgrid_free():
    """Running 2 x 5 iterations equals 10 iterations (no hidden state)."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "rk4_f64_periodic.npz"))
    case = json.loads(str(z["params"]))
    f = O.fields_from_golden(z)
    a, _ = O.run(case, f, max_steps=10)
    b, _ = O.run(case, f, max_steps=5)
    f2 = dict(f, psi_plus=b["psi_plus"], n_plus=b["n_plus"])
    case2 = dict(case, t0=5 * case["dt"])
    c, _ = O.run(case2, f2, max_steps=5)
    np.testing.assert_allclose(c["psi_plus"], a["psi_plus"], rtol=0, atol=1e-13)
