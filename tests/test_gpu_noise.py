"""Stochastic noise on the GPU, bit for bit against the oracle.

The kernels draw the noise of every point and iteration from the same
counter-based generator as the oracle (Philox4x32-10 + Box-Muller with
separately rounded series), add the stochastic drift to the right-hand side
and the dw term to every stage sum, so noisy runs are compared exactly; the
statistical link to the reference is tests/test_noise.py.
"""
import json
import os

import numpy as np
import pytest

import phoenix_b200 as pb
from oracle import phx_oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return json.loads(str(z["params"])), O.fields_from_golden(z)


def run_gpu(case, fields, steps=None):
    sp = pb.system_from_case(case)
    with pb.Solver(sp) as s:
        pb.load_case_fields(s, case, fields)
        info = s.run() if steps is None else s.run(steps)
        comps = ["plus", "minus"] if sp.use_twin_mode else ["plus"]
        out = {}
        for c in comps:
            out[f"psi_{c}"] = s.get_field(f"psi_{c}")
            if sp.use_reservoir:
                out[f"n_{c}"] = s.get_field(f"n_{c}")
        return out, info


CASES = {
    "rk4_f64_periodic": dict(dw=0.05, seed=3),
    "rk4_f32_periodic": dict(dw=0.05, seed=4),
    "rk4_f64_zero": dict(dw=0.05, seed=5),
    "rk4_f64_mixed_rect": dict(dw=0.05, seed=6),
    "rk4_f64_nores": dict(dw=0.05, seed=7),
    "tetm_f64_periodic": dict(dw=0.05, seed=8),
    "tetm_f64_zero": dict(dw=0.05, seed=9),
    "dp45_f64_fixed": dict(dw=0.05, seed=10),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_noise_matches_oracle_bitwise(require_gpu, name):
    case, fields = load(name)
    case.update(CASES[name])
    out, info = run_gpu(case, fields)
    ref, rec = O.run(case, fields)
    assert info.iterations == rec["steps"]
    quiet, _ = O.run(dict(case, dw=0.0), fields)
    assert not np.array_equal(ref["psi_plus"], quiet["psi_plus"])  # the noise is on
    for k in out:
        want = ref[k] if k.startswith("psi") else np.real(ref[k])
        np.testing.assert_array_equal(out[k], want, err_msg=f"{name}: {k}")


def test_gpu_noise_dp45_adaptive_matches_oracle(require_gpu):
    """Adaptive DP45 with noise: the noise enters the stage values whose
    halo-padded norm steers dt, so the error control must see it too."""
    case, fields = load("dp45_f64_adaptive")
    case.update(dw=0.02, seed=11)
    out, info = run_gpu(case, fields)
    ref, rec = O.run(case, fields)
    assert info.iterations == rec["steps"]
    assert (info.accepted, info.rejected) == (rec["accepted"], rec["rejected"])
    for k in out:
        want = ref[k] if k.startswith("psi") else np.real(ref[k])
        err = float(np.linalg.norm(out[k] - want) / np.linalg.norm(want))
        assert err <= 1e-12, (k, err)


def test_gpu_noise_does_not_depend_on_launch_shape(require_gpu, monkeypatch):
    case, fields = load("rk4_f32_periodic")
    case.update(dw=0.05, seed=12)
    outs = []
    for shape in range(4):
        monkeypatch.setenv("PHX_STAGE_SHAPE", str(shape))
        outs.append(run_gpu(case, fields)[0])
    for o in outs[1:]:
        for k in o:
            np.testing.assert_array_equal(o[k], outs[0][k])


def test_gpu_noise_iteration_counter_continues_across_calls(require_gpu):
    """Noise is keyed by the iteration count of the handle, so 10 + 30
    iterations equal 40 in one call."""
    case, fields = load("rk4_f64_periodic")
    case.update(dw=0.05, seed=13)
    one, _ = run_gpu(case, fields, steps=40)
    sp = pb.system_from_case(case)
    with pb.Solver(sp) as s:
        pb.load_case_fields(s, case, fields)
        s.run(10)
        s.run(30)
        np.testing.assert_array_equal(s.get_field("psi_plus"), one["psi_plus"])
