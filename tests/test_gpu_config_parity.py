"""GPU parity at the benchmark configurations' own sizes, through the C ABI.

Cases and reference digests: tests/golden/config_cases.py and
config_digests.json (the reference binary's outputs, hashed).
- Fixed-step cases without a k-space filter (1024^2 scalar FP32 with disorder;
  TE/TM 1024^2 FP64 and FP32, 4096^2 FP32): the library's outputs hash to the
  reference's SHA-256, i.e. they are bit-identical over the whole grid.
- The k-space filter (cuFFT here, the reference's FFT routine there) and the
  adaptive Dormand-Prince steps (FP64 tree reductions here, the reference's
  sequential sums there) cannot be bit-identical: those cases are compared
  with the oracle run here on the same inputs (rel-L2 <= 1e-12 on psi and n,
  the same accepted and rejected step counts) and with the reference's
  stored sample of values.  The oracle itself hashes to the reference's
  digests (tests/test_config_oracle.py).
"""
import json
import os
import sys

import numpy as np
import pytest

import phoenix_b200 as pb
from oracle import phx_oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import config_cases as CC  # noqa: E402

pytestmark = pytest.mark.gpu

DB = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "config_digests.json")))
EXACT = [n for n in sorted(DB) if not DB[n]["case"].get("mask_cut") and not DB[n]["case"].get("adaptive")]
BOUNDED = [n for n in sorted(DB) if n not in EXACT]


def expected_iterations(case):
    """Solver::iterate calls until t >= t_max with t accumulated in the build
    precision, as the reference does (an FP32 clock can take one more)."""
    ft = np.float32 if case["dtype"] == "f32" else np.float64
    t, dt, t_max, k = ft(0), ft(case["dt"]), ft(case["t_max"]), 0
    while t < t_max:
        t = ft(t + dt)
        k += 1
    return k


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_gpu(name):
    case = CC.oracle_case(name)
    fields = CC.inputs(name)
    assert CC.input_digest(fields) == DB[name]["inputs_sha256"], "seeded inputs differ from the ones the reference ran"
    sp = pb.system_from_case(case)
    out = {}
    with pb.SolverFactory.create(sp) as s:
        pb.load_case_fields(s, case, fields)
        info = s.run()
        for comp in (["plus", "minus"] if case.get("tetm") else ["plus"]):
            out[f"psi_{comp}"] = s.get_field(f"psi_{comp}")
            out[f"n_{comp}"] = s.get_field(f"n_{comp}")
    return case, fields, out, info


@pytest.mark.parametrize("name", EXACT)
def test_gpu_bit_identical_to_reference_at_config_size(require_gpu, name):
    case, _, out, info = run_gpu(name)
    assert info.iterations == expected_iterations(case)
    for key, d in DB[name]["outputs"].items():
        a = out[key].astype(np.dtype(d["dtype"])) + 0.0
        assert CC.digest(a) == d["sha256"], (
            f"{key}: not bit-identical to the reference (l2 {np.linalg.norm(a)!r} vs {d['l2']!r}, "
            f"sample rel-L2 {rel_l2(CC.sample(a), np.array(d['sample_re']) + 1j * np.array(d['sample_im'])):.3e})")


@pytest.mark.parametrize("name", BOUNDED)
def test_gpu_matches_oracle_and_reference_sample_at_config_size(require_gpu, name):
    case, fields, out, info = run_gpu(name)
    ref, rec = O.run(case, fields)
    assert info.iterations == rec["steps"]
    if case.get("adaptive"):
        assert (info.accepted, info.rejected) == (rec["accepted"], rec["rejected"])
        assert rec["accepted"] >= 20
    if case.get("mask_cut"):
        assert info.fft_filters == rec["fft_applied"] >= 1
    for key, d in DB[name]["outputs"].items():
        r = ref[key] if key.startswith("psi") else np.real(ref[key])
        err = rel_l2(out[key], r)
        assert err <= 1e-12, f"{key}: rel-L2 {err:.3e} against the oracle"
        sref = np.array(d["sample_re"]) + 1j * np.array(d["sample_im"])
        serr = rel_l2(CC.sample(out[key]), sref)
        assert serr <= 1e-12, f"{key}: sample rel-L2 {serr:.3e} against the reference"
