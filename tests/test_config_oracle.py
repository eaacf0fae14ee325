"""The C restatement oracle at the benchmark configurations' own sizes,
against digests of the reference binary's outputs (tests/golden/config_cases.py,
tests/golden/config_digests.json, made by tests/golden/make_config_golden.py).

The oracle and the reference CPU build share the FFT routine and keep the
same operand order, so every output, k-space filter and adaptive steps
included, must hash to the same SHA-256.  The 4096^2 TE/TM case is checked on
the GPU only (the oracle takes minutes there)."""
import json
import os
import sys

import numpy as np
import pytest

from oracle import phx_oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import config_cases as CC  # noqa: E402

DIGESTS = os.path.join(os.path.dirname(__file__), "golden", "config_digests.json")
DB = json.load(open(DIGESTS)) if os.path.exists(DIGESTS) else {}
CPU_CASES = [n for n in sorted(DB) if DB[n]["case"]["N_c"] <= 1024]


def test_digests_cover_every_config_case():
    assert set(DB) == set(CC.cases())


@pytest.mark.parametrize("name", CPU_CASES)
def test_oracle_matches_reference_at_config_size(name):
    rec = DB[name]
    fields = CC.inputs(name)
    assert CC.input_digest(fields) == rec["inputs_sha256"], "seeded inputs differ from the ones the reference ran"
    out, info = O.run(CC.oracle_case(name), fields)
    assert info["steps"] > 0
    for key, d in rec["outputs"].items():
        a = out[key] if key.startswith("psi") else np.real(out[key])
        a = a.astype(np.dtype(d["dtype"])) + 0.0
        assert CC.digest(a) == d["sha256"], f"{key}: oracle differs from the reference (l2 {np.linalg.norm(a)} vs {d['l2']})"
