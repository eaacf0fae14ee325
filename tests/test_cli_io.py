"""The command line's file formats and envelope evaluation (libphx_io.so)
against files the reference executable wrote (tests/golden/cli/, made by
tests/golden/make_cli_golden.py): no GPU needed.

* every reference output file, decoded and encoded again, gives the same bytes
  (text with its header, npy, the PHOENIX .ash binary, MATLAB v4);
* the envelopes of each command line (positional and named forms, charges,
  rings, momenta, local coordinates, polarisations) evaluate to exactly the
  matrices the reference wrote (pump, potential, pulse, k-space mask).
"""
import glob
import json
import os

import numpy as np
import pytest

from phoenix_b200 import io as pio

CLI = os.path.join(os.path.dirname(__file__), "golden", "cli")
CASES = sorted(d for d in os.listdir(CLI) if os.path.isdir(os.path.join(CLI, d)))


def case(name):
    with open(os.path.join(CLI, name, "case.json")) as f:
        return json.load(f)


def ref_files(name):
    root = os.path.join(CLI, name, "ref")
    return [p for p in sorted(glob.glob(os.path.join(root, "**", "*"), recursive=True))
            if os.path.isfile(p) and not p.endswith("scalar.txt")]


def header_of(path):
    with open(path) as f:
        m = pio._HEADER.match(f.readline())
    toks = m.group(3).split()
    vals = dict(zip(toks[0::2], toks[1::2]))
    if "OSC" in toks:
        k = toks.index("OSC")
        vals.update(dict(zip(toks[k + 1::2], toks[k + 2::2])))
    return [float(vals.get(k, 0)) for k in ("LX", "LY", "DX", "DY", "TIME", "T0", "FREQ", "SIGMA")]


@pytest.mark.parametrize("name", CASES)
def test_reference_files_encode_to_the_same_bytes(name):
    c = case(name)
    prec = c["precision"]
    args = c["args"]
    digits = int(args[args.index("--fileoutPrecision") + 1]) if "--fileoutPrecision" in args else -1
    checked = 0
    for path in ref_files(name):
        ext = os.path.splitext(path)[1][1:]
        with open(path, "rb") as f:
            want = f.read()
        if ext == "txt":
            if digits != 17:
                continue  # six digits do not give the values back
            a, _ = pio.read_txt(path)
            a = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64)
            if prec == "fp32":
                a = a.astype(np.complex64 if np.iscomplexobj(a) else np.float32)
            complex_file = open(path).read().count("\n") - 1 == 2 * a.shape[0]
            if complex_file and not np.iscomplexobj(a):
                a = a.astype(np.complex128)
            got = pio.encode_matrix("txt", a, header_of(path), precision=digits)
        else:
            a = pio.read_matrix(path)
            if ext == "mat" and prec == "fp32":
                a = a.astype(np.complex64 if np.iscomplexobj(a) else np.float32)
            got = pio.encode_matrix(ext, a)
        assert got == want, f"{os.path.relpath(path, CLI)} differs"
        checked += 1
    assert checked >= 3


def envelope_matrix(name, file):
    path = os.path.join(CLI, name, "ref", file)
    return pio.read_matrix(path)


def test_envelopes_positional_named_and_temporal_groups_fp64():
    c = case("rk4_txt_fp64")
    pump = pio.evaluate_envelope(c["args"], "pump", "f64", 0, "plus")
    np.testing.assert_array_equal(pump.real, envelope_matrix("rk4_txt_fp64", "pump_plus.txt"))
    pot = pio.evaluate_envelope(c["args"], "potential", "f64", 0, "plus")
    np.testing.assert_array_equal(pot.real, envelope_matrix("rk4_txt_fp64", "potential_plus.txt"))


def test_envelopes_named_local_mask_and_loaded_fp64():
    c = case("dp45_npy_fp64")
    pump = pio.evaluate_envelope(c["args"], "pump", "f64", 0, "plus")
    np.testing.assert_array_equal(pump.real, envelope_matrix("dp45_npy_fp64", "pump_plus.npy"))
    mask = pio.evaluate_envelope(c["args"], "fftMask", "f64", -1, "plus", default=1.0).real
    n_r, n_c = mask.shape
    shifted = np.roll(np.roll(mask, n_r // 2, axis=0), n_c // 2, axis=1)
    np.testing.assert_array_equal(shifted, envelope_matrix("dp45_npy_fp64", "fft_mask_plus.npy"))


def test_envelopes_fp32_pulse_momenta_and_polarisations():
    c = case("tetm_mat_fp32")
    for pol in ("plus", "minus"):
        pulse = pio.evaluate_envelope(c["args"], "pulse", "f32", 0, pol)
        np.testing.assert_array_equal(pulse, envelope_matrix("tetm_mat_fp32", f"pulse_{pol}.mat").astype(np.complex64))
        pump = pio.evaluate_envelope(c["args"], "pump", "f32", 0, pol)
        np.testing.assert_array_equal(pump.real, envelope_matrix("tetm_mat_fp32", f"pump_{pol}.mat").astype(np.float32))


def test_envelopes_ring_with_charge():
    c = case("heun3_ash_fp64")
    pot = pio.evaluate_envelope(c["args"], "potential", "f64", 0, "plus")
    np.testing.assert_array_equal(pot.real, envelope_matrix("heun3_ash_fp64", "run_potential_plus.ash").real)


def test_envelope_errors_are_reported():
    with pytest.raises(ValueError, match="unknown"):
        pio.evaluate_envelope(["--N", "8", "8", "--pump", "1", "add", "1", "1", "0", "0", "both", "1", "none", "bogus"],
                              "pump")
