"""The C ABI library: it loads without a GPU, exports every function that
include/phx.h declares, and rejects bad arguments before touching a device."""
import ctypes as C

import pytest

import phoenix_b200 as pb
from phoenix_b200 import _lib as L


def test_header_declares_the_abi():
    names = L.header_symbols()
    for required in ("phx_create", "phx_destroy", "phx_set_field", "phx_get_field", "phx_set_temporal", "phx_step",
                     "phx_get_time", "phx_set_time", "phx_sum_abs2", "phx_field_device_ptr", "phx_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = L.load()
    for name in L.header_symbols():
        assert hasattr(lib, name), f"{name} declared in include/phx.h but not exported"


def test_abi_version_and_build_info():
    lib = L.load()
    assert lib.phx_abi_version() == L.ABI_VERSION
    assert b"sm_100a" in lib.phx_build_info()


def test_status_strings():
    lib = L.load()
    assert lib.phx_status_string(0) == b"ok"
    assert lib.phx_status_string(6) == b"unsupported"


def test_create_rejects_bad_parameters_without_device_work():
    lib = L.load()
    h = C.c_void_p()
    p = pb.SystemParameters(N_c=4, N_r=4, dt=0.01).to_abi()
    st = lib.phx_create(C.byref(p), C.byref(h))
    assert st == 1 and not h.value
    assert b"8 x 8" in lib.phx_last_error(None)
    p = pb.SystemParameters(N_c=32, N_r=32, dt=0.01).to_abi()
    p.abi_version = 99
    assert lib.phx_create(C.byref(p), C.byref(h)) == 1
    p = pb.SystemParameters(N_c=33, N_r=32, dt=0.01, dtype="f32").to_abi()
    assert lib.phx_create(C.byref(p), C.byref(h)) == 6


def test_imaginary_time_parameters_are_checked_without_device_work():
    lib = L.load()
    h = C.c_void_p()
    # the complex step would make the reservoir complex: Runge-Kutta iterators refuse it
    p = pb.SystemParameters(N_c=32, N_r=32, dt=0.01, imag_time_amplitude=1.0, use_reservoir=True).to_abi()
    assert lib.phx_create(C.byref(p), C.byref(h)) == 6 and not h.value
    assert b"reservoir" in lib.phx_last_error(None)
    p = pb.SystemParameters(N_c=32, N_r=32, dt=0.01, imag_time_amplitude=1.0, use_reservoir=False,
                            iterator="DP85").to_abi()
    assert lib.phx_create(C.byref(p), C.byref(h)) == 6
    p = pb.SystemParameters(N_c=32, N_r=32, dt=0.01, imag_time_amplitude=float("nan"), use_reservoir=False).to_abi()
    assert lib.phx_create(C.byref(p), C.byref(h)) == 1
    assert b"imag_time_amplitude" in lib.phx_last_error(None)


def test_null_handle_calls_fail_cleanly():
    lib = L.load()
    assert lib.phx_step(None, 1, None) == 1
    assert lib.phx_destroy(None) == 0


def test_unknown_iterator_is_rejected_like_the_factory():
    with pytest.raises(KeyError):
        pb.SystemParameters(iterator="RK17").to_abi()


def _batch_status(systems):
    lib = L.load()
    b = C.c_void_p()
    arr = (L.Params * len(systems))(*[s.to_abi() for s in systems])
    st = lib.phx_batch_create(arr, len(systems), C.byref(b))
    assert not b.value
    return st, lib.phx_batch_last_error(None).decode()


def test_batch_rejects_unsupported_instances_without_device_work():
    ok = pb.SystemParameters(N_c=64, N_r=64, dt=0.01, dtype="f32", use_reservoir=True)
    cases = [
        (pb.SystemParameters(N_c=64, N_r=64, dt=0.01, dtype="f64", use_reservoir=True), 1, "dtype"),
        (pb.SystemParameters(N_c=64, N_r=64, dt=0.01, dtype="f32", use_reservoir=False), 1, "use_reservoir"),
        (pb.SystemParameters(N_c=64, N_r=64, dt=0.01, dtype="f32", use_reservoir=True, iterator="DP45"), 6, "RK4"),
        (pb.SystemParameters(N_c=64, N_r=64, dt=0.01, dtype="f32", use_reservoir=True, use_twin_mode=True), 6, "scalar"),
        (pb.SystemParameters(N_c=63, N_r=64, dt=0.01, dtype="f32", use_reservoir=True), 6, "even"),
        (pb.SystemParameters(N_c=4, N_r=64, dt=0.01, dtype="f32", use_reservoir=True), 1, "8 x 8"),
        (pb.SystemParameters(N_c=64, N_r=64, dt=0.01, dtype="f32", use_reservoir=True, imag_time_amplitude=1.0), 6,
         "real time"),
    ]
    for bad, status, words in cases:
        st, msg = _batch_status([ok, bad])
        assert st == status, (msg, status)
        assert msg.startswith("instance 1") and words in msg, msg
    lib = L.load()
    b = C.c_void_p()
    assert lib.phx_batch_create(None, 1, C.byref(b)) == 1
    assert lib.phx_batch_step(None, 1, None) == 1
    assert lib.phx_batch_destroy(None) == 0
