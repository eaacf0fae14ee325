"""The library's failure contract, exercised without faulting the GPU.

- A bounded wait that gives up: the one-kernel TMA iteration's wait for a
  tile's data is given a limit of zero polls (phx_set_wait_limit), so every
  CTA gives up at its first tile, drains the loads it has in flight with the
  normal bound and leaves; the next call that reads results returns
  PHX_ERR_TIMEOUT, and the handle then steps normally again.
- Non-finite values: a NaN in psi makes phx_sum_abs2 return
  PHX_ERR_NONFINITE, and makes Dormand-Prince step-size control give up with
  PHX_ERR_NONFINITE once dt has shrunk to dt_min.
- A host-side abort: phx_request_abort from another thread stops a long
  phx_step between iterations (PHX_ERR_ABORTED); the handle stays usable.
"""
import ctypes as C
import threading
import time

import numpy as np
import pytest

import phoenix_b200 as pb
from phoenix_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _system(n=256, **kw):
    base = dict(N_c=n, N_r=n, L_x=100.0, L_y=100.0, h_bar_s=0.6582, m_eff=3.184, gamma_c=0.15, gamma_r=0.225,
                g_c=6e-6, g_r=1.2e-5, R=0.01, periodic_boundary_x=True, periodic_boundary_y=True, dtype="f32",
                dt=0.04, t_max=1e12, fft_every=1e12, pump_temporal=[pb.Temporal()])
    base.update(kw)
    return pb.SystemParameters(**base)


def _inputs(n=256, seed=5):
    rng = np.random.default_rng(seed)
    x = np.linspace(-50, 50, n)
    X, Y = np.meshgrid(x, x)
    psi = 0.1 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    pump = 5.0 * np.exp(-(X ** 2 + Y ** 2) / 200.0)
    return psi, pump


def _load(s, psi, pump):
    s.set_field("psi_plus", psi)
    s.set_field("n_plus", np.zeros(psi.shape))
    s.set_field("pump_plus", pump, 0)


# the TMA-fed one-kernel iterations: 64 x 16 tiles, and column strips 8 rows per step
@pytest.mark.parametrize("shape", [10, 14])
def test_tma_wait_that_gives_up_returns_timeout_and_the_handle_recovers(require_gpu, monkeypatch, shape):
    monkeypatch.setenv("PHX_STAGE_SHAPE", str(shape))
    psi, pump = _inputs()
    with pb.Solver(_system()) as ref:
        _load(ref, psi, pump)
        ref.run(5)
        want = ref.get_field("psi_plus")
    with pb.Solver(_system()) as s:
        _load(s, psi, pump)
        s.set_wait_limit(0)
        info = s.run(1)
        assert info.launch_shape == shape
        with pytest.raises(pb.PhxError) as e:
            s.get_field("psi_plus")
        assert e.value.status == L.STATUS_CODES["PHX_ERR_TIMEOUT"]
        # the flag is consumed by that report; with the default bound the
        # handle runs normally from fresh inputs
        s.set_wait_limit(-1)
        _load(s, psi, pump)
        s.set_time(0.0, 0.04)
        s.run(5)
        np.testing.assert_array_equal(s.get_field("psi_plus"), want)


def test_nan_field_makes_sum_abs2_nonfinite(require_gpu):
    psi, pump = _inputs(64)
    psi[7, 9] = np.nan
    with pb.Solver(_system(64)) as s:
        _load(s, psi, pump)
        with pytest.raises(pb.PhxError) as e:
            s.sum_abs2("psi_plus")
        assert e.value.status == L.STATUS_CODES["PHX_ERR_NONFINITE"]
        psi[7, 9] = 0.0
        s.set_field("psi_plus", psi)
        assert np.isfinite(s.sum_abs2("psi_plus"))


def test_nan_state_makes_adaptive_step_control_give_up(require_gpu):
    psi, pump = _inputs(64)
    psi[3, 4] = np.nan
    sp = _system(64, dtype="f64", iterator="DP45", use_adaptive_timestep=True, tolerance=1e-6, dt_min=1e-3,
                 dt_max=0.05, dt=0.04)
    with pb.Solver(sp) as s:
        _load(s, psi, pump)
        with pytest.raises(pb.PhxError) as e:
            s.run(1)
        assert e.value.status == L.STATUS_CODES["PHX_ERR_NONFINITE"]
        assert s.dt <= 1e-3 * (1 + 1e-12)


def test_abort_request_stops_a_running_step(require_gpu):
    psi, pump = _inputs(512)
    with pb.Solver(_system(512)) as s:
        _load(s, psi, pump)
        s.run(240)  # tuned
        lib, h = L.load(), s._h
        info = L.StepInfo()
        box = {}

        def long_run():
            box["status"] = lib.phx_step(h, C.c_int64(1 << 40), C.byref(info))

        th = threading.Thread(target=long_run)
        th.start()
        time.sleep(0.5)
        s.request_abort()
        th.join(timeout=60)
        assert not th.is_alive()
        assert box["status"] == L.STATUS_CODES["PHX_ERR_ABORTED"]
        assert 0 < info.iterations < 1 << 40
        # the record of the stopped call is filled in: its clock is the handle's
        assert info.t == s.t and info.t > 200 * 0.04
        # the request was consumed: the handle keeps stepping
        assert s.run(3).iterations == 3
        assert np.isfinite(s.sum_abs2("psi_plus"))
