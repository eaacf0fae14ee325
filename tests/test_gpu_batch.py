"""Batched RK4 (phx_batch_*) against the oracle and against single-simulation
handles.

A batch advances instances of different grid sizes, boundary conditions and
physical parameters together; every instance must come out bit-identical to
the oracle (small grids) and to a single-simulation Solver (larger grids),
through the autotuning iterations, the captured-graph chunks from either
ping-pong plane and the single launches that follow.
"""
import numpy as np
import pytest

import phoenix_b200 as pb
from oracle import phx_oracle as O

pytestmark = pytest.mark.gpu

STRONG = dict(h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.05, g_r=0.08, R=0.04, g_pm=0.0,
              delta_LT=0.0)
BASE = dict(h_bar_s=0.6582, m_eff=3.1840, gamma_c=0.15, gamma_r=0.225, g_c=6e-6, g_r=1.2e-5, R=0.01, g_pm=0.0,
            delta_LT=0.0)


def make_instance(seed, N_c, N_r, dtype, px=1, py=1, pump=True, pot=True, phys=STRONG, L=20.0, dt=0.01):
    rng = np.random.default_rng(seed)
    x = -L / 2 + L / (N_c - 1) * np.arange(N_c)
    y = -L / 2 + L / (N_r - 1) * np.arange(N_r)
    X, Y = np.meshgrid(x, y)
    amp = 4.0 if phys is STRONG else 1.5 * 0.15 * 0.225 / 0.01
    case = dict(N_c=N_c, N_r=N_r, L_x=L, L_y=L, dtype=dtype, iterator="RK4", dt=dt, t_max=1e9, periodic_x=px,
                periodic_y=py, n0_amp=1.0, **phys)
    fields = {"psi_plus": 0.3 * (rng.standard_normal((N_r, N_c)) + 1j * rng.standard_normal((N_r, N_c))),
              "n_plus": np.abs(rng.standard_normal((N_r, N_c)))}
    if pump:
        case["pumps"] = [(amp, 3.0, 0.0)]
        fields["pump_0"] = amp * np.exp(-(X ** 2 + Y ** 2) / (2 * (L / 6) ** 2))
    if pot:
        case["potentials"] = [0.2]
        fields["potential_0"] = 0.2 * rng.standard_normal((N_r, N_c))
    return case, fields


def load_batch(b, i, case, fields):
    b.set_field(i, "psi_plus", fields["psi_plus"])
    b.set_field(i, "n_plus", fields["n_plus"])
    if case.get("pumps"):
        b.set_field(i, "pump_plus", fields["pump_0"])
    if case.get("potentials"):
        b.set_field(i, "potential_plus", fields["potential_0"])


def small_mix(dtype):
    return [make_instance(1, 64, 64, dtype),
            make_instance(2, 48, 32, dtype, px=1, py=0, pot=False),
            make_instance(3, 96, 72, dtype, px=0, py=0, pump=False),
            make_instance(4, 200, 136, dtype, phys=BASE, L=100.0, dt=0.04),
            make_instance(5, 40, 24, dtype, px=0, py=1, pump=False, pot=False)]


@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_batch_matches_oracle_bitwise(require_gpu, dtype):
    inst = small_mix(dtype)
    with pb.BatchSolver([pb.system_from_case(c) for c, _ in inst]) as b:
        for i, (c, f) in enumerate(inst):
            load_batch(b, i, c, f)
        i1 = b.run(43)  # 20 tuning iterations, one 16-iteration graph from plane 0, seven single launches
        i2 = b.run(37)  # graphs from plane 1
        assert i1.iterations == 43 and i2.iterations == 37
        assert i1.launch_shape in (0, 1, 2, 3, 4)
        for i, (c, f) in enumerate(inst):
            ref, rec = O.run(c, f, max_steps=80)
            assert rec["steps"] == 80
            np.testing.assert_array_equal(b.get_field(i, "psi_plus"), ref["psi_plus"], err_msg=f"instance {i} psi")
            np.testing.assert_array_equal(b.get_field(i, "n_plus"), np.real(ref["n_plus"]), err_msg=f"instance {i} n")


@pytest.mark.parametrize("shape", [0, 1, 2, 3, 4])
def test_every_batch_tile_shape_matches_oracle(require_gpu, shape, monkeypatch):
    monkeypatch.setenv("PHX_BATCH_SHAPE", str(shape))
    inst = small_mix("f32")[:3]
    with pb.BatchSolver([pb.system_from_case(c) for c, _ in inst]) as b:
        for i, (c, f) in enumerate(inst):
            load_batch(b, i, c, f)
        info = b.run(21)
        assert info.launch_shape == shape
        for i, (c, f) in enumerate(inst):
            ref, _ = O.run(c, f, max_steps=21)
            np.testing.assert_array_equal(b.get_field(i, "psi_plus"), ref["psi_plus"])
            np.testing.assert_array_equal(b.get_field(i, "n_plus"), np.real(ref["n_plus"]))


RAGGED = [(256, 256), (192, 160), (224, 96), (160, 200), (256, 128), (96, 256), (200, 200), (256, 192),
          (128, 224), (176, 144), (240, 240), (144, 112)]


@pytest.mark.parametrize("shape", [0, 1, 2, 3, 4])
def test_every_batch_tile_shape_with_more_tiles_than_ctas(require_gpu, shape, monkeypatch):
    """12 ragged instances with mixed boundaries: 445-859 tiles per shape, more than the
    296 or 592 resident CTAs and not a multiple of them, so every CTA walks a run of
    several tiles across instance borders; one 16-iteration graph and nine single
    launches, bit-identical to the oracle."""
    monkeypatch.setenv("PHX_BATCH_SHAPE", str(shape))
    inst = [make_instance(500 + k, c, r, "f32", px=k % 2, py=(k // 2) % 2) for k, (c, r) in enumerate(RAGGED)]
    with pb.BatchSolver([pb.system_from_case(c) for c, _ in inst]) as b:
        for i, (c, f) in enumerate(inst):
            load_batch(b, i, c, f)
        info = b.run(25)
        assert info.launch_shape == shape and info.kernel_launches == 25
        for i, (c, f) in enumerate(inst):
            ref, _ = O.run(c, f, max_steps=25)
            np.testing.assert_array_equal(b.get_field(i, "psi_plus"), ref["psi_plus"], err_msg=f"instance {i} psi")
            np.testing.assert_array_equal(b.get_field(i, "n_plus"), np.real(ref["n_plus"]), err_msg=f"instance {i} n")


def test_batch_matches_single_solvers_ragged_fp32(require_gpu):
    """Sweep-shaped batch: grid sizes from {128, 256, 512, 1024}, pump 0.8-3.0x
    threshold, disorder 0.05-0.2 meV rms; each instance equals its own Solver."""
    rng = np.random.default_rng(11)
    sizes = [128, 1024, 256, 512, 128, 256, 512, 128]
    pth = 0.15 * 0.225 / 0.01
    inst = []
    for k, n in enumerate(sizes):
        case, fields = make_instance(100 + k, n, n, "f32", phys=BASE, L=100.0, dt=0.02)
        p = rng.uniform(0.8, 3.0) * pth
        case["pumps"] = [(p, 10.0, 0.0)]
        x = -50.0 + 100.0 / (n - 1) * np.arange(n)
        X, Y = np.meshgrid(x, x)
        fields["pump_0"] = p * np.exp(-(X ** 2 + Y ** 2) / (2 * 10.0 ** 2))
        fields["potential_0"] = rng.uniform(0.05, 0.2) * rng.standard_normal((n, n))
        fields["psi_plus"] = 1e-2 * fields["psi_plus"]
        fields["n_plus"] = np.zeros((n, n))
        inst.append((case, fields))
    iters = 120
    with pb.BatchSolver([pb.system_from_case(c) for c, _ in inst]) as b:
        for i, (c, f) in enumerate(inst):
            load_batch(b, i, c, f)
        b.run(iters)
        got = [(b.get_field(i, "psi_plus"), b.get_field(i, "n_plus"), b.time(i)) for i in range(len(inst))]
    for i, (c, f) in enumerate(inst):
        with pb.Solver(pb.system_from_case(c)) as s:
            pb.load_case_fields(s, c, f)
            s.run(iters)
            np.testing.assert_array_equal(got[i][0], s.get_field("psi_plus"), err_msg=f"instance {i} psi")
            np.testing.assert_array_equal(got[i][1], s.get_field("n_plus"), err_msg=f"instance {i} n")
            assert got[i][2][0] == s.t


def test_batch_field_errors(require_gpu):
    inst = small_mix("f32")[:2]
    with pb.BatchSolver([pb.system_from_case(c) for c, _ in inst]) as b:
        with pytest.raises(IndexError):
            b.set_field(2, "psi_plus", inst[0][1]["psi_plus"])
        buf = np.zeros(64 * 64 * 2, np.float32)
        lib = pb.load()
        assert lib.phx_batch_set_field(b._b, 2, 0, 0, buf.ctypes.data, buf.size, 0) == 1  # instance out of range
        assert b"instance out of range" in lib.phx_batch_last_error(b._b)
        assert lib.phx_batch_get_field(b._b, -1, 0, 0, buf.ctypes.data, buf.size, 0) == 1
        with pytest.raises(ValueError):
            b.set_field(0, "psi_plus", np.zeros((3, 3), np.complex64))
        with pytest.raises(pb.PhxError) as e:
            b.get_field(0, "pulse_plus")
        assert e.value.status == 6
        with pytest.raises(pb.PhxError) as e:
            b.set_field(1, "potential_plus", np.zeros((32, 48)))  # instance 1 has no potential group
        assert e.value.status == 1
