"""GPU parity through the C ABI against the reference's own outputs.

Every golden fixture (tests/golden/*.npz, written by the PHOENIX CPU build)
is replayed through phoenix_b200 -> libphx.so on the GPU.  The kernels use
explicitly rounded operations in the reference's operand order, so FP64 and
FP32 results are expected to be bit-identical to the reference CPU build;
the asserted bounds are the north star's (rel-L2 <= 1e-12 for FP64) and
1e-6 for FP32.  The k-space filter goes through cuFFT instead of FFTW, and
DP45 and the imaginary-time normalisation sum their norms in FP64 instead
of the build precision, so those cases are held to the bound, not to bit
equality.
"""
import glob
import json
import os

import numpy as np
import pytest

import phoenix_b200 as pb
from oracle import phx_oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
# imaginary time with a reservoir makes the reservoir complex; the library
# refuses it (PHX_ERR_UNSUPPORTED, tests/test_abi.py) and the oracle covers it
SUPPORTED = [g for g in GOLDEN if os.path.basename(g) != "imag_rk4_f64_reservoir.npz"]


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_gpu(case, fields, **over):
    sp = pb.system_from_case(case, **over)
    with pb.SolverFactory.create(sp) as s:
        pb.load_case_fields(s, case, fields)
        info = s.run()
        comps = ["plus", "minus"] if sp.use_twin_mode else ["plus"]
        out = {}
        for c in comps:
            out[f"psi_{c}"] = s.get_field(f"psi_{c}")
            if sp.use_reservoir:
                out[f"n_{c}"] = s.get_field(f"n_{c}")
        return out, info, s.t


@pytest.mark.parametrize("path", SUPPORTED, ids=[os.path.basename(p)[:-4] for p in SUPPORTED])
def test_gpu_matches_reference_golden(require_gpu, path):
    z = np.load(path)
    case = json.loads(str(z["params"]))
    fields = O.fields_from_golden(z)
    out, info, t = run_gpu(case, fields)
    _, rec = O.run(case, fields)
    assert info.iterations == rec["steps"]
    # the reference's DP85 with fixed dt never changes the state (its branches
    # are swapped, dormand_prince.cu:182-190), so nothing needs to run
    assert info.kernel_launches > 0 or (case["iterator"] == "DP85" and not case.get("adaptive"))
    tol = 1e-12 if case["dtype"] == "f64" else 1e-6
    for k in ("psi_plus", "n_plus", "psi_minus", "n_minus"):
        gk = "out_" + k
        if gk not in z.files or k not in out:
            continue
        ref = z[gk] if k.startswith("psi") else np.real(z[gk])
        err = rel_l2(out[k], ref)
        assert err <= tol, f"{k}: rel-L2 {err:.3e} > {tol}"
        # the imaginary-time norm is summed in FP64 here, in the build precision
        # (and another order) there: its factor agrees to rounding only
        exact = not case.get("mask_cut") and not case.get("adaptive") and not case.get("imag_time")
        if exact:
            np.testing.assert_array_equal(out[k], ref, err_msg=f"{k} not bit-identical to the reference")


def test_config1_256_fp64_1000_steps_matches_oracle(require_gpu):
    """North-star parity: 256^2 periodic, FP64, RK4, dt 0.04, 1000 steps, Gaussian
    pump at 1.5x threshold, complex white-noise psi0 of amplitude 1e-2."""
    N, L = 256, 100.0
    rng = np.random.default_rng(1)
    x = -L / 2 + L / (N - 1) * np.arange(N)
    X, Y = np.meshgrid(x, x)
    pth = 0.15 * 0.225 / 0.01
    case = dict(N_c=N, N_r=N, L_x=L, L_y=L, h_bar_s=0.6582, m_eff=3.1840, gamma_c=0.15, gamma_r=0.225, g_c=6e-6,
                g_r=1.2e-5, R=0.01, g_pm=0.0, delta_LT=0.0, dtype="f64", iterator="RK4", dt=0.04,
                t_max=1000 * 0.04 * (1 - 1e-9), periodic_x=1, periodic_y=1, pumps=[(1.5 * pth, 10.0, 0.0)])
    fields = {"psi_plus": 1e-2 * (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))),
              "pump_0": 1.5 * pth * np.exp(-(X ** 2 + Y ** 2) / (2 * 10.0 ** 2))}
    out, info, t = run_gpu(case, fields)
    ref, rec = O.run(case, fields)
    assert info.iterations == rec["steps"] == 1000
    for k in ("psi_plus", "n_plus"):
        r = ref[k] if k.startswith("psi") else np.real(ref[k])
        err = rel_l2(out[k], r)
        assert err <= 1e-12, f"{k}: rel-L2 {err:.3e}"


def test_periodic_translation_equivariance_1024_fp32(require_gpu):
    """Full-size property: with periodic boundaries a cyclic shift of every input
    field shifts the result by the same amount, bit for bit."""
    N = 1024
    rng = np.random.default_rng(3)
    psi = 0.1 * (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N)))
    pump = 5.0 * rng.random((N, N))
    pot = 0.1 * rng.standard_normal((N, N))
    sp = pb.SystemParameters(N_c=N, N_r=N, L_x=100.0, L_y=100.0, h_bar_s=0.6582, m_eff=3.184, g_c=6e-6, g_r=1.2e-5,
                             periodic_boundary_x=True, periodic_boundary_y=True, dtype="f32", dt=0.02, t_max=1e9,
                             fft_every=1e9, pump_temporal=[pb.Temporal()], potential_temporal=[pb.Temporal()])
    shift = (37, 501)
    res = []
    for s_ in ((0, 0), shift):
        with pb.Solver(sp) as s:
            s.set_field("psi_plus", np.roll(psi, s_, (0, 1)))
            s.set_field("n_plus", np.zeros((N, N)))
            s.set_field("pump_plus", np.roll(pump, s_, (0, 1)))
            s.set_field("potential_plus", np.roll(pot, s_, (0, 1)))
            s.run(20)
            res.append(s.get_field("psi_plus"))
    np.testing.assert_array_equal(np.roll(res[0], shift, (0, 1)), res[1])


def test_fp32_vs_fp64_error_is_bounded(require_gpu):
    """FP32 error against the FP64 path on the 64^2 baseline-physics golden case,
    over the same number of iterations (with t_max as the stop criterion the
    FP32 clock, accumulated in FP32 as in the reference, can take one more
    iteration than the FP64 one).  The oracle gives 2.6e-7 for this case."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "rk4_f64_baseline_phys.npz"))
    case = dict(json.loads(str(z["params"])), t_max=1e9)
    fields = O.fields_from_golden(z)
    res = {}
    for dt_ in ("f64", "f32"):
        sp = pb.system_from_case(dict(case, dtype=dt_))
        with pb.Solver(sp) as s:
            pb.load_case_fields(s, case, fields)
            s.run(100)
            res[dt_] = (s.get_field("psi_plus"), s.get_field("n_plus"))
    o32, _ = O.run(dict(case, dtype="f32"), fields, max_steps=100)
    assert rel_l2(res["f32"][0], res["f64"][0]) < 1e-6
    assert rel_l2(res["f32"][1], res["f64"][1]) < 1e-6
    np.testing.assert_array_equal(res["f32"][0], o32["psi_plus"])


SHAPE_CASES = ["rk4_f64_zero", "rk4_f64_periodic", "rk4_f64_mixed_rect", "rk4_f32_periodic", "rk4_f64_mask",
               "rk4_f64_temporal", "rk4_f64_nores"]


@pytest.mark.parametrize("shape", list(range(15)))
@pytest.mark.parametrize("name", SHAPE_CASES)
def test_every_launch_shape_gives_identical_results(require_gpu, shape, name, monkeypatch):
    """The autotuner may pick any launch shape (0-3: one kernel per RK stage,
    4-14: the whole RK4 iteration in one kernel); all of them must reproduce the
    reference bit for bit (the mask case through cuFFT: to 1e-12)."""
    monkeypatch.setenv("PHX_STAGE_SHAPE", str(shape))
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    case = json.loads(str(z["params"]))
    out, info, _ = run_gpu(case, O.fields_from_golden(z))
    fused_ok = len(case.get("pulses", [])) == 0
    if shape < 4 or fused_ok:
        assert info.launch_shape == shape
    for k in ("psi_plus", "n_plus"):
        if "out_" + k not in z.files or k not in out:
            continue
        ref = z["out_" + k] if k.startswith("psi") else np.real(z["out_" + k])
        if case.get("mask_cut"):
            assert rel_l2(out[k], ref) <= 1e-12
        else:
            np.testing.assert_array_equal(out[k], ref)


def test_fused_iteration_matches_stage_kernels_1024_fp32(require_gpu, monkeypatch):
    """Full-size: the one-kernel RK4 iteration and the four stage kernels give
    the same bits on the 1024^2 benchmark workload (periodic, pump, disorder)."""
    import bench as B

    n = 1024
    wl = B.workload(n)
    res = {}
    for shape in (2,) + tuple(range(4, 15)):
        monkeypatch.setenv("PHX_STAGE_SHAPE", str(shape))
        sp = B.system(pb, n, "f32", 0)
        sp.fft_every = 1e12
        with pb.Solver(sp) as s:
            s.set_field("psi_plus", wl["psi0"])
            s.set_field("n_plus", np.zeros((n, n)))
            s.set_field("pump_plus", wl["pump"], 0)
            s.set_field("potential_plus", wl["potential"], 0)
            info = s.run(25)
            assert info.launch_shape == shape
            res[shape] = (s.get_field("psi_plus"), s.get_field("n_plus"))
    for shape in range(4, 15):
        np.testing.assert_array_equal(res[2][0], res[shape][0])
        np.testing.assert_array_equal(res[2][1], res[shape][1])


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("px,py", [(True, False), (False, True), (True, True)])
def test_tma_iterations_on_ragged_grids(require_gpu, monkeypatch, dtype, px, py):
    """The persistent TMA iterations (shapes 8-14, 14 walking column strips) on a grid whose sides are
    multiples of no tile side (tiles reach past the grid, the TMA boxes past
    the planes): bit-identical to the stage kernels after 7 iterations, with
    periodic and zero boundaries."""
    import bench as B

    n_c, n_r = 200, 140  # no multiple of 16, 32 or 64
    rng = np.random.default_rng(11)
    psi0 = 1e-1 * (rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c)))
    pump = 2.0 * rng.random((n_r, n_c))
    pot = 0.1 * rng.standard_normal((n_r, n_c))
    n0 = rng.random((n_r, n_c))
    res = {}
    for shape in (2, 8, 9, 10, 11, 12, 13, 14):
        monkeypatch.setenv("PHX_STAGE_SHAPE", str(shape))
        sp = pb.SystemParameters(N_c=n_c, N_r=n_r, L_x=60.0, L_y=40.0, **B.PHYS, periodic_boundary_x=px,
                                 periodic_boundary_y=py, dtype=dtype, iterator="RK4", dt=0.01, t0=0.0, t_max=1e12,
                                 fft_every=1e12, pump_temporal=[pb.Temporal()], potential_temporal=[pb.Temporal()],
                                 device=0)
        with pb.Solver(sp) as s:
            s.set_field("psi_plus", psi0)
            s.set_field("n_plus", n0)
            s.set_field("pump_plus", pump, 0)
            s.set_field("potential_plus", pot, 0)
            info = s.run(7)
            assert info.launch_shape == shape
            res[shape] = (s.get_field("psi_plus"), s.get_field("n_plus"))
    for shape in (8, 9, 10, 11, 12, 13, 14):
        np.testing.assert_array_equal(res[2][0], res[shape][0])
        np.testing.assert_array_equal(res[2][1], res[shape][1])


def test_autotuning_across_every_shape_is_bit_identical(require_gpu, monkeypatch):
    """The first iterations of a handle cycle through every candidate launch
    shape (TMA tile shapes of different sizes among them, whose tensor maps
    differ): the result equals a run on one fixed shape."""
    import bench as B

    monkeypatch.setenv("PHX_TUNE_CACHE", "0")  # tune in this handle, whatever ran before
    n = 256
    wl = B.workload(n)
    outs = []
    for shape in (None, "2"):
        if shape is None:
            monkeypatch.delenv("PHX_STAGE_SHAPE", raising=False)
        else:
            monkeypatch.setenv("PHX_STAGE_SHAPE", shape)
        sp = B.system(pb, n, "f32", 0)
        sp.fft_every = 1e12
        with pb.Solver(sp) as s:
            s.set_field("psi_plus", wl["psi0"])
            s.set_field("n_plus", np.zeros((n, n)))
            s.set_field("pump_plus", wl["pump"], 0)
            s.set_field("potential_plus", wl["potential"], 0)
            info = s.run(240)  # 11 candidates x 6 rounds x 3 iterations of tuning, then more
            if shape is None:
                assert info.launch_shape >= 0  # tuning finished within the run
            outs.append((s.get_field("psi_plus"), s.get_field("n_plus")))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])


def test_tuned_shape_is_remembered_per_configuration(require_gpu, monkeypatch):
    """A second handle of the same configuration starts with the shape the
    first one tuned (no tuning iterations); another grid tunes anew; with
    PHX_TUNE_CACHE=0 every handle tunes."""
    import bench as B

    monkeypatch.delenv("PHX_STAGE_SHAPE", raising=False)

    def first_shape(n):
        sp = B.system(pb, n, "f32", 0)
        sp.fft_every = 1e12
        with pb.Solver(sp) as s:
            s.set_field("psi_plus", np.zeros((n, n)))
            first = s.run(1).launch_shape
            last = s.run(239).launch_shape
        return first, last

    tuned = first_shape(192)[1]
    assert tuned >= 4
    assert first_shape(192) == (tuned, tuned)
    assert first_shape(200)[0] == -1
    monkeypatch.setenv("PHX_TUNE_CACHE", "0")
    assert first_shape(192)[0] == -1


def test_tuning_reports_medians_and_keeps_the_incumbent_within_margin(require_gpu, monkeypatch):
    """The tuner reports a median time for every candidate shape; the shape it
    keeps is the fastest one, or the incumbent (shape 10) when that is within
    3 % of the fastest."""
    import bench as B

    monkeypatch.setenv("PHX_TUNE_CACHE", "0")
    monkeypatch.delenv("PHX_STAGE_SHAPE", raising=False)
    n = 512
    sp = B.system(pb, n, "f32", 0)
    sp.fft_every = 1e12
    with pb.Solver(sp) as s:
        s.set_field("psi_plus", np.zeros((n, n)))
        assert s.tune_report() == {}
        k = B.tune(s)
        assert k == 11 * 6 * 3
        rep = s.tune_report()
        chosen = s.run(0).launch_shape
    assert sorted(rep) == list(range(4, 15))
    assert all(v > 0 for v in rep.values())
    best = min(rep.values())
    assert rep[chosen] == best or (chosen == 10 and rep[10] <= best * 1.03)


def test_bad_field_shape_is_rejected(require_gpu):
    sp = pb.SystemParameters(N_c=32, N_r=32, dt=0.01)
    with pb.Solver(sp) as s:
        with pytest.raises(ValueError):
            s.set_field("psi_plus", np.zeros((16, 16)))
        with pytest.raises(pb.PhxError):
            s.get_field("pump_plus", 0)  # no pump groups configured


def test_fft_filter_in_place_matches_contiguous_path(require_gpu, monkeypatch):
    """Square grids filter the padded state plane in place (advanced cuFFT
    layout); the contiguous gather/FFT/scatter path gives the same field to
    rounding (FP64, 1e-13)."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "rk4_f64_mask.npz"))
    case = json.loads(str(z["params"]))
    fields = O.fields_from_golden(z)
    a, _, _ = run_gpu(case, fields)
    monkeypatch.setenv("PHX_FFT_CONTIGUOUS", "1")
    b, _, _ = run_gpu(case, fields)
    assert rel_l2(a["psi_plus"], b["psi_plus"]) <= 1e-13
