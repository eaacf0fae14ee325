"""The fused multiply-add arithmetic of the one-kernel RK4 iteration
(phx_params.fma, FP32 only).

Every operation of that arithmetic is an explicitly rounded fma / mul / add,
so all launch shapes (and the batch kernel, which runs the same tile loop)
compute the same bits; against FP64 its error is of the size of the
bit-exact FP32 path's (both are FP32 rounding), which this file measures on
the 1024^2 workload with disorder (500 iterations, no filter).
"""
import numpy as np
import pytest

import phoenix_b200 as pb

pytestmark = pytest.mark.gpu


def _bench():
    import bench as B

    return B


def _run(n, dtype, fma, iters, wl, shape=None, monkeypatch=None):
    B = _bench()
    if monkeypatch is not None:
        if shape is None:
            monkeypatch.delenv("PHX_STAGE_SHAPE", raising=False)
        else:
            monkeypatch.setenv("PHX_STAGE_SHAPE", str(shape))
    sp = B.system(pb, n, dtype, 0)
    sp.fft_every = 1e12
    sp.fma = fma
    with pb.Solver(sp) as s:
        s.set_field("psi_plus", wl["psi0"])
        s.set_field("n_plus", np.zeros((n, n)))
        s.set_field("pump_plus", wl["pump"], 0)
        s.set_field("potential_plus", wl["potential"], 0)
        info = s.run(iters)
        return s.get_field("psi_plus"), s.get_field("n_plus"), info


def test_fma_results_do_not_depend_on_the_launch_shape(require_gpu, monkeypatch):
    n = 320  # not a multiple of the 64-wide tiles
    wl = _bench().workload(n)
    ref = None
    for shape in range(4, 15):
        psi, nres, info = _run(n, "f32", True, 12, wl, shape, monkeypatch)
        assert info.launch_shape == shape
        if ref is None:
            ref = (psi, nres)
            continue
        np.testing.assert_array_equal(psi, ref[0], err_msg=f"shape {shape}")
        np.testing.assert_array_equal(nres, ref[1], err_msg=f"shape {shape}")


def test_fma_changes_bits_but_not_accuracy_at_1024(require_gpu, monkeypatch):
    n, iters = 1024, 500
    wl = _bench().workload(n)
    p64, n64, _ = _run(n, "f64", False, iters, wl, 10, monkeypatch)
    pe, ne, _ = _run(n, "f32", False, iters, wl, 10, monkeypatch)
    pf, nf, _ = _run(n, "f32", True, iters, wl, 10, monkeypatch)
    rel = lambda a, b: float(np.linalg.norm(a.astype(np.complex128) - b) / np.linalg.norm(b))  # noqa: E731
    e_exact, e_fma = rel(pe, p64), rel(pf, p64)
    en_exact, en_fma = rel(ne, n64), rel(nf, n64)
    print(f"1024^2, {iters} RK4 iterations, FP32 vs FP64 rel-L2: psi exact {e_exact:.3e} fma {e_fma:.3e}; "
          f"n exact {en_exact:.3e} fma {en_fma:.3e}")
    assert not np.array_equal(pe, pf)  # the arithmetic is a different one
    assert e_fma <= 2e-5 and e_fma <= 3 * e_exact
    assert en_fma <= 2e-5 and en_fma <= 3 * en_exact + 1e-7


def test_fma_is_refused_in_fp64(require_gpu):
    sp = pb.SystemParameters(N_c=64, N_r=64, dtype="f64", dt=0.01, fma=True)
    with pytest.raises(pb.PhxError) as e:
        pb.Solver(sp)
    assert "FP32" in str(e.value)


def test_fma_batch_matches_single_fma_runs(require_gpu):
    B = _bench()
    sizes = (128, 192, 256)
    wls = [B.workload(n, seed=20 + k) for k, n in enumerate(sizes)]
    systems = []
    for n in sizes:
        sp = B.system(pb, n, "f32", 0)
        sp.fft_every = 1e12
        sp.fma = True
        systems.append(sp)
    with pb.BatchSolver(systems) as b:
        for k, wl in enumerate(wls):
            b.set_field(k, "psi_plus", wl["psi0"])
            b.set_field(k, "n_plus", np.zeros(wl["psi0"].shape))
            b.set_field(k, "pump_plus", wl["pump"], 0)
            b.set_field(k, "potential_plus", wl["potential"], 0)
        b.run(15)
        got = [b.get_field(k, "psi_plus") for k in range(len(sizes))]
    for k, (n, wl) in enumerate(zip(sizes, wls)):
        with pb.Solver(systems[k]) as s:
            s.set_field("psi_plus", wl["psi0"])
            s.set_field("n_plus", np.zeros((n, n)))
            s.set_field("pump_plus", wl["pump"], 0)
            s.set_field("potential_plus", wl["potential"], 0)
            s.run(15)
            np.testing.assert_array_equal(got[k], s.get_field("psi_plus"), err_msg=f"instance {k}")
