"""phx_sum_abs2_noalloc: the FP64 norm for callers that cannot allocate.

Callers inside another runtime's CUDA-graph capture, callers whose device
memory belongs to their own allocator, and loops that cannot pay for the
synchronisation of cudaMalloc need a reduction that allocates nothing.  This
test calls that entry point through the C ABI on a field owned by a solver
handle, twice in a row, and checks both results against the handle's own
phx_sum_abs2 (same FP64 accumulation, different summation order: 1e-12).
A pitched, non-square field whose last chunk is partial is checked against
numpy's FP64 sum, and a field above the stated 4096 x 4096 limit is refused.
The file sorts last so that a run stopping at the first failure has run
every other test first; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import phoenix_b200 as pb
from phoenix_b200 import _lib as L

pytestmark = pytest.mark.gpu


def test_noalloc_norm_matches_handle_norm_twice(require_gpu):
    import torch

    lib = L.load()
    n = 256
    rng = np.random.default_rng(11)
    for dtype in ("f32", "f64"):
        sp = pb.SystemParameters(N_c=n, N_r=n, dt=0.01, dtype=dtype, periodic_boundary_x=True,
                                 periodic_boundary_y=True, pump_temporal=[pb.Temporal()])
        with pb.Solver(sp) as s:
            s.set_field("psi_plus", rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
            s.set_field("n_plus", rng.random((n, n)))
            s.set_field("pump_plus", rng.random((n, n)), 0)
            s.run(3)
            for name, cplx in (("psi_plus", 1), ("n_plus", 0)):
                want = s.sum_abs2(name)
                ptr, pitch = s.device_ptr(name)
                out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda:0")
                for k in range(2):
                    st = lib.phx_sum_abs2_noalloc(C.c_void_p(ptr), L.F32 if dtype == "f32" else L.F64, cplx, n, n,
                                                  pitch, C.c_void_p(out.data_ptr() + 8 * k), C.c_void_p(s.stream))
                    assert st == 0, lib.phx_last_error(None)
                torch.cuda.synchronize()
                got = out.cpu().numpy()
                for k in range(2):
                    assert got[k] == pytest.approx(want, rel=1e-12), (dtype, name, k, got[k], want)


def test_noalloc_norm_of_a_pitched_non_square_field(require_gpu):
    """A 300 x 257 field inside a wider allocation (row pitch 320 elements):
    77,100 points, so the last block's chunk is partial.  Against numpy's FP64
    sum of the same values, twice in a row."""
    import torch

    lib = L.load()
    n_r, n_c, pitch = 300, 257, 320
    rng = np.random.default_rng(12)
    for dtype, tdt in (("f32", torch.float32), ("f64", torch.float64)):
        for cplx in (1, 0):
            width = 2 * pitch if cplx else pitch
            base = torch.full((n_r, width), float("nan"), dtype=tdt, device="cuda:0")  # padding never read
            vals = rng.standard_normal((n_r, 2 * n_c if cplx else n_c))
            base[:, : vals.shape[1]] = torch.tensor(vals, dtype=tdt, device="cuda:0")
            want = float(np.sum(base[:, : vals.shape[1]].double().cpu().numpy() ** 2))
            out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda:0")
            for k in range(2):
                st = lib.phx_sum_abs2_noalloc(C.c_void_p(base.data_ptr()), L.F32 if dtype == "f32" else L.F64, cplx,
                                              n_r, n_c, pitch, C.c_void_p(out.data_ptr() + 8 * k), None)
                assert st == 0, lib.phx_last_error(None)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            for k in range(2):
                assert got[k] == pytest.approx(want, rel=1e-12), (dtype, cplx, k, got[k], want)


def test_noalloc_rejects_fields_beyond_the_scratch_limit(require_gpu):
    import torch

    lib = L.load()
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    field = torch.zeros(16, dtype=torch.float32, device="cuda:0")
    st = lib.phx_sum_abs2_noalloc(C.c_void_p(field.data_ptr()), L.F32, 0, 4097, 4096, 4096,
                                  C.c_void_p(out.data_ptr()), None)
    assert st == 1  # PHX_ERR_INVALID_ARG
    assert b"4096 x 4096" in lib.phx_last_error(None)
