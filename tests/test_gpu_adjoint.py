"""Adjoint RK4 gradients (phx_adjoint_*, phoenix_b200.adjoint.evolve).

* FP64 adjoint against a PyTorch-autograd FP64 reference of the same map
  (tests/gp_torch.py) on 64 x 64;
* FP64 adjoint against FP64 central differences in seeded random directions;
* the inverse-design configuration: 512 x 512 FP32, T = 500 iterations,
  dt = 0.04 ps, loss sum (|psi_T|^2 - rho)^2 dV with rho seven Gaussian
  spots (sigma 4 um) on a hexagonal lattice of spacing 15 um, parameter the
  pump P(x, y) started as a 1.2x threshold disc of radius 30 um; the FP32
  adjoint gradient against FP64 central differences on 16 seeded random
  directions;
* gradients do not depend on the checkpoint spacing (bit for bit).
"""
import numpy as np
import pytest
import torch

import phoenix_b200 as pb
from phoenix_b200.adjoint import evolve

from gp_torch import rk4

pytestmark = pytest.mark.gpu

PHYS = dict(h_bar_s=0.6582, m_eff=3.1840, gamma_c=0.15, gamma_r=0.225, g_c=6e-6, g_r=1.2e-5, R=0.01)
P_TH = 0.15 * 0.225 / 0.01


def system(n, L, dtype, dt, pot=True):
    return pb.SystemParameters(N_c=n, N_r=n, L_x=L, L_y=L, **PHYS, g_pm=0.0, delta_LT=0.0, periodic_boundary_x=True,
                               periodic_boundary_y=True, dtype=dtype, iterator="RK4", dt=dt, t_max=1e9,
                               fft_every=1e12, pump_temporal=[pb.Temporal()],
                               potential_temporal=[pb.Temporal()] if pot else [])


def grid(n, L):
    x = -L / 2 + L / (n - 1) * np.arange(n)
    return np.meshgrid(x, x)


def inverse_design_inputs(n, L):
    X, Y = grid(n, L)
    pump = np.where(X ** 2 + Y ** 2 <= 30.0 ** 2, 1.2 * P_TH, 0.0)
    rho = np.zeros((n, n))
    spots = [(0.0, 0.0)] + [(15.0 * np.cos(a), 15.0 * np.sin(a)) for a in np.arange(6) * np.pi / 3]
    for x0, y0 in spots:
        rho += 5.0 * np.exp(-((X - x0) ** 2 + (Y - y0) ** 2) / (2 * 4.0 ** 2))
    rng = np.random.default_rng(6)
    psi0 = 1e-2 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    return pump, rho, psi0


def loss_np(psi, rho, dV):
    return float(np.sum((np.abs(psi) ** 2 - rho) ** 2) * dV)


def forward_loss(sp, pump, psi0, n0, pot, rho, iters):
    with pb.Solver(sp) as s:
        s.set_field("psi_plus", psi0)
        s.set_field("n_plus", n0)
        s.set_field("pump_plus", pump, 0)
        if pot is not None:
            s.set_field("potential_plus", pot, 0)
        s.run(iters)
        psi = s.get_field("psi_plus")
    dV = (sp.L_x / (sp.N_c - 1)) * (sp.L_y / (sp.N_r - 1))
    return loss_np(psi.astype(np.complex128), rho, dV)


def adjoint_grads(sp, pump, psi0, n0, pot, rho, iters, every=0):
    dev = "cuda:0"
    f32 = sp.dtype == "f32"
    cdt, rdt = (torch.complex64, torch.float32) if f32 else (torch.complex128, torch.float64)
    with pb.Solver(sp) as s:
        if pot is not None:
            s.set_field("potential_plus", pot, 0)
        P = torch.tensor(pump, dtype=rdt, device=dev, requires_grad=True)
        z0 = torch.tensor(psi0, dtype=cdt, device=dev, requires_grad=True)
        m0 = torch.tensor(n0, dtype=rdt, device=dev, requires_grad=True)
        psi_T, n_T = evolve(s, P, z0, m0, iters, every)
        dV = (sp.L_x / (sp.N_c - 1)) * (sp.L_y / (sp.N_r - 1))
        rho_t = torch.tensor(rho, dtype=rdt, device=dev)
        L = (((psi_T.real ** 2 + psi_T.imag ** 2) - rho_t) ** 2).sum() * dV
        L.backward()
        torch.cuda.synchronize()
        return float(L.detach()), P.grad.cpu().numpy(), z0.grad.cpu().numpy(), m0.grad.cpu().numpy()


def test_adjoint_matches_torch_autograd_fp64_64(require_gpu):
    n, L, iters = 64, 100.0, 60
    pump, rho, psi0 = inverse_design_inputs(n, L)
    rng = np.random.default_rng(3)
    psi0 = psi0 + 0.5 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    n0 = rng.random((n, n))
    pot = 0.1 * rng.standard_normal((n, n))
    sp = system(n, L, "f64", 0.04)
    Lg, gP, gpsi, gn = adjoint_grads(sp, pump, psi0, n0, pot, rho, iters)
    case = dict(N_c=n, N_r=n, L_x=L, L_y=L, **PHYS, dt=0.04)
    t = lambda a: torch.tensor(a, dtype=torch.complex128 if np.iscomplexobj(a) else torch.float64,  # noqa: E731
                               requires_grad=True)
    P, z0, m0, V = t(pump), t(psi0), t(n0), torch.tensor(pot)
    psi, _ = rk4(case, z0, m0, P, V, iters)
    dV = (L / (n - 1)) ** 2
    Lt = (((psi.real ** 2 + psi.imag ** 2) - torch.tensor(rho)) ** 2).sum() * dV
    Lt.backward()
    assert abs(Lg - float(Lt)) <= 1e-12 * abs(float(Lt))
    for ours, ref in ((gP, P.grad.numpy()), (gpsi, z0.grad.numpy()), (gn, m0.grad.numpy())):
        err = np.linalg.norm(ours - ref) / np.linalg.norm(ref)
        assert err < 1e-10, err


def test_adjoint_fp64_matches_central_differences(require_gpu):
    n, L, iters = 96, 100.0, 80
    pump, rho, psi0 = inverse_design_inputs(n, L)
    rng = np.random.default_rng(4)
    psi0 = psi0 + 0.5 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    n0 = rng.random((n, n))
    sp = system(n, L, "f64", 0.04, pot=False)
    _, gP, gpsi, gn = adjoint_grads(sp, pump, psi0, n0, None, rho, iters)
    eps = 1e-4
    for k in range(4):
        v = np.random.default_rng(100 + k).standard_normal((n, n))
        fd = (forward_loss(sp, pump + eps * v, psi0, n0, None, rho, iters) -
              forward_loss(sp, pump - eps * v, psi0, n0, None, rho, iters)) / (2 * eps)
        assert abs(np.sum(gP * v) - fd) <= 1e-6 * abs(fd), (k, np.sum(gP * v), fd)
        w = np.random.default_rng(200 + k).standard_normal((n, n)) + 1j * np.random.default_rng(300 + k).standard_normal((n, n))
        fd = (forward_loss(sp, pump, psi0 + eps * w, n0, None, rho, iters) -
              forward_loss(sp, pump, psi0 - eps * w, n0, None, rho, iters)) / (2 * eps)
        assert abs(np.sum(gpsi.real * w.real + gpsi.imag * w.imag) - fd) <= 1e-6 * abs(fd)
        fd = (forward_loss(sp, pump, psi0, n0 + eps * v, None, rho, iters) -
              forward_loss(sp, pump, psi0, n0 - eps * v, None, rho, iters)) / (2 * eps)
        assert abs(np.sum(gn * v) - fd) <= 1e-6 * abs(fd)


def test_adjoint_gradient_independent_of_checkpoint_spacing(require_gpu):
    n, L, iters = 64, 100.0, 37
    pump, rho, psi0 = inverse_design_inputs(n, L)
    psi0 = psi0 + 0.3
    sp = system(n, L, "f32", 0.04, pot=False)
    base = adjoint_grads(sp, pump, psi0, np.zeros((n, n)), None, rho, iters, every=0)
    for every in (1, 5, 37):
        g = adjoint_grads(sp, pump, psi0, np.zeros((n, n)), None, rho, iters, every=every)
        for a, b in zip(base[1:], g[1:]):
            np.testing.assert_array_equal(a, b)


def test_inverse_design_512_fp32_gradient_vs_fp64_central_differences(require_gpu):
    n, L, iters = 512, 100.0, 500
    pump, rho, psi0 = inverse_design_inputs(n, L)
    n0 = np.zeros((n, n))
    _, gP, _, _ = adjoint_grads(system(n, L, "f32", 0.04, pot=False), pump, psi0, n0, None, rho, iters)
    sp64 = system(n, L, "f64", 0.04, pot=False)
    eps = 1e-3
    errs = []
    for k in range(16):
        v = np.random.default_rng(7000 + k).standard_normal((n, n))
        fd = (forward_loss(sp64, pump + eps * v, psi0, n0, None, rho, iters) -
              forward_loss(sp64, pump - eps * v, psi0, n0, None, rho, iters)) / (2 * eps)
        errs.append(abs(float(np.sum(gP.astype(np.float64) * v)) - fd) / abs(fd))
    print("inverse design 512^2: FP32 adjoint vs FP64 central differences, rel. errors", errs)
    assert max(errs) < 1e-2, errs


def test_fused_adjoint_kernel_matches_stage_kernels(require_gpu, monkeypatch):
    """The one-launch adjoint iteration and the four stage launches compute the
    same vector-Jacobian products (summed in a different order): FP64 to 1e-12,
    on a grid that is not a multiple of the tile."""
    n, L, iters = 72, 100.0, 30
    pump, rho, psi0 = inverse_design_inputs(n, L)
    rng = np.random.default_rng(9)
    psi0 = psi0 + 0.5 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    n0 = rng.random((n, n))
    pot = 0.1 * rng.standard_normal((n, n))
    sp = system(n, L, "f64", 0.04)
    fused = adjoint_grads(sp, pump, psi0, n0, pot, rho, iters)
    monkeypatch.setenv("PHX_ADJOINT_STAGES", "1")
    staged = adjoint_grads(sp, pump, psi0, n0, pot, rho, iters)
    for a, b in zip(fused[1:], staged[1:]):
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b)
