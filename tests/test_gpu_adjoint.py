"""Adjoint RK4 gradients (phx_adjoint_*, phoenix_b200.adjoint.evolve).

* FP64 adjoint against a PyTorch-autograd FP64 reference of the same map
  (tests/gp_torch.py) on 64 x 64: dL/dP, dL/dV, dL/dpsi_0, dL/dn_0;
* FP64 adjoint against FP64 central differences in seeded random directions;
* the inverse-design configuration: 512 x 512, T = 500 iterations,
  dt = 0.04 ps, loss sum (|psi_T|^2 - rho)^2 dV with rho seven Gaussian
  spots (sigma 4 um) on a hexagonal lattice of spacing 15 um, parameter the
  pump P(x, y) started as a 1.2x threshold disc of radius 30 um (and a
  potential, zero, to differentiate against); the FP64 adjoint against FP64
  central differences (Richardson-extrapolated) on 16 seeded random pump
  directions and 4 potential directions to 1e-6, and the FP32 adjoint on
  the same directions;
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


def central_difference(f, eps):
    """Directional derivative of f(t) at t = 0 by central differences at eps
    and eps / 2, Richardson-extrapolated (truncation error O(eps^4))."""
    d1 = (f(eps) - f(-eps)) / (2 * eps)
    d2 = (f(eps / 2) - f(-eps / 2)) / eps
    return (4 * d2 - d1) / 3


def adjoint_grads(sp, pump, psi0, n0, pot, rho, iters, every=0):
    """(L, dL/dP, dL/dpsi_0, dL/dn_0, dL/dV or None) through evolve()."""
    dev = "cuda:0"
    f32 = sp.dtype == "f32"
    cdt, rdt = (torch.complex64, torch.float32) if f32 else (torch.complex128, torch.float64)
    with pb.Solver(sp) as s:
        P = torch.tensor(pump, dtype=rdt, device=dev, requires_grad=True)
        z0 = torch.tensor(psi0, dtype=cdt, device=dev, requires_grad=True)
        m0 = torch.tensor(n0, dtype=rdt, device=dev, requires_grad=True)
        V = torch.tensor(pot, dtype=rdt, device=dev, requires_grad=True) if pot is not None else None
        psi_T, n_T = evolve(s, P, z0, m0, iters, every, potential=V)
        dV = (sp.L_x / (sp.N_c - 1)) * (sp.L_y / (sp.N_r - 1))
        rho_t = torch.tensor(rho, dtype=rdt, device=dev)
        L = (((psi_T.real ** 2 + psi_T.imag ** 2) - rho_t) ** 2).sum() * dV
        L.backward()
        torch.cuda.synchronize()
        return (float(L.detach()), P.grad.cpu().numpy(), z0.grad.cpu().numpy(), m0.grad.cpu().numpy(),
                None if V is None else V.grad.cpu().numpy())


def test_adjoint_matches_torch_autograd_fp64_64(require_gpu):
    n, L, iters = 64, 100.0, 60
    pump, rho, psi0 = inverse_design_inputs(n, L)
    rng = np.random.default_rng(3)
    psi0 = psi0 + 0.5 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    n0 = rng.random((n, n))
    pot = 0.1 * rng.standard_normal((n, n))
    sp = system(n, L, "f64", 0.04)
    Lg, gP, gpsi, gn, gV = adjoint_grads(sp, pump, psi0, n0, pot, rho, iters)
    case = dict(N_c=n, N_r=n, L_x=L, L_y=L, **PHYS, dt=0.04)
    t = lambda a: torch.tensor(a, dtype=torch.complex128 if np.iscomplexobj(a) else torch.float64,  # noqa: E731
                               requires_grad=True)
    P, z0, m0, V = t(pump), t(psi0), t(n0), t(pot)
    psi, _ = rk4(case, z0, m0, P, V, iters)
    dV = (L / (n - 1)) ** 2
    Lt = (((psi.real ** 2 + psi.imag ** 2) - torch.tensor(rho)) ** 2).sum() * dV
    Lt.backward()
    assert abs(Lg - float(Lt)) <= 1e-12 * abs(float(Lt))
    for name, ours, ref in (("P", gP, P.grad.numpy()), ("psi0", gpsi, z0.grad.numpy()), ("n0", gn, m0.grad.numpy()),
                            ("V", gV, V.grad.numpy())):
        err = np.linalg.norm(ours - ref) / np.linalg.norm(ref)
        assert err < 1e-10, (name, err)


def test_adjoint_fp64_matches_central_differences(require_gpu):
    n, L, iters = 96, 100.0, 80
    pump, rho, psi0 = inverse_design_inputs(n, L)
    rng = np.random.default_rng(4)
    psi0 = psi0 + 0.5 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    n0 = rng.random((n, n))
    pot = 0.1 * rng.standard_normal((n, n))
    sp = system(n, L, "f64", 0.04)
    _, gP, gpsi, gn, gV = adjoint_grads(sp, pump, psi0, n0, pot, rho, iters)
    f = lambda dP=0, dz=0, dn=0, dv=0: forward_loss(sp, pump + dP, psi0 + dz, n0 + dn, pot + dv, rho, iters)  # noqa: E731
    for k in range(4):
        v = np.random.default_rng(100 + k).standard_normal((n, n))
        w = np.random.default_rng(200 + k).standard_normal((n, n)) + 1j * np.random.default_rng(300 + k).standard_normal((n, n))
        checks = [("P", np.sum(gP * v), central_difference(lambda e: f(dP=e * v), 1e-3)),
                  ("V", np.sum(gV * v), central_difference(lambda e: f(dv=e * v), 1e-3)),
                  ("psi0", np.sum(gpsi.real * w.real + gpsi.imag * w.imag), central_difference(lambda e: f(dz=e * w), 1e-3)),
                  ("n0", np.sum(gn * v), central_difference(lambda e: f(dn=e * v), 1e-3))]
        for name, adj, fd in checks:
            assert abs(adj - fd) <= 1e-6 * abs(fd), (k, name, adj, fd)


def test_adjoint_gradient_independent_of_checkpoint_spacing(require_gpu):
    n, L, iters = 64, 100.0, 37
    pump, rho, psi0 = inverse_design_inputs(n, L)
    psi0 = psi0 + 0.3
    sp = system(n, L, "f32", 0.04, pot=False)
    base = adjoint_grads(sp, pump, psi0, np.zeros((n, n)), None, rho, iters, every=0)
    for every in (1, 5, 37):
        g = adjoint_grads(sp, pump, psi0, np.zeros((n, n)), None, rho, iters, every=every)
        for a, b in zip(base[1:4], g[1:4]):
            np.testing.assert_array_equal(a, b)


def inverse_design_directions(n):
    pump_dirs = [np.random.default_rng(7000 + k).standard_normal((n, n)) for k in range(16)]
    pot_dirs = [np.random.default_rng(8000 + k).standard_normal((n, n)) for k in range(4)]
    return pump_dirs, pot_dirs


def inverse_design_errors(dtype):
    """The adjoint's directional derivatives (dtype) against FP64 central
    differences on the inverse-design configuration, per family: the relative
    errors |adj - fd| / |fd|, the scaled errors |adj - fd| / max(|fd|, |g|)
    (|g| the gradient's 2-norm, the size of a directional derivative along a
    direction of unit-variance normal entries), the derivatives |fd| and |g|.
    The scaled error matters for directions nearly orthogonal to the gradient,
    where |fd| is far below |g| and the differences' own rounding (about
    1e-14 of the loss, over 2 eps) dominates the relative error."""
    n, L, iters = 512, 100.0, 500
    pump, rho, psi0 = inverse_design_inputs(n, L)
    n0, pot = np.zeros((n, n)), np.zeros((n, n))
    _, gP, _, _, gV = adjoint_grads(system(n, L, dtype, 0.04), pump, psi0, n0, pot, rho, iters)
    sp64 = system(n, L, "f64", 0.04)
    pump_dirs, pot_dirs = inverse_design_directions(n)
    out = {}
    for fam, g, dirs, perturb in (
            ("pump", gP, pump_dirs, lambda e, v: forward_loss(sp64, pump + e * v, psi0, n0, pot, rho, iters)),
            ("potential", gV, pot_dirs, lambda e, v: forward_loss(sp64, pump, psi0, n0, pot + e * v, rho, iters))):
        rel, scaled, mag = [], [], []
        gn = float(np.linalg.norm(g.astype(np.float64)))
        for v in dirs:
            fd = central_difference(lambda e: perturb(e, v), 1e-2)
            d = abs(float(np.sum(g.astype(np.float64) * v)) - fd)
            rel.append(d / abs(fd))
            scaled.append(d / max(abs(fd), gn))
            mag.append(abs(fd))
        out[fam] = {"rel": rel, "scaled": scaled, "fd": mag, "grad_norm": gn}
    return out


def test_inverse_design_512_fp64_adjoint_vs_fp64_central_differences(require_gpu):
    errs = inverse_design_errors("f64")
    print("inverse design 512^2, T = 500: FP64 adjoint vs FP64 central differences", errs)
    for fam, e in errs.items():
        assert max(e["scaled"]) <= 1e-6, (fam, e)
        # all but directions nearly orthogonal to the gradient also meet 1e-6 relative
        assert sum(r <= 1e-6 for r in e["rel"]) >= len(e["rel"]) - 1, (fam, e)


def test_inverse_design_512_fp32_adjoint_vs_fp64_central_differences(require_gpu):
    errs = inverse_design_errors("f32")
    print("inverse design 512^2, T = 500: FP32 adjoint vs FP64 central differences", errs)
    for fam, e in errs.items():
        assert max(e["scaled"]) <= 1e-4, (fam, e)


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
    assert fused[4] is not None and np.linalg.norm(fused[4]) > 0
