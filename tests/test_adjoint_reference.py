"""The PyTorch FP64 twin of the RK4 map (tests/gp_torch.py), which supplies
autograd reference gradients for the adjoint, is the same discrete map as the
oracle; and torch's complex-gradient convention is dL/du + i dL/dv."""
import numpy as np
import torch

from oracle import phx_oracle as O
from gp_torch import rk4

CASE = dict(N_c=48, N_r=40, L_x=30.0, L_y=25.0, h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.05,
            g_r=0.08, R=0.04, g_pm=0.0, delta_LT=0.0, dtype="f64", iterator="RK4", dt=0.01, periodic_x=1,
            periodic_y=1, pumps=[(4.0, 3.0, 0.0)], potentials=[0.2])


def test_torch_twin_matches_oracle():
    rng = np.random.default_rng(5)
    shape = (CASE["N_r"], CASE["N_c"])
    psi0 = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    n0 = rng.random(shape)
    pump = 4.0 * rng.random(shape)
    pot = 0.2 * rng.standard_normal(shape)
    steps = 20
    case = dict(CASE, t_max=steps * CASE["dt"] * (1 - 1e-9))
    ref, rec = O.run(case, {"psi_plus": psi0, "n_plus": n0, "pump_0": pump, "potential_0": pot})
    assert rec["steps"] == steps
    t = lambda a: torch.tensor(a)  # noqa: E731
    psi, n = rk4(CASE, t(psi0), t(n0), t(pump), t(pot), steps)
    assert np.linalg.norm(psi.numpy() - ref["psi_plus"]) / np.linalg.norm(ref["psi_plus"]) < 1e-13
    assert np.linalg.norm(n.numpy() - np.real(ref["n_plus"])) / np.linalg.norm(np.real(ref["n_plus"])) < 1e-13


def test_torch_complex_gradient_convention():
    z = torch.tensor([1.0 + 2.0j, -0.5 + 0.25j], dtype=torch.complex128, requires_grad=True)
    (z.real ** 2 + z.imag ** 2 + 3.0 * z.imag).sum().backward()
    # dL/du + i dL/dv = 2u + i (2v + 3)
    np.testing.assert_allclose(z.grad.numpy(), np.array([2.0 + 7.0j, -1.0 + 3.5j]))
