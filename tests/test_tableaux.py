"""The fixed-step tableaux of the oracle (the reference's registered
iterators) converge with their order on a problem with an exact discrete
solution: linear, damped Schroedinger dynamics on a periodic grid, where the
5-point Laplacian is diagonal in Fourier space.  This pins the two tableaux
whose reference output is undefined (RK3, Ralston4) to their methods and
checks every other table entry as well."""
import numpy as np
import pytest

from oracle import phx_oracle as O

ORDERS = {"Newton": 1, "MP": 2, "Heun2": 2, "Ralston": 2, "RK3": 3, "SSPRK3": 3, "Heun3": 3, "HW": 3,
          "Ralston3": 3, "RK4": 4, "Rule38": 4, "Ralston4": 4, "Nystroem": 5}
N, L, T_END = 32, 20.0, 0.4
PHYS = dict(h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.0, g_r=0.0, R=0.0, g_pm=0.0, delta_LT=0.0)


def exact(psi0):
    dx = L / (N - 1)
    odx2 = 1.0 / (dx * dx)
    k = 2 * np.pi * np.fft.fftfreq(N)
    KX, KY = np.meshgrid(k, k)
    lam = -4 * odx2 + 2 * odx2 * (np.cos(KX) + np.cos(KY))  # eigenvalues of the 5-point Laplacian
    meff = -0.5 * PHYS["h_bar_s"] ** 2 / PHYS["m_eff"]
    rate = -1j * meff * lam / PHYS["h_bar_s"] - 0.5 * PHYS["gamma_c"]
    return np.fft.ifft2(np.exp(rate * T_END) * np.fft.fft2(psi0))


def error(it, steps, psi0):
    dt = T_END / steps
    case = dict(N_c=N, N_r=N, L_x=L, L_y=L, **PHYS, dtype="f64", iterator=it, dt=dt, t_max=T_END - 0.5 * dt,
                periodic_x=1, periodic_y=1)
    out, rec = O.run(case, {"psi_plus": psi0})
    assert rec["steps"] == steps
    return np.linalg.norm(out["psi_plus"] - exact(psi0)) / np.linalg.norm(psi0)


@pytest.mark.parametrize("it", sorted(ORDERS))
def test_tableau_converges_with_its_order(it):
    rng = np.random.default_rng(1)
    x = -L / 2 + L / (N - 1) * np.arange(N)
    X, Y = np.meshgrid(x, x)
    psi0 = np.exp(-(X ** 2 + Y ** 2) / 8.0) * np.exp(0.5j * X) + 0.05 * rng.standard_normal((N, N))
    p = ORDERS[it]
    n1 = {1: 400, 2: 100, 3: 40, 4: 20, 5: 10}[p]
    e1, e2 = error(it, n1, psi0), error(it, 2 * n1, psi0)
    observed = np.log2(e1 / e2)
    assert abs(observed - p) < 0.3, (it, e1, e2, observed)
