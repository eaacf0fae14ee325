"""A PyTorch restatement of one RK4 iteration of the scalar GP equation with
reservoir on a periodic grid, for autograd reference gradients (FP64, CPU or
GPU).  Same discrete map as RungeKutta4::step with gp_scalar
(runge_kutta.cu:74-94, kernel_gp_compute.cuh:37-111): the 5-point Laplacian
with 1/dx^2, 1/dy^2 and -2(1/dx^2 + 1/dy^2) (dx = L/(N-1), system.cpp:116-160),
constant pump and potential.  Test infrastructure only.
"""
from __future__ import annotations

import torch


def constants(case):
    dx = case["L_x"] / (case["N_c"] - 1)
    dy = case["L_y"] / (case["N_r"] - 1)
    odx2, ody2 = 1.0 / (dx * dx), 1.0 / (dy * dy)
    return dict(dx=dx, dy=dy, dV=dx * dy, odx2=odx2, ody2=ody2, m2=-2.0 * (odx2 + ody2),
                meff=-0.5 * case["h_bar_s"] * case["h_bar_s"] / case["m_eff"], ohb=1.0 / case["h_bar_s"])


def rhs(case, k, psi, n, pump, pot):
    lap = k["m2"] * psi + k["ody2"] * (torch.roll(psi, -1, 0) + torch.roll(psi, 1, 0)) + \
        k["odx2"] * (torch.roll(psi, -1, 1) + torch.roll(psi, 1, 1))
    mi = -1j * psi
    norm = psi.real ** 2 + psi.imag ** 2
    wf = k["ohb"] * (-1j) * (k["meff"] * lap)
    wf = wf + k["ohb"] * case["g_c"] * norm * mi - 0.5 * case["gamma_c"] * psi
    wf = wf + k["ohb"] * case["g_r"] * n * mi + 0.5 * case["R"] * n * psi
    if pot is not None:
        wf = wf + k["ohb"] * pot * mi
    rv = -(case["gamma_r"] + case["R"] * norm) * n
    if pump is not None:
        rv = rv + pump
    return wf, rv


def rk4(case, psi, n, pump, pot, steps):
    k = constants(case)
    dt = case["dt"]
    for _ in range(steps):
        k1p, k1n = rhs(case, k, psi, n, pump, pot)
        k2p, k2n = rhs(case, k, psi + 0.5 * dt * k1p, n + 0.5 * dt * k1n, pump, pot)
        k3p, k3n = rhs(case, k, psi + 0.5 * dt * k2p, n + 0.5 * dt * k2n, pump, pot)
        k4p, k4n = rhs(case, k, psi + dt * k3p, n + dt * k3n, pump, pot)
        psi = psi + dt * (k1p / 6 + k2p / 3 + k3p / 3 + k4p / 6)
        n = n + dt * (k1n / 6 + k2n / 3 + k3n / 3 + k4n / 6)
    return psi, n
