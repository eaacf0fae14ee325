"""The split-step Fourier iterator of the oracle (the reference's SSFM,
split_step_fourier_method.cu:24-72).  The reference's CPU build ends its
first SSFM step with a segmentation fault, so its output cannot pin this
path; instead, for linear dynamics (g_c = 0, no reservoir) the split step is
exact for the reference's spectral operator hbar/2m (kx^2 + ky^2) with
k = 2 pi j / L (its kernel uses the literal 3.1415926535): the result must
equal the closed-form solution to rounding."""
import numpy as np

from oracle import phx_oracle as O

PHYS = dict(h_bar_s=0.6582, m_eff=0.5, gamma_c=0.2, gamma_r=0.3, g_c=0.0, g_r=0.0, R=0.0, g_pm=0.0, delta_LT=0.0)


def test_ssfm_linear_step_is_exact():
    n_c, n_r, L_x, L_y, dt, steps = 32, 24, 20.0, 15.0, 0.01, 30
    rng = np.random.default_rng(2)
    psi0 = rng.standard_normal((n_r, n_c)) + 1j * rng.standard_normal((n_r, n_c))
    case = dict(N_c=n_c, N_r=n_r, L_x=L_x, L_y=L_y, **PHYS, dtype="f64", iterator="SSFM", dt=dt,
                t_max=steps * dt * (1 - 1e-9), periodic_x=1, periodic_y=1)
    out, rec = O.run(case, {"psi_plus": psi0})
    assert rec["steps"] == steps
    # the (N_c, N_r) plan on the row-major N_r x N_c matrix is a 2-D DFT of the
    # same memory seen as N_c rows of N_r; the kernel's phase uses the row /
    # column of the N_r x N_c view
    pi = 3.1415926535
    col = np.arange(n_c)
    row = np.arange(n_r)
    kx = 2 * pi * np.where(col <= n_c // 2, col, col - n_c) / L_x
    ky = 2 * pi * np.where(row <= n_r // 2, row, row - n_r) / L_y
    KX, KY = np.meshgrid(kx, ky)
    lin = PHYS["h_bar_s"] / 2.0 / PHYS["m_eff"] * (KX ** 2 + KY ** 2)
    f = psi0.reshape(n_c, n_r)
    for _ in range(steps):
        for half in range(2):
            spec = np.fft.fft2(f).reshape(n_r, n_c) / (n_c * n_r) * np.exp(-1j * lin * dt / 2)
            f = np.fft.ifft2(spec.reshape(n_c, n_r)) * (n_c * n_r)
            if half == 0:
                f = f * np.exp(-0.5 * PHYS["gamma_c"] * dt)
    want = f.reshape(n_r, n_c)
    assert np.linalg.norm(out["psi_plus"] - want) / np.linalg.norm(want) < 1e-12


def test_ssfm_reservoir_and_nonlinearity_run():
    """With every term on (reservoir, pump, potential, noise), the oracle's
    SSFM stays finite and its reservoir follows dn/dt = -(gamma_r + R|psi|^2) n + P."""
    n = 32
    rng = np.random.default_rng(3)
    phys = dict(PHYS, g_c=0.05, g_r=0.08, R=0.04)
    case = dict(N_c=n, N_r=n, L_x=20.0, L_y=20.0, **phys, dtype="f64", iterator="SSFM", dt=0.005,
                t_max=20 * 0.005 * (1 - 1e-9), periodic_x=1, periodic_y=1, pumps=[(4.0, 3.0, 0.0)],
                potentials=[0.2], dw=0.02, seed=5)
    fields = {"psi_plus": rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)), "n_plus": rng.random((n, n)),
              "pump_0": 4.0 * rng.random((n, n)), "potential_0": 0.2 * rng.standard_normal((n, n))}
    out, rec = O.run(case, fields)
    assert rec["steps"] == 20
    assert np.isfinite(out["psi_plus"]).all() and np.isfinite(out["n_plus"]).all()
    assert np.abs(np.imag(out["n_plus"])).max() == 0.0
