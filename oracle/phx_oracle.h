/*
 * phx_oracle -- CPU restatement of the PHOENIX RK time-stepping path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this library, and only as the
 * checker.  The product library (phoenix_b200/libphx.so) never links it.
 *
 * It restates, for a single subgrid (the reference's `--subgrids 1 1`), the
 * algorithm of:
 *   Solver::iterate           source/cuda_solver/solver/solver.cu:22-70
 *   Solver::adaptTimeStep     source/cuda_solver/solver/solver.cu:72-105
 *   Solver::updateKernelTime  source/cuda_solver/solver/iterator/solver_iterator.cu:11-28
 *   RungeKutta4::step         source/cuda_solver/solver/iterator/runge_kutta.cu:74-94
 *   DormandPrince45::step     source/cuda_solver/solver/iterator/dormand_prince.cu:37-95
 *   the fixed-step tableaux   runge_kutta.cu:33-47 (RK3), SSPRK3.cu:27-41, explicit_mp.cu:28-38,
 *                             heun.cu:31-41,66-80, houwen_wray.cu:27-41, newton.cu:24-30,
 *                             nystroem.cu:30-56, ralston.cu:31-41,66-80,106-124, rule38.cu:28-47
 *   the adaptive tableaux     bogacki.cu:27-76, cash_karp.cu:31-84, fehlberg.cu:33-73,100-153,
 *                             dormand_prince.cu:128-204, NSRK78.cu:37-117
 *   SSFM::step                split_step_fourier_method.cu:24-72 with the SSFM kernels
 *                             (kernel_gp_compute.cuh:244-440)
 *   gp_scalar                 include/kernel/kernel_gp_compute.cuh:18-236
 *   runge_sum_to_input_k / runge_add_to_input_k / runge_sum_to_error
 *                             include/kernel/kernel_summation.cuh:66-289
 *   synchronize_halos         include/kernel/kernel_halo.cuh:50-76
 *   applyFFTFilter            source/cuda_solver/solver/solver_fft.cu:67-119
 *   fft_shift_2D / kernel_mask_fft  include/kernel/kernel_fft.cuh:16-39
 *   calculateAuto             source/system/system.cpp:116-160
 * in the reference's storage layout (halo-padded arrays, complex reservoir,
 * k-stack), so halo-cell behaviour (zero boundaries, DP45 error norms over
 * padded cells, buffer swaps) is reproduced as the reference has it.
 * Stochastic noise (--dw) is restated with the reference's distribution and
 * placement (gp_scalar stochastic terms, the dw term of the stage sums,
 * kernel_summation.cuh:216-224, one complex normal field per iteration
 * shared by both polarisations) but drawn from a counter-based generator
 * (phx_oracle.c), since the reference's cuRAND / mt19937 stream is not
 * reproducible.  Imaginary-time propagation is not on the path.
 */
#ifndef PHX_ORACLE_H
#define PHX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* iterator keys: the reference's REGISTER_SOLVER names, numbered as in include/phx.h */
enum {
    PHX_ORACLE_RK4 = 0, PHX_ORACLE_DP45 = 1, PHX_ORACLE_RK3 = 2, PHX_ORACLE_SSPRK3 = 3, PHX_ORACLE_MP = 4,
    PHX_ORACLE_HEUN2 = 5, PHX_ORACLE_HEUN3 = 6, PHX_ORACLE_HW = 7, PHX_ORACLE_NEWTON = 8, PHX_ORACLE_NYSTROEM = 9,
    PHX_ORACLE_RALSTON = 10, PHX_ORACLE_RALSTON3 = 11, PHX_ORACLE_RALSTON4 = 12, PHX_ORACLE_RULE38 = 13,
    PHX_ORACLE_BOSHA = 14, PHX_ORACLE_CASHKARP = 15, PHX_ORACLE_FEHLBERG2 = 16, PHX_ORACLE_FEHLBERG5 = 17,
    PHX_ORACLE_DP85 = 18, PHX_ORACLE_NSRK78 = 19, PHX_ORACLE_SSFM = 20
};
enum { PHX_ORACLE_T_CONSTANT = 0, PHX_ORACLE_T_IEXP = 1, PHX_ORACLE_T_COS = 2, PHX_ORACLE_T_GAUSS = 3 };

#define PHX_ORACLE_MAX_GROUPS 8

typedef struct {
    int kind; /* PHX_ORACLE_T_* */
    double t0, sigma, freq;
} phx_oracle_temporal;

typedef struct {
    int32_t N_c, N_r;
    double L_x, L_y;
    double h_bar_s, m_eff; /* already scaled units (--hbarscaled, --meff) */
    double gamma_c, gamma_r, g_c, g_r, R, g_pm, delta_LT;
    int32_t periodic_x, periodic_y;
    int32_t tetm;
    int32_t use_reservoir;
    int32_t iterator; /* PHX_ORACLE_* */
    int32_t adaptive; /* DP45 only */
    double dt, t0, t_max;
    double tol, dt_min, dt_max;
    double fft_every;
    int32_t use_fft_mask;
    int32_t n_pump, n_potential, n_pulse; /* temporal groups */
    phx_oracle_temporal pump_t[PHX_ORACLE_MAX_GROUPS];
    phx_oracle_temporal potential_t[PHX_ORACLE_MAX_GROUPS];
    phx_oracle_temporal pulse_t[PHX_ORACLE_MAX_GROUPS];
    double stochastic_amplitude; /* --dw; noise is on when > 0 */
    uint64_t seed;
    double imag_time_amplitude;  /* --imagTime; imaginary-time propagation when != 0 */
} phx_oracle_params;

/* Derived kernel constants as calculateAuto computes them (system.cpp:116-160),
 * rounded to the build precision the way the reference rounds them. */
typedef struct {
    double dx, dy, dV, one_over_dx2, one_over_dy2, m2_over_dx2_p_dy2, m_eff_scaled, one_over_h_bar_s;
} phx_oracle_derived;

typedef struct {
    double t, dt;
    int64_t steps, accepted, rejected, fft_applied;
} phx_oracle_result;

void phx_oracle_derive_f64(const phx_oracle_params* p, phx_oracle_derived* d);
/* the noise generator: Philox4x32-10 in place on ctr, and one normal pair */
void phx_oracle_philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1);
void phx_oracle_noise_normal2(uint64_t seed, uint64_t iteration, uint32_t point, float* z0, float* z1);
void phx_oracle_derive_f32(const phx_oracle_params* p, phx_oracle_derived* d);

/* Fields are full N_r x N_c row-major grids (column index fastest).  Complex
 * fields are interleaved (re, im).  psi_* and n_* are updated in place;
 * n_* is complex like the reference's reservoir.  pump/potential are
 * n_groups x N real, pulse n_groups x N complex, fft_mask N real in
 * real-space order (the oracle applies the reference's fft shift).  Minus
 * arrays may be NULL unless tetm.  Runs `iterate` until t >= t_max or
 * max_steps calls, whichever comes first.  Returns 0 on success. */
int phx_oracle_run_f64(const phx_oracle_params* p, double* psi_p, double* n_p, double* psi_m, double* n_m,
                       const double* pump_p, const double* pump_m, const double* pot_p, const double* pot_m,
                       const double* pulse_p, const double* pulse_m, const double* fft_mask_p,
                       const double* fft_mask_m, int64_t max_steps, phx_oracle_result* res);
int phx_oracle_run_f32(const phx_oracle_params* p, float* psi_p, float* n_p, float* psi_m, float* n_m,
                       const float* pump_p, const float* pump_m, const float* pot_p, const float* pot_m,
                       const float* pulse_p, const float* pulse_m, const float* fft_mask_p,
                       const float* fft_mask_m, int64_t max_steps, phx_oracle_result* res);

#ifdef __cplusplus
}
#endif
#endif
