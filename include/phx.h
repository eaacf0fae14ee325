/*
 * phx.h -- C ABI of the B200 time-stepping library for the driven-dissipative
 * Gross-Pitaevskii equation with reservoir (the PHOENIX RK hot path).
 *
 * The reference has no library API: its plug-in point is the C++ class
 * `PHOENIX::Solver` (include/solver/solver.hpp:22-170) selected by string
 * through `SolverFactory` / `REGISTER_SOLVER` (include/solver/solver_factory.hpp:31-84),
 * fed by `SystemParameters` (include/system/system_parameters.hpp:22-131) and
 * reached from the CLI (source/main.cu:46-135) or by pyphoenix as a
 * subprocess (pyphoenix/pyphoenix.py:162-216).  Each entry point below
 * names the reference interface it replaces.
 *
 * Conventions
 *  - Every call returns phx_status; no exception, exit() or abort() crosses
 *    the ABI.  phx_last_error() gives a message for the last failure.
 *  - A handle owns all of its device memory.  Host pointers passed in are
 *    borrowed for the duration of the call only.
 *  - A handle is not thread safe; distinct handles are independent.  All of
 *    a handle's GPU work is ordered on its stream.
 *  - Grids are N_r rows x N_c columns, row-major with the column index
 *    fastest (the reference's full-grid order, index = row * N_c + col).
 *    Complex values are interleaved (re, im).
 */
#ifndef PHX_H
#define PHX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHX_ABI_VERSION 3

#if defined(__GNUC__)
#define PHX_API __attribute__((visibility("default")))
#else
#define PHX_API
#endif

typedef enum {
    PHX_OK = 0,
    PHX_ERR_INVALID_ARG = 1,  /* bad size, pointer, enum or parameter      */
    PHX_ERR_OOM = 2,          /* device or host allocation failed          */
    PHX_ERR_CUDA = 3,         /* a CUDA / cuFFT call failed                 */
    PHX_ERR_NONFINITE = 4,    /* NaN or Inf found in a reduction            */
    PHX_ERR_TIMEOUT = 5,      /* a bounded wait gave up                     */
    PHX_ERR_UNSUPPORTED = 6,  /* valid request this build does not support  */
    PHX_ERR_STATE = 7,        /* call not valid in the handle's state       */
    PHX_ERR_ABORTED = 8       /* stopped by phx_request_abort               */
} phx_status;

typedef enum { PHX_F32 = 0, PHX_F64 = 1 } phx_dtype;

/* iterator keys of REGISTER_SOLVER: "RK4" (runge_kutta.cu:96), "DP45" (dormand_prince.cu:97) */
/* REGISTER_SOLVER keys of the reference (the .cu files of source/cuda_solver/solver/iterator) */
typedef enum {
    PHX_ITER_RK4 = 0,       /* "RK4"      runge_kutta.cu:96 */
    PHX_ITER_DP45 = 1,      /* "DP45"     dormand_prince.cu:97 (adaptive) */
    PHX_ITER_RK3 = 2,       /* "RK3"      runge_kutta.cu:51 */
    PHX_ITER_SSPRK3 = 3,    /* "SSPRK3"   SSPRK3.cu:45 */
    PHX_ITER_MP = 4,        /* "MP"       explicit_mp.cu:42 */
    PHX_ITER_HEUN2 = 5,     /* "Heun2"    heun.cu:45 */
    PHX_ITER_HEUN3 = 6,     /* "Heun3"    heun.cu:84 */
    PHX_ITER_HW = 7,        /* "HW"       houwen_wray.cu:45 */
    PHX_ITER_NEWTON = 8,    /* "Newton"   newton.cu:36 (explicit Euler) */
    PHX_ITER_NYSTROEM = 9,  /* "Nystroem" nystroem.cu:60 */
    PHX_ITER_RALSTON = 10,  /* "Ralston"  ralston.cu:45 */
    PHX_ITER_RALSTON3 = 11, /* "Ralston3" ralston.cu:84 */
    PHX_ITER_RALSTON4 = 12, /* "Ralston4" ralston.cu:128 */
    PHX_ITER_RULE38 = 13,   /* "Rule38"   rule38.cu:51 */
    PHX_ITER_BOSHA = 14,    /* "BoSha"     bogacki.cu:78 (adaptive) */
    PHX_ITER_CASHKARP = 15, /* "CashKarp"  cash_karp.cu:86 (adaptive) */
    PHX_ITER_FEHLBERG2 = 16,/* "Fehlberg2" fehlberg.cu:75 (adaptive) */
    PHX_ITER_FEHLBERG5 = 17,/* "Fehlberg5" fehlberg.cu:155 (adaptive) */
    PHX_ITER_DP85 = 18,     /* "DP85"      dormand_prince.cu:206 (adaptive) */
    PHX_ITER_NSRK78 = 19,   /* "NSRK78"    NSRK78.cu:119 (adaptive) */
    PHX_ITER_SSFM = 20      /* "SSFM"      split_step_fourier_method.cu:74 (split-step Fourier, periodic) */
} phx_iterator;

/* Norms of the adaptive error control and of the imaginary-time
 * normalisation.  PHX_NORM_REFERENCE reproduces the reference's sums over
 * the halo-padded buffer of a single subgrid (cuda_matrix.cuh:614-632,699-705,
 * solver.cu:73-75, solver_normalize_imag_time.cu:14-25); PHX_NORM_INTERIOR
 * sums over grid points only. */
typedef enum { PHX_NORM_REFERENCE = 0, PHX_NORM_INTERIOR = 1 } phx_norm_mode;

/* Fields of MatrixContainer (include/solver/matrix_container.cuh:16-53) that
 * are inputs or state of the iteration. */
typedef enum {
    PHX_PSI_PLUS = 0,        /* wavefunction_plus   complex          */
    PHX_PSI_MINUS = 1,       /* wavefunction_minus  complex (TE/TM)  */
    PHX_N_PLUS = 2,          /* reservoir_plus      real             */
    PHX_N_MINUS = 3,         /* reservoir_minus     real (TE/TM)     */
    PHX_PUMP_PLUS = 4,       /* pump_plus           real, per group  */
    PHX_PUMP_MINUS = 5,      /* pump_minus          real, per group  */
    PHX_POTENTIAL_PLUS = 6,  /* potential_plus      real, per group  */
    PHX_POTENTIAL_MINUS = 7, /* potential_minus     real, per group  */
    PHX_PULSE_PLUS = 8,      /* pulse_plus          complex, per group */
    PHX_PULSE_MINUS = 9,     /* pulse_minus         complex, per group */
    PHX_FFT_MASK_PLUS = 10,  /* fft_mask_plus       real, real-space order */
    PHX_FFT_MASK_MINUS = 11, /* fft_mask_minus      real, real-space order */
    PHX_FFT_PLUS = 12,       /* fft_plus            complex, read only: the k-space field of the
                                last filter time (phx_set_spectrum_output) */
    PHX_FFT_MINUS = 13       /* fft_minus           complex, read only */
} phx_field;

/* Temporal envelope kinds (include/system/envelope.hpp:63-69,165-175) */
typedef enum {
    PHX_TEMPORAL_CONSTANT = 0,
    PHX_TEMPORAL_IEXP = 1,
    PHX_TEMPORAL_COS = 2,
    PHX_TEMPORAL_GAUSS = 3,
    PHX_TEMPORAL_LOADED = 4 /* a table of (t, re, im), phx_set_temporal_table */
} phx_temporal_kind;

/* Which temporal-envelope family a group belongs to */
typedef enum { PHX_ENV_PUMP = 0, PHX_ENV_POTENTIAL = 1, PHX_ENV_PULSE = 2 } phx_envelope;

/* Replaces SystemParameters (system_parameters.hpp:22-131) for the
 * iteration: the physics and numerics flags of system_initialization.cpp:13-261
 * after calculateAuto (system.cpp:116-160).  h_bar_s and m_eff are the
 * scaled values (--hbarscaled, --meff); the library derives dx = L/(N-1),
 * dV, 1/dx^2, -2(1/dx^2+1/dy^2), -hbar^2/2m and 1/hbar exactly as
 * calculateAuto does in the chosen precision. */
typedef struct {
    int32_t abi_version; /* PHX_ABI_VERSION */
    int32_t N_c, N_r;
    double L_x, L_y;
    double h_bar_s, m_eff;
    double gamma_c, gamma_r, g_c, g_r, R, g_pm, delta_LT;
    int32_t periodic_x, periodic_y; /* --boundary; 0 = zero (reference default) */
    int32_t tetm;                   /* -tetm */
    int32_t use_reservoir;          /* reservoir present (pump or initReservoir, not -noReservoir) */
    int32_t dtype;                  /* phx_dtype: the build precision of the reference */
    int32_t iterator;               /* phx_iterator */
    int32_t adaptive;               /* -adaptive (DP45) */
    int32_t norm_mode;              /* phx_norm_mode (adaptive error, imaginary-time norm) */
    double dt, t0, t_max;           /* --dt, --t0, --tmax */
    double tol, dt_min, dt_max;     /* --tol, --rkvdt */
    double fft_every;               /* --fftEvery (ps) */
    double stochastic_amplitude;    /* --dw ; 0 = deterministic */
    uint64_t seed;                  /* noise seed */
    int32_t n_pump_groups, n_potential_groups, n_pulse_groups;
    int32_t device;                 /* CUDA device ordinal */
    double imag_time_amplitude;     /* --imagTime A: imaginary-time propagation (complex step
                                       (0, -dt) in every stage sum, then every field scaled to
                                       sum |f|^2 dV = A after each iteration); 0 = real time.
                                       Runge-Kutta iterators need use_reservoir = 0 (the complex
                                       step makes the reservoir complex); SSFM takes both */
    int32_t fma;                    /* 1: the one-kernel scalar RK4 iteration (and the batch) evaluates
                                       the right-hand side and the stage sums with fused multiply-adds,
                                       regrouped (FP32 only; no reference counterpart).  About 40 %
                                       fewer instructions per point; results then differ from the
                                       reference FP32 build in the last bits (their FP32-vs-FP64
                                       error is of the same size).  0: every operation rounded
                                       separately in the reference's order (bit-identical). */
} phx_params;

typedef struct {
    double t, dt;                   /* simulated time and current dt after the call */
    int64_t iterations;             /* Solver::iterate calls made by this call */
    int64_t accepted, rejected;     /* DP45 attempts */
    int64_t fft_filters;            /* k-space mask applications */
    int64_t kernel_launches;        /* this library's kernels launched */
    int32_t launch_shape;           /* launch shape in use: 0-3 per-stage kernels, 4-7 the fused
                                       RK4 iteration (tile shapes), 8-13 its persistent TMA-fed
                                       tile variants, 14 the TMA-fed column-strip walk, -1 while
                                       the first iterations time them */
    int32_t reserved;
} phx_step_info;

typedef struct phx_handle phx_handle;

/* Replaces SolverFactory::create + Solver::initialize (solver_factory.hpp:53-60,
 * solver_initialization.cu:13-35): allocate and zero all state for `p`. */
PHX_API phx_status phx_create(const phx_params* p, phx_handle** out);

/* Frees every device buffer and stream of the handle (no reference
 * counterpart: the reference never frees).  NULL is accepted. */
PHX_API phx_status phx_destroy(phx_handle* h);

/* Replaces the host->device upload of one matrix
 * (initializeMatricesFromSystem, solver_initialization.cu:37-174, and
 * CUDAMatrix::hostToDeviceSync, cuda_matrix.cuh:281-306).  `host` holds
 * count = N_c*N_r values (complex fields: 2*N_c*N_r reals) of type
 * host_dtype; group selects the temporal group of pump/potential/pulse. */
PHX_API phx_status phx_set_field(phx_handle* h, int32_t field, int32_t group, const void* host, int64_t count, int32_t host_dtype);

/* Replaces CUDAMatrix::getFullMatrix (device->host, cuda_matrix.cuh:375-403,
 * used by outputMatrices, solver_output_matrices.cu:20-70). */
PHX_API phx_status phx_get_field(phx_handle* h, int32_t field, int32_t group, void* host, int64_t count, int32_t host_dtype);

/* Replaces Envelope::addTemporal (envelope.cpp:88-120) for one group. */
PHX_API phx_status phx_set_temporal(phx_handle* h, int32_t envelope, int32_t group, int32_t kind, double t0, double sigma,
                            double freq);

/* A loaded temporal envelope (`time load <file>`, Envelope::addTemporal(path)
 * and updateTemporal, envelope.cpp:106-120,472-489): the amplitude at t is
 * interpolated linearly between the table's points (t ascending, n >= 2),
 * and is the last value after the table's end.  Pump tables must be real. */
PHX_API phx_status phx_set_temporal_table(phx_handle* h, int32_t envelope, int32_t group, const double* t,
                                          const double* re, const double* im, int64_t n);

/* Replaces the main loop's calls of Solver::iterate (main.cu:80-117,
 * solver.cu:22-70): run iterate() until t >= t_max or max_iterations calls. */
PHX_API phx_status phx_step(phx_handle* h, int64_t max_iterations, phx_step_info* info);

/* One Solver::iterate(force_fixed_time_step) call: info->iterations is 0 once
 * t >= t_max.  force_fixed_time_step != 0 runs an adaptive iterator once with
 * the current dt and no step-size control, as the main loop does for the
 * step that lands on an output time (main.cu:86-101). */
PHX_API phx_status phx_iterate(phx_handle* h, int32_t force_fixed_time_step, phx_step_info* info);

/* Keep the k-space field of every fft_every time (Solver::applyFFTFilter,
 * solver_fft.cu:67-100): the forward transform of psi, times mask / N where a
 * mask is set, readable as PHX_FFT_PLUS / PHX_FFT_MINUS (N_r x N_c complex, the
 * transform's own order).  Without a mask the transform is taken and psi is
 * left as it is, as in the reference.  Off by default (no extra work). */
PHX_API phx_status phx_set_spectrum_output(phx_handle* h, int32_t enable);

/* Current t and dt (SystemParameters::p.t / p.dt). */
PHX_API phx_status phx_get_time(phx_handle* h, double* t, double* dt);

/* Overwrite t and dt (--t0 / --dt, and the main loop's last-step dt
 * adjustment, main.cu:86-101). */
PHX_API phx_status phx_set_time(phx_handle* h, double t, double dt);

/* Sum over grid points of |field|^2 accumulated in FP64 (the reference's
 * transformReduce with transform_abs2, cuda_matrix.cuh:614-632, without
 * halo cells).  Real fields sum their squares. */
PHX_API phx_status phx_sum_abs2(phx_handle* h, int32_t field, double* out);

/* Borrow the device pointer of a field for zero-copy interop (e.g. torch):
 * pointer to grid point (0,0), row pitch in elements.  Valid until the
 * handle is destroyed; the caller must order its own work on the handle's
 * stream (phx_get_stream). */
PHX_API phx_status phx_field_device_ptr(phx_handle* h, int32_t field, int32_t group, void** dev_ptr, int64_t* row_pitch_elems);

/* Kernel families for phx_profile_read */
typedef enum {
    PHX_KERNEL_RK4_FIRST = 0,   /* fused RK4 stage 1                         */
    PHX_KERNEL_RK4_MID = 1,     /* fused RK4 stages 2 and 3                  */
    PHX_KERNEL_RK4_LAST = 2,    /* fused RK4 stage 4 (in-place update)       */
    PHX_KERNEL_STAGE = 3,       /* fused k-stack stage (DP45 stages 1-6)     */
    PHX_KERNEL_STAGE_FINAL = 4, /* fused k-stack final stage (fixed DP45)    */
    PHX_KERNEL_STAGE_ERROR = 5, /* DP45 k7 + error / norm reduction          */
    PHX_KERNEL_FILTER = 6,      /* k-space filter passes (without cuFFT)     */
    PHX_KERNEL_OTHER = 7,       /* rings, reductions                         */
    PHX_KERNEL_RK4_FUSED = 8,   /* whole RK4 iteration in one launch         */
    PHX_KERNEL_DP45_FUSED = 9,  /* whole DP45 attempt in one launch          */
    PHX_KERNEL_KINDS = 10
} phx_kernel_kind;

/* Per-launch CUDA-event timing of this handle's kernels (no reference
 * counterpart: the reference only times its whole loop, misc/timeit.hpp:27-35).
 * While enabled every launch is bracketed by events on the handle's stream;
 * enabling resets the totals. */
PHX_API phx_status phx_profile_enable(phx_handle* h, int32_t enable);

/* Totals since phx_profile_enable(h, 1) for one phx_kernel_kind: device
 * milliseconds, launches, and the algorithmic bytes those launches must move
 * to or from HBM (each input and output plane touched once per point). */
PHX_API phx_status phx_profile_read(phx_handle* h, int32_t kind, double* total_ms, int64_t* launches, double* bytes);

/* Ask a running (or the next) phx_step / phx_iterate on this handle to stop
 * before its next iteration; that call then returns PHX_ERR_ABORTED with
 * its phx_step_info filled in and the state of the last completed iteration
 * (no reference counterpart: the reference's main loop runs to t_max).  The
 * one call that may come from another thread while the handle is in use;
 * the request is consumed by the call it stops. */
PHX_API phx_status phx_request_abort(phx_handle* h);

/* Bound of the one-kernel RK4 iteration's wait for a tile's data (no
 * reference counterpart): the number of polls of the tile's mbarrier before
 * the wait gives up, also capped at about one second of device clock.  A wait
 * that gives up makes the step return PHX_ERR_TIMEOUT; the iteration's result
 * is then invalid, the handle stays usable.  polls < 0 restores the default
 * (2^26); 0 makes every such wait give up at once, which exercises the error
 * path without any fault. */
PHX_API phx_status phx_set_wait_limit(phx_handle* h, int32_t polls);

/* Result of the launch-shape autotuning (no reference counterpart): the
 * candidate shapes the handle timed and the median device time of one
 * iteration with each, in microseconds (count = 0 before tuning has ended or
 * when the configuration has no shape choice).  Up to `capacity` entries are
 * written; *count receives the number available. */
PHX_API phx_status phx_tune_read(phx_handle* h, int32_t capacity, int32_t* shapes, double* median_us, int32_t* count);

/* The handle's cudaStream_t, as void*. */
PHX_API phx_status phx_get_stream(phx_handle* h, void** stream);

/* ---------------------------------------------------------------- device memory
 * No counterpart in the reference (its fields move through host matrices,
 * cuda_matrix.cuh:445-476).  Copy one field between the handle and a
 * caller-owned contiguous N_r x N_c device array in the build precision
 * (complex fields as interleaved (re, im)); `count` is the number of real
 * values.  Ordered on the handle's stream; an upload rebuilds the plane's
 * ring (periodic images / zeros).  For torch tensors and other device-side
 * callers. */
PHX_API phx_status phx_set_field_device(phx_handle* h, int32_t field, int32_t group, const void* dev, int64_t count);
PHX_API phx_status phx_get_field_device(phx_handle* h, int32_t field, int32_t group, void* dev, int64_t count);

/* ---------------------------------------------------------------- adjoint
 * No counterpart in the reference.  Reverse-mode gradients of scalar
 * fixed-step RK4 (periodic boundaries, constant envelopes, at most one pump
 * and one potential group, no pulse, no filter, no noise).
 * phx_adjoint_forward runs `iterations` iterations from the handle's state
 * (as phx_step does) and keeps a checkpoint of the state every
 * `checkpoint_every` iterations (<= 0: ceil(sqrt(iterations))).
 * phx_adjoint_backward takes dL/dpsi_T (and dL/dn_T, or NULL for zero) of
 * the final state and writes dL/dpsi_0, dL/dn_0, dL/dP (pump group 0) and
 * dL/dV (potential group 0) -- each may be NULL -- by recomputing the
 * checkpoint segments last to first.  The pump and the potential enter the
 * right-hand side as in gp_scalar (include/kernel/kernel_gp_compute.cuh:86-98):
 * dL/dP through the reservoir's gain P c_P(t), dL/dV through
 * (c_V(t) / hbar) V (-i psi).
 * The recompute of the next segment runs on a second stream that the call
 * creates, beside the current segment's gradient sweep, so two segments'
 * states and stage values are held at once; the call returns after both
 * streams' work is done.  All arrays are contiguous N_r x N_c device arrays in
 * the build precision; the adjoint of a complex value u + iv is
 * dL/du + i dL/dv. */
PHX_API phx_status phx_adjoint_forward(phx_handle* h, int64_t iterations, int64_t checkpoint_every);
PHX_API phx_status phx_adjoint_backward(phx_handle* h, const void* dpsi_T, const void* dn_T, void* dpsi_0, void* dn_0,
                                        void* dpump, void* dpotential);

/* ---------------------------------------------------------------- batches
 * Many independent RK4 simulations -- pump-power sweeps, disorder
 * realisations -- with their own grid sizes and parameters, advanced
 * together.  The reference runs one simulation per process; the batch
 * replaces n sequential runs of its main loop (source/main.cu:80-117).
 * Every instance: scalar RK4, at most one pump and one potential group,
 * constant temporal envelopes, no pulse, no k-space filter, one shared
 * dtype.  One batch iteration advances every instance by one RK4 iteration
 * in a single launch of a persistent kernel that walks the tiles of all
 * instances; phx_batch_step replays a captured CUDA graph of it. */
typedef struct phx_batch phx_batch;

PHX_API phx_status phx_batch_create(const phx_params* instances, int32_t n_instances, phx_batch** out);
PHX_API phx_status phx_batch_destroy(phx_batch* b);
/* as phx_set_field / phx_get_field for one instance */
PHX_API phx_status phx_batch_set_field(phx_batch* b, int32_t instance, int32_t field, int32_t group, const void* host,
                                       int64_t count, int32_t host_dtype);
PHX_API phx_status phx_batch_get_field(phx_batch* b, int32_t instance, int32_t field, int32_t group, void* host,
                                       int64_t count, int32_t host_dtype);
/* `iterations` batch iterations (every instance advances by that many RK4
 * iterations; t_max is not consulted).  info->t / dt are instance 0's. */
PHX_API phx_status phx_batch_step(phx_batch* b, int64_t iterations, phx_step_info* info);
/* t and dt of one instance */
PHX_API phx_status phx_batch_get_time(phx_batch* b, int32_t instance, double* t, double* dt);
/* the batch's cudaStream_t, as void* */
PHX_API phx_status phx_batch_get_stream(phx_batch* b, void** stream);
/* message of the last failed call on this batch */
PHX_API const char* phx_batch_last_error(const phx_batch* b);

/* Message of the last failed call on this handle (or, when h is NULL, of
 * the last failed call in this thread that takes no handle: phx_create,
 * phx_sum_abs2_noalloc). */
PHX_API const char* phx_last_error(const phx_handle* h);

PHX_API const char* phx_status_string(int32_t status);

/* No counterpart in the reference.  FP64 sum of |z|^2 (complex field) or
 * x^2 (real field) over an N_r x N_c device field with the given row pitch
 * (elements), written to *out_dev (device memory), queued on `stream`
 * (a cudaStream_t; NULL for the legacy default stream).  It allocates
 * nothing, for callers that cannot call cudaMalloc: code running while
 * another runtime captures a CUDA graph, hosts whose device memory belongs
 * to their own allocator or pool, and loops that cannot take the device
 * synchronisation of cudaMalloc / cudaFree.  Its scratch (the per-block
 * partial sums) is a fixed 32 KiB array inside the library that every GPU
 * loading the library keeps until exit, so fields are limited to
 * 16,777,216 points (4096 x 4096); larger ones return PHX_ERR_INVALID_ARG.
 * The first call on a device looks up that array's device address (with
 * the device current); make that first call before any stream capture.
 * All calls share the array: calls whose kernels overlap on the GPU race.
 * Errors: phx_last_error(NULL). */
PHX_API phx_status phx_sum_abs2_noalloc(const void* field_dev, int32_t dtype, int32_t is_complex, int32_t N_r,
                                        int32_t N_c, int64_t row_pitch_elems, double* out_dev, void* stream);

/* ABI version and build description ("sm_100a ..."). */
PHX_API int32_t phx_abi_version(void);
PHX_API const char* phx_build_info(void);

#ifdef __cplusplus
}
#endif
#endif
