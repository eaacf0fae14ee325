/*
 * Minimal FFTW3-compatible interface used only to compile the PHOENIX CPU
 * build as a parity oracle (test infrastructure; never linked into the
 * product library).  FFTW itself is not installed in this image.
 *
 * Only the calls made by source/cuda_solver/solver/solver_fft.cu:108-117 are
 * provided: fftw[f]_plan_dft_2d, fftw[f]_execute, fftw[f]_destroy_plan.
 * Convention (FFTW's): forward uses exp(-2*pi*i*k*n/N), backward exp(+...),
 * no normalisation; row-major n0 x n1 with n1 contiguous.
 */
#ifndef PHX_ORACLE_FFTW_SHIM_H
#define PHX_ORACLE_FFTW_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef float fftwf_complex[2];

typedef struct phx_shim_plan_s* fftw_plan;
typedef struct phx_shim_planf_s* fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE (0U)

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif
#endif
