/*
 * phx_oracle.c -- CPU restatement of the PHOENIX RK time-stepping path.
 * TEST INFRASTRUCTURE ONLY (see phx_oracle.h for scope and citations).
 * The precision-generic body lives in phx_oracle_body.inc and is compiled
 * once for double (Type::real of the FP64 build) and once for float
 * (the FP32 build, -DUSE_32_BIT_PRECISION).  Build with
 * -ffp-contract=off so no multiply-add is fused (oracle/Makefile).
 */
#include "phx_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

#define PCAT2(a, b) a##b
#define PCAT(a, b) PCAT2(a, b)

/* 2-D transforms through the same FFTW-convention shim the reference CPU
 * build is linked against (solver_fft.cu:108-117: plan (N_c, N_r)). */
static void dft2d_f64(double* buf, int n0, int n1, int sign) {
    fftw_plan pl = fftw_plan_dft_2d(n0, n1, (fftw_complex*)buf, (fftw_complex*)buf,
                                    sign < 0 ? FFTW_FORWARD : FFTW_BACKWARD, FFTW_ESTIMATE);
    fftw_execute(pl);
    fftw_destroy_plan(pl);
}
static void dft2d_f32(float* buf, int n0, int n1, int sign) {
    fftwf_plan pl = fftwf_plan_dft_2d(n0, n1, (fftwf_complex*)buf, (fftwf_complex*)buf,
                                      sign < 0 ? FFTW_FORWARD : FFTW_BACKWARD, FFTW_ESTIMATE);
    fftwf_execute(pl);
    fftwf_destroy_plan(pl);
}

#define REAL double
#define SFX _f64
#define PHX_ORACLE_F32 0
#include "phx_oracle_body.inc"
#undef REAL
#undef SFX
#undef PHX_ORACLE_F32

#define REAL float
#define SFX _f32
#define PHX_ORACLE_F32 1
#include "phx_oracle_body.inc"
#undef REAL
#undef SFX
#undef PHX_ORACLE_F32
