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
#include <stdint.h>
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

/* ---- stochastic noise (the reference's --dw) ------------------------------
 * The reference draws a complex normal field per iteration from cuRAND
 * XORWOW (kernel_random_numbers.cu:17-26, called from solver.cu:36-45), one
 * value per padded subgrid point, shared by both polarisations; that stream
 * is not reproducible.  This restatement and the product draw the same
 * distribution from a counter-based generator instead, so the two agree bit
 * for bit:
 *   Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 *   easy as 1, 2, 3", SC 2011): key (seed low, seed high), counter
 *   (point id, iteration low, iteration high, 0);
 *   two uniforms u1 = (x0 >> 8 + 1) 2^-24 in (0, 1], u2 = (x1 >> 8) 2^-24;
 *   Box-Muller (1958): z0 = r cos(2 pi u2), z1 = r sin(2 pi u2),
 *   r = sqrt(-2 ln u1), with ln, cos and sin evaluated by the series below
 *   in float, each operation rounded on its own (no contraction).
 * The point id numbers the padded coordinates (row + 16) (N_c + 32) + col + 16
 * after wrapping periodic axes, so periodic images draw their point's value. */
static void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int round = 0; round < 10; ++round) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c[0] = n0, c[1] = n1, c[2] = n2, c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}
/* ln u for u in (0, 1]: u = m 2^e with m in [1/sqrt2, sqrt2),
 * ln m = 2 atanh(t), t = (m - 1) / (m + 1), |t| <= 0.1716 (series to t^9) */
static float noise_log(float u) {
    uint32_t b;
    memcpy(&b, &u, 4);
    int e = (int)((b >> 23) & 0xffu) - 127;
    const uint32_t mb = (b & 0x7fffffu) | 0x3f800000u;
    float m;
    memcpy(&m, &mb, 4);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    const float t = (m - 1.0f) / (m + 1.0f);
    const float t2 = t * t;
    float q = t2 * 0.111111111f + 0.142857143f;
    q = q * t2 + 0.2f;
    q = q * t2 + 0.333333333f;
    q = q * t2 + 1.0f;
    return 2.0f * t * q + (float)e * 0.693147181f;
}
/* (cos, sin) of 2 pi k 2^-24 for k in [0, 2^24): nearest quadrant q from the
 * integer, remainder x in [-pi/4, pi/4), Taylor series to x^10 / x^9 */
static void noise_cossin(uint32_t k, float* co, float* si) {
    const uint32_t q = (k + (1u << 21)) >> 22;
    const int32_t f = (int32_t)k - (int32_t)(q << 22);
    const float x = (float)f * 3.74507028e-7f; /* (pi / 2) 2^-22 */
    const float x2 = x * x;
    float s = x2 * 2.75573192e-6f + -1.98412698e-4f;
    s = s * x2 + 8.33333333e-3f;
    s = s * x2 + -0.166666667f;
    const float sn = x + x * x2 * s;
    float c = x2 * -2.75573192e-7f + 2.48015873e-5f;
    c = c * x2 + -1.38888889e-3f;
    c = c * x2 + 4.16666667e-2f;
    c = c * x2 + -0.5f;
    const float cs = 1.0f + x2 * c;
    switch (q & 3u) {
        case 0: *co = cs, *si = sn; break;
        case 1: *co = -sn, *si = cs; break;
        case 2: *co = -cs, *si = -sn; break;
        default: *co = sn, *si = -cs; break;
    }
}
/* standard normal pair of one point and iteration */
static void noise_normal2(uint64_t seed, uint64_t iteration, uint32_t point, float* z0, float* z1) {
    uint32_t c[4] = {point, (uint32_t)iteration, (uint32_t)(iteration >> 32), 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const float u1 = (float)((c[0] >> 8) + 1u) * 0x1p-24f;
    const float r = sqrtf(-2.0f * noise_log(u1));
    float co, si;
    noise_cossin(c[1] >> 8, &co, &si);
    *z0 = r * co;
    *z1 = r * si;
}

/* exported for the generator's own tests */
void phx_oracle_philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) { philox4x32_10(ctr, k0, k1); }
void phx_oracle_noise_normal2(uint64_t seed, uint64_t iteration, uint32_t point, float* z0, float* z1) {
    noise_normal2(seed, iteration, point, z0, z1);
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
