/*
 * FFTW3-compatible 2-D complex DFT for the parity oracle (test
 * infrastructure only).  Written from the DFT definition: an iterative
 * radix-2 Cooley-Tukey transform for power-of-two lengths and a direct
 * O(n^2) sum for every other length.  All arithmetic is done in double;
 * the float entry points convert on the way in and out.
 *
 * Used by (a) the PHOENIX CPU build compiled from the reference sources
 * (oracle/Makefile), which calls it from
 * source/cuda_solver/solver/solver_fft.cu:108-117, and (b) the C
 * restatement oracle/phx_oracle.c for the k-space mask filter, so both
 * CPU paths share one transform.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct phx_shim_plan_s {
    int n0, n1, sign;
    double* in;
    double* out;
};
struct phx_shim_planf_s {
    int n0, n1, sign;
    float* in;
    float* out;
};

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place 1-D transform of n complex values spaced `stride` apart. */
static void dft1d(double* data, int n, int stride, int sign, double* scratch) {
    if (n <= 1) return;
    const double two_pi = 6.283185307179586476925286766559;
    if (is_pow2(n)) {
        /* gather, bit-reverse permute, butterflies, scatter */
        for (int i = 0; i < n; ++i) {
            scratch[2 * i] = data[2 * (size_t)i * stride];
            scratch[2 * i + 1] = data[2 * (size_t)i * stride + 1];
        }
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) {
                double tr = scratch[2 * i], ti = scratch[2 * i + 1];
                scratch[2 * i] = scratch[2 * j];
                scratch[2 * i + 1] = scratch[2 * j + 1];
                scratch[2 * j] = tr;
                scratch[2 * j + 1] = ti;
            }
        }
        for (int len = 2; len <= n; len <<= 1) {
            const int half = len >> 1;
            for (int k = 0; k < half; ++k) {
                const double ang = sign * two_pi * (double)k / (double)len;
                const double wr = cos(ang), wi = sin(ang);
                for (int s = 0; s < n; s += len) {
                    double* a = scratch + 2 * (s + k);
                    double* b = scratch + 2 * (s + k + half);
                    const double br = b[0] * wr - b[1] * wi;
                    const double bi = b[0] * wi + b[1] * wr;
                    b[0] = a[0] - br;
                    b[1] = a[1] - bi;
                    a[0] = a[0] + br;
                    a[1] = a[1] + bi;
                }
            }
        }
        for (int i = 0; i < n; ++i) {
            data[2 * (size_t)i * stride] = scratch[2 * i];
            data[2 * (size_t)i * stride + 1] = scratch[2 * i + 1];
        }
        return;
    }
    for (int k = 0; k < n; ++k) {
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < n; ++j) {
            const double ang = sign * two_pi * (double)(((long long)k * j) % n) / (double)n;
            const double wr = cos(ang), wi = sin(ang);
            const double xr = data[2 * (size_t)j * stride], xi = data[2 * (size_t)j * stride + 1];
            sr += xr * wr - xi * wi;
            si += xr * wi + xi * wr;
        }
        scratch[2 * k] = sr;
        scratch[2 * k + 1] = si;
    }
    for (int k = 0; k < n; ++k) {
        data[2 * (size_t)k * stride] = scratch[2 * k];
        data[2 * (size_t)k * stride + 1] = scratch[2 * k + 1];
    }
}

/* 2-D transform of an n0 x n1 row-major array (n1 contiguous), in place. */
static void dft2d(double* data, int n0, int n1, int sign) {
    const int nmax = n0 > n1 ? n0 : n1;
    double* scratch = (double*)malloc(sizeof(double) * 2 * (size_t)nmax);
    for (int r = 0; r < n0; ++r) dft1d(data + 2 * (size_t)r * n1, n1, 1, sign, scratch);
    for (int c = 0; c < n1; ++c) dft1d(data + 2 * (size_t)c, n0, n1, sign, scratch);
    free(scratch);
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
    (void)flags;
    fftw_plan p = (fftw_plan)malloc(sizeof(struct phx_shim_plan_s));
    p->n0 = n0;
    p->n1 = n1;
    p->sign = sign;
    p->in = (double*)in;
    p->out = (double*)out;
    return p;
}

void fftw_execute(const fftw_plan p) {
    const size_t n = (size_t)p->n0 * p->n1;
    if (p->out != p->in) memcpy(p->out, p->in, sizeof(double) * 2 * n);
    dft2d(p->out, p->n0, p->n1, p->sign < 0 ? -1 : 1);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags) {
    (void)flags;
    fftwf_plan p = (fftwf_plan)malloc(sizeof(struct phx_shim_planf_s));
    p->n0 = n0;
    p->n1 = n1;
    p->sign = sign;
    p->in = (float*)in;
    p->out = (float*)out;
    return p;
}

void fftwf_execute(const fftwf_plan p) {
    const size_t n = (size_t)p->n0 * p->n1;
    double* tmp = (double*)malloc(sizeof(double) * 2 * n);
    for (size_t i = 0; i < 2 * n; ++i) tmp[i] = (double)p->in[i];
    dft2d(tmp, p->n0, p->n1, p->sign < 0 ? -1 : 1);
    for (size_t i = 0; i < 2 * n; ++i) p->out[i] = (float)tmp[i];
    free(tmp);
}

void fftwf_destroy_plan(fftwf_plan p) { free(p); }
