// Stochastic noise of the --dw option, drawn in the kernels that use it.
//
// The reference fills a complex normal field per iteration from cuRAND
// XORWOW (kernel_random_numbers.cu:17-26, called from solver.cu:36-45): one
// value per padded point, amplitude dw*sqrt(dt) per component, shared by
// both polarisations and reused by every stage of the iteration.  That
// stream cannot be reproduced; the same distribution is drawn here from a
// counter-based generator, so no noise plane is stored or read and any
// kernel can recompute the value of any point:
//   Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
//   easy as 1, 2, 3", SC 2011), key (seed low, seed high), counter
//   (point id, iteration low, iteration high, 0);
//   u1 = (x0 >> 8 + 1) 2^-24 in (0, 1], u2 = (x1 >> 8) 2^-24 in [0, 1);
//   Box-Muller (1958): z0 = r cos(2 pi u2), z1 = r sin(2 pi u2),
//   r = sqrt(-2 ln u1); ln, cos and sin by the series below, in float, every
//   operation rounded on its own so that results do not depend on the
//   compiler's contraction choices.
// The point id numbers padded coordinates (row + 16)(N_c + 32) + col + 16
// after wrapping periodic axes (rings up to 15 deep): a periodic image draws
// its point's value.
#pragma once

#include <cstdint>

#include "phx_device.cuh"

namespace phx {

struct NoiseParams {
    uint32_t key0, key1;    // seed
    uint32_t it_lo, it_hi;  // iteration counter (Solver::iterate calls)
    int on;                 // stochastic_amplitude > 0
};

__device__ __forceinline__ void philox4x32_10(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3, uint32_t k0,
                                              uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0, c1 = lo1, c2 = n2, c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// ln u, u in (0, 1]: u = m 2^e, m in [1/sqrt2, sqrt2); ln m = 2 atanh(t),
// t = (m - 1) / (m + 1), |t| <= 0.1716, atanh series to t^9
__device__ __forceinline__ float noise_log(float u) {
    const uint32_t b = __float_as_uint(u);
    int e = (int)((b >> 23) & 0xffu) - 127;
    float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
    if (m > 1.41421356f) {
        m = __fmul_rn(m, 0.5f);
        e += 1;
    }
    const float t = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
    const float t2 = __fmul_rn(t, t);
    float q = __fadd_rn(__fmul_rn(t2, 0.111111111f), 0.142857143f);
    q = __fadd_rn(__fmul_rn(q, t2), 0.2f);
    q = __fadd_rn(__fmul_rn(q, t2), 0.333333333f);
    q = __fadd_rn(__fmul_rn(q, t2), 1.0f);
    return __fadd_rn(__fmul_rn(__fmul_rn(2.0f, t), q), __fmul_rn((float)e, 0.693147181f));
}

// (cos, sin) of 2 pi k 2^-24, k in [0, 2^24): nearest quadrant from the
// integer, remainder x in [-pi/4, pi/4), Taylor series to x^10 / x^9
__device__ __forceinline__ void noise_cossin(uint32_t k, float& co, float& si) {
    const uint32_t q = (k + (1u << 21)) >> 22;
    const int32_t f = (int32_t)k - (int32_t)(q << 22);
    const float x = __fmul_rn((float)f, 3.74507028e-7f);  // (pi / 2) 2^-22
    const float x2 = __fmul_rn(x, x);
    float s = __fadd_rn(__fmul_rn(x2, 2.75573192e-6f), -1.98412698e-4f);
    s = __fadd_rn(__fmul_rn(s, x2), 8.33333333e-3f);
    s = __fadd_rn(__fmul_rn(s, x2), -0.166666667f);
    const float sn = __fadd_rn(x, __fmul_rn(__fmul_rn(x, x2), s));
    float c = __fadd_rn(__fmul_rn(x2, -2.75573192e-7f), 2.48015873e-5f);
    c = __fadd_rn(__fmul_rn(c, x2), -1.38888889e-3f);
    c = __fadd_rn(__fmul_rn(c, x2), 4.16666667e-2f);
    c = __fadd_rn(__fmul_rn(c, x2), -0.5f);
    const float cs = __fadd_rn(1.0f, __fmul_rn(x2, c));
    switch (q & 3u) {
        case 0: co = cs, si = sn; break;
        case 1: co = -sn, si = cs; break;
        case 2: co = -cs, si = -sn; break;
        default: co = sn, si = -cs; break;
    }
}

// standard normal pair of one point in one iteration
__device__ __forceinline__ void noise_normal2(const NoiseParams& N, uint32_t point, float& z0, float& z1) {
    uint32_t c0 = point, c1 = N.it_lo, c2 = N.it_hi, c3 = 0u;
    philox4x32_10(c0, c1, c2, c3, N.key0, N.key1);
    const float u1 = __fmul_rn((float)((c0 >> 8) + 1u), 0x1p-24f);
    const float r = __fsqrt_rn(__fmul_rn(-2.0f, noise_log(u1)));
    float co, si;
    noise_cossin(c1 >> 8, co, si);
    z0 = __fmul_rn(r, co);
    z1 = __fmul_rn(r, si);
}

// point id of interior coordinates (r, c), possibly in the ring
__device__ __forceinline__ uint32_t noise_point(int r, int c, int N_r, int N_c, int periodic_x, int periodic_y) {
    if (periodic_y) r = r < 0 ? r + N_r : (r >= N_r ? r - N_r : r);
    if (periodic_x) c = c < 0 ? c + N_c : (c >= N_c ? c - N_c : c);
    return (uint32_t)(r + 16) * (uint32_t)(N_c + 32) + (uint32_t)(c + 16);
}

// xi = (z0, z1) * amp: the reference's random_number[i]
template <typename T>
__device__ __forceinline__ cx<T> noise_xi(const NoiseParams& N, uint32_t point, T amp) {
    float z0, z1;
    noise_normal2(N, point, z0, z1);
    return mk(rmul((T)z0, amp), rmul((T)z1, amp));
}

}  // namespace phx
