// Split-step Fourier iterator (the reference's "SSFM",
// source/cuda_solver/solver/iterator/split_step_fourier_method.cu:24-72 with
// the kernels of include/kernel/kernel_gp_compute.cuh:244-440).  Halo 0: the
// wavefunction is worked on as a contiguous N_r x N_c array between four
// unnormalised cuFFT transforms per iteration, with the (N_c, N_r) plan of
// solver_fft.cu:102-118; the reservoir stays in its halo-padded plane.
//   linear half step   psi <- F^-1[ F[psi] / N2 exp(-i lin dt / 2) ],
//                      lin = hbar / 2 / m (kx^2 + ky^2), k = 2 pi j / L with
//                      the reference's literal pi = 3.1415926535
//   nonlinear step     psi <- psi exp(-i/hbar (g_c|psi|^2 - i hbar/2 gamma_c
//                      + V + g_r n + i hbar/2 R n) dt),  n_new = n + f_n dt
//   linear half step   again
//   independent step   psi <- psi + dt/hbar pulse amp + dw
// The reference's complex arithmetic order is kept; its complex exponential
// is std::exp / CUDA's, here exp(re) (cos im, sin im) from CUDA's functions,
// so results agree with the oracle to rounding, not bit for bit.
#pragma once

#include "phx_device.cuh"
#include "phx_noise.cuh"

namespace phx {

template <typename T>
struct SsfmParams {
    int N_r, N_c;
    long long pitch;     // of the padded planes
    int tetm, res;
    T hbs, meff, Lx, Ly, dt, N2;
    T g_c, g_r, R, gamma_c, gamma_r, g_pm, ohb, dV;
    int n_pump, n_pot, n_pulse;
    long long plane;     // group stride of the padded input planes
    const T* pump[2];    // padded planes (interior origin), [component]
    const T* pot[2];
    const cx<T>* pulse[2];
    cx<T> amp_pump[kMaxGroups], amp_pot[kMaxGroups], amp_pulse[kMaxGroups];
    // stochastic terms
    NoiseParams noise;
    T noise_amp;
    int periodic_x, periodic_y;
};

template <typename T>
__device__ __forceinline__ cx<T> cexp_dev(cx<T> z) {
    T s, c;
    if constexpr (sizeof(T) == 4)
        sincosf(z.im, &s, &c);
    else
        sincos(z.im, &s, &c);
    const T e = sizeof(T) == 4 ? (T)expf((float)z.re) : (T)exp((double)z.re);
    return mk(e * c, e * s);
}

// gp_scalar_linear_fourier: out = in / N2 * exp(minus_i * lin * dt / 2)
template <typename T>
__global__ void ssfm_linear_kernel(const __grid_constant__ SsfmParams<T> S, const cx<T>* __restrict__ in,
                                   cx<T>* __restrict__ out) {
    const long long N = (long long)S.N_r * S.N_c;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const T row = (T)(unsigned)(i / S.N_c), col = (T)(unsigned)(i % S.N_c);
        const T kx = (T)(2.0 * 3.1415926535 * (double)(col <= (T)((unsigned)S.N_c / 2) ? col : -(T)S.N_c + col) / (double)S.Lx);
        const T ky = (T)(2.0 * 3.1415926535 * (double)(row <= (T)((unsigned)S.N_r / 2) ? row : -(T)S.N_r + row) / (double)S.Ly);
        const T lin = (T)((double)S.hbs / 2.0 / (double)S.meff * (double)radd(rmul(kx, kx), rmul(ky, ky)));
        cx<T> z = mk(rmul((T)0.0, lin), rmul((T)-1.0, lin));
        z = mk(rmul(z.re, S.dt), rmul(z.im, S.dt));
        z = mk(rdiv(z.re, (T)2.0), rdiv(z.im, (T)2.0));
        const cx<T> a = in[i];
        out[i] = cmul(mk(rdiv(a.re, S.N2), rdiv(a.im, S.N2)), cexp_dev(z));
    }
}

template <typename T>
__device__ __forceinline__ void ssfm_nonlinear_one(const SsfmParams<T>& S, int comp, long long pi, cx<T> in_wf, T in_rv, T cross_norm,
                                                   cx<T>& out_wf, T& out_rv) {
    const T norm = abs2(in_wf);
    cx<T> result = mk(rmul(S.g_c, norm), rmul(rmul(-S.hbs, (T)0.5), S.gamma_c));
    for (int k = 0; k < S.n_pot; ++k) result = cadd(result, smul(S.pot[comp][pi + k * S.plane], S.amp_pot[k]));
    const cx<T> rv = mk(in_rv, (T)0);
    result = cadd(result, smul(S.g_r, rv));
    {
        cx<T> ih = mk(rmul((T)0.0, S.hbs), rmul((T)1.0, S.hbs));
        ih = smul((T)0.5, ih);
        ih = smul(S.R, ih);
        result = cadd(result, cmul(ih, rv));
    }
    if (S.noise.on) result = csub(result, mk(rdiv(S.g_c, S.dV), (T)0));
    cx<T> z;
    if (!S.tetm) {
        result = mk(result.im, rmul((T)-1.0f, result.re));
        z = smul(S.dt, smul(S.ohb, result));
    } else {
        const cx<T> mioh = mk((T)0.0, rdiv((T)-1.0, S.hbs));
        z = smul(S.dt, cmul(mioh, cadd(result, mk(rmul(S.g_pm, cross_norm), (T)0))));
    }
    out_wf = cmul(in_wf, cexp_dev(z));
    // reservoir (stored real: every term keeps its imaginary part 0)
    T r = rmul(-S.gamma_r, in_rv);
    r = rsub(r, rmul(rmul(S.R, norm), in_rv));
    for (int k = 0; k < S.n_pump; ++k) r = radd(r, rmul(S.pump[comp][pi + k * S.plane], S.amp_pump[k].re));
    if (S.noise.on) r = radd(r, rdiv(rmul(S.R, in_rv), S.dV));
    out_rv = radd(in_rv, rmul(S.dt, r));
}

// gp_scalar_nonlinear: (fft, rv) -> (wf, buffer rv)
template <typename T>
__global__ void ssfm_nonlinear_kernel(const __grid_constant__ SsfmParams<T> S, const cx<T>* __restrict__ fp,
                                      const cx<T>* __restrict__ fm, const T* __restrict__ rvp, const T* __restrict__ rvm,
                                      cx<T>* __restrict__ wp, cx<T>* __restrict__ wm, T* __restrict__ brvp,
                                      T* __restrict__ brvm) {
    const long long N = (long long)S.N_r * S.N_c;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / S.N_c, c = i - r * S.N_c, pi = r * S.pitch + c;
        if (!S.tetm) {
            cx<T> o;
            T on;
            ssfm_nonlinear_one(S, 0, pi, fp[i], S.res ? rvp[pi] : (T)0, (T)0, o, on);
            wp[i] = o;
            if (S.res) brvp[pi] = on;
        } else {
            const cx<T> a = fp[i], b = fm[i];
            cx<T> o;
            T on;
            ssfm_nonlinear_one(S, 0, pi, a, rvp[pi], abs2(b), o, on);
            wp[i] = o;
            brvp[pi] = on;
            ssfm_nonlinear_one(S, 1, pi, b, rvm[pi], abs2(a), o, on);
            wm[i] = o;
            brvm[pi] = on;
        }
    }
}

// gp_scalar_independent: psi = fft + pulse + dw into the padded state plane;
// the scalar branch copies the buffer reservoir back, the TE/TM branch does not
template <typename T>
__global__ void ssfm_independent_kernel(const __grid_constant__ SsfmParams<T> S, const cx<T>* __restrict__ fp,
                                        const cx<T>* __restrict__ fm, T* __restrict__ rvp, const T* __restrict__ brvp,
                                        const T* __restrict__ brvm, cx<T>* __restrict__ psip, cx<T>* __restrict__ psim) {
    const long long N = (long long)S.N_r * S.N_c;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / S.N_c, c = i - r * S.N_c, pi = r * S.pitch + c;
        cx<T> ap = mk((T)0, (T)0), am = mk((T)0, (T)0);
        for (int k = 0; k < S.n_pulse; ++k) {
            if (!S.tetm) {
                ap = cadd(ap, cmul(smul(rmul(S.ohb, S.dt), S.pulse[0][pi + k * S.plane]), S.amp_pulse[k]));
            } else {
                const cx<T> m = smul(S.dt, mk((T)0.0, rdiv((T)-1.0, S.hbs)));
                ap = cadd(ap, cmul(cmul(m, S.pulse[0][pi + k * S.plane]), S.amp_pulse[k]));
                am = cadd(am, cmul(cmul(m, S.pulse[1][pi + k * S.plane]), S.amp_pulse[k]));
            }
        }
        if (S.noise.on) {
            const cx<T> xi = noise_xi(S.noise, noise_point((int)r, (int)c, S.N_r, S.N_c, S.periodic_x, S.periodic_y), S.noise_amp);
            const T nrp = S.res ? (!S.tetm ? rvp[pi] : brvp[pi]) : (T)0;
            const T scp = rsqrt_rn(rdiv(radd(rmul(S.R, nrp), S.gamma_c), rmul((T)4.0, S.dV)));
            ap = cadd(ap, mk(rmul(xi.re, scp), rmul(xi.im, scp)));
            if (S.tetm) {
                const T scm = rsqrt_rn(rdiv(radd(rmul(S.R, brvm[pi]), S.gamma_c), rmul((T)4.0, S.dV)));
                am = cadd(am, mk(rmul(xi.re, scm), rmul(xi.im, scm)));
            }
        }
        psip[pi] = cadd(fp[i], ap);
        if (S.tetm) psim[pi] = cadd(fm[i], am);
        else if (S.res) rvp[pi] = brvp[pi];
    }
}

}  // namespace phx
