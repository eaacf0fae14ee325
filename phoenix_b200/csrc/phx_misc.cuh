// Small kernels around the stage kernels: ring maintenance of padded planes,
// the k-space mask filter's gather / mask / scatter passes, and the final
// FP64 reduction of per-block partial sums.
#pragma once

#include "phx_device.cuh"
#include "phx_noise.cuh"

namespace phx {

// Zero the ring of a padded plane along non-periodic axes (what
// synchronize_halos does for a zero boundary, kernel_halo.cuh:68-70) and
// write ring-1 periodic images along periodic axes.  Grid-stride over the
// ring cells only: top/bottom bands of G rows (full padded width) and
// left/right bands of G columns (interior rows).
template <typename V>
__global__ void ring_fill_kernel(V* base, int N_r, int N_c, long long pitch, int G, int periodic_x, int periodic_y) {
    const long long W = N_c + 2LL * G;
    const long long band_tb = (long long)G * W;      // one of top / bottom
    const long long band_lr = (long long)N_r * G;    // one of left / right
    const long long total = 2 * band_tb + 2 * band_lr;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int r, c;
        if (t < 2 * band_tb) {
            const long long u = t % band_tb;
            const int rr = (int)(u / W);
            c = (int)(u % W) - G;
            r = t < band_tb ? -G + rr : N_r + rr;
        } else {
            const long long u = (t - 2 * band_tb) % band_lr;
            r = (int)(u / G);
            const int cc = (int)(u % G);
            c = (t - 2 * band_tb) < band_lr ? -G + cc : N_c + cc;
        }
        const bool out_r = r < 0 || r >= N_r;
        const bool out_c = c < 0 || c >= N_c;
        bool zero = (out_r && !periodic_y) || (out_c && !periodic_x);
        V v{};
        if (!zero) {
            // periodic image; only ring 1 is ever read by the stencil, deeper
            // rings along periodic axes are filled with images as well.
            const int sr = out_r ? (r + N_r) % N_r : r;
            const int sc = out_c ? (c + N_c) % N_c : c;
            v = base[(long long)sr * pitch + sc];
        }
        base[(long long)r * pitch + c] = v;
    }
}

// padded interior -> contiguous N_r x N_c (full_grid layout, index r*N_c + c)
template <typename T>
__global__ void gather_interior_kernel(const cx<T>* __restrict__ src, long long pitch, int N_r, int N_c, cx<T>* __restrict__ dst) {
    const long long n = (long long)N_r * N_c;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / N_c), c = (int)(i % N_c);
        dst[i] = src[(long long)r * pitch + c];
    }
}

// kernel_mask_fft (kernel_fft.cuh:35-39): data = data / N * mask
template <typename T>
__global__ void mask_kernel(cx<T>* __restrict__ data, const T* __restrict__ mask, long long n) {
    const T fn = (T)n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const cx<T> d = data[i];
        const T m = mask[i];
        data[i] = mk(rmul(rdiv(d.re, fn), m), rmul(rdiv(d.im, fn), m));
    }
}

// the same, on the interior of a halo-padded plane (in-place transform)
template <typename T>
__global__ void mask_padded_kernel(cx<T>* __restrict__ base, long long pitch, int N_r, int N_c, const T* __restrict__ mask) {
    const long long n = (long long)N_r * N_c;
    const T fn = (T)n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / N_c, c = i - r * N_c;
        cx<T>* p = base + r * pitch + c;
        const cx<T> d = *p;
        const T m = mask[i];
        *p = mk(rmul(rdiv(d.re, fn), m), rmul(rdiv(d.im, fn), m));
    }
}

// contiguous -> padded interior, plus periodic images
template <typename T>
__global__ void scatter_interior_kernel(const cx<T>* __restrict__ src, cx<T>* __restrict__ dst, long long pitch, int N_r,
                                        int N_c, int periodic_x, int periodic_y) {
    const long long n = (long long)N_r * N_c;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / N_c), c = (int)(i % N_c);
        const cx<T> v = src[i];
        dst[(long long)r * pitch + c] = v;
        // periodic images four deep, as the stage kernels write them
        const bool lx = periodic_x && c < 4, hx = periodic_x && c >= N_c - 4;
        const bool ly = periodic_y && r < 4, hy = periodic_y && r >= N_r - 4;
        const bool ex = lx || hx, ey = ly || hy;
        const int ci = lx ? c + N_c : c - N_c;
        const int ri = ly ? r + N_r : r - N_r;
        if (ex) dst[(long long)r * pitch + ci] = v;
        if (ey) dst[(long long)ri * pitch + c] = v;
        if (ex && ey) dst[(long long)ri * pitch + ci] = v;
    }
}

// ---- Adaptive error norm as the reference takes it over one halo-padded
// subgrid (halo H = k_max; adaptTimeStep sums rk_error and
// |buffer_wavefunction_plus|^2 over every padded cell, solver.cu:73-75,
// cuda_matrix.cuh:614-632,699-705).  Stage s computes k_s out to ring H - s
// and intermediate sum m writes Y_{m+1} out to ring H - m, so a padded point
// at ring distance rho (1..H-1) holds Y_{m+1} of sum m = min(S, H - rho) and
// only k_1..k_{H-rho} were ever computed there: its error term uses those.
// Along periodic axes those cells are exact copies of the wrapped interior
// point; along zero axes they are the computed ring values, stored in place.
template <typename T>
struct RingParams {
    const cx<T>* psi0;  // state (y0)
    const cx<T>* k;     // k-stack, plane stride
    long long pitch, plane;
    int N_r, N_c, periodic_x, periodic_y;
    int H, S, E;       // halo, solution-sum index, error weights
    T dt;
    T dtw1;            // dt * a21 (single-weight first stage sum)
    T a[kMaxStages][kMaxStages];  // stage-sum weights, row m-1 builds Y_{m+1} (row S-1: the solution)
    int nw[kMaxStages];
    T e[kMaxStages];   // error weights
    int passes;        // 1, or 2 where the reference counts the plus error twice
    double* partials;  // per-block (error, norm)
    // stochastic dw term of the stage sums (as in the stage kernels)
    NoiseParams noise;
    T noise_amp, w_sum[kMaxStages], R, gamma_c, four_dV, noise_scale;
    const T* n0;       // state reservoir, or nullptr without reservoir
    int imag;          // imaginary time: the sums' complex step (0, -dt), as in the stage kernels
    T dtw_final;       // final_ring_kernel: dt * b_1 for a one-weight final sum
};

template <typename T>
__device__ __forceinline__ cx<T> ring_inc(const RingParams<T>& R, cx<T> v) {
    return R.imag ? mi(v) : v;
}

template <typename T>
__global__ void dp45_ring_kernel(const __grid_constant__ RingParams<T> R) {
    const int B = R.H - 1;
    const long long W = R.N_c + 2LL * B;
    const long long band_tb = (long long)B * W, band_lr = (long long)R.N_r * B;
    const long long total = 2 * band_tb + 2 * band_lr;
    double err = 0.0, nrm = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int r, c;
        if (t < 2 * band_tb) {
            const long long u = t % band_tb;
            r = (t < band_tb ? -B : R.N_r) + (int)(u / W);
            c = (int)(u % W) - B;
        } else {
            const long long u = (t - 2 * band_tb) % band_lr;
            r = (int)(u / B);
            c = ((t - 2 * band_tb) < band_lr ? -B : R.N_c) + (int)(u % B);
        }
        const int dr = r < 0 ? -r : (r >= R.N_r ? r - R.N_r + 1 : 0);
        const int dc = c < 0 ? -c : (c >= R.N_c ? c - R.N_c + 1 : 0);
        const int rho = max(dr, dc);
        const int sr = (dr && R.periodic_y) ? (r + R.N_r) % R.N_r : r;
        const int sc = (dc && R.periodic_x) ? (c + R.N_c) % R.N_c : c;
        const long long idx = (long long)sr * R.pitch + sc;
        const int kv = R.H - rho;           // k_1..k_kv exist here
        const int m = min(R.S, kv);         // buffer holds Y_{m+1}
        cx<T> e = mk((T)0, (T)0);
        for (int j = 0; j < min(R.E, kv); ++j) {
            if (R.e[j] == (T)0) continue;
            e = cadd(e, smul(R.e[j], R.k[(long long)j * R.plane + idx]));
        }
        err += (double)abs2(smul(R.dt, e)) * (double)R.passes;
        const cx<T> y0 = R.psi0[idx];
        cx<T> y;
        if (m == 1) {
            y = cadd(y0, ring_inc(R, smul(R.dtw1, R.k[idx])));
        } else {
            // as the stage kernels: up to 7 weights left to right, more nested from the right
            const int n = R.nw[m - 1];
            const bool wide = n > 7;
            cx<T> acc = mk((T)0, (T)0);
            bool have = false;
            for (int u = 0; u < n; ++u) {
                const int q = wide ? n - 1 - u : u;
                if (wide && R.a[m - 1][q] == (T)0) continue;
                const cx<T> tq = smul(R.a[m - 1][q], R.k[(long long)q * R.plane + idx]);
                acc = !have ? tq : (wide ? cadd(tq, acc) : cadd(acc, tq));
                have = true;
            }
            y = cadd(y0, ring_inc(R, smul(R.dt, acc)));
        }
        if (R.noise.on) {
            const cx<T> xi = noise_xi(R.noise, noise_point(r, c, R.N_r, R.N_c, R.periodic_x, R.periodic_y), R.noise_amp);
            const T s_ = R.n0 ? rsqrt_rn(rdiv(radd(rmul(R.R, R.n0[idx]), R.gamma_c), R.four_dV)) : R.noise_scale;
            y = cadd(y, mk(rmul(rmul(R.w_sum[m - 1], xi.re), s_), rmul(rmul(R.w_sum[m - 1], xi.im), s_)));
        }
        nrm += (double)abs2(y);
    }
    for (int o = 16; o > 0; o >>= 1) {
        err += __shfl_down_sync(0xffffffffu, err, o);
        nrm += __shfl_down_sync(0xffffffffu, nrm, o);
    }
    __shared__ double s[64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s[2 * warp] = err;
        s[2 * warp + 1] = nrm;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) {
            a += s[2 * w];
            b += s[2 * w + 1];
        }
        R.partials[2 * blockIdx.x] = a;
        R.partials[2 * blockIdx.x + 1] = b;
    }
}

// The halo rings 1..H of the state after an in-place final sum
// (FINAL_SUM_K over the whole padded subgrid, cuda_macro.cuh:200-229), for
// the imaginary-time normalisation over the padded buffer
// (solver_normalize_imag_time.cu:14-25).  A cell at ring distance rho holds
// y0 + dt sum_q b_q k_q with only k_1..k_{H-rho} ever computed there (the
// others stay zero, so they add nothing), plus the dw term; y0 is the
// synchronised halo of the step's start (images along periodic axes, zero
// outside a zero axis), read from the state before the final sum replaces
// it.  Rows: R.a[R.S - 1] / R.nw[R.S - 1] hold the final weights.
// Per-block partials (norm, 0).
template <typename T>
__global__ void final_ring_kernel(const __grid_constant__ RingParams<T> R) {
    const int B = R.H;
    const long long W = R.N_c + 2LL * B;
    const long long band_tb = (long long)B * W, band_lr = (long long)R.N_r * B;
    const long long total = 2 * band_tb + 2 * band_lr;
    const int m = R.S;  // the final sum's row
    const int n = R.nw[m - 1];
    double nrm = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int r, c;
        if (t < 2 * band_tb) {
            const long long u = t % band_tb;
            r = (t < band_tb ? -B : R.N_r) + (int)(u / W);
            c = (int)(u % W) - B;
        } else {
            const long long u = (t - 2 * band_tb) % band_lr;
            r = (int)(u / B);
            c = ((t - 2 * band_tb) < band_lr ? -B : R.N_c) + (int)(u % B);
        }
        const int dr = r < 0 ? -r : (r >= R.N_r ? r - R.N_r + 1 : 0);
        const int dc = c < 0 ? -c : (c >= R.N_c ? c - R.N_c + 1 : 0);
        const int rho = max(dr, dc);
        const int sr = (dr && R.periodic_y) ? (r + R.N_r) % R.N_r : r;
        const int sc = (dc && R.periodic_x) ? (c + R.N_c) % R.N_c : c;
        const long long idx = (long long)sr * R.pitch + sc;
        const int kv = min(n, R.H - rho);  // weights whose k exists here
        cx<T> y = R.psi0[idx];
        if (n == 1) {
            if (kv >= 1) y = cadd(y, ring_inc(R, smul(R.dtw_final, R.k[idx])));
        } else if (kv >= 1) {
            const bool wide = n > 7;
            cx<T> acc = mk((T)0, (T)0);
            bool have = false;
            for (int u = 0; u < kv; ++u) {
                const int q = wide ? kv - 1 - u : u;
                if (wide && R.a[m - 1][q] == (T)0) continue;
                const cx<T> tq = smul(R.a[m - 1][q], R.k[(long long)q * R.plane + idx]);
                acc = !have ? tq : (wide ? cadd(tq, acc) : cadd(acc, tq));
                have = true;
            }
            if (have) y = cadd(y, ring_inc(R, smul(R.dt, acc)));
        }
        if (R.noise.on) {
            const cx<T> xi = noise_xi(R.noise, noise_point(r, c, R.N_r, R.N_c, R.periodic_x, R.periodic_y), R.noise_amp);
            const T s_ = R.n0 ? rsqrt_rn(rdiv(radd(rmul(R.R, R.n0[idx]), R.gamma_c), R.four_dV)) : R.noise_scale;
            y = cadd(y, mk(rmul(rmul(R.w_sum[m - 1], xi.re), s_), rmul(rmul(R.w_sum[m - 1], xi.im), s_)));
        }
        nrm += (double)abs2(y);
    }
    for (int o = 16; o > 0; o >>= 1) nrm += __shfl_down_sync(0xffffffffu, nrm, o);
    __shared__ double s[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s[warp] = nrm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) a += s[w];
        R.partials[2 * blockIdx.x] = a;
        R.partials[2 * blockIdx.x + 1] = 0.0;
    }
}

// Imaginary-time factor sqrt(A / (s dV)) of one field, s = the sum of the
// first slots of n partial pairs rounded to T, 1 when below 1e-10
// (solver_normalize_imag_time.cu:18-25).  One block.
template <typename T>
__global__ void imag_factor_kernel(const double* __restrict__ partials, long long n, T A, T dV, T* __restrict__ factor) {
    __shared__ double s[32];
    double a = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) a += partials[2 * i];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s[warp] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) v += s[w];
        T sum = (T)v;
        if ((double)sum < 1e-10) sum = (T)1.0;
        *factor = rsqrt_rn(rdiv(A, rmul(sum, dV)));
    }
}

// every element of a padded plane (n values of T; a complex plane as 2 n)
// times the factor: complex * real is (re f, im f)
template <typename T>
__global__ void scale_plane_kernel(T* __restrict__ base, long long n, const T* __restrict__ factor, T host_factor) {
    const T f = factor ? *factor : host_factor;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        base[i] = rmul(base[i], f);
}

// Outer ring (rho == H) of the state's synchronised halo: images along
// periodic axes, zero outside any zero axis.  The reference's buffer keeps
// this ring from the state of the previous accepted step (buffers swap on
// accept, solver.cu:107-114), so the host carries the value one step.
template <typename T>
__global__ void ring7_kernel(const cx<T>* __restrict__ psi0, long long pitch, int N_r, int N_c, int periodic_x,
                             int periodic_y, int H, double* __restrict__ out) {
    const int B = H;
    const long long W = N_c + 2LL * B;
    const long long total = 2 * W + 2LL * (N_r + 2 * (B - 1));
    double a = 0.0;
    for (long long t = threadIdx.x; t < total; t += blockDim.x) {
        int r, c;
        if (t < 2 * W) {
            r = t < W ? -B : N_r + B - 1;
            c = (int)(t % W) - B;
        } else {
            const long long u = (t - 2 * W) % (N_r + 2LL * (B - 1));
            r = (int)u - (B - 1);
            c = (t - 2 * W) < (N_r + 2LL * (B - 1)) ? -B : N_c + B - 1;
        }
        const bool out_r = r < 0 || r >= N_r, out_c = c < 0 || c >= N_c;
        if ((out_r && !periodic_y) || (out_c && !periodic_x)) continue;
        const int sr = out_r ? (r + N_r) % N_r : r, sc = out_c ? (c + N_c) % N_c : c;
        a += (double)abs2(psi0[(long long)sr * pitch + sc]);
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    __shared__ double s[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s[warp] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) v += s[w];
        *out = v;
    }
}

static __global__ void finalize_pairs_kernel(const double* __restrict__ partials, long long n, double* __restrict__ out) {
    __shared__ double sa[32], sb[32];
    double a = 0.0, b = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        a += partials[2 * i];
        b += partials[2 * i + 1];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sa[warp] = a;
        sb[warp] = b;
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) / 32;
        a = lane < nw ? sa[lane] : 0.0;
        b = lane < nw ? sb[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (lane == 0) {
            out[0] = a;
            out[1] = b;
        }
    }
}

// Sum over interior points of |z|^2 (complex) or x^2 (real), FP64, two-pass:
// per-block partials (second slot unused) then finalize_pairs_kernel.
template <typename T, bool COMPLEX>
__global__ void sum_abs2_kernel(const T* __restrict__ base, long long pitch, int N_r, int N_c, double* __restrict__ partials) {
    double a = 0.0;
    const long long n = (long long)N_r * N_c;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / N_c), c = (int)(i % N_c);
        if (COMPLEX) {
            const T re = base[2 * ((long long)r * pitch + c)], im = base[2 * ((long long)r * pitch + c) + 1];
            a += (double)re * (double)re + (double)im * (double)im;
        } else {
            const T x = base[(long long)r * pitch + c];
            a += (double)x * (double)x;
        }
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    __shared__ double s[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s[warp] = a;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) / 32;
        a = lane < nw ? s[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) {
            partials[2 * blockIdx.x] = a;
            partials[2 * blockIdx.x + 1] = 0.0;
        }
    }
}

}  // namespace phx
