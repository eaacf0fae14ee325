// Reverse-mode (adjoint) RK4 for the scalar GP equation with reservoir.
//
// The reference has no adjoint.  For one RK4 iteration
//   Y1 = y, Y2 = y + dt/2 k1, Y3 = y + dt/2 k2, Y4 = y + dt k3,
//   y' = y + dt (b1 k1 + b2 k2 + b3 k3 + b4 k4),   k_s = f(Y_s),
// the vector-Jacobian product with the adjoint lam' of y' is
//   kbar_4 = dt b4 lam',  kbar_s = dt b_s lam' + a_s dt Ybar_{s+1} (s = 3, 2, 1),
//   Ybar_s = J_f(Y_s)^T kbar_s,  lam = lam' + Ybar_1 + ... + Ybar_4,
//   Pbar  += sum_s c_s kbar_s^n               (dk_n / dP = c_s, the pump envelope)
// with a_1 = a_2 = 1/2, a_3 = 1.  One launch evaluates one stage s over the
// interior; Ybar_{s+1} and lam' are read with a 5-point stencil because
// J^T contains the (symmetric) Laplacian.
//
// Complex components are carried as real pairs: the adjoint of psi = u + iv
// is dL/du + i dL/dv (the convention of torch.autograd for real losses).
// For f_psi = -i (A lap(psi) + W psi) + B psi and f_n = -(gamma_r + R|psi|^2) n + P c,
//   A = m_eff_scaled / hbar,  W = (g_c |psi|^2 + g_r n + V c_V) / hbar,
//   B = (R n - gamma_c) / 2,
// J^T (mu, m) is
//   psi: i (A lap(mu) + W mu) + B mu + 2 (g_c/hbar) Im(conj(mu) psi) psi - 2 R n m psi
//   n:   (g_r/hbar) Im(conj(mu) psi) + (R/2) Re(conj(mu) psi) - (gamma_r + R|psi|^2) m
// Periodic boundaries only: every plane keeps 1-deep periodic images, and the
// forward map is then a function of the interior points alone.
#pragma once

#include "phx_device.cuh"

namespace phx {

template <typename T>
struct AdjParams {
    int N_r, N_c;
    long long pitch;
    const cx<T>* Ypsi;   // Y_s (stage input state)
    const T* Yn;
    const cx<T>* lam_psi;  // lam' (adjoint of y'), with images
    const T* lam_n;
    const cx<T>* ybar_in_psi;  // Ybar_{s+1}, with images (s < 4)
    const T* ybar_in_n;
    cx<T>* ybar_out_psi;       // Ybar_s (s > 1), images written
    T* ybar_out_n;
    const cx<T>* acc_in_psi;  // running lam' + Ybar_4 + ... (s < 4)
    const T* acc_in_n;
    cx<T>* acc_psi;  // running sum out; at s == 1 the new lam (with images)
    T* acc_n;
    const T* pot;    // potential plane or nullptr
    const T* pump;   // pump plane or nullptr (only its presence matters: dP accumulates)
    T* pbar;         // dL/dP accumulator (interior), or nullptr
    T c_pot, c_pump; // envelope coefficients of this stage
    T dt_b, a_dt;    // dt b_s and a_s dt (0 for s == 4)
    T A, ohb, ohb_gc, ohb_gr, half_R, half_gamma_c, gamma_r, R;
    T m2, odx2, ody2;
    int s;           // stage 1..4
    int res;         // reservoir present
};

template <typename T>
__device__ __forceinline__ void adj_images(const AdjParams<T>& Q, cx<T>* base_c, T* base_r, int r, int c, cx<T> v,
                                           T w) {
    // 1-deep periodic images (the stencil of the next stage reads them)
    const bool lx = c == 0, hx = c == Q.N_c - 1, ly = r == 0, hy = r == Q.N_r - 1;
    if (!(lx || hx || ly || hy)) return;
    const int ci = lx ? Q.N_c : -1, ri = ly ? Q.N_r : -1;
    const long long p = Q.pitch;
    if (lx || hx) {
        base_c[(long long)r * p + ci] = v;
        if (base_r) base_r[(long long)r * p + ci] = w;
    }
    if (ly || hy) {
        base_c[(long long)ri * p + c] = v;
        if (base_r) base_r[(long long)ri * p + c] = w;
    }
    if ((lx || hx) && (ly || hy)) {
        base_c[(long long)ri * p + ci] = v;
        if (base_r) base_r[(long long)ri * p + ci] = w;
    }
}

template <typename T>
__device__ __forceinline__ cx<T> adj_kbar(const AdjParams<T>& Q, long long i) {
    cx<T> k = Q.lam_psi[i];
    k.re *= Q.dt_b;
    k.im *= Q.dt_b;
    if (Q.s < 4) {
        const cx<T> y = Q.ybar_in_psi[i];
        k.re += Q.a_dt * y.re;
        k.im += Q.a_dt * y.im;
    }
    return k;
}

template <typename T>
__global__ void __launch_bounds__(256) adj_stage_kernel(const __grid_constant__ AdjParams<T> Q) {
    const int c = blockIdx.x * 32 + (threadIdx.x & 31);
    const int r = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (r >= Q.N_r || c >= Q.N_c) return;
    const long long p = Q.pitch, i = (long long)r * p + c;
    // kbar_s (psi part with its 5-point stencil, n part pointwise)
    const cx<T> mu = adj_kbar(Q, i);
    const cx<T> mu_u = adj_kbar(Q, i - p), mu_d = adj_kbar(Q, i + p);
    const cx<T> mu_l = adj_kbar(Q, i - 1), mu_r = adj_kbar(Q, i + 1);
    T m = (T)0;
    if (Q.res) {
        m = Q.dt_b * Q.lam_n[i];
        if (Q.s < 4) m += Q.a_dt * Q.ybar_in_n[i];
    }
    const cx<T> psi = Q.Ypsi[i];
    const T n = Q.res ? Q.Yn[i] : (T)0;
    const T norm = psi.re * psi.re + psi.im * psi.im;
    cx<T> lap;
    lap.re = Q.m2 * mu.re + Q.ody2 * (mu_u.re + mu_d.re) + Q.odx2 * (mu_l.re + mu_r.re);
    lap.im = Q.m2 * mu.im + Q.ody2 * (mu_u.im + mu_d.im) + Q.odx2 * (mu_l.im + mu_r.im);
    T W = Q.ohb_gc * norm;
    T B = -Q.half_gamma_c;
    if (Q.res) {
        W += Q.ohb_gr * n;
        B += Q.half_R * n;
    }
    if (Q.pot) W += Q.ohb * (Q.pot[i] * Q.c_pot);
    // h = A lap(mu) + W mu; i h = (-h.im, h.re)
    const T hre = Q.A * lap.re + W * mu.re, him = Q.A * lap.im + W * mu.im;
    const T im_mbar_psi = mu.re * psi.im - mu.im * psi.re;  // Im(conj(mu) psi)
    const T re_mbar_psi = mu.re * psi.re + mu.im * psi.im;  // Re(conj(mu) psi)
    const T sp = (T)2 * Q.ohb_gc * im_mbar_psi - (Q.res ? (T)2 * Q.R * n * m : (T)0);
    cx<T> g;
    g.re = -him + B * mu.re + sp * psi.re;
    g.im = hre + B * mu.im + sp * psi.im;
    T gn = (T)0;
    if (Q.res) gn = Q.ohb_gr * im_mbar_psi + Q.half_R * re_mbar_psi - (Q.gamma_r + Q.R * norm) * m;
    if (Q.pbar) Q.pbar[i] += Q.c_pump * m;
    // lam = lam' + Ybar_4 + Ybar_3 + Ybar_2 + Ybar_1
    cx<T> acc;
    T accn = (T)0;
    if (Q.s == 4) {
        acc = Q.lam_psi[i];
        if (Q.res) accn = Q.lam_n[i];
    } else {
        acc = Q.acc_in_psi[i];
        if (Q.res) accn = Q.acc_in_n[i];
    }
    acc.re += g.re;
    acc.im += g.im;
    accn += gn;
    Q.acc_psi[i] = acc;
    if (Q.res) Q.acc_n[i] = accn;
    if (Q.s == 1) adj_images(Q, Q.acc_psi, Q.res ? Q.acc_n : nullptr, r, c, acc, accn);
    if (Q.s > 1) {
        Q.ybar_out_psi[i] = g;
        if (Q.res) Q.ybar_out_n[i] = gn;
        adj_images(Q, Q.ybar_out_psi, Q.res ? Q.ybar_out_n : nullptr, r, c, g, gn);
    }
}

// copies between a contiguous N_r x N_c array and the interior of a padded
// plane (device to device), with the periodic images of the plane
template <typename V>
__global__ void pack_interior_kernel(const V* __restrict__ plane, long long pitch, int N_r, int N_c, V* __restrict__ dense) {
    const long long n = (long long)N_r * N_c;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long r = k / N_c, c = k - r * N_c;
        dense[k] = plane[r * pitch + c];
    }
}
template <typename V>
__global__ void unpack_interior_kernel(const V* __restrict__ dense, V* __restrict__ plane, long long pitch, int N_r, int N_c) {
    const long long n = (long long)N_r * N_c;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long r = k / N_c, c = k - r * N_c;
        plane[r * pitch + c] = dense[k];
    }
}

}  // namespace phx
