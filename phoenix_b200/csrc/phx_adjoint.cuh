// Reverse-mode (adjoint) RK4 for the scalar GP equation with reservoir.
//
// The reference has no adjoint.  For one RK4 iteration
//   Y1 = y, Y2 = y + dt/2 k1, Y3 = y + dt/2 k2, Y4 = y + dt k3,
//   y' = y + dt (b1 k1 + b2 k2 + b3 k3 + b4 k4),   k_s = f(Y_s),
// the vector-Jacobian product with the adjoint lam' of y' is
//   kbar_4 = dt b4 lam',  kbar_s = dt b_s lam' + a_s dt Ybar_{s+1} (s = 3, 2, 1),
//   Ybar_s = J_f(Y_s)^T kbar_s,  lam = lam' + Ybar_1 + ... + Ybar_4,
//   Pbar  += sum_s c_s kbar_s^n               (dk_n / dP = c_s, the pump envelope)
//   Vbar  += sum_s (c_V,s / hbar) Im(conj(kbar_s^psi) Y_s^psi)
//                                  (dk_psi / dV = (c_V,s / hbar) (-i psi), the potential term
//                                   of gp_scalar, kernel_gp_compute.cuh:93-98)
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
    T* vbar;         // dL/dV accumulator (interior), or nullptr
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
    if (Q.vbar) Q.vbar[i] += Q.ohb * Q.c_pot * im_mbar_psi;
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

namespace phx {

// The four vector-Jacobian stages of one iteration in one launch.  A block
// owns a TW x TH tile; lam' is staged in shared memory with a 4-cell halo,
// Ybar_s (psi part, needed with a stencil by stage s - 1) ping-pongs between
// two shared buffers, stage s evaluated on the tile plus a (s - 1)-cell halo
// (4: 3 cells, ..., 1: none).  The n parts are pointwise and stay in
// registers, as do the running sum of Ybar and the pump gradient.  The new
// lam is written with 4-deep periodic images (the next iteration reads it
// with a 4-cell halo).  Same arithmetic as adj_stage_kernel, periodic
// boundaries only.
template <typename T>
struct AdjFusedParams {
    int N_r, N_c;
    long long pitch;
    const cx<T>* Ypsi[4];  // Y_1 .. Y_4
    const T* Yn[4];
    const cx<T>* lam_psi;  // lam' (4-deep images)
    const T* lam_n;
    cx<T>* out_psi;        // lam (another plane)
    T* out_n;
    const T* pot;
    T* pbar;
    T* vbar;               // dL/dV accumulator, or nullptr
    T c_pot[4], c_pump[4];
    T dt_b[4], a_dt[4];    // dt b_s; a_s dt (a_4 unused)
    T A, ohb, ohb_gc, ohb_gr, half_R, half_gamma_c, gamma_r, R;
    T m2, odx2, ody2;
    int res;
};

template <typename V>
__device__ __forceinline__ void adj_images4(int N_r, int N_c, long long pitch, V* base, int r, int c, V v) {
    const bool lx = c < 4, hx = c >= N_c - 4, ly = r < 4, hy = r >= N_r - 4;
    if (!(lx || hx || ly || hy)) return;
    const int cs = lx ? c + N_c : c - N_c;
    const int rs = ly ? r + N_r : r - N_r;
    if (lx || hx) base[(long long)r * pitch + cs] = v;
    if (ly || hy) base[(long long)rs * pitch + c] = v;
    if ((lx || hx) && (ly || hy)) base[(long long)rs * pitch + cs] = v;
}

// MINB: CTAs per SM the register allocation must leave room for
template <typename T, int TW, int TH, int NT, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) adj_fused_kernel(const __grid_constant__ AdjFusedParams<T> Q) {
    constexpr int W4 = TW + 8, H4 = TH + 8;  // lam' with a 4-cell halo
    constexpr int W3 = TW + 6, H3 = TH + 6;  // Ybar regions (3-cell halo at most)
    constexpr int NP = W3 * H3;
    constexpr int OWN = (NP + NT - 1) / NT;
    __shared__ cx<T> sL[H4 * W4];
    __shared__ cx<T> sB[2][H3 * W3];
    const int ty0 = blockIdx.y * TH, tx0 = blockIdx.x * TW;
    const long long p = Q.pitch;
    // every load stays within rows / columns [-4, N + 4) of the padded planes
    // (ring >= 8); cells beyond feed no output point of this tile
    for (int k = threadIdx.x; k < H4 * W4; k += NT) {
        const int y = k / W4, x = k - y * W4;
        const int r = ty0 - 4 + y, c = tx0 - 4 + x;
        sL[k] = (r < Q.N_r + 4 && c < Q.N_c + 4) ? Q.lam_psi[(long long)r * p + c] : mk((T)0, (T)0);
    }
    __syncthreads();
    T ybn[OWN], accn[OWN], pb[OWN], vb[OWN];
    cx<T> acc[OWN];
#pragma unroll
    for (int j = 0; j < OWN; ++j) {
        ybn[j] = (T)0, accn[j] = (T)0, pb[j] = (T)0, vb[j] = (T)0;
        acc[j] = mk((T)0, (T)0);
    }
#pragma unroll
    for (int s = 4; s >= 1; --s) {
        const int h = s - 1;  // halo of this stage's region
        const cx<T>* prev = sB[(s + 1) & 1];
        cx<T>* cur = sB[s & 1];
        const T dtb = Q.dt_b[s - 1], adt = s < 4 ? Q.a_dt[s - 1] : (T)0;
        // this stage's global values of every owned point, loaded before any
        // arithmetic so that the loads are in flight together
        cx<T> ypsi[OWN];
        T yn[OWN], lamn[OWN], potv[OWN];
#pragma unroll
        for (int j = 0; j < OWN; ++j) {
            const int q = threadIdx.x + NT * j;
            const int qy = q / W3, qx = q - qy * W3;
            const int dy = qy - 3, dx = qx - 3;
            const int r = ty0 + dy, c = tx0 + dx;
            const bool live = q < NP && dy >= -h && dy < TH + h && dx >= -h && dx < TW + h && r < Q.N_r + 4 && c < Q.N_c + 4;
            const long long i = (long long)r * p + c;
            ypsi[j] = live ? Q.Ypsi[s - 1][i] : mk((T)0, (T)0);
            yn[j] = (live && Q.res) ? Q.Yn[s - 1][i] : (T)0;
            lamn[j] = (live && Q.res) ? Q.lam_n[i] : (T)0;
            potv[j] = (live && Q.pot) ? Q.pot[i] : (T)0;
        }
        auto mu_at = [&](int qy, int qx) {  // kbar_s psi at W3-grid point (qy, qx) (may be a halo-4 point)
            cx<T> m = sL[(qy + 1) * W4 + qx + 1];
            m.re *= dtb;
            m.im *= dtb;
            if (s < 4) {
                const cx<T> y = prev[qy * W3 + qx];
                m.re += adt * y.re;
                m.im += adt * y.im;
            }
            return m;
        };
#pragma unroll
        for (int j = 0; j < OWN; ++j) {
            const int q = threadIdx.x + NT * j;
            if (q >= NP) continue;
            const int qy = q / W3, qx = q - qy * W3;  // W3 grid: tile offset -3
            const int dy = qy - 3, dx = qx - 3;      // offset from the tile origin
            if (dy < -h || dy >= TH + h || dx < -h || dx >= TW + h) continue;
            const int r = ty0 + dy, c = tx0 + dx;
            if (r >= Q.N_r + 4 || c >= Q.N_c + 4) {
                cur[qy * W3 + qx] = mk((T)0, (T)0);
                ybn[j] = (T)0;
                continue;
            }
            const cx<T> mu = mu_at(qy, qx);
            // neighbours: stage 4 reads lam' only (halo 4 in sL); lower stages read Ybar_{s+1}
            // on its region, one cell wider than this one
            cx<T> mu_u, mu_d, mu_l, mu_r;
            if (s == 4) {
                auto lam_mu = [&](int yy, int xx) {
                    cx<T> m = sL[(yy + 1) * W4 + xx + 1];
                    m.re *= dtb;
                    m.im *= dtb;
                    return m;
                };
                mu_u = lam_mu(qy - 1, qx), mu_d = lam_mu(qy + 1, qx), mu_l = lam_mu(qy, qx - 1), mu_r = lam_mu(qy, qx + 1);
            } else {
                mu_u = mu_at(qy - 1, qx), mu_d = mu_at(qy + 1, qx), mu_l = mu_at(qy, qx - 1), mu_r = mu_at(qy, qx + 1);
            }
            T m = (T)0;
            if (Q.res) m = dtb * lamn[j] + adt * ybn[j];
            const cx<T> psi = ypsi[j];
            const T n = yn[j];
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
            if (Q.pot) W += Q.ohb * (potv[j] * Q.c_pot[s - 1]);
            const T hre = Q.A * lap.re + W * mu.re, him = Q.A * lap.im + W * mu.im;
            const T im_mbar_psi = mu.re * psi.im - mu.im * psi.re;
            const T re_mbar_psi = mu.re * psi.re + mu.im * psi.im;
            const T sp = (T)2 * Q.ohb_gc * im_mbar_psi - (Q.res ? (T)2 * Q.R * n * m : (T)0);
            cx<T> g;
            g.re = -him + B * mu.re + sp * psi.re;
            g.im = hre + B * mu.im + sp * psi.im;
            T gn = (T)0;
            if (Q.res) gn = Q.ohb_gr * im_mbar_psi + Q.half_R * re_mbar_psi - (Q.gamma_r + Q.R * norm) * m;
            cur[qy * W3 + qx] = g;
            ybn[j] = gn;
            if (dy >= 0 && dy < TH && dx >= 0 && dx < TW) {
                acc[j].re += g.re;
                acc[j].im += g.im;
                accn[j] += gn;
                pb[j] += Q.c_pump[s - 1] * m;
                if (Q.vbar) vb[j] += Q.ohb * Q.c_pot[s - 1] * im_mbar_psi;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < OWN; ++j) {
        const int q = threadIdx.x + NT * j;
        if (q >= NP) continue;
        const int qy = q / W3, qx = q - qy * W3;
        const int dy = qy - 3, dx = qx - 3;
        if (dy < 0 || dy >= TH || dx < 0 || dx >= TW) continue;
        const int r = ty0 + dy, c = tx0 + dx;
        if (r >= Q.N_r || c >= Q.N_c) continue;
        const long long i = (long long)r * p + c;
        cx<T> l = sL[(qy + 1) * W4 + qx + 1];
        l.re += acc[j].re;
        l.im += acc[j].im;
        Q.out_psi[i] = l;
        adj_images4(Q.N_r, Q.N_c, p, Q.out_psi, r, c, l);
        if (Q.vbar) Q.vbar[i] += vb[j];
        if (Q.res) {
            const T ln = Q.lam_n[i] + accn[j];
            Q.out_n[i] = ln;
            adj_images4(Q.N_r, Q.N_c, p, Q.out_n, r, c, ln);
            if (Q.pbar) Q.pbar[i] += pb[j];
        }
    }
}

}  // namespace phx
