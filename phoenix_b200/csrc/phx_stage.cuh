// Fused Runge-Kutta stage kernels for the scalar GP equation + reservoir.
//
// One launch = one RK stage over a rectangle of grid points.  Each launch
// evaluates the right-hand side of gp_scalar (scalar branch,
// include/kernel/kernel_gp_compute.cuh:37-111) at every point and, in the
// same pass, the stage accumulation that the reference runs as separate
// kernels (runge_sum_to_input_k / runge_add_to_input_k,
// include/kernel/kernel_summation.cuh:66-258).  Halo cells are resolved in
// registers: a warp owns a strip of rows of 32*CPT columns, keeps the rows
// above/below in a sliding register window and gets left/right neighbours by
// warp shuffles, so no halo-exchange kernel runs (kernel_halo.cuh:50-76 is
// replaced by writing the periodic images of border points as they are
// produced).
#pragma once

#include "phx_device.cuh"
#include "phx_noise.cuh"

namespace phx {

// Launch shapes (rows per warp, warps per block) the stage kernels are
// instantiated for; the runtime times them on the first steps of a handle
// and keeps the fastest.
constexpr int kShapes = 4;
constexpr int kShapeRB[kShapes] = {1, 2, 4, 8};
constexpr int kShapeWarps[kShapes] = {8, 8, 4, 4};
constexpr int kDefaultShape = 0;

enum StageKind : int {
    kRk4First = 0,  // k1 = f(y0); A = b1 k1; y1 = y0 + (dt a) k1
    kRk4Mid = 1,    // k = f(y_s); A += b k;  y_{s+1} = y0 + (dt a) k
    kRk4Last = 2,   // k4 = f(y3); y0 <- y0 + dt (A + b4 k4)        (in place)
    kStack = 3,     // k_s = f(y_s) stored;   y_{s+1} = y0 + dt sum_j w_j k_j
    kStackFinal = 4,// k_s = f(y_s);          y0 <- y0 + dt sum_j w_j k_j (in place)
    kStackError = 5 // k_s = f(y_s);          error / norm reduction (DP45 k7)
};

template <typename T>
struct StageParams {
    int r0, r1, c0, c1;  // compute rectangle [r0,r1) x [c0,c1), interior coordinates
    int N_r, N_c;
    int img_x, img_y;    // write ring-1 periodic images of psi_out along x / y
    long long pitch;     // elements per padded row
    long long plane;     // elements per padded plane (group / stage stride)
    const cx<T>* psi_in; // y_s wavefunction (stencil input)
    const T* n_in;       // y_s reservoir
    const cx<T>* psi0;   // y_0
    const T* n0;
    cx<T>* psi_out;      // y_{s+1}, or the state itself for the in-place kinds
    T* n_out;
    cx<T>* acc_psi;      // RK4 accumulator A
    T* acc_n;
    cx<T>* k_psi;        // k-stack, stage j at k_psi + (j-1)*plane
    T* k_n;
    const T* pump;       // n_pump planes
    const T* pot;        // n_pot planes
    const cx<T>* pulse;  // n_pulse planes
    int n_pump, n_pot, n_pulse;
    int stage;           // 1-based stage index (k-stack slot stage-1)
    int nw;              // weights of the stage sum (kStack / kStackFinal / kStackError)
    cx<T> pump_c[kMaxGroups];   // amp*(1-w) + w*amp_next for this stage
    cx<T> pot_c[kMaxGroups];
    cx<T> pulse_c[kMaxGroups];
    T w[kMaxStages];
    // Type::real kernel constants (system_parameters.hpp:25-64, system.cpp:116-160)
    T m2, odx2, ody2, meff, ohb;
    T ohb_gc, half_gamma_c, ohb_gr, half_R, gamma_r, R;
    T b;    // accumulator weight of this stage (RK4)
    T dtw;  // dt * a_{s+1,s} for single-weight stage sums
    T dt;
    double* partials;    // kStackError: per-block (error, norm) pairs
    int error_passes;    // 1, or 2 for the TE/TM double count
    // stochastic terms (noise.on): drift in the right-hand side, dw in the
    // stage sums (kernel_summation.cuh:216-224)
    NoiseParams noise;
    T noise_amp;         // dw * sqrt(dt) of this iteration
    T w_sum;             // right fold of this stage sum's weights
    T dV, four_dV;       // dV, 4 dV
    T gamma_c;
    T noise_scale;       // sqrt(gamma_c / (4 dV)), the scale without reservoir
    // imaginary time (--imagTime): the k-stack sums take the complex step
    // (0, -dt): ((0, -dt) w) k = -i (dt w) k and (0, -dt) a = -i (dt a),
    // the same bits as the complex products of the complex_dt branches
    // (kernel_summation.cuh:66-190) up to the sign of an exact zero; the
    // wavefunction only (no reservoir runs with it)
    int imag;
};

template <typename T>
__device__ __forceinline__ cx<T> step_inc(const StageParams<T>& P, cx<T> v) {
    return P.imag ? mi(v) : v;
}

// ---- 16-byte packs: CPT grid points per lane ----
template <typename T>
struct Pack {
    static constexpr int CPT = 16 / (int)sizeof(cx<T>);
    cx<T> v[CPT];
};
template <typename T>
struct RPack {
    static constexpr int CPT = 16 / (int)sizeof(cx<T>);
    T v[CPT];
};

template <typename T>
__device__ __forceinline__ Pack<T> ldp(const cx<T>* p) {
    Pack<T> r;
    const float4 u = __ldg(reinterpret_cast<const float4*>(p));
    static_assert(sizeof(Pack<T>) == 16, "pack");
    *reinterpret_cast<float4*>(&r) = u;
    return r;
}
template <typename T>
__device__ __forceinline__ Pack<T> ldp_rw(const cx<T>* p) {
    Pack<T> r;
    *reinterpret_cast<float4*>(&r) = *reinterpret_cast<const float4*>(p);
    return r;
}
template <typename T>
__device__ __forceinline__ void stp(cx<T>* p, const Pack<T>& v) {
    *reinterpret_cast<float4*>(p) = *reinterpret_cast<const float4*>(&v);
}
template <typename T>
__device__ __forceinline__ RPack<T> ldr(const T* p) {
    RPack<T> r;
    static_assert(sizeof(RPack<T>) == 8, "rpack");
    *reinterpret_cast<float2*>(&r) = __ldg(reinterpret_cast<const float2*>(p));
    return r;
}
template <typename T>
__device__ __forceinline__ RPack<T> ldr_rw(const T* p) {
    RPack<T> r;
    *reinterpret_cast<float2*>(&r) = *reinterpret_cast<const float2*>(p);
    return r;
}
template <typename T>
__device__ __forceinline__ void str(T* p, const RPack<T>& v) {
    *reinterpret_cast<float2*>(p) = *reinterpret_cast<const float2*>(&v);
}
template <typename T>
__device__ __forceinline__ cx<T> ld1(const cx<T>* p) {
    return *p;
}
template <typename T>
__device__ __forceinline__ cx<T> shfl_up1(cx<T> z) {
    return mk(__shfl_up_sync(0xffffffffu, z.re, 1), __shfl_up_sync(0xffffffffu, z.im, 1));
}
template <typename T>
__device__ __forceinline__ cx<T> shfl_dn1(cx<T> z) {
    return mk(__shfl_down_sync(0xffffffffu, z.re, 1), __shfl_down_sync(0xffffffffu, z.im, 1));
}

// amp * (1 - w) + w * amp_next, folded on the host per stage: a complex
// temporal coefficient c.  Reservoir n is stored real; pump coefficients are
// real (checked on the host), so every reservoir expression below is the
// reference's complex one with a zero imaginary part carried exactly.

// (one_over_h_bar_s g_c) (-i psi) / dV: the stochastic drift of psi
template <typename T>
__device__ __forceinline__ cx<T> noise_drift(const StageParams<T>& P, cx<T> in_wf_mi) {
    const cx<T> d = smul(P.ohb_gc, in_wf_mi);
    return mk(rdiv(d.re, P.dV), rdiv(d.im, P.dV));
}

// Right-hand side of gp_scalar, scalar branch, one grid point.
template <typename T, bool RES>
__device__ __forceinline__ void rhs_scalar(const StageParams<T>& P, long long idx, cx<T> in_wf, cx<T> up, cx<T> dn,
                                           cx<T> left, cx<T> right, T in_rv, cx<T>& k_wf, T& k_rv) {
    const cx<T> in_wf_mi = mi(in_wf);
    const T in_psi_norm = abs2(in_wf);
    // m_eff_scaled * ( m2 * psi + (psi[i+ro] + psi[i-ro]) / dy^2 + (psi[i+1] + psi[i-1]) / dx^2 )
    cx<T> wf = smul(P.meff, cadd(cadd(smul(P.m2, in_wf), smul(P.ody2, cadd(dn, up))), smul(P.odx2, cadd(right, left))));
    wf = smul(P.ohb, mi(wf));
    wf = cadd(wf, smul(rmul(P.ohb_gc, in_psi_norm), in_wf_mi));
    wf = csub(wf, smul(P.half_gamma_c, in_wf));
    if constexpr (RES) {
        const cx<T> rv = mk(in_rv, (T)0);
        wf = cadd(wf, cmul(smul(P.ohb_gr, rv), in_wf_mi));
        wf = cadd(wf, cmul(smul(P.half_R, rv), in_wf));
        const T s = -radd(P.gamma_r, rmul(P.R, in_psi_norm));
        T krv = rmul(s, in_rv);
        for (int g = 0; g < P.n_pump; ++g) krv = radd(krv, rmul(__ldg(P.pump + idx + g * P.plane), P.pump_c[g].re));
        k_rv = krv;
    }
    for (int g = 0; g < P.n_pot; ++g) {
        const T v = __ldg(P.pot + idx + g * P.plane);
        const cx<T> pot = smul(v, P.pot_c[g]);
        wf = cadd(wf, cmul(smul(P.ohb, pot), in_wf_mi));
    }
    for (int g = 0; g < P.n_pulse; ++g) {
        const cx<T> pulse = ld1(P.pulse + idx + g * P.plane);
        wf = cadd(wf, cmul(smul(P.ohb, pulse), P.pulse_c[g]));
    }
    if (P.noise.on) {
        // stochastic drift (kernel_gp_compute.cuh:82-84, 101-103)
        wf = csub(wf, noise_drift(P, in_wf_mi));
        if constexpr (RES) k_rv = radd(k_rv, rdiv(rmul(P.R, in_rv), P.dV));
    }
    k_wf = wf;
}

// dw term of a stage sum at interior point (r, c): w_sum * xi * sqrt((R n0 +
// gamma_c) / (4 dV)) with n0 the state reservoir (kernel_summation.cuh:216-224);
// the reference's product with the complex square root (x, 0) keeps each
// component's two roundings
template <typename T>
__device__ __forceinline__ cx<T> stage_xi(const StageParams<T>& P, int r, int c) {
    return noise_xi(P.noise, noise_point(r, c, P.N_r, P.N_c, P.img_x, P.img_y), P.noise_amp);
}
template <typename T, bool RES>
__device__ __forceinline__ cx<T> stage_noise_of(const StageParams<T>& P, cx<T> xi, T n0) {
    const T sc = RES ? rsqrt_rn(rdiv(radd(rmul(P.R, n0), P.gamma_c), P.four_dV)) : P.noise_scale;
    return mk(rmul(rmul(P.w_sum, xi.re), sc), rmul(rmul(P.w_sum, xi.im), sc));
}
template <typename T, bool RES>
__device__ __forceinline__ cx<T> stage_noise(const StageParams<T>& P, int r, int c, T n0) {
    return stage_noise_of<T, RES>(P, stage_xi(P, r, c), n0);
}

// Periodic images of a produced point (wavefunction and reservoir): every
// point within kImgDepth of a periodic border is also written into the ring
// on the opposite side, so the ring always holds images kImgDepth deep (the
// fused iteration evaluates stage values on a 3-4 cell halo read straight
// from the ring, as the reference does on its halo-padded subgrids).
constexpr int kImgDepth = 4;
template <typename T, typename V>
__device__ __forceinline__ void write_images(const StageParams<T>& P, V* base, int r, int c, V v) {
    const bool lx = P.img_x && c >= 0 && c < kImgDepth, hx = P.img_x && c >= P.N_c - kImgDepth && c < P.N_c;
    const bool ly = P.img_y && r >= 0 && r < kImgDepth, hy = P.img_y && r >= P.N_r - kImgDepth && r < P.N_r;
    const bool ex = lx || hx, ey = ly || hy;
    if (!(ex || ey)) return;
    const int ci = lx ? c + P.N_c : c - P.N_c;
    const int ri = ly ? r + P.N_r : r - P.N_r;
    if (ex) base[(long long)r * P.pitch + ci] = v;
    if (ey) base[(long long)ri * P.pitch + c] = v;
    if (ex && ey) base[(long long)ri * P.pitch + ci] = v;
}

template <int BLOCK>
__device__ __forceinline__ void block_reduce2(double& a, double& b, double* smem) {
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        smem[2 * warp] = a;
        smem[2 * warp + 1] = b;
    }
    __syncthreads();
    if (warp == 0) {
        a = lane < BLOCK / 32 ? smem[2 * lane] : 0.0;
        b = lane < BLOCK / 32 ? smem[2 * lane + 1] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
    }
}

// Launch: block (32*WARPS), grid (ceil(W / (32*CPT)), ceil(H / (WARPS*RB))).
// Each warp owns RB consecutive rows of 32*CPT columns.
template <typename T, int KIND, bool RES, int RB, int WARPS>
__global__ void __launch_bounds__(32 * WARPS) stage_scalar_kernel(const __grid_constant__ StageParams<T> P) {
    constexpr int CPT = Pack<T>::CPT;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int c_base = P.c0 + blockIdx.x * (32 * CPT);
    const int c = c_base + lane * CPT;
    const int rs = P.r0 + (blockIdx.y * WARPS + warp) * RB;
    const int re = min(rs + RB, P.r1);
    const bool active = c < P.c1;
    const int cl = min(c, P.c1);  // columns [c1, c1+CPT) are allocated, so clamped loads stay in bounds
    const int c_left = c_base - 1;
    const int c_right = min(c_base + 32 * CPT, P.c1);
    const long long pitch = P.pitch;

    double err_acc = 0.0, norm_acc = 0.0;

    if (rs < P.r1) {
        Pack<T> up = ldp(P.psi_in + (long long)(rs - 1) * pitch + cl);
        Pack<T> ce = ldp(P.psi_in + (long long)rs * pitch + cl);
        for (int r = rs; r < re; ++r) {
            const long long rowo = (long long)r * pitch;
            const Pack<T> dn = ldp(P.psi_in + rowo + pitch + cl);
            // left / right neighbours of this lane's points
            cx<T> lft = shfl_up1(ce.v[CPT - 1]);
            cx<T> rgt = shfl_dn1(ce.v[0]);
            if (lane == 0) lft = ld1(P.psi_in + rowo + c_left);
            if (lane == 31) rgt = ld1(P.psi_in + rowo + c_right);
            const long long idx = rowo + cl;
            RPack<T> nin;
            if constexpr (RES) nin = ldr(P.n_in + idx);
            if (active) {
                Pack<T> out_wf;
                RPack<T> out_rv;
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    const cx<T> L = j == 0 ? lft : ce.v[j - 1];
                    const cx<T> Rt = j == CPT - 1 ? rgt : ce.v[j + 1];
                    cx<T> kw;
                    T kr = (T)0;
                    rhs_scalar<T, RES>(P, idx + j, ce.v[j], up.v[j], dn.v[j], L, Rt, RES ? nin.v[j] : (T)0, kw, kr);
                    out_wf.v[j] = kw;
                    out_rv.v[j] = kr;
                }
                // ---- stage accumulation (kernel_summation.cuh) ----
                if constexpr (KIND == kRk4First || KIND == kRk4Mid || KIND == kRk4Last) {
                    const Pack<T> y0 = KIND == kRk4First ? ce : ldp(P.psi0 + idx);
                    RPack<T> n0;
                    if constexpr (RES) n0 = KIND == kRk4First ? nin : ldr(P.n0 + idx);
                    Pack<T> acc;
                    RPack<T> accn;
                    if constexpr (KIND != kRk4First) {
                        acc = ldp_rw(P.acc_psi + idx);
                        if constexpr (RES) accn = ldr_rw(P.acc_n + idx);
                    }
#pragma unroll
                    for (int j = 0; j < CPT; ++j) {
                        const cx<T> k = out_wf.v[j];
                        if constexpr (KIND == kRk4First) {
                            acc.v[j] = smul(P.b, k);
                            out_wf.v[j] = cadd(y0.v[j], smul(P.dtw, k));
                            if constexpr (RES) {
                                accn.v[j] = rmul(P.b, out_rv.v[j]);
                                out_rv.v[j] = radd(n0.v[j], rmul(P.dtw, out_rv.v[j]));
                            }
                        } else if constexpr (KIND == kRk4Mid) {
                            acc.v[j] = cadd(acc.v[j], smul(P.b, k));
                            out_wf.v[j] = cadd(y0.v[j], smul(P.dtw, k));
                            if constexpr (RES) {
                                accn.v[j] = radd(accn.v[j], rmul(P.b, out_rv.v[j]));
                                out_rv.v[j] = radd(n0.v[j], rmul(P.dtw, out_rv.v[j]));
                            }
                        } else {
                            out_wf.v[j] = cadd(y0.v[j], smul(P.dt, cadd(acc.v[j], smul(P.b, k))));
                            if constexpr (RES)
                                out_rv.v[j] = radd(n0.v[j], rmul(P.dt, radd(accn.v[j], rmul(P.b, out_rv.v[j]))));
                        }
                        if (P.noise.on) {
                            T nn = (T)0;
                            if constexpr (RES) nn = n0.v[j];
                            out_wf.v[j] = cadd(out_wf.v[j], stage_noise<T, RES>(P, r, c + j, nn));
                        }
                    }
                    if constexpr (KIND != kRk4Last) {
                        stp(P.acc_psi + idx, acc);
                        if constexpr (RES) str(P.acc_n + idx, accn);
                    }
                } else {
                    // k-stack tableau (DP45 and general explicit RK)
                    const long long kofs = (long long)(P.stage - 1) * P.plane;
                    if constexpr (KIND == kStack) {
                        stp(P.k_psi + kofs + idx, out_wf);
                        if constexpr (RES) str(P.k_n + kofs + idx, out_rv);
                    }
                    const Pack<T> y0 = P.stage == 1 ? ce : ldp(P.psi0 + idx);
                    RPack<T> n0;
                    if constexpr (RES) n0 = P.stage == 1 ? nin : ldr(P.n0 + idx);
                    if constexpr (KIND == kStackError) {
                        // runge_sum_to_error (kernel_summation.cuh:260-289): error = sum e_j k_j (nonzero e_j)
#pragma unroll
                        for (int j = 0; j < CPT; ++j) {
                            cx<T> e = mk((T)0, (T)0);
                            for (int q = 0; q < P.nw; ++q) {
                                if (P.w[q] == (T)0) continue;
                                const cx<T> kq = (q == P.stage - 1) ? out_wf.v[j]
                                                                     : ld1(P.k_psi + (long long)q * P.plane + idx + j);
                                e = cadd(e, smul(P.w[q], kq));
                            }
                            const T ee = abs2(smul(P.dt, e));
                            err_acc += (double)ee * (double)P.error_passes;
                            norm_acc += (double)abs2(ce.v[j]);
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < CPT; ++j) {
                            if (P.nw == 1) {
                                out_wf.v[j] = cadd(y0.v[j], step_inc(P, smul(P.dtw, out_wf.v[j])));
                                if constexpr (RES) out_rv.v[j] = radd(n0.v[j], rmul(P.dtw, out_rv.v[j]));
                            } else {
                                // up to 7 weights: left to right, zeros included
                                // (runge_sum_to_input_k2..k7); more: zeros dropped, nested
                                // from the right (sum_single_k, kernel_summation.cuh:7-29)
                                const bool wide = P.nw > 7;
                                cx<T> a = mk((T)0, (T)0);
                                T an = (T)0;
                                bool have = false;
                                for (int u = 0; u < P.nw; ++u) {
                                    const int q = wide ? P.nw - 1 - u : u;
                                    if (wide && P.w[q] == (T)0) continue;
                                    cx<T> kq;
                                    T kqn = (T)0;
                                    if (q == P.stage - 1) {
                                        kq = out_wf.v[j];
                                        kqn = out_rv.v[j];
                                    } else {
                                        kq = ld1(P.k_psi + (long long)q * P.plane + idx + j);
                                        if constexpr (RES) kqn = P.k_n[(long long)q * P.plane + idx + j];
                                    }
                                    const cx<T> tq = smul(P.w[q], kq);
                                    const T tn = rmul(P.w[q], kqn);
                                    if (!have) {
                                        a = tq, an = tn, have = true;
                                    } else if (wide) {
                                        a = cadd(tq, a), an = radd(tn, an);
                                    } else {
                                        a = cadd(a, tq), an = radd(an, tn);
                                    }
                                }
                                out_wf.v[j] = cadd(y0.v[j], step_inc(P, smul(P.dt, a)));
                                if constexpr (RES) out_rv.v[j] = radd(n0.v[j], rmul(P.dt, an));
                            }
                            if (P.noise.on) {
                                T nn = (T)0;
                                if constexpr (RES) nn = n0.v[j];
                                out_wf.v[j] = cadd(out_wf.v[j], stage_noise<T, RES>(P, r, c + j, nn));
                            }
                        }
                    }
                }
                if constexpr (KIND != kStackError) {
                    stp(P.psi_out + idx, out_wf);
                    if constexpr (RES) str(P.n_out + idx, out_rv);
                    if (P.img_x | P.img_y) {
#pragma unroll
                        for (int j = 0; j < CPT; ++j) {
                            write_images(P, P.psi_out, r, c + j, out_wf.v[j]);
                            if constexpr (RES) write_images(P, P.n_out, r, c + j, out_rv.v[j]);
                        }
                    }
                }
            }
            up = ce;
            ce = dn;
        }
    }
    if constexpr (KIND == kStackError) {
        __shared__ double red[2 * WARPS];
        block_reduce2<32 * WARPS>(err_acc, norm_acc, red);
        if (threadIdx.x == 0) {
            const long long b = (long long)blockIdx.y * gridDim.x + blockIdx.x;
            P.partials[2 * b] = err_acc;
            P.partials[2 * b + 1] = norm_acc;
        }
    }
}

}  // namespace phx
