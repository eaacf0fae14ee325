// One launch per RK4 iteration: all four stages of RungeKutta4::step
// (source/cuda_solver/solver/iterator/runge_kutta.cu:74-94) fused on an
// on-chip tile.
//
// The reference evaluates a step on subgrids padded by a halo as wide as the
// number of stages and lets every stage shrink the evaluated region by one
// cell (GENERATE_SUBGRID_INDEX / CALCULATE_K, include/cuda/cuda_macro.cuh:43-49,
// 110-134).  This kernel does the same with a TW x TH output tile: the state
// is read once over the tile plus a 4-cell halo into shared memory, stage s
// is evaluated over the tile plus (4 - s) cells, the stencil input of each
// stage lives in shared memory (two ping-pong buffers) and the pointwise
// values (y0, n, accumulator, pump, potential) stay in registers of the
// thread that owns the point.  Every point is computed with the same
// operations, in the same order, as by the per-stage kernels, so the result
// is bit-identical to them and to the reference CPU build; HBM traffic per
// point drops from the 236 B of four stage passes (FP32) to the compulsory
// 32 B (read psi, n, pump, potential; write psi, n).
//
// The halo is read straight from the padded planes: along periodic axes the
// rings of psi, n, pump and potential hold periodic images at least 4 deep
// (uploads fill them; this kernel and the stage kernels write them for the
// state they produce), along zero axes they hold zeros, which is exactly the
// reference's halo after synchronize_halos (kernel_halo.cuh:50-76; pump and
// potential halos are synchronised once at initialisation,
// solver_initialization.cu:105-146).
#pragma once

#include "phx_device.cuh"
#include "phx_stage.cuh"

namespace phx {

template <typename T>
struct FusedParams {
    int N_r, N_c;
    int img_x, img_y;  // periodic axes: write images of outputs within kImg of a border
    long long pitch;
    const cx<T>* psi0;  // state in  (interior origin, padded plane)
    const T* n0;
    cx<T>* psi1;        // state out (a different plane)
    T* n1;
    const T* pump;      // one plane or nullptr
    const T* pot;       // one plane or nullptr
    T pump_c[4];        // real temporal coefficient of stage s
    T pot_c[4];
    T m2, odx2, ody2, meff, ohb;
    T ohb_gc, half_gamma_c, ohb_gr, half_R, gamma_r, R;
    T b[4];
    T dtw[3];
    T dt;
    cx<T>* st_psi[3];  // STORE: the stage values Y2..Y4 (with images), for the adjoint
    T* st_n[3];
};

constexpr int kImg = kImgDepth;

// gp_scalar right-hand side with real temporal coefficients (constant / cos /
// gauss envelopes) and the reservoir stored real.  The reference multiplies
// complex numbers whose imaginary part is exactly zero here
// ((g_r n) * (-i psi), (R/2 n) * psi, (V c) * (-i psi)); this keeps only the
// products that are not with that zero, which changes no result except,
// possibly, the sign of an exact zero.
// (PP: any parameter struct with these constants and per-stage pump_c / pot_c)
template <typename T, bool RES, typename PP>
__device__ __forceinline__ void rhs_fused(const PP& P, int s, cx<T> in_wf, cx<T> up, cx<T> dn, cx<T> left,
                                          cx<T> right, T in_rv, T pump, T pot, bool has_pump, bool has_pot, cx<T>& k_wf,
                                          T& k_rv) {
    const cx<T> in_wf_mi = mi(in_wf);
    const T in_psi_norm = abs2(in_wf);
    cx<T> wf = smul(P.meff, cadd(cadd(smul(P.m2, in_wf), smul(P.ody2, cadd(dn, up))), smul(P.odx2, cadd(right, left))));
    wf = smul(P.ohb, mi(wf));
    wf = cadd(wf, smul(rmul(P.ohb_gc, in_psi_norm), in_wf_mi));
    wf = csub(wf, smul(P.half_gamma_c, in_wf));
    if constexpr (RES) {
        wf = cadd(wf, smul(rmul(P.ohb_gr, in_rv), in_wf_mi));
        wf = cadd(wf, smul(rmul(P.half_R, in_rv), in_wf));
        T krv = rmul(-radd(P.gamma_r, rmul(P.R, in_psi_norm)), in_rv);
        if (has_pump) krv = radd(krv, rmul(pump, P.pump_c[s]));
        k_rv = krv;
    }
    if (has_pot) wf = cadd(wf, smul(rmul(P.ohb, rmul(pot, P.pot_c[s])), in_wf_mi));
    k_wf = wf;
}

// ---- fused multiply-add arithmetic (opt-in, phx_params.fma; FP32 only) ----
// The same right-hand side and stage sums as rhs_fused and the bit-exact
// stage updates, regrouped around explicitly rounded fused multiply-adds:
//   k_psi = -i (A lap(psi) + W psi) + B psi,  A = m_eff_scaled / hbar,
//   W = (g_c |psi|^2 + g_r n + V c_V) / hbar,  B = (R n - gamma_c) / 2,
//   k_n   = -(gamma_r + R |psi|^2) n + P c_P.
// Every operation is an explicit __fmaf_rn / __fmul_rn / __fadd_rn, so the
// compiler contracts nothing further and every launch shape computes the
// same bits; they differ from the reference's separately rounded products
// and sums in the last bits (about 40 % fewer instructions per point).
__device__ __forceinline__ float fm(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fm(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T, bool RES>
__device__ __forceinline__ void rhs_fma(const FusedParams<T>& P, int s, cx<T> psi, cx<T> up, cx<T> dn, cx<T> left,
                                        cx<T> right, T n, T pump, T pot, bool has_pump, bool has_pot, cx<T>& k, T& kn) {
    const T norm = fm(psi.re, psi.re, rmul(psi.im, psi.im));
    const cx<T> sv = cadd(dn, up), sh = cadd(right, left);
    const T lre = fm(P.odx2, sh.re, fm(P.ody2, sv.re, rmul(P.m2, psi.re)));
    const T lim = fm(P.odx2, sh.im, fm(P.ody2, sv.im, rmul(P.m2, psi.im)));
    T W = rmul(P.ohb_gc, norm);
    T B = -P.half_gamma_c;
    if constexpr (RES) {
        W = fm(P.ohb_gr, n, W);
        B = fm(P.half_R, n, B);
    }
    if (has_pot) W = fm(rmul(P.ohb, P.pot_c[s]), pot, W);
    const T A = rmul(P.ohb, P.meff);
    k.re = fm(A, lim, fm(W, psi.im, rmul(B, psi.re)));
    k.im = fm(-A, lre, fm(-W, psi.re, rmul(B, psi.im)));
    if constexpr (RES) {
        const T g = fm(P.R, norm, P.gamma_r);
        kn = has_pump ? fm(-g, n, rmul(pump, P.pump_c[s])) : rmul(-g, n);
    }
}

// the right-hand side of stage s in the chosen arithmetic
template <typename T, bool RES, bool FMA>
__device__ __forceinline__ void rhs_iter(const FusedParams<T>& P, int s, cx<T> in_wf, cx<T> up, cx<T> dn, cx<T> left,
                                         cx<T> right, T in_rv, T pump, T pot, bool has_pump, bool has_pot, cx<T>& k_wf,
                                         T& k_rv) {
    if constexpr (FMA)
        rhs_fma<T, RES>(P, s, in_wf, up, dn, left, right, in_rv, pump, pot, has_pump, has_pot, k_wf, k_rv);
    else
        rhs_fused<T, RES>(P, s, in_wf, up, dn, left, right, in_rv, pump, pot, has_pump, has_pot, k_wf, k_rv);
}
// y + a k
template <bool FMA, typename T>
__device__ __forceinline__ cx<T> axpy(T a, cx<T> k, cx<T> y) {
    if constexpr (FMA) return mk(fm(a, k.re, y.re), fm(a, k.im, y.im));
    else return cadd(y, smul(a, k));
}
template <bool FMA, typename T>
__device__ __forceinline__ T raxpy(T a, T k, T y) {
    if constexpr (FMA) return fm(a, k, y);
    else return radd(y, rmul(a, k));
}
// y + dt (acc + b k): the last stage's update
template <bool FMA, typename T>
__device__ __forceinline__ cx<T> final_update(T dt, T b, cx<T> acc, cx<T> k, cx<T> y) {
    if constexpr (FMA) return axpy<true>(dt, axpy<true>(b, k, acc), y);
    else return cadd(y, smul(dt, cadd(acc, smul(b, k))));
}
template <bool FMA, typename T>
__device__ __forceinline__ T rfinal_update(T dt, T b, T acc, T k, T y) {
    if constexpr (FMA) return fm(dt, fm(b, k, acc), y);
    else return radd(y, rmul(dt, radd(acc, rmul(b, k))));
}

template <typename T, typename V>
__device__ __forceinline__ void fused_images(const FusedParams<T>& P, V* base, int r, int c, V v) {
    const bool lx = P.img_x && c < kImg, hx = P.img_x && c >= P.N_c - kImg;
    const bool ly = P.img_y && r < kImg, hy = P.img_y && r >= P.N_r - kImg;
    if (!(lx || hx || ly || hy)) return;
    const int cs = lx ? c + P.N_c : c - P.N_c;
    const int rs = ly ? r + P.N_r : r - P.N_r;
    if (lx || hx) base[(long long)r * P.pitch + cs] = v;
    if (ly || hy) base[(long long)rs * P.pitch + c] = v;
    if ((lx || hx) && (ly || hy)) base[(long long)rs * P.pitch + cs] = v;
}

// Block: NT threads, one TW x TH output tile.  Grid: (ceil(N_c/TW), ceil(N_r/TH)).
// A thread owns horizontal pairs of points of tile + 3 (R3) for all four
// stages: their y0, reservoir, accumulators, pump and potential stay in its
// registers; the stencil input of each stage is in shared memory.  Shared
// planes are stored with one leading pad column so that every pair starts on
// a 16-byte boundary.
template <typename T, bool RES, int TW, int TH, int NT, bool STORE = false, bool FMA = false>
__global__ void __launch_bounds__(NT) rk4_fused_kernel(const __grid_constant__ FusedParams<T> P) {
    static_assert(TW % 2 == 0, "pairs");
    constexpr int W4 = TW + 8, H4 = TH + 8;    // tile + 4-cell halo (stage-1 stencil input)
    constexpr int SW = W4 + 2;                 // shared row: pad + W4 + pad
    constexpr int W3 = TW + 6, H3 = TH + 6;    // tile + 3 (points of stage 1)
    constexpr int PW = W3 / 2;                 // pairs per R3 row
    constexpr int NP = PW * H3;
    constexpr int OWN = (NP + NT - 1) / NT;    // pairs owned by a thread
    __shared__ __align__(16) cx<T> sA[H4 * SW];
    __shared__ __align__(16) cx<T> sB[H4 * SW];
    const int tx0 = blockIdx.x * TW, ty0 = blockIdx.y * TH;
    const long long pitch = P.pitch;
    const bool has_pump = P.pump != nullptr, has_pot = P.pot != nullptr;
    const int rmax = P.N_r + kRing - 1, cmax = P.N_c + kRing - 1;
    pdl_wait();  // the previous iteration's kernel has completed

    // 1) psi0 over tile + 4 into sA; R4 point (ry, rx) at sA[ry * SW + rx + 1].
    // The loads (and those of the pointwise values below) are all issued
    // before the first shared store, so that their latencies overlap.
    constexpr int NL = (H4 * W4 + NT - 1) / NT;
    cx<T> v[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const int i = threadIdx.x + k * NT;
        if (i < H4 * W4) {
            const int ry = i / W4, rx = i - ry * W4;
            v[k] = P.psi0[(long long)min(ty0 - 4 + ry, rmax) * pitch + min(tx0 - 4 + rx, cmax)];
        }
    }
    // 2) pointwise values of the owned pairs; R3 pair (qy, qx..qx+1)
    cx<T> y0[OWN][2], acc[OWN][2];
    T n0[OWN][2], ns[OWN][2], an[OWN][2], pu[OWN][2], po[OWN][2];
#pragma unroll
    for (int j = 0; j < OWN; ++j) {
        const int p = threadIdx.x + NT * j;
        const int qy = p / PW, qx = 2 * (p - qy * PW);
        const bool own = p < NP;
        const int gy = min(ty0 - 3 + qy, rmax);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int gx = min(tx0 - 3 + qx + h, cmax);
            const long long g = (long long)gy * pitch + gx;
            n0[j][h] = (RES && own) ? __ldg(P.n0 + g) : (T)0;
            pu[j][h] = (RES && has_pump && own) ? __ldg(P.pump + g) : (T)0;
            po[j][h] = (has_pot && own) ? __ldg(P.pot + g) : (T)0;
            ns[j][h] = n0[j][h];
        }
    }
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const int i = threadIdx.x + k * NT;
        if (i < H4 * W4) {
            const int ry = i / W4, rx = i - ry * W4;
            sA[ry * SW + rx + 1] = v[k];
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < OWN; ++j) {
        const int p = threadIdx.x + NT * j;
        const int qy = p / PW, qx = 2 * (p - qy * PW);
        const int e = (qy + 1) * SW + qx + 2;  // shared index of the pair's first point
        y0[j][0] = p < NP ? sA[e] : mk((T)0, (T)0);
        y0[j][1] = p < NP ? sA[e + 1] : mk((T)0, (T)0);
    }

    // 3) stages; stage s (0-based) covers R3 [s, H3 - s) x [s, W3 - s).  A pair
    // straddling the x edge computes both points: the outer one is never read
    // by a later stage nor stored.
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const cx<T>* in = (s & 1) ? sB : sA;
        cx<T>* out = (s & 1) ? sA : sB;
#pragma unroll
        for (int j = 0; j < OWN; ++j) {
            const int p = threadIdx.x + NT * j;
            const int qy = p / PW, qx = 2 * (p - qy * PW);
            if (p >= NP || qy < s || qy >= H3 - s || qx + 1 < s || qx >= W3 - s) continue;
            const int e = (qy + 1) * SW + qx + 2;
            cx<T> c0, c1;
            if (s == 0) {
                c0 = y0[j][0];
                c1 = y0[j][1];
            } else {
                c0 = in[e];
                c1 = in[e + 1];
            }
            const cx<T> u0 = in[e - SW], u1 = in[e - SW + 1];
            const cx<T> d0 = in[e + SW], d1 = in[e + SW + 1];
            const cx<T> lft = in[e - 1], rgt = in[e + 2];
            cx<T> kw[2];
            T kr[2] = {(T)0, (T)0};
            rhs_iter<T, RES, FMA>(P, s, c0, u0, d0, lft, c1, ns[j][0], pu[j][0], po[j][0], has_pump, has_pot, kw[0],
                                  kr[0]);
            rhs_iter<T, RES, FMA>(P, s, c1, u1, d1, c0, rgt, ns[j][1], pu[j][1], po[j][1], has_pump, has_pot, kw[1],
                                  kr[1]);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (s == 0) {
                    acc[j][h] = smul(P.b[0], kw[h]);
                    an[j][h] = rmul(P.b[0], kr[h]);
                } else if (s < 3) {
                    acc[j][h] = axpy<FMA>(P.b[s], kw[h], acc[j][h]);
                    an[j][h] = raxpy<FMA>(P.b[s], kr[h], an[j][h]);
                }
                if (s < 3) {
                    const cx<T> o = axpy<FMA>(P.dtw[s], kw[h], y0[j][h]);
                    out[e + h] = o;
                    if constexpr (RES) ns[j][h] = raxpy<FMA>(P.dtw[s], kr[h], n0[j][h]);
                    if constexpr (STORE) {
                        const int gy = ty0 - 3 + qy, gx = tx0 - 3 + qx + h;
                        if (qy >= 3 && qy < H3 - 3 && qx + h >= 3 && qx + h < W3 - 3 && gy < P.N_r && gx < P.N_c) {
                            const long long g = (long long)gy * pitch + gx;
                            P.st_psi[s][g] = o;
                            if (P.img_x | P.img_y) fused_images(P, P.st_psi[s], gy, gx, o);
                            if constexpr (RES) {
                                P.st_n[s][g] = ns[j][h];
                                if (P.img_x | P.img_y) fused_images(P, P.st_n[s], gy, gx, ns[j][h]);
                            }
                        }
                    }
                } else {
                    const int gy = ty0 - 3 + qy, gx = tx0 - 3 + qx + h;
                    if (qx + h >= 3 && qx + h < W3 - 3 && gy < P.N_r && gx < P.N_c) {
                        const cx<T> ynew = final_update<FMA>(P.dt, P.b[3], acc[j][h], kw[h], y0[j][h]);
                        const long long g = (long long)gy * pitch + gx;
                        P.psi1[g] = ynew;
                        if (P.img_x | P.img_y) fused_images(P, P.psi1, gy, gx, ynew);
                        if constexpr (RES) {
                            const T nnew = rfinal_update<FMA>(P.dt, P.b[3], an[j][h], kr[h], n0[j][h]);
                            P.n1[g] = nnew;
                            if (P.img_x | P.img_y) fused_images(P, P.n1, gy, gx, nnew);
                        }
                    }
                }
            }
        }
        if (s < 3) __syncthreads();
    }
}

}  // namespace phx
