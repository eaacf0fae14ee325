// The whole RK4 iteration of the TE/TM spinor (psi+, psi-, n+, n-) in one
// kernel: the four stage evaluations of stage_tetm_kernel
// (phx_stage_tetm.cuh) on one tile, with the stage values of tile + halo in
// shared memory instead of global stage planes.
//
// Block: NT threads, one TW x TH output tile.  Both components of psi over
// tile + 4 are staged in shared memory; stage s (0-based) evaluates tile +
// (3 - s), so every stencil point of the next stage -- the nine-point stencil
// of the TE-TM term reads the diagonal neighbours -- was computed here.  The
// accumulators, reservoirs and the iteration's noise values of tile + 3 stay
// in shared memory as well; each stage spreads its points evenly over the
// threads, one point per item, with a single inlined copy of the two-component
// right-hand side (more copies overflow the instruction cache).  Halo points along
// periodic axes are evaluated from the images in the ring (the same values
// as the wrapped points), along zero axes from the zero ring, as the
// reference's extended stage regions are.  Each point's right-hand side,
// stage sums and noise terms are stage_tetm_kernel's (rhs_tetm, the kRk4*
// sums), so results are bit-identical to the per-stage kernels.
#pragma once

#include "phx_stage_tetm.cuh"

namespace phx {

template <typename T>
struct TetmFusedParams {
    TetmParams<T> st[4];  // stage s: the per-stage parameters (coefficients, b, dtw, w_sum, planes)
    const cx<T>* psi0[2];  // state in, [component]
    const T* n0[2];
    cx<T>* psi1[2];        // state out (other planes)
    T* n1[2];
};

template <typename T, int TW, int TH>
struct TetmFusedLayout {
    static constexpr int W4 = TW + 8, H4 = TH + 8;  // tile + 4
    static constexpr int SW = W4 + 2;               // pad + W4 + pad
    static constexpr int plane = SW * H4;           // points of one psi buffer
    static constexpr int W3 = TW + 6, H3 = TH + 6;  // tile + 3: the points of stage 0
    static constexpr int NR = W3 * H3;
    // psi: 3 buffers (A = y0, B, C) x 2 components; per tile + 3 point: the
    // accumulators of psi+- (complex), the noise value (complex), and n0,
    // stage n and accumulator of n+- (real)
    static constexpr int psi_bytes = 6 * plane * (int)sizeof(cx<T>);
    static constexpr int acc_off = psi_bytes;
    static constexpr int xi_off = acc_off + 2 * NR * (int)sizeof(cx<T>);
    static constexpr int n_off = xi_off + NR * (int)sizeof(cx<T>);
    // group 0 of the pump and of the potential, both components
    static constexpr int in_off = n_off + 6 * NR * (int)sizeof(T);
    static constexpr int bytes = in_off + 4 * NR * (int)sizeof(T);
};

// Pointwise inputs of a tile + 3 point: group 0 of the pump and potential
// from the CTA's shared copy, other groups and pulses from the global planes
template <typename T>
struct TetmTileSrc {
    const TetmParams<T>& Q;
    long long idx;
    const T* in;  // [pump+, pump-, pot+, pot-][NR] at this point: in + q
    int NR;
    __device__ __forceinline__ T pump(int c, int g) const {
        return g == 0 ? in[c * NR] : __ldg((c ? Q.pump : Q.p.pump) + idx + g * Q.p.plane);
    }
    __device__ __forceinline__ T pot(int c, int g) const {
        return g == 0 ? in[(2 + c) * NR] : __ldg((c ? Q.pot : Q.p.pot) + idx + g * Q.p.plane);
    }
    __device__ __forceinline__ cx<T> pulse(int c, int g) const { return ld1((c ? Q.pulse : Q.p.pulse) + idx + g * Q.p.plane); }
};

template <typename T, int TW, int TH, int NT>
__global__ void __launch_bounds__(NT) rk4_tetm_fused_kernel(const __grid_constant__ TetmFusedParams<T> F) {
    using Lay = TetmFusedLayout<T, TW, TH>;
    constexpr int W4 = Lay::W4, H4 = Lay::H4, SW = Lay::SW, W3 = Lay::W3, H3 = Lay::H3, NR = Lay::NR;
    extern __shared__ __align__(16) unsigned char tetm_smem[];
    cx<T>* psi = reinterpret_cast<cx<T>*>(tetm_smem);
    cx<T>* acc = reinterpret_cast<cx<T>*>(tetm_smem + Lay::acc_off);  // [2][NR]
    cx<T>* xis = reinterpret_cast<cx<T>*>(tetm_smem + Lay::xi_off);   // [NR]
    T* nv = reinterpret_cast<T*>(tetm_smem + Lay::n_off);             // [6][NR]: n0+, n0-, ns+, ns-, an+, an-
    T* tin = reinterpret_cast<T*>(tetm_smem + Lay::in_off);           // [4][NR]: pump+, pump-, pot+, pot- (group 0)
    // psi buffer b (0 = A = y0, 1 = B, 2 = C) of component q
    auto pbuf = [&](int b, int q) { return psi + (2 * b + q) * Lay::plane; };

    const StageParams<T>& P0 = F.st[0].p;
    const long long pitch = P0.pitch;
    const int N_r = P0.N_r, N_c = P0.N_c;
    const int tx0 = blockIdx.x * TW, ty0 = blockIdx.y * TH;
    const int rmax = N_r + kRing - 1, cmax = N_c + kRing - 1;
    pdl_wait();  // the previous iteration's kernel has completed

    // 1) psi0 of both components over tile + 4 into A; reservoirs and the
    // inputs of group 0 over tile + 3.  A thread issues all its loads before
    // its first shared store, so that their latencies overlap (a load-store
    // loop waits for each in turn).
    constexpr int NL0 = (H4 * W4 + NT - 1) / NT, NL1 = (NR + NT - 1) / NT;
    cx<T> vp[NL0], vm[NL0];
#pragma unroll
    for (int k = 0; k < NL0; ++k) {
        const int i = threadIdx.x + k * NT;
        if (i < H4 * W4) {
            const int ry = i / W4, rx = i - ry * W4;
            const long long g = (long long)min(ty0 - 4 + ry, rmax) * pitch + min(tx0 - 4 + rx, cmax);
            vp[k] = F.psi0[0][g];
            vm[k] = F.psi0[1][g];
        }
    }
    T va[NL1], vb[NL1], vi[4][NL1];
#pragma unroll
    for (int k = 0; k < NL1; ++k) {
        const int i = threadIdx.x + k * NT;
        if (i < NR) {
            const int qy = i / W3, qx = i - qy * W3;
            const long long g = (long long)min(ty0 - 3 + qy, rmax) * pitch + min(tx0 - 3 + qx, cmax);
            va[k] = __ldg(F.n0[0] + g), vb[k] = __ldg(F.n0[1] + g);
            if (P0.n_pump > 0) vi[0][k] = __ldg(P0.pump + g), vi[1][k] = __ldg(F.st[0].pump + g);
            if (P0.n_pot > 0) vi[2][k] = __ldg(P0.pot + g), vi[3][k] = __ldg(F.st[0].pot + g);
        }
    }
#pragma unroll
    for (int k = 0; k < NL0; ++k) {
        const int i = threadIdx.x + k * NT;
        if (i < H4 * W4) {
            const int ry = i / W4, rx = i - ry * W4;
            pbuf(0, 0)[ry * SW + rx + 1] = vp[k];
            pbuf(0, 1)[ry * SW + rx + 1] = vm[k];
        }
    }
#pragma unroll
    for (int k = 0; k < NL1; ++k) {
        const int i = threadIdx.x + k * NT;
        if (i < NR) {
            const int qy = i / W3, qx = i - qy * W3;
            nv[i] = va[k], nv[NR + i] = vb[k], nv[2 * NR + i] = va[k], nv[3 * NR + i] = vb[k];
            if (P0.noise.on) xis[i] = stage_xi(P0, ty0 - 3 + qy, tx0 - 3 + qx);
            if (P0.n_pump > 0) tin[i] = vi[0][k], tin[NR + i] = vi[1][k];
            if (P0.n_pot > 0) tin[2 * NR + i] = vi[2][k], tin[3 * NR + i] = vi[3][k];
        }
    }
    __syncthreads();

    // 2) stages: stage s evaluates tile + (3 - s); A -> B, B -> C, C -> B, B -> state.
    // One point per work item, items spread evenly over the threads; the
    // point's accumulators and reservoirs live in shared memory.  The four
    // stages are unrolled (their buffers, regions and sums become constants;
    // the item loop inside stays rolled, four copies of the right-hand side).
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const TetmParams<T>& Q = F.st[s];
        const StageParams<T>& P = Q.p;
        const int ib = s == 0 ? 0 : (s == 2 ? 2 : 1), ob = s == 1 ? 2 : 1;
        const cx<T>* ip = pbuf(ib, 0);
        const cx<T>* im = pbuf(ib, 1);
        cx<T>* op = pbuf(ob, 0);
        cx<T>* om = pbuf(ob, 1);
        const int ws = W3 - 2 * s, n_items = ws * (H3 - 2 * s);
        // the item's (row, column) in the stage's region, advanced by NT items
        // per pass without a division per item
        const int adv_r = NT / ws, adv_c = NT - adv_r * ws;
        int ir = threadIdx.x / ws, ic = threadIdx.x - ir * ws;
#pragma unroll 1
        for (int it = threadIdx.x; it < n_items; it += NT) {
            const int qy = s + ir, qx = s + ic;
            ir += adv_r, ic += adv_c;
            if (ic >= ws) ic -= ws, ++ir;
            const int q = qy * W3 + qx;                // tile + 3 index
            const int e = (qy + 1) * SW + qx + 2;      // shared psi index
            const int gy = ty0 - 3 + qy, gx = tx0 - 3 + qx;
            const long long idx = (long long)min(gy, rmax) * pitch + min(gx, cmax);
            cx<T> kwp, kwm;
            T krp, krm;
            rhs_tetm_src<T>(Q, TetmTileSrc<T>{Q, idx, tin + q, NR}, ip[e], ip[e - SW], ip[e + SW], ip[e - 1], ip[e + 1],
                            ip[e - SW - 1], ip[e - SW + 1], ip[e + SW - 1], ip[e + SW + 1], im[e], im[e - SW], im[e + SW],
                            im[e - 1], im[e + 1], im[e - SW - 1], im[e - SW + 1], im[e + SW - 1], im[e + SW + 1],
                            nv[2 * NR + q], nv[3 * NR + q], kwp, krp, kwm, krm);
            const cx<T> y0p = pbuf(0, 0)[e], y0m = pbuf(0, 1)[e];
            const T n0p = nv[q], n0m = nv[NR + q];
            // the kRk4First / kRk4Mid / kRk4Last sums of stage_tetm_kernel
            cx<T> ap, am;
            T anp, anm;
            if (s == 0) {
                ap = smul(P.b, kwp);
                am = smul(P.b, kwm);
                anp = rmul(P.b, krp);
                anm = rmul(P.b, krm);
            } else {
                ap = acc[q], am = acc[NR + q], anp = nv[4 * NR + q], anm = nv[5 * NR + q];
                if (s < 3) {
                    ap = cadd(ap, smul(P.b, kwp));
                    am = cadd(am, smul(P.b, kwm));
                    anp = radd(anp, rmul(P.b, krp));
                    anm = radd(anm, rmul(P.b, krm));
                }
            }
            cx<T> owp, owm;
            T orp, orm;
            if (s < 3) {
                owp = cadd(y0p, smul(P.dtw, kwp));
                owm = cadd(y0m, smul(P.dtw, kwm));
                orp = radd(n0p, rmul(P.dtw, krp));
                orm = radd(n0m, rmul(P.dtw, krm));
            } else {
                owp = cadd(y0p, smul(P.dt, cadd(ap, smul(P.b, kwp))));
                owm = cadd(y0m, smul(P.dt, cadd(am, smul(P.b, kwm))));
                orp = radd(n0p, rmul(P.dt, radd(anp, rmul(P.b, krp))));
                orm = radd(n0m, rmul(P.dt, radd(anm, rmul(P.b, krm))));
            }
            if (P.noise.on) {
                // one noise value for both polarisations, scaled by the plus
                // reservoir; the last sum sees the updated n+ for psi-
                const cx<T> xi = xis[q];
                owp = cadd(owp, stage_noise_of<T, true>(P, xi, n0p));
                owm = cadd(owm, stage_noise_of<T, true>(P, xi, s == 3 ? orp : n0p));
            }
            if (s < 3) {
                op[e] = owp;
                om[e] = owm;
                nv[2 * NR + q] = orp;
                nv[3 * NR + q] = orm;
                acc[q] = ap, acc[NR + q] = am, nv[4 * NR + q] = anp, nv[5 * NR + q] = anm;
            } else if (gy < N_r && gx < N_c) {
                const long long g = (long long)gy * pitch + gx;
                F.psi1[0][g] = owp;
                F.psi1[1][g] = owm;
                F.n1[0][g] = orp;
                F.n1[1][g] = orm;
                if (P.img_x | P.img_y) {
                    write_images(P, F.psi1[0], gy, gx, owp);
                    write_images(P, F.psi1[1], gy, gx, owm);
                    write_images(P, F.n1[0], gy, gx, orp);
                    write_images(P, F.n1[1], gy, gx, orm);
                }
            }
        }
        if (s < 3) __syncthreads();
    }
}

}  // namespace phx

namespace phx {

// The scalar model's whole RK4 iteration for the cases rk4_tma_kernel does
// not take (noise, pulses, several pump or potential groups, complex
// temporal coefficients): the same shared-memory scheme as
// rk4_tetm_fused_kernel with one component, and the per-stage kernel's
// right-hand side (rhs_scalar) and RK4 sums, so results are bit-identical to
// stage_scalar_kernel's.
template <typename T>
struct ScalarFusedParams {
    StageParams<T> st[4];  // stage s: coefficients, b, dtw, w_sum, input planes
    const cx<T>* psi0;
    const T* n0;
    cx<T>* psi1;
    T* n1;
};

template <typename T, int TW, int TH>
struct ScalarFusedLayout {
    static constexpr int W4 = TW + 8, H4 = TH + 8, SW = W4 + 2, plane = SW * H4;
    static constexpr int W3 = TW + 6, H3 = TH + 6, NR = W3 * H3;
    // psi: 3 buffers (A = y0, B, C); per tile + 3 point: accumulator and noise
    // value (complex), n0, stage n and accumulator of n (real)
    static constexpr int psi_bytes = 3 * plane * (int)sizeof(cx<T>);
    static constexpr int acc_off = psi_bytes;
    static constexpr int xi_off = acc_off + NR * (int)sizeof(cx<T>);
    static constexpr int n_off = xi_off + NR * (int)sizeof(cx<T>);
    static constexpr int bytes = n_off + 3 * NR * (int)sizeof(T);
};

template <typename T, bool RES, int TW, int TH, int NT>
__global__ void __launch_bounds__(NT) rk4_scalar_general_kernel(const __grid_constant__ ScalarFusedParams<T> F) {
    using Lay = ScalarFusedLayout<T, TW, TH>;
    constexpr int W4 = Lay::W4, H4 = Lay::H4, SW = Lay::SW, W3 = Lay::W3, H3 = Lay::H3, NR = Lay::NR;
    extern __shared__ __align__(16) unsigned char gen_smem[];
    cx<T>* psi = reinterpret_cast<cx<T>*>(gen_smem);
    cx<T>* acc = reinterpret_cast<cx<T>*>(gen_smem + Lay::acc_off);
    cx<T>* xis = reinterpret_cast<cx<T>*>(gen_smem + Lay::xi_off);
    T* nv = reinterpret_cast<T*>(gen_smem + Lay::n_off);  // [3][NR]: n0, stage n, accumulator
    auto pbuf = [&](int b) { return psi + b * Lay::plane; };

    const StageParams<T>& P0 = F.st[0];
    const long long pitch = P0.pitch;
    const int N_r = P0.N_r, N_c = P0.N_c;
    const int tx0 = blockIdx.x * TW, ty0 = blockIdx.y * TH;
    const int rmax = N_r + kRing - 1, cmax = N_c + kRing - 1;
    pdl_wait();  // the previous iteration's kernel has completed

    // psi0 over tile + 4, n0 over tile + 3: every load of a thread issued
    // before its first shared store (latencies overlap)
    constexpr int NL0 = (H4 * W4 + NT - 1) / NT, NL1 = (NR + NT - 1) / NT;
    cx<T> vp[NL0];
    T va[NL1];
#pragma unroll
    for (int k = 0; k < NL0; ++k) {
        const int i = threadIdx.x + k * NT;
        if (i < H4 * W4) {
            const int ry = i / W4, rx = i - ry * W4;
            vp[k] = F.psi0[(long long)min(ty0 - 4 + ry, rmax) * pitch + min(tx0 - 4 + rx, cmax)];
        }
    }
#pragma unroll
    for (int k = 0; k < NL1; ++k) {
        const int i = threadIdx.x + k * NT;
        if (i < NR) {
            const int qy = i / W3, qx = i - qy * W3;
            va[k] = RES ? __ldg(F.n0 + (long long)min(ty0 - 3 + qy, rmax) * pitch + min(tx0 - 3 + qx, cmax)) : (T)0;
        }
    }
#pragma unroll
    for (int k = 0; k < NL0; ++k) {
        const int i = threadIdx.x + k * NT;
        if (i < H4 * W4) {
            const int ry = i / W4, rx = i - ry * W4;
            pbuf(0)[ry * SW + rx + 1] = vp[k];
        }
    }
#pragma unroll
    for (int k = 0; k < NL1; ++k) {
        const int i = threadIdx.x + k * NT;
        if (i < NR) {
            const int qy = i / W3, qx = i - qy * W3;
            nv[i] = va[k], nv[NR + i] = va[k];
            if (P0.noise.on) xis[i] = stage_xi(P0, ty0 - 3 + qy, tx0 - 3 + qx);
        }
    }
    __syncthreads();

#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const StageParams<T>& P = F.st[s];
        const int ib = s == 0 ? 0 : (s == 2 ? 2 : 1), ob = s == 1 ? 2 : 1;
        const cx<T>* in = pbuf(ib);
        cx<T>* out = pbuf(ob);
        const int ws = W3 - 2 * s, n_items = ws * (H3 - 2 * s);
        const int adv_r = NT / ws, adv_c = NT - adv_r * ws;
        int ir = threadIdx.x / ws, ic = threadIdx.x - ir * ws;
#pragma unroll 1
        for (int it = threadIdx.x; it < n_items; it += NT) {
            const int qy = s + ir, qx = s + ic;
            ir += adv_r, ic += adv_c;
            if (ic >= ws) ic -= ws, ++ir;
            const int q = qy * W3 + qx;
            const int e = (qy + 1) * SW + qx + 2;
            const int gy = ty0 - 3 + qy, gx = tx0 - 3 + qx;
            const long long idx = (long long)min(gy, rmax) * pitch + min(gx, cmax);
            cx<T> kw;
            T kr = (T)0;
            rhs_scalar<T, RES>(P, idx, in[e], in[e - SW], in[e + SW], in[e - 1], in[e + 1], nv[NR + q], kw, kr);
            const cx<T> y0 = pbuf(0)[e];
            const T n0 = nv[q];
            // the kRk4First / kRk4Mid / kRk4Last sums of stage_scalar_kernel
            cx<T> a;
            T an = (T)0;
            if (s == 0) {
                a = smul(P.b, kw);
                if constexpr (RES) an = rmul(P.b, kr);
            } else {
                a = acc[q];
                if constexpr (RES) an = nv[2 * NR + q];
                if (s < 3) {
                    a = cadd(a, smul(P.b, kw));
                    if constexpr (RES) an = radd(an, rmul(P.b, kr));
                }
            }
            cx<T> o;
            T on = (T)0;
            if (s < 3) {
                o = cadd(y0, smul(P.dtw, kw));
                if constexpr (RES) on = radd(n0, rmul(P.dtw, kr));
            } else {
                o = cadd(y0, smul(P.dt, cadd(a, smul(P.b, kw))));
                if constexpr (RES) on = radd(n0, rmul(P.dt, radd(an, rmul(P.b, kr))));
            }
            if (P.noise.on) o = cadd(o, stage_noise_of<T, RES>(P, xis[q], n0));
            if (s < 3) {
                out[e] = o;
                acc[q] = a;
                if constexpr (RES) {
                    nv[NR + q] = on;
                    nv[2 * NR + q] = an;
                }
            } else if (gy < N_r && gx < N_c) {
                const long long g = (long long)gy * pitch + gx;
                F.psi1[g] = o;
                if (P.img_x | P.img_y) write_images(P, F.psi1, gy, gx, o);
                if constexpr (RES) {
                    F.n1[g] = on;
                    if (P.img_x | P.img_y) write_images(P, F.n1, gy, gx, on);
                }
            }
        }
        if (s < 3) __syncthreads();
    }
}

}  // namespace phx

