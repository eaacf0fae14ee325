// The whole RK4 iteration of the TE/TM spinor (psi+, psi-, n+, n-) in one
// kernel: the four stage evaluations of stage_tetm_kernel
// (phx_stage_tetm.cuh) on one tile, with the stage values of tile + halo in
// shared memory instead of global stage planes.
//
// Block: NT threads, one TW x TH output tile.  Both components of psi over
// tile + 4 are staged in shared memory; stage s (0-based) evaluates tile +
// (3 - s), so every stencil point of the next stage -- the nine-point stencil
// of the TE-TM term reads the diagonal neighbours -- was computed here.  A
// thread owns horizontal point pairs of tile + 3: their y0, reservoirs and
// accumulators stay in registers for the four stages.  Halo points along
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
    static constexpr int plane = SW * H4;           // points of one buffer
    static constexpr int bytes = 4 * plane * (int)sizeof(cx<T>);  // A/B x plus/minus
};

template <typename T, int TW, int TH, int NT>
__global__ void __launch_bounds__(NT) rk4_tetm_fused_kernel(const __grid_constant__ TetmFusedParams<T> F) {
    static_assert(TW % 2 == 0, "pairs");
    using Lay = TetmFusedLayout<T, TW, TH>;
    constexpr int W4 = Lay::W4, H4 = Lay::H4, SW = Lay::SW;
    constexpr int W3 = TW + 6, H3 = TH + 6;
    constexpr int PW = W3 / 2;
    constexpr int NP = PW * H3;
    constexpr int OWN = (NP + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char tetm_smem[];
    cx<T>* buf = reinterpret_cast<cx<T>*>(tetm_smem);
    // buffer b (0 = A, 1 = B) of component q
    auto sbuf = [&](int b, int q) { return buf + (2 * b + q) * Lay::plane; };

    const StageParams<T>& P0 = F.st[0].p;
    const long long pitch = P0.pitch;
    const int N_r = P0.N_r, N_c = P0.N_c;
    const int tx0 = blockIdx.x * TW, ty0 = blockIdx.y * TH;
    const int rmax = N_r + kRing - 1, cmax = N_c + kRing - 1;

    // 1) psi0 of both components over tile + 4 into A
    for (int i = threadIdx.x; i < H4 * W4; i += NT) {
        const int ry = i / W4, rx = i - ry * W4;
        const int gy = min(ty0 - 4 + ry, rmax), gx = min(tx0 - 4 + rx, cmax);
        const long long g = (long long)gy * pitch + gx;
        sbuf(0, 0)[ry * SW + rx + 1] = F.psi0[0][g];
        sbuf(0, 1)[ry * SW + rx + 1] = F.psi0[1][g];
    }
    // 2) reservoirs of the owned pairs
    T n0p[OWN][2], n0m[OWN][2], nsp[OWN][2], nsm[OWN][2], anp[OWN][2], anm[OWN][2];
    cx<T> y0p[OWN][2], y0m[OWN][2], ap[OWN][2], am[OWN][2];
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
            n0p[j][h] = own ? __ldg(F.n0[0] + g) : (T)0;
            n0m[j][h] = own ? __ldg(F.n0[1] + g) : (T)0;
            nsp[j][h] = n0p[j][h];
            nsm[j][h] = n0m[j][h];
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < OWN; ++j) {
        const int p = threadIdx.x + NT * j;
        const int qy = p / PW, qx = 2 * (p - qy * PW);
        const int e = (qy + 1) * SW + qx + 2;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            y0p[j][h] = p < NP ? sbuf(0, 0)[e + h] : mk((T)0, (T)0);
            y0m[j][h] = p < NP ? sbuf(0, 1)[e + h] : mk((T)0, (T)0);
        }
    }

    // 3) stages: s reads buffer s & 1 and writes the other
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const TetmParams<T>& Q = F.st[s];
        const StageParams<T>& P = Q.p;
        const cx<T>* ip = sbuf(s & 1, 0);
        const cx<T>* im = sbuf(s & 1, 1);
        cx<T>* op = sbuf((s + 1) & 1, 0);
        cx<T>* om = sbuf((s + 1) & 1, 1);
#pragma unroll
        for (int j = 0; j < OWN; ++j) {
            const int p = threadIdx.x + NT * j;
            const int qy = p / PW, qx = 2 * (p - qy * PW);
            if (p >= NP || qy < s || qy >= H3 - s || qx + 1 < s || qx >= W3 - s) continue;
            const int e0 = (qy + 1) * SW + qx + 2;
            const int gy = ty0 - 3 + qy;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int e = e0 + h;
                const int gx = tx0 - 3 + qx + h;
                const long long idx = (long long)min(gy, rmax) * pitch + min(gx, cmax);
                cx<T> kwp, kwm;
                T krp, krm;
                rhs_tetm<T>(Q, idx, ip[e], ip[e - SW], ip[e + SW], ip[e - 1], ip[e + 1], ip[e - SW - 1], ip[e - SW + 1],
                            ip[e + SW - 1], ip[e + SW + 1], im[e], im[e - SW], im[e + SW], im[e - 1], im[e + 1],
                            im[e - SW - 1], im[e - SW + 1], im[e + SW - 1], im[e + SW + 1], nsp[j][h], nsm[j][h], kwp, krp,
                            kwm, krm);
                // the kRk4First / kRk4Mid / kRk4Last sums of stage_tetm_kernel
                cx<T> owp, owm;
                T orp, orm;
                if (s == 0) {
                    ap[j][h] = smul(P.b, kwp);
                    am[j][h] = smul(P.b, kwm);
                    anp[j][h] = rmul(P.b, krp);
                    anm[j][h] = rmul(P.b, krm);
                } else if (s < 3) {
                    ap[j][h] = cadd(ap[j][h], smul(P.b, kwp));
                    am[j][h] = cadd(am[j][h], smul(P.b, kwm));
                    anp[j][h] = radd(anp[j][h], rmul(P.b, krp));
                    anm[j][h] = radd(anm[j][h], rmul(P.b, krm));
                }
                if (s < 3) {
                    owp = cadd(y0p[j][h], smul(P.dtw, kwp));
                    owm = cadd(y0m[j][h], smul(P.dtw, kwm));
                    orp = radd(n0p[j][h], rmul(P.dtw, krp));
                    orm = radd(n0m[j][h], rmul(P.dtw, krm));
                } else {
                    owp = cadd(y0p[j][h], smul(P.dt, cadd(ap[j][h], smul(P.b, kwp))));
                    owm = cadd(y0m[j][h], smul(P.dt, cadd(am[j][h], smul(P.b, kwm))));
                    orp = radd(n0p[j][h], rmul(P.dt, radd(anp[j][h], rmul(P.b, krp))));
                    orm = radd(n0m[j][h], rmul(P.dt, radd(anm[j][h], rmul(P.b, krm))));
                }
                if (P.noise.on) {
                    // one noise value for both polarisations, scaled by the plus
                    // reservoir; the last sum sees the updated n+ for psi-
                    const cx<T> xi = stage_xi(P, gy, gx);
                    owp = cadd(owp, stage_noise_of<T, true>(P, xi, n0p[j][h]));
                    owm = cadd(owm, stage_noise_of<T, true>(P, xi, s == 3 ? orp : n0p[j][h]));
                }
                if (s < 3) {
                    op[e] = owp;
                    om[e] = owm;
                    nsp[j][h] = orp;
                    nsm[j][h] = orm;
                } else if (qx + h >= 3 && qx + h < W3 - 3 && gy < N_r && gx < N_c) {
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
        }
        if (s < 3) __syncthreads();
    }
}

}  // namespace phx
