// The fused RK4 iteration (phx_step_fused.cuh) walking down column strips.
//
// A CTA owns a segment of a strip TW points wide and advances TH rows per
// step.  Step k (output rows r0 .. r0 + TH - 1) evaluates stage s (0-based)
// on rows r0 + 3 - s .. r0 + TH + 2 - s, so every stage computes TH new rows
// per step and the rows above them -- the vertical halo that a tile kernel
// recomputes for every tile -- come from the previous step.  Only the first
// step of a segment (the prologue) evaluates the rows above the segment, as
// a tile would.  Stage evaluations per output point: 4.25 per step at
// TW = 64 (the horizontal halo), against 5.1 for 64 x 14 tiles.
//
// Ownership: thread (i, c), i < TH, c < (TW + 6) / 2, owns the point pair of
// columns 2c, 2c + 1 of the strip + 3 and, in stage s, the row r0 + i when
// i >= 3 - s, else r0 + TH + i (a row the later stages reach only in the next
// step).  A point's stages therefore all run in one thread: its y0, n0,
// accumulators and stage reservoir stay in that thread's registers.  A thread
// with i < 3 holds two rows: it starts r0 + TH + i in the first 3 - i stages
// and finishes r0 + i in the others, keeping the row it is not working on in
// a second register set (one save at stage 0, one swap, one move at the end
// of the step).  Every thread evaluates one pair per stage.
//
// Shared memory: rings of 3 TH rows for psi, n, pump and potential (the
// tensor-memory-accelerator loads of a step's TH new rows land in one
// third while the step reads the other two), and rings of YP rows
// (>= TH + 2) for the stage values Y2, Y3, Y4.  Every point is computed with
// the operations, in the order, of rk4_tma_kernel: results are bit-identical
// to it and to the stage kernels.  Waits on mbarriers are bounded, loads
// never use multicast (the alignment argument of phx_step_tma.cuh holds: the
// boxes start 4 points left of a strip whose origin is a multiple of 64).
#pragma once

#include "phx_step_tma.cuh"

namespace phx {

template <typename T>
struct StreamParams {
    CUtensorMap psi_map;   // boxes of TW + 8 points x TH rows
    CUtensorMap n_map;
    CUtensorMap pump_map;
    CUtensorMap pot_map;
    FusedParams<T> f;
    int has_pump, has_pot;
    int strips;            // ceil(N_c / TW)
    int seg_steps;         // steps of TH rows per segment
    int n_segs;            // strips * segments per strip
    int* err;
    int wait_polls;
};

__host__ __device__ constexpr int stream_pow2_at_least(int v) {
    int p = 1;
    while (p < v) p *= 2;
    return p;
}

template <typename T, int TW, int TH>
struct StreamLayout {
    static constexpr int W4 = TW + 8;                        // box / ring row width (points)
    static constexpr int RP = 3 * TH;                        // input ring rows
    static constexpr int YP = stream_pow2_at_least(TH + 2);  // stage ring rows
    static constexpr int SW = W4 + 2;                        // stage ring row: pad + W4 + pad
    static constexpr int al(int b) { return (b + 127) / 128 * 128; }
    static constexpr int psi_box = W4 * TH * 2 * (int)sizeof(T);
    static constexpr int real_box = W4 * TH * (int)sizeof(T);
    static constexpr int psi_off = 0;
    static constexpr int n_off = al(3 * psi_box);
    static constexpr int pump_off = n_off + al(3 * real_box);
    static constexpr int pot_off = pump_off + al(3 * real_box);
    static constexpr int y_bytes = YP * SW * 2 * (int)sizeof(T);
    static constexpr int y_off = pot_off + al(3 * real_box);  // Y2, Y3, Y4
    static constexpr int bar_off = y_off + 3 * al(y_bytes);   // three mbarriers, one per ring third
    static constexpr int total = bar_off + 3 * 8 + 128;       // + slack to align the base to 128 bytes
};

// the point pair's per-row state (a step's own row, or the next step's)
template <typename T>
struct StreamRow {
    cx<T> y0[2], acc[2];
    T n0[2], ns[2], an[2];
};

template <typename T, bool RES, int TW, int TH, int NT, int MINB = 1, bool FMA = false>
__global__ void __launch_bounds__(NT, MINB) rk4_stream_kernel(const __grid_constant__ StreamParams<T> Q) {
    using Lay = StreamLayout<T, TW, TH>;
    constexpr int W4 = Lay::W4, RP = Lay::RP, YP = Lay::YP, SW = Lay::SW;
    constexpr int W3 = TW + 6;
    constexpr int PW = W3 / 2;
    static_assert(TH * PW <= NT, "one thread per (row offset, pair column)");
    // the prologue reads the four rows above the segment from one ring third
    static_assert(TH >= 8, "rows per step");
    // every ring third, a load's destination, starts on a 128-byte boundary
    static_assert(Lay::psi_box % 128 == 0 && Lay::real_box % 128 == 0, "ring thirds on 128-byte boundaries");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + Lay::bar_off);
    const cx<T>* s_psi = reinterpret_cast<const cx<T>*>(smem + Lay::psi_off);
    const T* s_n = reinterpret_cast<const T*>(smem + Lay::n_off);
    const T* s_pu = reinterpret_cast<const T*>(smem + Lay::pump_off);
    const T* s_po = reinterpret_cast<const T*>(smem + Lay::pot_off);
    auto yring = [&](int k) { return reinterpret_cast<cx<T>*>(smem + Lay::y_off + k * Lay::al(Lay::y_bytes)); };

    const FusedParams<T>& P = Q.f;
    const bool has_pump = Q.has_pump != 0, has_pot = Q.has_pot != 0;
    const long long pitch = P.pitch;
    const int ti = threadIdx.x / PW, tc = threadIdx.x - (threadIdx.x / PW) * PW;
    const bool slot = threadIdx.x < TH * PW;
    const int qx = 2 * tc;  // strip + 3 column of the pair

    if (threadIdx.x == 0) {
        for (int k = 0; k < 3; ++k) mbar_init(&bars[k], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    pdl_wait();  // the previous iteration's kernel has completed
    __syncthreads();
    unsigned phase = 0;  // bit t: parity of the next phase of ring third t's mbarrier
    // step m of a segment (m = 0: the prologue) has base row R + (m - 1) TH;
    // its new rows -- psi r0 + 4 .., n, pump, potential r0 + 3 .., TH each --
    // land in ring third (m + 2) % 3
    auto issue = [&](int tx0, int R, int m) {
        const int third = (m + 2) % 3;
        const int r0 = R + (m - 1) * TH;
        unsigned char* base = smem;
        const unsigned bytes = (unsigned)Lay::psi_box + (unsigned)Lay::real_box * (RES ? 1u : 0u) +
                               (unsigned)Lay::real_box * ((RES && has_pump) ? 1u : 0u) +
                               (unsigned)Lay::real_box * (has_pot ? 1u : 0u);
        mbar_expect_tx(&bars[third], bytes);
        tma_load_2d(base + Lay::psi_off + third * Lay::psi_box, &Q.psi_map, 2 * (tx0 - 4 + kRing), r0 + 4 + kRing,
                    &bars[third]);
        if (RES)
            tma_load_2d(base + Lay::n_off + third * Lay::real_box, &Q.n_map, tx0 - 4 + kRing, r0 + 3 + kRing,
                        &bars[third]);
        if (RES && has_pump)
            tma_load_2d(base + Lay::pump_off + third * Lay::real_box, &Q.pump_map, tx0 - 4 + kRing, r0 + 3 + kRing,
                        &bars[third]);
        if (has_pot)
            tma_load_2d(base + Lay::pot_off + third * Lay::real_box, &Q.pot_map, tx0 - 4 + kRing, r0 + 3 + kRing,
                        &bars[third]);
    };

    for (int seg = blockIdx.x; seg < Q.n_segs; seg += gridDim.x) {
        const int sx = seg % Q.strips, sy = seg / Q.strips;
        const int tx0 = sx * TW, R = sy * Q.seg_steps * TH;
        const int steps = min(Q.seg_steps, (P.N_r - R + TH - 1) / TH);
        // S: the row this stage works on; O: the thread's other row (i < 3)
        StreamRow<T> S, O;
        if (threadIdx.x == 0) issue(tx0, R, 0);
        for (int m = 0; m <= steps; ++m) {
            const int r0 = R + (m - 1) * TH;
            const int third = (m + 2) % 3;
            // the next step's rows go into the third this step does not read
            // (the previous step's reads of it ended at its closing barrier)
            const bool pending = m + 1 <= steps;
            if (threadIdx.x == 0 && pending) issue(tx0, R, m + 1);
            const unsigned parity = (phase >> third) & 1u;
            const bool ok = threadIdx.x == 0 ? mbar_wait_bounded(&bars[third], parity, Q.wait_polls) : true;
            if (__syncthreads_or(!ok)) {
                if (threadIdx.x == 0) {
                    atomicExch(Q.err, 1);
                    // drain the loads still in flight before leaving
                    (void)mbar_wait_bounded(&bars[third], parity);
                    if (pending) {
                        const int nt = (m + 3) % 3;
                        (void)mbar_wait_bounded(&bars[nt], (phase >> nt) & 1u);
                    }
                }
                return;
            }
            phase ^= 1u << third;
            // ring rows of absolute row q: psi (q - R - 4) mod RP, real planes
            // (q - R - 3) mod RP, stage rings q mod YP
            const int pbase = (m - 1) * TH - 4;  // ring row of r0 in the psi ring, before the modulo
            const int nbase = (m - 1) * TH - 3;
            auto prow = [&](int o) {
                int v = (pbase + o) % RP;
                return v < 0 ? v + RP : v;
            };
            auto nrow = [&](int o) {
                int v = (nbase + o) % RP;
                return v < 0 ? v + RP : v;
            };
            auto yrow = [&](int q) { return q & (YP - 1); };
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const bool ahead = ti < 3 - s;  // this stage's row belongs to the next step
                if (s == 0) {
                    if (ti < 3) O = S;  // this step's own row waits; stage 0 starts the next step's
                } else if (ti == 3 - s) {
                    const StreamRow<T> t = S;  // back to this step's own row
                    S = O;
                    O = t;
                }
                const int o = ahead ? ti + TH : ti;
                const int q = r0 + o;
                // the prologue evaluates only the rows the segment needs
                const bool active = slot && qx + 1 >= s && qx < W3 - s && (m > 0 || o >= TH - 3 + s);
                if (active) {
                    const int er = nrow(o) * W4 + qx + 1;
                    cx<T> c0, c1, u0, u1, d0, d1, lft, rgt;
                    if (s == 0) {
                        const cx<T>* rc = s_psi + prow(o) * W4 + qx + 1;
                        const cx<T>* ru = s_psi + prow(o - 1) * W4 + qx + 1;
                        const cx<T>* rd = s_psi + prow(o + 1) * W4 + qx + 1;
                        c0 = rc[0], c1 = rc[1];
                        u0 = ru[0], u1 = ru[1];
                        d0 = rd[0], d1 = rd[1];
                        lft = rc[-1], rgt = rc[2];
                        S.y0[0] = c0, S.y0[1] = c1;
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            S.n0[h] = RES ? s_n[er + h] : (T)0;
                            S.ns[h] = S.n0[h];
                        }
                    } else {
                        const cx<T>* in = yring(s - 1);
                        const int ep = yrow(q) * SW + qx + 2;
                        lds_pair(in + ep, c0, c1);
                        lds_pair(in + yrow(q - 1) * SW + qx + 2, u0, u1);
                        lds_pair(in + yrow(q + 1) * SW + qx + 2, d0, d1);
                        lft = in[ep - 1], rgt = in[ep + 2];
                    }
                    const T pu0 = (RES && has_pump) ? s_pu[er] : (T)0, pu1 = (RES && has_pump) ? s_pu[er + 1] : (T)0;
                    const T po0 = has_pot ? s_po[er] : (T)0, po1 = has_pot ? s_po[er + 1] : (T)0;
                    cx<T> kw[2];
                    T kr[2] = {(T)0, (T)0};
                    rhs_iter<T, RES, FMA>(P, s, c0, u0, d0, lft, c1, S.ns[0], pu0, po0, has_pump, has_pot, kw[0], kr[0]);
                    rhs_iter<T, RES, FMA>(P, s, c1, u1, d1, c0, rgt, S.ns[1], pu1, po1, has_pump, has_pot, kw[1], kr[1]);
                    cx<T> o2[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        if (s == 0) {
                            S.acc[h] = smul(P.b[0], kw[h]);
                            S.an[h] = rmul(P.b[0], kr[h]);
                        } else if (s < 3) {
                            S.acc[h] = axpy<FMA>(P.b[s], kw[h], S.acc[h]);
                            S.an[h] = raxpy<FMA>(P.b[s], kr[h], S.an[h]);
                        }
                        if (s < 3) {
                            o2[h] = axpy<FMA>(P.dtw[s], kw[h], S.y0[h]);
                            if constexpr (RES) S.ns[h] = raxpy<FMA>(P.dtw[s], kr[h], S.n0[h]);
                        } else {
                            const int gx = tx0 - 3 + qx + h;
                            if (qx + h >= 3 && qx + h < W3 - 3 && q < P.N_r && gx < P.N_c) {
                                const cx<T> ynew = final_update<FMA>(P.dt, P.b[3], S.acc[h], kw[h], S.y0[h]);
                                const long long g = (long long)q * pitch + gx;
                                P.psi1[g] = ynew;
                                if (P.img_x | P.img_y) fused_images(P, P.psi1, q, gx, ynew);
                                if constexpr (RES) {
                                    const T nnew = rfinal_update<FMA>(P.dt, P.b[3], S.an[h], kr[h], S.n0[h]);
                                    P.n1[g] = nnew;
                                    if (P.img_x | P.img_y) fused_images(P, P.n1, q, gx, nnew);
                                }
                            }
                        }
                    }
                    if (s < 3) sts_pair(yring(s) + yrow(q) * SW + qx + 2, o2[0], o2[1]);
                }
                __syncthreads();
            }
            // the rows this step started are the next step's own rows
            if (ti < 3) S = O;
            // the ring third refilled by the next issue was read by this step's
            // generic-proxy loads: order them before the async-proxy writes
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
        }
    }
}

}  // namespace phx
