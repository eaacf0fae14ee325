// The fused RK4 iteration (phx_step_fused.cuh) as a persistent, TMA-fed
// kernel.
//
// Each CTA loops over output tiles.  While its threads evaluate the four
// stages of one tile, one thread has already issued the tensor-memory-
// accelerator loads (cp.async.bulk.tensor.2d) of the next tile's boxes --
// psi over tile + 4, and n, pump, potential over tile + 3 -- into the other
// of two shared-memory slots; an mbarrier with a transaction count signals
// their arrival.  The global-load latency that stalls the non-persistent
// kernel is thereby hidden behind the previous tile's arithmetic.  The
// per-point arithmetic is the same as in rk4_fused_kernel (bit-identical
// results).
//
// TMA alignment: every box starts at an x coordinate whose byte offset is a
// multiple of 16 (tile origins are multiples of the tile width; the psi box
// starts 4 points left of the tile in a plane whose ring is 8 wide, the real
// boxes 4 points left, one more than the 3 needed), and every box row is a
// multiple of 16 bytes.  Loads never use multicast.
//
// Every wait on an mbarrier is bounded: when it gives up the CTA sets the
// error flag, waits (again bounded) for the load it may still have in
// flight and leaves; the host turns the flag into PHX_ERR_TIMEOUT.
#pragma once

#include <cuda.h>

#include "phx_step_fused.cuh"

namespace phx {

template <typename T>
struct TmaParams {
    CUtensorMap psi_map;   // state psi plane as 2D T[rows][2*pitch]
    CUtensorMap n_map;     // state n plane, T[rows][pitch]
    CUtensorMap pump_map;  // pump plane (used when has_pump)
    CUtensorMap pot_map;   // potential plane (used when has_pot)
    FusedParams<T> f;      // outputs, constants, stage coefficients
    int has_pump, has_pot;
    int tiles_x, n_tiles;
    int* err;              // set to 1 when a bounded wait gave up
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: gives up after ~1 s of device clock
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
    const long long t0 = clock64();
    for (int it = 0; it < (1 << 26); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (clock64() - t0 > 2000000000LL) break;
    }
    return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// shared-memory layout of one slot (byte offsets; every box 128-byte aligned)
template <typename T, int TW, int TH>
struct TmaLayout {
    static constexpr int W4 = TW + 8, H4 = TH + 8;  // psi box (points)
    static constexpr int WR = TW + 8, HR = TH + 6;  // real boxes (points)
    static constexpr int psi_bytes = W4 * H4 * 2 * (int)sizeof(T);
    static constexpr int real_bytes = WR * HR * (int)sizeof(T);
    static constexpr int al(int b) { return (b + 127) / 128 * 128; }
    static constexpr int psi_off = 0;
    static constexpr int n_off = al(psi_bytes);
    static constexpr int pump_off = n_off + al(real_bytes);
    static constexpr int pot_off = pump_off + al(real_bytes);
    static constexpr int slot_bytes = pot_off + al(real_bytes);
    static constexpr int b_off = 2 * slot_bytes;            // stage ping-pong buffer B
    static constexpr int bar_off = b_off + al(psi_bytes);   // two mbarriers
    static constexpr int total = bar_off + 16 + 128;  // + slack to align the base to 128 bytes
};

template <typename T, bool RES, int TW, int TH, int NT>
__global__ void __launch_bounds__(NT) rk4_tma_kernel(const __grid_constant__ TmaParams<T> Q) {
    using Lay = TmaLayout<T, TW, TH>;
    constexpr int W4 = Lay::W4, WR = Lay::WR;
    constexpr int W3 = TW + 6, H3 = TH + 6;
    constexpr int PW = W3 / 2;
    constexpr int NP = PW * H3;
    constexpr int OWN = (NP + NT - 1) / NT;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // TMA destinations are 128-byte aligned: round the dynamic base up
    unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + Lay::bar_off);
    cx<T>* sB = reinterpret_cast<cx<T>*>(smem + Lay::b_off);
    const FusedParams<T>& P = Q.f;
    const bool has_pump = Q.has_pump != 0, has_pot = Q.has_pot != 0;
    const long long pitch = P.pitch;
    const unsigned tx_bytes = (unsigned)Lay::psi_bytes + (unsigned)Lay::real_bytes * (RES ? 1u : 0u) +
                              (unsigned)Lay::real_bytes * ((RES && has_pump) ? 1u : 0u) +
                              (unsigned)Lay::real_bytes * (has_pot ? 1u : 0u);

    auto issue = [&](int slot, int tile) {
        unsigned char* base = smem + slot * Lay::slot_bytes;
        const int ty0 = (tile / Q.tiles_x) * TH, tx0 = (tile % Q.tiles_x) * TW;
        mbar_expect_tx(&bars[slot], tx_bytes);
        // psi: x in T units (2 per point) of the padded plane, ring kRing
        tma_load_2d(base + Lay::psi_off, &Q.psi_map, 2 * (tx0 - 4 + kRing), ty0 - 4 + kRing, &bars[slot]);
        if (RES) tma_load_2d(base + Lay::n_off, &Q.n_map, tx0 - 4 + kRing, ty0 - 3 + kRing, &bars[slot]);
        if (RES && has_pump) tma_load_2d(base + Lay::pump_off, &Q.pump_map, tx0 - 4 + kRing, ty0 - 3 + kRing, &bars[slot]);
        if (has_pot) tma_load_2d(base + Lay::pot_off, &Q.pot_map, tx0 - 4 + kRing, ty0 - 3 + kRing, &bars[slot]);
    };

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    int tile = blockIdx.x;
    if (threadIdx.x == 0 && tile < Q.n_tiles) issue(0, tile);
    int it = 0;
    bool pending_next = false;  // thread 0: a load into the other slot is in flight
    for (; tile < Q.n_tiles; tile += gridDim.x, ++it) {
        const int slot = it & 1;
        const unsigned parity = (unsigned)((it >> 1) & 1);
        const int next = tile + gridDim.x;
        if (threadIdx.x == 0) {
            pending_next = next < Q.n_tiles;
            if (pending_next) issue(slot ^ 1, next);
        }
        const bool ok = mbar_wait_bounded(&bars[slot], parity);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicExch(Q.err, 1);
                // drain this CTA's loads still in flight before leaving
                (void)mbar_wait_bounded(&bars[slot], parity);
                if (pending_next) (void)mbar_wait_bounded(&bars[slot ^ 1], (unsigned)(((it + 1) >> 1) & 1));
            }
            return;
        }
        unsigned char* base = smem + slot * Lay::slot_bytes;
        cx<T>* sA = reinterpret_cast<cx<T>*>(base + Lay::psi_off);
        const T* s_n = reinterpret_cast<const T*>(base + Lay::n_off);
        const T* s_pu = reinterpret_cast<const T*>(base + Lay::pump_off);
        const T* s_po = reinterpret_cast<const T*>(base + Lay::pot_off);
        const int ty0 = (tile / Q.tiles_x) * TH, tx0 = (tile % Q.tiles_x) * TW;

        cx<T> y0[OWN][2], acc[OWN][2];
        T n0[OWN][2], ns[OWN][2], an[OWN][2];
#pragma unroll
        for (int j = 0; j < OWN; ++j) {
            const int p = threadIdx.x + NT * j;
            const int qy = p / PW, qx = 2 * (p - qy * PW);
            const bool own = p < NP;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                y0[j][h] = own ? sA[(qy + 1) * W4 + qx + 1 + h] : mk((T)0, (T)0);
                n0[j][h] = (RES && own) ? s_n[qy * WR + qx + 1 + h] : (T)0;
                ns[j][h] = n0[j][h];
            }
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const cx<T>* in = (s & 1) ? sB : sA;
            cx<T>* out = (s & 1) ? sA : sB;
#pragma unroll
            for (int j = 0; j < OWN; ++j) {
                const int p = threadIdx.x + NT * j;
                const int qy = p / PW, qx = 2 * (p - qy * PW);
                if (p >= NP || qy < s || qy >= H3 - s || qx + 1 < s || qx >= W3 - s) continue;
                const int e = (qy + 1) * W4 + qx + 1;
                const int er = qy * WR + qx + 1;
                cx<T> c0, c1;
                if (s == 0) {
                    c0 = y0[j][0];
                    c1 = y0[j][1];
                } else {
                    c0 = in[e];
                    c1 = in[e + 1];
                }
                const cx<T> u0 = in[e - W4], u1 = in[e - W4 + 1];
                const cx<T> d0 = in[e + W4], d1 = in[e + W4 + 1];
                const cx<T> lft = in[e - 1], rgt = in[e + 2];
                const T pu0 = (RES && has_pump) ? s_pu[er] : (T)0, pu1 = (RES && has_pump) ? s_pu[er + 1] : (T)0;
                const T po0 = has_pot ? s_po[er] : (T)0, po1 = has_pot ? s_po[er + 1] : (T)0;
                cx<T> kw[2];
                T kr[2] = {(T)0, (T)0};
                rhs_fused<T, RES>(P, s, c0, u0, d0, lft, c1, ns[j][0], pu0, po0, has_pump, has_pot, kw[0], kr[0]);
                rhs_fused<T, RES>(P, s, c1, u1, d1, c0, rgt, ns[j][1], pu1, po1, has_pump, has_pot, kw[1], kr[1]);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (s == 0) {
                        acc[j][h] = smul(P.b[0], kw[h]);
                        an[j][h] = rmul(P.b[0], kr[h]);
                    } else if (s < 3) {
                        acc[j][h] = cadd(acc[j][h], smul(P.b[s], kw[h]));
                        an[j][h] = radd(an[j][h], rmul(P.b[s], kr[h]));
                    }
                    if (s < 3) {
                        out[e + h] = cadd(y0[j][h], smul(P.dtw[s], kw[h]));
                        if constexpr (RES) ns[j][h] = radd(n0[j][h], rmul(P.dtw[s], kr[h]));
                    } else {
                        const int gy = ty0 - 3 + qy, gx = tx0 - 3 + qx + h;
                        if (qx + h >= 3 && qx + h < W3 - 3 && gy < P.N_r && gx < P.N_c) {
                            const cx<T> ynew = cadd(y0[j][h], smul(P.dt, cadd(acc[j][h], smul(P.b[3], kw[h]))));
                            const long long g = (long long)gy * pitch + gx;
                            P.psi1[g] = ynew;
                            if (P.img_x | P.img_y) fused_images(P, P.psi1, gy, gx, ynew);
                            if constexpr (RES) {
                                const T nnew = radd(n0[j][h], rmul(P.dt, radd(an[j][h], rmul(P.b[3], kr[h]))));
                                P.n1[g] = nnew;
                                if (P.img_x | P.img_y) fused_images(P, P.n1, gy, gx, nnew);
                            }
                        }
                    }
                }
            }
            __syncthreads();
        }
        // this slot is refilled by the async proxy two tiles later: order this
        // tile's shared-memory accesses before that
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
    }
}

}  // namespace phx
