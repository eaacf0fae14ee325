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
// flight and leaves; the host turns the flag into PHX_ERR_TIMEOUT.  Only
// thread 0 polls the mbarrier; the other threads wait at the CTA barrier
// that follows.
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
    int wait_polls;        // polls of a tile's mbarrier before the wait gives up (0: at once)
};

// polls of an mbarrier before a bounded wait gives up (also capped at ~1 s of
// device clock)
constexpr int kWaitPolls = 1 << 26;

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
// bounded wait: gives up after max_polls polls or ~1 s of device clock
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, int max_polls = kWaitPolls) {
    const long long t0 = clock64();
    for (int it = 0; it < max_polls; ++it) {
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
    // stage buffers B and C: rows of SW points with one leading pad point, so
    // that the point pairs a thread owns start on 16-byte boundaries
    static constexpr int SW = W4 + 2;
    static constexpr int pad_bytes = SW * H4 * 2 * (int)sizeof(T);
    static constexpr int b_off = 2 * slot_bytes;
    static constexpr int c_off = b_off + al(pad_bytes);
    static constexpr int bar_off = c_off + al(pad_bytes);  // two mbarriers
    static constexpr int total = bar_off + 16 + 128;       // + slack to align the base to 128 bytes
};

// Order earlier generic-proxy writes of a tensor map in global memory before
// this thread's uses of it by the tensor-map proxy.  The maps are written by
// a host copy, hence system scope.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* m) {
    asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(m) : "memory");
}

// 16-byte shared-memory access to the point pair at an even index
template <typename T>
__device__ __forceinline__ void lds_pair(const cx<T>* p, cx<T>& a, cx<T>& b) {
    if constexpr (sizeof(T) == 4) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        a = mk(v.x, v.y);
        b = mk(v.z, v.w);
    } else {
        a = p[0];
        b = p[1];
    }
}
template <typename T>
__device__ __forceinline__ void sts_pair(cx<T>* p, cx<T> a, cx<T> b) {
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(a.re, a.im, b.re, b.im);
    } else {
        p[0] = a;
        p[1] = b;
    }
}

// What one tile needs: its tensor maps, its parameters and its origin.
template <typename T>
struct TileRef {
    const CUtensorMap* psi_map;
    const CUtensorMap* n_map;
    const CUtensorMap* pump_map;
    const CUtensorMap* pot_map;
    const FusedParams<T>* f;
    int has_pump, has_pot;
    int tx0, ty0;
};

// Persistent tile loop shared by the single-simulation and the batched
// kernel; `tile_of(g)` returns the TileRef of global tile g.  BATCH: the
// tensor maps and parameters live in global memory (one set per instance);
// the maps are acquired for the tensor-map proxy before use and the tile's
// parameters are staged in shared memory.
// wait_polls bounds the wait for each tile's boxes (the error path gives up
// there); the drain of loads still in flight after a failed wait always uses
// the full bound, so no bulk copy lands in the shared memory of a CTA that
// has left.
template <typename T, bool RES, int TW, int TH, int NT, bool BATCH, bool STORE, bool FMA, typename TileOf>
__device__ __forceinline__ void tma_tile_loop(const TileOf& tile_of, int n_tiles, int* err, int wait_polls) {
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
    cx<T>* sC = reinterpret_cast<cx<T>*>(smem + Lay::c_off);
    constexpr int SW = Lay::SW;

    __shared__ FusedParams<T> sP;  // BATCH: this tile's parameters

    // BATCH, thread 0: the psi map of the instance whose maps it acquired
    // last.  An acquire orders the issuing thread's later uses of a map, so
    // a run of tiles of one instance needs one (fencing the same maps again
    // for every tile made a batch of one 1024^2 instance take 39.5 instead
    // of 35.0 us per iteration).
    const CUtensorMap* acquired = nullptr;
    auto issue = [&](int slot, int g) {
        const TileRef<T> R = tile_of(g);
        if constexpr (BATCH) {
            if (R.psi_map != acquired) {
                tensormap_acquire(R.psi_map);
                if (RES) tensormap_acquire(R.n_map);
                if (RES && R.has_pump) tensormap_acquire(R.pump_map);
                if (R.has_pot) tensormap_acquire(R.pot_map);
                acquired = R.psi_map;
            }
        }
        unsigned char* base = smem + slot * Lay::slot_bytes;
        const unsigned tx_bytes = (unsigned)Lay::psi_bytes + (unsigned)Lay::real_bytes * (RES ? 1u : 0u) +
                                  (unsigned)Lay::real_bytes * ((RES && R.has_pump) ? 1u : 0u) +
                                  (unsigned)Lay::real_bytes * (R.has_pot ? 1u : 0u);
        mbar_expect_tx(&bars[slot], tx_bytes);
        // psi: x in T units (2 per point) of the padded plane, ring kRing
        tma_load_2d(base + Lay::psi_off, R.psi_map, 2 * (R.tx0 - 4 + kRing), R.ty0 - 4 + kRing, &bars[slot]);
        if (RES) tma_load_2d(base + Lay::n_off, R.n_map, R.tx0 - 4 + kRing, R.ty0 - 3 + kRing, &bars[slot]);
        if (RES && R.has_pump) tma_load_2d(base + Lay::pump_off, R.pump_map, R.tx0 - 4 + kRing, R.ty0 - 3 + kRing, &bars[slot]);
        if (R.has_pot) tma_load_2d(base + Lay::pot_off, R.pot_map, R.tx0 - 4 + kRing, R.ty0 - 3 + kRing, &bars[slot]);
    };

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    // the previous iteration's state (and the plane this one writes, which the
    // previous one read) are settled only once its kernel has completed
    pdl_wait();
    __syncthreads();
    int tile = blockIdx.x;
    if (threadIdx.x == 0 && tile < n_tiles) issue(0, tile);
    int it = 0;
    bool pending_next = false;  // thread 0: a load into the other slot is in flight
    for (; tile < n_tiles; tile += gridDim.x, ++it) {
        const int slot = it & 1;
        const unsigned parity = (unsigned)((it >> 1) & 1);
        const int next = tile + gridDim.x;
        const TileRef<T> R = tile_of(tile);
        if constexpr (BATCH) {
            // the previous tile's reads of sP ended at its closing barrier
            constexpr int kWords = (int)(sizeof(FusedParams<T>) / sizeof(int));
            static_assert(sizeof(FusedParams<T>) % sizeof(int) == 0, "FusedParams copied as words");
            const int* src = reinterpret_cast<const int*>(R.f);
            int* dst = reinterpret_cast<int*>(&sP);
            for (int w = threadIdx.x; w < kWords; w += NT) dst[w] = __ldg(src + w);
        }
        // thread 0 waits for the tile's boxes; the others wait at the barrier
        // (no issue slots spent spinning), which also orders the data thread 0
        // observed before their reads
        const bool ok = threadIdx.x == 0 ? mbar_wait_bounded(&bars[slot], parity, wait_polls) : true;
        // the next tile's boxes go into the other slot once this tile's are in
        // (its reads of that slot ended at the previous tile's closing
        // barrier): at the start of a launch, when every CTA's first loads
        // come from DRAM at once, the first tiles do not share the bandwidth
        // with the second ones; later the current boxes have long arrived
        if (threadIdx.x == 0) {
            pending_next = ok && next < n_tiles;
            if (pending_next) issue(slot ^ 1, next);
        }
        // this CTA's last tile: the next iteration's kernel may be scheduled
        // (every CTA of this persistent grid is resident already, so its CTAs
        // only take the slots these leave; they wait in pdl_wait() for this
        // grid to complete)
        if (next >= n_tiles) pdl_trigger();
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicExch(err, 1);
                // drain this CTA's loads still in flight before leaving
                (void)mbar_wait_bounded(&bars[slot], parity);
                if (pending_next) (void)mbar_wait_bounded(&bars[slot ^ 1], (unsigned)(((it + 1) >> 1) & 1));
            }
            return;
        }
        const FusedParams<T>& P = BATCH ? sP : *R.f;
        const bool has_pump = R.has_pump != 0, has_pot = R.has_pot != 0;
        const long long pitch = P.pitch;
        unsigned char* base = smem + slot * Lay::slot_bytes;
        cx<T>* sA = reinterpret_cast<cx<T>*>(base + Lay::psi_off);
        const T* s_n = reinterpret_cast<const T*>(base + Lay::n_off);
        const T* s_pu = reinterpret_cast<const T*>(base + Lay::pump_off);
        const T* s_po = reinterpret_cast<const T*>(base + Lay::pot_off);
        const int ty0 = R.ty0, tx0 = R.tx0;

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
        // stage 0 reads the TMA box sA (row W4, unpadded); stages 1-3 ping-pong
        // between the padded buffers: 0: sA -> sB, 1: sB -> sC, 2: sC -> sB, 3: sB -> global
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const cx<T>* in = s == 0 ? sA : (s == 2 ? sC : sB);
            cx<T>* out = s == 1 ? sC : sB;
#pragma unroll
            for (int j = 0; j < OWN; ++j) {
                const int p = threadIdx.x + NT * j;
                const int qy = p / PW, qx = 2 * (p - qy * PW);
                if (p >= NP || qy < s || qy >= H3 - s || qx + 1 < s || qx >= W3 - s) continue;
                const int ep = (qy + 1) * SW + qx + 2;  // padded index of the pair (even)
                const int er = qy * WR + qx + 1;
                cx<T> c0, c1, u0, u1, d0, d1, lft, rgt;
                if (s == 0) {
                    const int e = (qy + 1) * W4 + qx + 1;
                    c0 = y0[j][0];
                    c1 = y0[j][1];
                    u0 = in[e - W4], u1 = in[e - W4 + 1];
                    d0 = in[e + W4], d1 = in[e + W4 + 1];
                    lft = in[e - 1], rgt = in[e + 2];
                } else {
                    lds_pair(in + ep, c0, c1);
                    lds_pair(in + ep - SW, u0, u1);
                    lds_pair(in + ep + SW, d0, d1);
                    lft = in[ep - 1], rgt = in[ep + 2];
                }
                const T pu0 = (RES && has_pump) ? s_pu[er] : (T)0, pu1 = (RES && has_pump) ? s_pu[er + 1] : (T)0;
                const T po0 = has_pot ? s_po[er] : (T)0, po1 = has_pot ? s_po[er + 1] : (T)0;
                cx<T> kw[2];
                T kr[2] = {(T)0, (T)0};
                rhs_iter<T, RES, FMA>(P, s, c0, u0, d0, lft, c1, ns[j][0], pu0, po0, has_pump, has_pot, kw[0], kr[0]);
                rhs_iter<T, RES, FMA>(P, s, c1, u1, d1, c0, rgt, ns[j][1], pu1, po1, has_pump, has_pot, kw[1], kr[1]);
                cx<T> o[2];
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
                        o[h] = axpy<FMA>(P.dtw[s], kw[h], y0[j][h]);
                        if constexpr (RES) ns[j][h] = raxpy<FMA>(P.dtw[s], kr[h], n0[j][h]);
                        if constexpr (STORE) {
                            const int gy = ty0 - 3 + qy, gx = tx0 - 3 + qx + h;
                            if (qy >= 3 && qy < H3 - 3 && qx + h >= 3 && qx + h < W3 - 3 && gy < P.N_r && gx < P.N_c) {
                                const long long g = (long long)gy * pitch + gx;
                                P.st_psi[s][g] = o[h];
                                if (P.img_x | P.img_y) fused_images(P, P.st_psi[s], gy, gx, o[h]);
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
                if (s < 3) sts_pair(out + ep, o[0], o[1]);
            }
            __syncthreads();
        }
        // this slot is refilled by the async proxy two tiles later: order this
        // tile's shared-memory accesses before that
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
    }
}

// MINB: CTAs per SM the register allocation must leave room for.  STORE: also
// write the stage values Y2..Y4 of the tile's points (f.st_psi / f.st_n, with
// periodic images), which the adjoint's backward sweep reads.
template <typename T, bool RES, int TW, int TH, int NT, int MINB = 1, bool STORE = false, bool FMA = false>
__global__ void __launch_bounds__(NT, MINB) rk4_tma_kernel(const __grid_constant__ TmaParams<T> Q) {
    auto tile_of = [&](int g) {
        TileRef<T> R;
        R.psi_map = &Q.psi_map;
        R.n_map = &Q.n_map;
        R.pump_map = &Q.pump_map;
        R.pot_map = &Q.pot_map;
        R.f = &Q.f;
        R.has_pump = Q.has_pump;
        R.has_pot = Q.has_pot;
        R.ty0 = (g / Q.tiles_x) * TH;
        R.tx0 = (g % Q.tiles_x) * TW;
        return R;
    };
    tma_tile_loop<T, RES, TW, TH, NT, false, STORE, FMA>(tile_of, Q.n_tiles, Q.err, Q.wait_polls);
}

// ---------------------------------------------------------------- batches
// Every instance of a batch owns two state planes (A, B); iteration k reads
// A and writes B when k is even, the other way round when odd.  Its tensor
// maps and parameters for both directions live in device memory.
template <typename T>
struct alignas(64) BatchInstance {
    CUtensorMap maps[2][4];  // [direction][psi, n, pump, potential]
    FusedParams<T> f[2];     // [direction]
    int has_pump, has_pot;
    int tiles_x, tile_begin;
};

template <typename T>
struct BatchParams {
    const BatchInstance<T>* inst;
    const int* tile_inst;  // global tile -> instance
    int n_tiles;
    int dir;
    int* err;
};

template <typename T, bool RES, int TW, int TH, int NT, int MINB = 1, bool FMA = false>
__global__ void __launch_bounds__(NT, MINB) rk4_batch_kernel(const __grid_constant__ BatchParams<T> B) {
    // the loop's g = b + k * gridDim.x (CTA b's k-th tile) is remapped to
    // tile b * q + min(b, r) + k (q, r: n_tiles / gridDim.x and remainder),
    // a bijection on [0, n_tiles) under which every CTA walks a contiguous
    // run of tiles, mostly of one instance, so that thread 0 seldom fences
    // a new instance's tensor maps
    const int q = B.n_tiles / (int)gridDim.x, r = B.n_tiles % (int)gridDim.x;
    auto tile_of = [&](int g) {
        const int cta = g % (int)gridDim.x, k = g / (int)gridDim.x;
        g = cta * q + min(cta, r) + k;
        const BatchInstance<T>& I = B.inst[__ldg(B.tile_inst + g)];
        TileRef<T> R;
        R.psi_map = &I.maps[B.dir][0];
        R.n_map = &I.maps[B.dir][1];
        R.pump_map = &I.maps[B.dir][2];
        R.pot_map = &I.maps[B.dir][3];
        R.f = &I.f[B.dir];
        R.has_pump = I.has_pump;
        R.has_pot = I.has_pot;
        const int local = g - I.tile_begin;
        R.ty0 = (local / I.tiles_x) * TH;
        R.tx0 = (local % I.tiles_x) * TW;
        return R;
    };
    tma_tile_loop<T, RES, TW, TH, NT, true, false, FMA>(tile_of, B.n_tiles, B.err, kWaitPolls);
}

}  // namespace phx
