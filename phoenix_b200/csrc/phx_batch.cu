// phx_batch.cu -- many independent RK4 simulations advanced together.
//
// The reference runs one simulation per process (source/main.cu:80-117); a
// pump-power sweep or a set of disorder realisations is n sequential runs of
// that main loop.  Here every instance keeps its own halo-padded planes
// (layout of phx_device.cuh), parameters and clock, and one batch iteration
// advances every instance by one RK4 iteration (the fused iteration of
// phx_step_fused.cuh, bit-identical to a single-simulation handle) in a
// single launch of the persistent TMA kernel rk4_batch_kernel, which walks
// the tiles of all instances through a tile -> instance table.  Launch
// sequences are captured once into CUDA graphs and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/phx.h"
#include "phx_host.hpp"
#include "phx_misc.cuh"
#include "phx_rt.hpp"
#include "phx_step_fused.cuh"
#include "phx_step_tma.cuh"

namespace phx {

// Tile shapes the batch autotuner chooses from: TW x TH points, NT threads.
// FP64 tiles are half as high (shared memory of the two TMA slots).
// MINB: CTAs per SM the register allocation leaves room for (the 12-warp
// shapes run two per SM).
constexpr int kBatchShapes = 5;
template <typename T>
struct BatchShape;
template <>
struct BatchShape<float> {
    static constexpr int TW[kBatchShapes] = {32, 64, 32, 32, 64};
    static constexpr int TH[kBatchShapes] = {32, 16, 16, 32, 16};
    static constexpr int NT[kBatchShapes] = {256, 256, 128, 384, 384};
    static constexpr int MINB[kBatchShapes] = {1, 1, 1, 2, 2};
};
template <>
struct BatchShape<double> {
    static constexpr int TW[kBatchShapes] = {32, 64, 32, 32, 64};
    static constexpr int TH[kBatchShapes] = {16, 8, 8, 16, 8};
    static constexpr int NT[kBatchShapes] = {256, 256, 128, 384, 384};
    static constexpr int MINB[kBatchShapes] = {1, 1, 1, 2, 2};
};

struct BatchBase {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    virtual ~BatchBase() = default;
    virtual void set_field(int inst, int field, int group, const void* host, int64_t count, int dtype) = 0;
    virtual void get_field(int inst, int field, int group, void* host, int64_t count, int dtype) = 0;
    virtual void step(int64_t iterations, phx_step_info* info) = 0;
    virtual void get_time(int inst, double* t, double* dt) = 0;
};

template <typename T>
struct BatchEngine final : BatchBase {
    static constexpr int G = kRing;
    using C = cx<T>;
    using SH = BatchShape<T>;

    struct Instance {
        phx_params P{};
        Derived<T> d{};
        long long pitch = 0, rows = 0, plane = 0;
        DevBuf psi[2], n[2];  // state ping-pong: cur holds the state
        DevBuf pump, pot;     // one group each, or empty
        T t = 0, dt = 0;
        C* cplane(DevBuf& b) { return reinterpret_cast<C*>(b.p) + G * pitch + G; }
        T* rplane(DevBuf& b) { return reinterpret_cast<T*>(b.p) + G * pitch + G; }
    };
    std::vector<std::unique_ptr<Instance>> inst;
    bool res = true;
    bool fma = false;  // fused multiply-add arithmetic (phx_params.fma)
    int cur = 0;  // which ping-pong plane holds every instance's state

    // per tile shape: instance table and tile -> instance map on the device
    DevBuf d_inst[kBatchShapes], d_tile[kBatchShapes];
    int n_tiles[kBatchShapes] = {};
    int blocks[kBatchShapes] = {};
    DevBuf err_flag;
    int sm_count = 0;

    // autotuning: the first kBatchTuneRounds * kBatchShapes iterations cycle
    // through the shapes (results do not depend on the shape).  The first
    // round warms up; each later one gives a sample per shape, and the median
    // sample ranks them.  The incumbent (32 x 32 tiles, 384 threads) is kept
    // unless the fastest median beats it by more than kBatchTuneMargin, so
    // that boxes whose timings differ by noise pick the same shape.
    static constexpr int kBatchTuneRounds = 4;
    static constexpr int kBatchIncumbent = 3;
    static constexpr double kBatchTuneMargin = 0.03;
    int shape = -1, tune_step = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> tune_ev[kBatchShapes];
    std::vector<cudaEvent_t> events;

    // graphs of kGraphIters iterations starting from state plane 0 / 1
    static constexpr int kGraphIters = 16;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int64_t launches = 0;

    ~BatchEngine() override {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto& v : tune_ev)
            for (auto& pr : v) {
                cudaEventDestroy(pr.first);
                cudaEventDestroy(pr.second);
            }
        for (auto e : events) cudaEventDestroy(e);
        inst.clear();
        if (stream) cudaStreamDestroy(stream);
    }

    void init(const phx_params* ps, int n) {
        device = ps[0].device;
        res = ps[0].use_reservoir != 0;
        fma = ps[0].fma != 0;
        PHX_CUDA(cudaSetDevice(device));
        PHX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        PHX_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device));
        for (int i = 0; i < n; ++i) {
            auto I = std::make_unique<Instance>();
            I->P = ps[i];
            I->d = derive<T>(ps[i]);
            I->pitch = ((ps[i].N_c + 2LL * G) + 31) / 32 * 32;
            I->rows = ps[i].N_r + 2LL * G;
            I->plane = I->pitch * I->rows;
            for (int b = 0; b < 2; ++b) {
                I->psi[b].alloc(sizeof(C) * I->plane, stream);
                if (res) I->n[b].alloc(sizeof(T) * I->plane, stream);
            }
            if (ps[i].n_pump_groups) I->pump.alloc(sizeof(T) * I->plane, stream);
            if (ps[i].n_potential_groups) I->pot.alloc(sizeof(T) * I->plane, stream);
            I->t = (T)ps[i].t0;
            I->dt = (T)ps[i].dt;
            inst.push_back(std::move(I));
        }
        err_flag.alloc(sizeof(int), stream);
        if (const char* e = std::getenv("PHX_BATCH_SHAPE")) {
            const int v = std::atoi(e);
            if (v >= 0 && v < kBatchShapes) shape = v;
        }
        build_tables();
        PHX_CUDA(cudaStreamSynchronize(stream));
    }

    // ------------------------------------------------------------ tables
    template <int S>
    void table(std::vector<BatchInstance<T>>& hi, std::vector<int>& tiles) {
        constexpr int TW = SH::TW[S], TH = SH::TH[S];
        static_assert(TW % 4 == 0, "TMA box x alignment needs tile origins on 16-byte boundaries");
        hi.assign(inst.size(), BatchInstance<T>{});
        tiles.clear();
        for (size_t i = 0; i < inst.size(); ++i) {
            Instance& I = *inst[i];
            BatchInstance<T>& B = hi[i];
            std::memset(&B, 0, sizeof(B));
            const int tx = (I.P.N_c + TW - 1) / TW, ty = (I.P.N_r + TH - 1) / TH;
            B.tiles_x = tx;
            B.tile_begin = (int)tiles.size();
            B.has_pump = I.P.n_pump_groups > 0;
            B.has_pot = I.P.n_potential_groups > 0;
            tiles.insert(tiles.end(), (size_t)tx * ty, (int)i);
            // a map that is never loaded still needs a valid encoding: the
            // real view of the first state plane stands in for it
            void* dummy = I.psi[0].p;
            for (int dir = 0; dir < 2; ++dir) {
                DevBuf& src_psi = I.psi[dir];
                DevBuf& src_n = I.n[dir];
                plane_tensor_map<T>(&B.maps[dir][0], src_psi.p, true, I.pitch, I.rows, TW + 8, TH + 8);
                plane_tensor_map<T>(&B.maps[dir][1], res ? src_n.p : dummy, false, I.pitch, I.rows, TW + 8, TH + 6);
                plane_tensor_map<T>(&B.maps[dir][2], B.has_pump ? I.pump.p : dummy, false, I.pitch, I.rows, TW + 8, TH + 6);
                plane_tensor_map<T>(&B.maps[dir][3], B.has_pot ? I.pot.p : dummy, false, I.pitch, I.rows, TW + 8, TH + 6);
                FusedParams<T>& F = B.f[dir];
                std::memset(&F, 0, sizeof(F));
                fused_constants<T>(F, I.P, I.d, I.dt, I.pitch);
                // constant temporal envelopes: amplitude 1 at every stage
                const T cw[4] = {(T)0.0, (T)0.5, (T)0.5, (T)1.0};
                const std::complex<T> one((T)1, (T)0);
                for (int s = 0; s < 4; ++s) {
                    F.pump_c[s] = interp<T>(one, one, cw[s]).real();
                    F.pot_c[s] = interp<T>(one, one, cw[s]).real();
                }
                F.psi0 = I.cplane(I.psi[dir]);
                F.psi1 = I.cplane(I.psi[dir ^ 1]);
                F.n0 = res ? I.rplane(I.n[dir]) : nullptr;
                F.n1 = res ? I.rplane(I.n[dir ^ 1]) : nullptr;
                F.pump = B.has_pump ? I.rplane(I.pump) : nullptr;
                F.pot = B.has_pot ? I.rplane(I.pot) : nullptr;
            }
        }
    }
    // the kernel of shape S for this batch (reservoir or not, bit-exact or
    // fused multiply-add arithmetic)
    template <int S>
    auto kernel_of() const {
        using K = void (*)(BatchParams<T>);
        K k = res ? (K)rk4_batch_kernel<T, true, SH::TW[S], SH::TH[S], SH::NT[S], SH::MINB[S]>
                  : (K)rk4_batch_kernel<T, false, SH::TW[S], SH::TH[S], SH::NT[S], SH::MINB[S]>;
        if constexpr (sizeof(T) == 4) {
            if (fma)
                k = res ? (K)rk4_batch_kernel<T, true, SH::TW[S], SH::TH[S], SH::NT[S], SH::MINB[S], true>
                        : (K)rk4_batch_kernel<T, false, SH::TW[S], SH::TH[S], SH::NT[S], SH::MINB[S], true>;
        }
        return k;
    }
    template <int S>
    void build_one() {
        std::vector<BatchInstance<T>> hi;
        std::vector<int> tiles;
        table<S>(hi, tiles);
        if (tiles.size() > (size_t)std::numeric_limits<int>::max() / 2) fail(PHX_ERR_INVALID_ARG, "batch has too many tiles");
        n_tiles[S] = (int)tiles.size();
        d_inst[S].alloc(sizeof(BatchInstance<T>) * hi.size(), stream);
        d_tile[S].alloc(sizeof(int) * tiles.size(), stream);
        PHX_CUDA(cudaMemcpyAsync(d_inst[S].p, hi.data(), sizeof(BatchInstance<T>) * hi.size(), cudaMemcpyHostToDevice, stream));
        PHX_CUDA(cudaMemcpyAsync(d_tile[S].p, tiles.data(), sizeof(int) * tiles.size(), cudaMemcpyHostToDevice, stream));
        PHX_CUDA(cudaStreamSynchronize(stream));  // host vectors die here
        auto kern = kernel_of<S>();
        const int smem = TmaLayout<T, SH::TW[S], SH::TH[S]>::total;
        PHX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int per_sm = 0;
        PHX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SH::NT[S], smem));
        if (per_sm < 1) fail(PHX_ERR_UNSUPPORTED, "batch iteration kernel does not fit on an SM");
        blocks[S] = std::max(1, std::min(n_tiles[S], per_sm * sm_count));
    }
    void build_tables() {
        build_one<0>();
        build_one<1>();
        build_one<2>();
        build_one<3>();
        build_one<4>();
        static_assert(kBatchShapes == 5, "every shape needs its tables");
    }

    // ------------------------------------------------------------ launches
    template <int S>
    void go(int dir) {
        BatchParams<T> B;
        B.inst = static_cast<const BatchInstance<T>*>(d_inst[S].p);
        B.tile_inst = static_cast<const int*>(d_tile[S].p);
        B.n_tiles = n_tiles[S];
        B.dir = dir;
        B.err = static_cast<int*>(err_flag.p);
        const int smem = TmaLayout<T, SH::TW[S], SH::TH[S]>::total;
        kernel_of<S>()<<<blocks[S], SH::NT[S], smem, stream>>>(B);
    }
    void launch(int sh, int dir) {
        switch (sh) {
            case 0: go<0>(dir); break;
            case 1: go<1>(dir); break;
            case 2: go<2>(dir); break;
            case 3: go<3>(dir); break;
            default: go<4>(dir); break;
        }
        PHX_CUDA(cudaGetLastError());
        ++launches;
    }
    // every instance's clock advances as in the single-simulation loop:
    // t = t + dt in the build precision, once per iteration
    void advance_clocks(int64_t k) {
        for (auto& I : inst)
            for (int64_t i = 0; i < k; ++i) I->t = I->t + I->dt;
    }
    cudaEvent_t event() {
        if (!events.empty()) {
            cudaEvent_t e = events.back();
            events.pop_back();
            return e;
        }
        cudaEvent_t e;
        PHX_CUDA(cudaEventCreate(&e));
        return e;
    }
    void tune_iteration() {
        const int sh = tune_step % kBatchShapes;
        cudaEvent_t a = event(), b = event();
        PHX_CUDA(cudaEventRecord(a, stream));
        launch(sh, cur);
        PHX_CUDA(cudaEventRecord(b, stream));
        tune_ev[sh].push_back({a, b});
        cur ^= 1;
        advance_clocks(1);
        if (++tune_step < kBatchTuneRounds * kBatchShapes) return;
        PHX_CUDA(cudaStreamSynchronize(stream));
        double best = 1e30, med[kBatchShapes];
        int best_sh = kBatchIncumbent;
        for (int s = 0; s < kBatchShapes; ++s) {
            std::vector<double> v;
            for (size_t i = 1; i < tune_ev[s].size(); ++i) {
                float m = 0.f;
                PHX_CUDA(cudaEventElapsedTime(&m, tune_ev[s][i].first, tune_ev[s][i].second));
                v.push_back(m);
            }
            std::sort(v.begin(), v.end());
            med[s] = v[v.size() / 2];
            if (med[s] < best) best = med[s], best_sh = s;
            for (auto& pr : tune_ev[s]) {
                events.push_back(pr.first);
                events.push_back(pr.second);
            }
            tune_ev[s].clear();
        }
        if (med[kBatchIncumbent] <= best * (1.0 + kBatchTuneMargin)) best_sh = kBatchIncumbent;
        shape = best_sh;
    }
    void capture(int start) {
        cudaGraph_t g = nullptr;
        PHX_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const int64_t l0 = launches;
        try {
            for (int i = 0; i < kGraphIters; ++i) launch(shape, (start + i) & 1);
        } catch (...) {
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        launches = l0;
        PHX_CUDA(cudaStreamEndCapture(stream, &g));
        const cudaError_t e = cudaGraphInstantiate(&graph[start], g, 0);
        cudaGraphDestroy(g);
        PHX_CUDA(e);
    }

    void step(int64_t iterations, phx_step_info* info) override {
        PHX_CUDA(cudaSetDevice(device));
        const int64_t l0 = launches;
        int64_t done = 0;
        while (done < iterations && shape < 0) {
            tune_iteration();
            ++done;
        }
        while (iterations - done >= kGraphIters) {
            if (!graph[cur]) capture(cur);
            PHX_CUDA(cudaGraphLaunch(graph[cur], stream));
            launches += kGraphIters;
            advance_clocks(kGraphIters);  // kGraphIters is even: cur is unchanged
            done += kGraphIters;
        }
        for (; done < iterations; ++done) {
            launch(shape, cur);
            cur ^= 1;
            advance_clocks(1);
        }
        if (info) {
            info->t = (double)inst[0]->t;
            info->dt = (double)inst[0]->dt;
            info->iterations = iterations;
            info->accepted = iterations;
            info->rejected = 0;
            info->fft_filters = 0;
            info->kernel_launches = launches - l0;
            info->launch_shape = shape;
            info->reserved = 0;
        }
    }

    // ------------------------------------------------------------ fields
    Instance& at(int i) {
        if (i < 0 || i >= (int)inst.size()) fail(PHX_ERR_INVALID_ARG, "instance out of range");
        return *inst[i];
    }
    // (plane, complex) of a field of instance I; the state planes are the
    // ones that currently hold the state
    std::pair<DevBuf*, bool> field_buf(Instance& I, int field, int group) {
        switch (field) {
            case PHX_PSI_PLUS: return {&I.psi[cur], true};
            case PHX_N_PLUS:
                if (!res) fail(PHX_ERR_INVALID_ARG, "reservoir field requires use_reservoir");
                return {&I.n[cur], false};
            case PHX_PUMP_PLUS:
                if (group != 0 || !I.P.n_pump_groups) fail(PHX_ERR_INVALID_ARG, "pump group out of range");
                return {&I.pump, false};
            case PHX_POTENTIAL_PLUS:
                if (group != 0 || !I.P.n_potential_groups) fail(PHX_ERR_INVALID_ARG, "potential group out of range");
                return {&I.pot, false};
            default:
                fail(PHX_ERR_UNSUPPORTED, "batch instances hold psi_plus, n_plus, pump_plus and potential_plus only");
        }
    }
    void set_field(int i, int field, int group, const void* host, int64_t count, int dtype) override {
        if (!host) fail(PHX_ERR_INVALID_ARG, "host pointer is NULL");
        if (dtype != PHX_F32 && dtype != PHX_F64) fail(PHX_ERR_INVALID_ARG, "bad host dtype");
        PHX_CUDA(cudaSetDevice(device));
        Instance& I = at(i);
        auto [buf, complex] = field_buf(I, field, group);
        const long long N = (long long)I.P.N_r * I.P.N_c;
        const long long want = complex ? 2 * N : N;
        if (count != want) fail(PHX_ERR_INVALID_ARG, "expected " + std::to_string(want) + " values, got " + std::to_string(count));
        std::vector<T> tmp;
        const void* src = host;
        if ((dtype == PHX_F64) != (sizeof(T) == 8)) {
            tmp.resize((size_t)want);
            if (dtype == PHX_F64)
                for (long long k = 0; k < want; ++k) tmp[k] = (T) static_cast<const double*>(host)[k];
            else
                for (long long k = 0; k < want; ++k) tmp[k] = (T) static_cast<const float*>(host)[k];
            src = tmp.data();
        }
        const size_t esz = complex ? sizeof(C) : sizeof(T);
        char* dst = reinterpret_cast<char*>(buf->p) + esz * (G * I.pitch + G);
        PHX_CUDA(cudaStreamSynchronize(stream));  // earlier iterations may still read this plane
        PHX_CUDA(cudaMemcpy2DAsync(dst, esz * I.pitch, src, esz * I.P.N_c, esz * I.P.N_c, I.P.N_r, cudaMemcpyHostToDevice,
                                   stream));
        if (complex)
            ring_fill_kernel<C><<<64, 256, 0, stream>>>(reinterpret_cast<C*>(dst), I.P.N_r, I.P.N_c, I.pitch, G,
                                                        I.P.periodic_x, I.P.periodic_y);
        else
            ring_fill_kernel<T><<<64, 256, 0, stream>>>(reinterpret_cast<T*>(dst), I.P.N_r, I.P.N_c, I.pitch, G,
                                                        I.P.periodic_x, I.P.periodic_y);
        PHX_CUDA(cudaGetLastError());
        PHX_CUDA(cudaStreamSynchronize(stream));
    }
    void check_err_flag() {
        int v = 0;
        PHX_CUDA(cudaMemcpy(&v, err_flag.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (v) {
            PHX_CUDA(cudaMemset(err_flag.p, 0, sizeof(int)));
            fail(PHX_ERR_TIMEOUT, "a bounded wait for TMA data gave up; the batch iteration's results are invalid");
        }
    }
    void get_field(int i, int field, int group, void* host, int64_t count, int dtype) override {
        if (!host) fail(PHX_ERR_INVALID_ARG, "host pointer is NULL");
        if (dtype != PHX_F32 && dtype != PHX_F64) fail(PHX_ERR_INVALID_ARG, "bad host dtype");
        PHX_CUDA(cudaSetDevice(device));
        PHX_CUDA(cudaStreamSynchronize(stream));
        check_err_flag();
        Instance& I = at(i);
        auto [buf, complex] = field_buf(I, field, group);
        const long long N = (long long)I.P.N_r * I.P.N_c;
        const long long want = complex ? 2 * N : N;
        if (count != want) fail(PHX_ERR_INVALID_ARG, "expected " + std::to_string(want) + " values");
        const size_t esz = complex ? sizeof(C) : sizeof(T);
        const char* src = reinterpret_cast<const char*>(buf->p) + esz * (G * I.pitch + G);
        const bool same = (dtype == PHX_F64) == (sizeof(T) == 8);
        std::vector<T> tmp(same ? 0 : (size_t)want);
        void* dst = same ? host : tmp.data();
        PHX_CUDA(cudaMemcpy2DAsync(dst, esz * I.P.N_c, src, esz * I.pitch, esz * I.P.N_c, I.P.N_r, cudaMemcpyDeviceToHost,
                                   stream));
        PHX_CUDA(cudaStreamSynchronize(stream));
        if (same) return;
        if (dtype == PHX_F64)
            for (long long k = 0; k < want; ++k) static_cast<double*>(host)[k] = (double)tmp[k];
        else
            for (long long k = 0; k < want; ++k) static_cast<float*>(host)[k] = (float)tmp[k];
    }
    void get_time(int i, double* t, double* dt) override {
        Instance& I = at(i);
        if (t) *t = (double)I.t;
        if (dt) *dt = (double)I.dt;
    }
};

}  // namespace phx

// ====================================================================== C ABI
struct phx_batch {
    std::unique_ptr<phx::BatchBase> eng;
};

namespace {

phx_status bguard(phx_batch* b, const std::function<void()>& f) {
    std::string& err = b ? b->eng->err : phx::g_create_error;
    try {
        f();
        if (b) err.clear();
        return PHX_OK;
    } catch (const phx::Error& e) {
        err = e.msg;
        return e.status;
    } catch (const std::bad_alloc&) {
        err = "host allocation failed";
        return PHX_ERR_OOM;
    } catch (const std::exception& e) {
        err = e.what();
        return PHX_ERR_INVALID_ARG;
    }
}

void validate_batch(const phx_params* ps, int n) {
    using phx::fail;
    if (n < 1) fail(PHX_ERR_INVALID_ARG, "a batch needs at least one instance");
    for (int i = 0; i < n; ++i) {
        const phx_params& p = ps[i];
        const std::string at = "instance " + std::to_string(i) + ": ";
        if (p.abi_version != PHX_ABI_VERSION) fail(PHX_ERR_INVALID_ARG, at + "abi_version mismatch");
        if (p.N_c < 8 || p.N_r < 8) fail(PHX_ERR_INVALID_ARG, at + "grid must be at least 8 x 8");
        if ((long long)p.N_c * p.N_r > (1LL << 28)) fail(PHX_ERR_INVALID_ARG, at + "grid too large for a batch instance");
        if (p.dtype != ps[0].dtype) fail(PHX_ERR_INVALID_ARG, at + "all instances share one dtype");
        if (p.fma != ps[0].fma) fail(PHX_ERR_INVALID_ARG, at + "all instances share one arithmetic (fma)");
        if (p.fma && p.dtype != PHX_F32) fail(PHX_ERR_UNSUPPORTED, at + "the fused multiply-add arithmetic is FP32 only");
        if (p.dtype != PHX_F32 && p.dtype != PHX_F64) fail(PHX_ERR_INVALID_ARG, at + "dtype must be PHX_F32 or PHX_F64");
        if (p.dtype == PHX_F32 && (p.N_c & 1)) fail(PHX_ERR_UNSUPPORTED, at + "FP32 grids need an even N_c");
        if (p.use_reservoir != ps[0].use_reservoir) fail(PHX_ERR_INVALID_ARG, at + "all instances share use_reservoir");
        if (p.device != ps[0].device) fail(PHX_ERR_INVALID_ARG, at + "all instances share one device");
        if (p.iterator != PHX_ITER_RK4 || p.adaptive) fail(PHX_ERR_UNSUPPORTED, at + "batches run fixed-step RK4");
        if (p.tetm) fail(PHX_ERR_UNSUPPORTED, at + "batches run the scalar model");
        if (p.imag_time_amplitude != 0.0) fail(PHX_ERR_UNSUPPORTED, at + "batches run real time");
        if (p.n_pump_groups > 1 || p.n_potential_groups > 1 || p.n_pulse_groups != 0)
            fail(PHX_ERR_UNSUPPORTED, at + "batch instances take at most one pump and one potential group and no pulse");
        if (p.n_pump_groups < 0 || p.n_potential_groups < 0) fail(PHX_ERR_INVALID_ARG, at + "negative group count");
        if (p.n_pump_groups > 0 && !p.use_reservoir) fail(PHX_ERR_INVALID_ARG, at + "pump groups need use_reservoir");
        if (p.stochastic_amplitude != 0.0) fail(PHX_ERR_UNSUPPORTED, at + "stochastic noise is not available in batches");
        if (!(p.L_x > 0) || !(p.L_y > 0) || !(p.h_bar_s > 0) || !(p.m_eff > 0))
            fail(PHX_ERR_INVALID_ARG, at + "L, h_bar_s and m_eff must be > 0");
        if (!(p.dt > 0)) fail(PHX_ERR_INVALID_ARG, at + "dt must be > 0");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        fail(PHX_ERR_CUDA, "no CUDA device available");
    }
    if (ps[0].device < 0 || ps[0].device >= ndev) fail(PHX_ERR_INVALID_ARG, "device ordinal out of range");
}

}  // namespace

extern "C" {

phx_status phx_batch_create(const phx_params* instances, int32_t n_instances, phx_batch** out) {
    if (!instances || !out) {
        phx::g_create_error = "NULL argument";
        return PHX_ERR_INVALID_ARG;
    }
    *out = nullptr;
    std::unique_ptr<phx_batch> b(new (std::nothrow) phx_batch());
    if (!b) return PHX_ERR_OOM;
    phx_status st = bguard(nullptr, [&] {
        validate_batch(instances, n_instances);
        if (instances[0].dtype == PHX_F64) {
            auto* e = new phx::BatchEngine<double>();
            b->eng.reset(e);
            e->init(instances, n_instances);
        } else {
            auto* e = new phx::BatchEngine<float>();
            b->eng.reset(e);
            e->init(instances, n_instances);
        }
    });
    if (st != PHX_OK) return st;
    *out = b.release();
    return PHX_OK;
}

phx_status phx_batch_destroy(phx_batch* b) {
    if (!b) return PHX_OK;
    if (b->eng) cudaSetDevice(b->eng->device);
    delete b;
    return PHX_OK;
}

phx_status phx_batch_set_field(phx_batch* b, int32_t instance, int32_t field, int32_t group, const void* host,
                               int64_t count, int32_t host_dtype) {
    if (!b) return PHX_ERR_INVALID_ARG;
    return bguard(b, [&] { b->eng->set_field(instance, field, group, host, count, host_dtype); });
}

phx_status phx_batch_get_field(phx_batch* b, int32_t instance, int32_t field, int32_t group, void* host, int64_t count,
                               int32_t host_dtype) {
    if (!b) return PHX_ERR_INVALID_ARG;
    return bguard(b, [&] { b->eng->get_field(instance, field, group, host, count, host_dtype); });
}

phx_status phx_batch_step(phx_batch* b, int64_t iterations, phx_step_info* info) {
    if (!b) return PHX_ERR_INVALID_ARG;
    return bguard(b, [&] {
        if (iterations < 0) phx::fail(PHX_ERR_INVALID_ARG, "iterations < 0");
        b->eng->step(iterations, info);
    });
}

phx_status phx_batch_get_time(phx_batch* b, int32_t instance, double* t, double* dt) {
    if (!b) return PHX_ERR_INVALID_ARG;
    return bguard(b, [&] { b->eng->get_time(instance, t, dt); });
}

phx_status phx_batch_get_stream(phx_batch* b, void** stream) {
    if (!b || !stream) return PHX_ERR_INVALID_ARG;
    *stream = (void*)b->eng->stream;
    return PHX_OK;
}

const char* phx_batch_last_error(const phx_batch* b) {
    if (!b) return phx::g_create_error.c_str();
    return b->eng ? b->eng->err.c_str() : "";
}

}  // extern "C"
