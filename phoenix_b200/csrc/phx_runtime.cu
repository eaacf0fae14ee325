// phx_runtime.cu -- the handle behind include/phx.h.
//
// Owns the device state of one simulation (halo-padded planes, see
// phx_device.cuh), runs the iteration loop of Solver::iterate
// (source/cuda_solver/solver/solver.cu:22-70) with t, dt and every host-side
// scalar kept in the build precision, launches one fused kernel per RK stage
// (phx_stage.cuh), performs DP45 step-size control with FP64 reductions
// (Solver::adaptTimeStep, solver.cu:72-105) and applies the k-space mask
// filter through cuFFT (Solver::applyFFTFilter, solver_fft.cu:67-119).
#include <cufft.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <limits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <type_traits>
#include <array>
#include <map>
#include <mutex>
#include <atomic>
#include <tuple>
#include <utility>
#include <vector>

#include "../../include/phx.h"
#include "phx_host.hpp"
#include "phx_misc.cuh"
#include "phx_stage.cuh"
#include "phx_stage_tetm.cuh"
#include "phx_step_fused.cuh"
#include "phx_step_tma.cuh"
#include "phx_step_stream.cuh"
#include "phx_step_tetm_fused.cuh"
#include "phx_rt.hpp"
#include "phx_adjoint.cuh"
#include "phx_ssfm.cuh"
#include "phx_dp45_fused.cuh"

namespace phx {

thread_local std::string g_create_error;

// ---------------------------------------------------------------- engine
struct EngineBase {
    phx_params P{};
    cudaStream_t stream = nullptr;
    int64_t launches = 0;
    std::string last_error;
    TemporalSpec pump_t[kMaxGroups], pot_t[kMaxGroups], pulse_t[kMaxGroups];
    bool force_fixed = false;  // phx_iterate(force_fixed_time_step): no step-size control this call
    std::vector<std::pair<int, double>> tune_medians;  // (shape, median us per iteration) of the last tuning
    // set by phx_request_abort (any thread); phx_step stops before its next iteration
    std::atomic<int> abort_requested{0};
    int wait_polls = kWaitPolls;  // bound of the TMA iteration's wait for a tile's data (phx_set_wait_limit)
    virtual ~EngineBase() = default;
    virtual void set_spectrum_output(bool enable) = 0;
    virtual void init() = 0;
    virtual void set_field(int field, int group, const void* host, int64_t count, int dtype) = 0;
    virtual void get_field(int field, int group, void* host, int64_t count, int dtype) = 0;
    virtual void step(int64_t max_iterations, phx_step_info* info) = 0;
    virtual void get_time(double* t, double* dt) = 0;
    virtual void set_time(double t, double dt) = 0;
    virtual double sum_abs2(int field) = 0;
    virtual void field_ptr(int field, int group, void** ptr, int64_t* pitch) = 0;
    virtual void field_device(int field, int group, void* dev, int64_t count, bool upload) = 0;
    virtual void adjoint_forward(int64_t iterations, int64_t every) = 0;
    virtual void adjoint_backward(const void* dpsi, const void* dn, void* dpsi0, void* dn0, void* dpump, void* dpot) = 0;

    // ---- per-launch event timing (phx_profile_*)
    bool profiling = false;
    struct Pending {
        int kind;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    double prof_ms[PHX_KERNEL_KINDS] = {};
    double prof_bytes[PHX_KERNEL_KINDS] = {};
    int64_t prof_count[PHX_KERNEL_KINDS] = {};
    cudaEvent_t get_event() {
        if (!event_pool.empty()) {
            cudaEvent_t e = event_pool.back();
            event_pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        PHX_CUDA(cudaEventCreate(&e));
        return e;
    }
    void prof_begin(cudaEvent_t& a) {
        if (!profiling) return;
        a = get_event();
        PHX_CUDA(cudaEventRecord(a, stream));
    }
    void prof_end(int kind, cudaEvent_t a, double bytes) {
        if (!profiling) return;
        cudaEvent_t b = get_event();
        PHX_CUDA(cudaEventRecord(b, stream));
        pending.push_back({kind, a, b, bytes});
    }
    void prof_harvest() {
        if (pending.empty()) return;
        PHX_CUDA(cudaStreamSynchronize(stream));
        for (auto& p : pending) {
            float ms = 0.f;
            PHX_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
            prof_ms[p.kind] += ms;
            prof_bytes[p.kind] += p.bytes;
            prof_count[p.kind] += 1;
            event_pool.push_back(p.a);
            event_pool.push_back(p.b);
        }
        pending.clear();
    }
    void prof_reset() {
        prof_harvest();
        for (int k = 0; k < PHX_KERNEL_KINDS; ++k) prof_ms[k] = prof_bytes[k] = 0, prof_count[k] = 0;
    }
};

template <typename T>
struct Engine final : EngineBase {
    int G = kRing;  // ring width of the padded planes: kRing, or H + 1 for wider halos
    static constexpr int CPT = Pack<T>::CPT;
    int shape = -1;                 // launch shape in use (kShapeRB / kShapeWarps), -1 = tuning
    int tune_step = 0;              // steps run while tuning
    static constexpr int kTuneRounds = 6;  // rounds over the candidates (the first untimed)
    static constexpr int kTuneIters = 3;   // consecutive iterations of one candidate per sample
    static constexpr double kTuneMargin = 0.03;  // a challenger must beat the incumbent by this fraction
    static constexpr int kFusedShape = kShapes;  // launch shapes 4-7: whole RK4 iteration in one kernel
    static constexpr int kFusedShapes = 11;      // shapes 8-13: persistent TMA-fed tiles, 14: column strips
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> tune_ev[kShapes + kFusedShapes];
    static constexpr int kRingBlocks = 256;  // blocks of the ring-norm kernels (their partial-sum slots follow the stage kernels')
    static constexpr int kNormBlocks = 296;
    // imaginary-time propagation (--imagTime): k-stack sums with the complex
    // step, then Solver::normalizeImaginaryTimePropagation after every iteration
    bool imag_time() const { return P.imag_time_amplitude != 0.0; }
    // step-size control this iteration (off for phx_iterate's forced fixed step)
    bool adaptive_now() const { return P.adaptive != 0 && !force_fixed; }
    DevBuf imag_f;           // the device-side normalisation factor (T)
    double imag_nrm = 0.0;   // adaptive stepping: the accepted attempt's norm
    using C = cx<T>;

    int N_r = 0, N_c = 0;
    long long pitch = 0, rows = 0, plane = 0;
    Derived<T> d{};
    int comps = 1;
    int H = 4;  // halo width the reference uses: k_max of the iterator
    Tableau tab;  // the fixed-step tableau of the other iterators

    // state and work planes (each allocation holds 1 or more planes)
    DevBuf psi[2], nres[2];            // state per component
    DevBuf sbuf_psi[2][2], sbuf_n[2][2];  // [component][ping-pong] stage values
    DevBuf acc_psi[2], acc_n[2];       // RK4 accumulators
    DevBuf k_psi[2], k_n[2];           // DP45 k-stack (7 planes)
    DevBuf pump[2], pot[2], pulse[2];  // input planes (groups)
    DevBuf mask[2];                    // fft-shifted mask, contiguous N_r*N_c
    DevBuf fft_x;                      // contiguous scratch for the filter
    DevBuf psi_alt, n_alt;             // second state plane for the fused RK4 iteration
    DevBuf err_flag;                   // set by kernels whose bounded waits gave up
    DevBuf partials, result;
    PinnedBuf host_result;
    cufftHandle plan = 0;
    bool have_plan = false;
    bool have_mask[2] = {false, false};

    // simulation clock, in the build precision (SystemParameters::p.t / p.dt)
    T t = 0, dt = 0, fft_cached_t = 0;
    // stochastic noise: Solver::iterate calls so far (the generator's counter)
    // and dw * sqrt(dt) of the current iteration (solver.cu:36-45)
    uint64_t noise_iteration = 0;
    T noise_amp = 0;
    double r7_prev = 0, r7_cur = 0;  // DP45 reference norm: outer halo ring carried between steps
    int64_t accepted_steps = 0;

    ~Engine() override {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        for (auto e : event_pool) cudaEventDestroy(e);
        if (have_plan) cufftDestroy(plan);
        if (have_ssfm_plan) cufftDestroy(ssfm_plan);
        if (stream) cudaStreamDestroy(stream);
    }

    C* cplane(DevBuf& b, int k = 0) { return reinterpret_cast<C*>(b.p) + G * pitch + G + (long long)k * plane; }
    T* rplane(DevBuf& b, int k = 0) { return reinterpret_cast<T*>(b.p) + G * pitch + G + (long long)k * plane; }

    void init() override {
        N_r = P.N_r;
        N_c = P.N_c;
        comps = P.tetm ? 2 : 1;
        if (P.iterator != PHX_ITER_RK4 && P.iterator != PHX_ITER_SSFM && !tableau_resolve(P.iterator, tab))
            fail(PHX_ERR_INVALID_ARG, "unknown iterator");
        // imaginary-time RK4 runs the k-stack stage kernels (complex step)
        if (P.iterator == PHX_ITER_RK4 && imag_time()) tableau_resolve(PHX_ITER_RK4, tab);
        // halo_size_ = k_max_ of the iterator's constructor (SSFM: 0); the ring holds it
        H = P.iterator == PHX_ITER_RK4 ? 4 : (P.iterator == PHX_ITER_SSFM ? 0 : tab.H);
        G = std::max(kRing, H + 1);
        pitch = ((N_c + 2LL * G) + 31) / 32 * 32;
        rows = N_r + 2LL * G;
        plane = pitch * rows;
        d = derive<T>(P);
        PHX_CUDA(cudaSetDevice(P.device));
        PHX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        const size_t cb = sizeof(C) * plane, rb = sizeof(T) * plane;
        for (int q = 0; q < comps; ++q) {
            psi[q].alloc(cb, stream);
            nres[q].alloc(rb, stream);
            for (int b = 0; b < 2; ++b) {
                sbuf_psi[q][b].alloc(cb, stream);
                sbuf_n[q][b].alloc(rb, stream);
            }
            if (P.iterator == PHX_ITER_RK4 && !imag_time()) {
                acc_psi[q].alloc(cb, stream);
                acc_n[q].alloc(rb, stream);
            } else {
                const int kp = std::max({7, tab.H, tab.nb, tab.E});
                k_psi[q].alloc(cb * kp, stream);
                k_n[q].alloc(rb * kp, stream);
            }
            pump[q].alloc(rb * std::max(1, P.n_pump_groups), stream);
            pot[q].alloc(rb * std::max(1, P.n_potential_groups), stream);
            pulse[q].alloc(cb * std::max(1, P.n_pulse_groups), stream);
        }
        long long min_rpb = rows_per_block(0);
        for (int sh = 1; sh < kShapes; ++sh) min_rpb = std::min(min_rpb, rows_per_block(sh));
        const long long max_blocks = grid_x(-(long long)G, N_c + G) * ((N_r + 2LL * G + min_rpb - 1) / min_rpb) + kRingBlocks;
        if (const char* e = std::getenv("PHX_STAGE_SHAPE")) {
            const int v = std::atoi(e);
            if (v >= 0 && v < kShapes) shape = v;
            if (v >= kFusedShape && v < kFusedShape + kFusedShapes && fused_eligible_static()) shape = v;
        }
        if (shape < 0 && shape_free()) shape = kDefaultShape;
        if (shape < 0 && tune_cache_on()) {
            std::lock_guard<std::mutex> lk(tune_cache_mu());
            auto it = tune_cache().find(tune_key());
            if (it != tune_cache().end()) shape = it->second;
        }
        partials.alloc(sizeof(double) * 2 * std::max<long long>(max_blocks, 1024), stream);
        result.alloc(sizeof(double) * 4, stream);
        host_result.alloc(sizeof(double) * 4);
        imag_f.alloc(sizeof(double) * 2, stream);
        t = (T)P.t0;
        dt = (T)P.dt;
        fft_cached_t = (T)0.0;
        PHX_CUDA(cudaStreamSynchronize(stream));
    }

    long long grid_x(long long c0, long long c1) const { return (c1 - c0 + 32 * CPT - 1) / (32 * CPT); }
    // autotuning candidates: the stage kernels' shapes 0-3, or, where the
    // one-kernel iteration applies, its shapes 4-14 (the stage kernels, four
    // launches and 236 B per point, never beat it there)
    int first_candidate() const { return fused_eligible_static() ? kFusedShape : 0; }
    int n_candidates() const { return fused_eligible_static() ? kFusedShapes : kShapes; }
    bool is_fused(int sh) const { return sh >= kFusedShape; }
    int cur_shape() const {
        return shape >= 0 ? shape : first_candidate() + (tune_step / kTuneIters) % n_candidates();
    }
    // the shape kept unless a challenger is clearly faster: 64 x 16 tiles of
    // the TMA iteration with two 12-warp CTAs per SM where the one-kernel
    // iteration applies (fastest at 1024^2 and 4096^2 on B200), else the
    // stage kernels' default
    int incumbent() const { return fused_eligible_static() ? kFusedShape + 6 : kDefaultShape; }
    // iterations whose kernels do not depend on the launch shape: no tuning
    bool shape_free() const {
        if (P.iterator == PHX_ITER_SSFM) return true;
        if (P.iterator != PHX_ITER_RK4 || imag_time()) return false;
        return (P.tetm && tetm_fused_on()) || (!P.tetm && !fused_eligible_static() && general_fused_on());
    }
    // the fused iteration handles scalar RK4 with at most one pump and one
    // potential group and no pulse (real temporal coefficients are checked
    // every iteration)
    bool fused_eligible_static() const {
        return P.iterator == PHX_ITER_RK4 && !P.tetm && P.n_pump_groups <= 1 && P.n_potential_groups <= 1 &&
               P.n_pulse_groups == 0 && !(P.stochastic_amplitude > 0.0) && !imag_time();
    }
    long long rows_per_block(int sh) const { return (long long)kShapeRB[sh] * kShapeWarps[sh]; }
    long long grid_y(long long r0, long long r1) const {
        const long long rpb = rows_per_block(is_fused(cur_shape()) ? kDefaultShape : cur_shape());
        return (r1 - r0 + rpb - 1) / rpb;
    }

    // ------------------------------------------------------------ fields
    struct FieldRef {
        DevBuf* buf;
        bool complex;
        int plane_index;
        int comp;
    };
    FieldRef field_ref(int field, int group) {
        const int comp = (field == PHX_PSI_MINUS || field == PHX_N_MINUS || field == PHX_PUMP_MINUS ||
                          field == PHX_POTENTIAL_MINUS || field == PHX_PULSE_MINUS || field == PHX_FFT_MASK_MINUS)
                             ? 1
                             : 0;
        if (comp == 1 && !P.tetm) fail(PHX_ERR_INVALID_ARG, "minus-component field requires tetm mode");
        switch (field) {
            case PHX_PSI_PLUS:
            case PHX_PSI_MINUS:
                return {&psi[comp], true, 0, comp};
            case PHX_N_PLUS:
            case PHX_N_MINUS:
                if (!P.use_reservoir) fail(PHX_ERR_INVALID_ARG, "reservoir field requires use_reservoir");
                return {&nres[comp], false, 0, comp};
            case PHX_PUMP_PLUS:
            case PHX_PUMP_MINUS:
                if (group < 0 || group >= P.n_pump_groups) fail(PHX_ERR_INVALID_ARG, "pump group out of range");
                return {&pump[comp], false, group, comp};
            case PHX_POTENTIAL_PLUS:
            case PHX_POTENTIAL_MINUS:
                if (group < 0 || group >= P.n_potential_groups) fail(PHX_ERR_INVALID_ARG, "potential group out of range");
                return {&pot[comp], false, group, comp};
            case PHX_PULSE_PLUS:
            case PHX_PULSE_MINUS:
                if (group < 0 || group >= P.n_pulse_groups) fail(PHX_ERR_INVALID_ARG, "pulse group out of range");
                return {&pulse[comp], true, group, comp};
            default:
                fail(PHX_ERR_INVALID_ARG, "unknown field " + std::to_string(field));
        }
        return {nullptr, false, 0, 0};
    }

    static void convert_in(const void* host, int dtype, size_t n, std::vector<T>& out) {
        out.resize(n);
        if (dtype == PHX_F64) {
            const double* s = static_cast<const double*>(host);
            for (size_t i = 0; i < n; ++i) out[i] = (T)s[i];
        } else {
            const float* s = static_cast<const float*>(host);
            for (size_t i = 0; i < n; ++i) out[i] = (T)s[i];
        }
    }

    void set_field(int field, int group, const void* host, int64_t count, int dtype) override {
        if (!host) fail(PHX_ERR_INVALID_ARG, "host pointer is NULL");
        if (dtype != PHX_F32 && dtype != PHX_F64) fail(PHX_ERR_INVALID_ARG, "bad host dtype");
        const long long N = (long long)N_r * N_c;
        if (field == PHX_FFT_MASK_PLUS || field == PHX_FFT_MASK_MINUS) {
            const int comp = field == PHX_FFT_MASK_MINUS ? 1 : 0;
            if (comp == 1 && !P.tetm) fail(PHX_ERR_INVALID_ARG, "minus mask requires tetm");
            if (count != N) fail(PHX_ERR_INVALID_ARG, "mask needs N_c*N_r values");
            std::vector<T> m;
            convert_in(host, dtype, (size_t)N, m);
            // fft_shift_2D (kernel_fft.cuh:16-32), done once on the host
            for (int k = 0; k < N_r / 2; ++k)
                for (int l = 0; l < N_c / 2; ++l) {
                    std::swap(m[(size_t)k * N_c + l], m[(size_t)(k + N_r / 2) * N_c + l + N_c / 2]);
                    std::swap(m[(size_t)k * N_c + l + N_c / 2], m[(size_t)(k + N_r / 2) * N_c + l]);
                }
            if (!mask[comp].p) mask[comp].alloc(sizeof(T) * N, stream);
            PHX_CUDA(cudaMemcpyAsync(mask[comp].p, m.data(), sizeof(T) * N, cudaMemcpyHostToDevice, stream));
            PHX_CUDA(cudaStreamSynchronize(stream));
            have_mask[comp] = true;
            ensure_fft();
            return;
        }
        FieldRef f = field_ref(field, group);
        const long long want = f.complex ? 2 * N : N;
        if (count != want) fail(PHX_ERR_INVALID_ARG, "expected " + std::to_string(want) + " values, got " + std::to_string(count));
        // same precision: copy straight from the caller's buffer (DMA when it is
        // pinned); otherwise convert through a host staging vector
        std::vector<T> tmp;
        const void* src = host;
        if ((dtype == PHX_F64) != (sizeof(T) == 8)) {
            convert_in(host, dtype, (size_t)want, tmp);
            src = tmp.data();
        }
        const size_t esz = f.complex ? sizeof(C) : sizeof(T);
        char* dst = reinterpret_cast<char*>(f.buf->p) + esz * (G * pitch + G + (long long)f.plane_index * plane);
        PHX_CUDA(cudaMemcpy2DAsync(dst, esz * pitch, src, esz * N_c, esz * N_c, N_r, cudaMemcpyHostToDevice, stream));
        // ring of the uploaded plane: zeros along zero axes, periodic images
        // along periodic axes (synchronize_halos after every upload,
        // solver_initialization.cu:81-146)
        if (f.complex)
            ring_fill_kernel<C><<<64, 256, 0, stream>>>(cplane(*f.buf, f.plane_index), N_r, N_c, pitch, G, P.periodic_x,
                                                        P.periodic_y);
        else
            ring_fill_kernel<T><<<64, 256, 0, stream>>>(rplane(*f.buf, f.plane_index), N_r, N_c, pitch, G, P.periodic_x,
                                                        P.periodic_y);
        PHX_CUDA(cudaGetLastError());
        PHX_CUDA(cudaStreamSynchronize(stream));
    }

    void get_field(int field, int group, void* host, int64_t count, int dtype) override {
        if (!host) fail(PHX_ERR_INVALID_ARG, "host pointer is NULL");
        PHX_CUDA(cudaStreamSynchronize(stream));
        check_err_flag();
        if (dtype != PHX_F32 && dtype != PHX_F64) fail(PHX_ERR_INVALID_ARG, "bad host dtype");
        if (field == PHX_FFT_MASK_PLUS || field == PHX_FFT_MASK_MINUS) fail(PHX_ERR_UNSUPPORTED, "mask read-back not provided");
        if (field == PHX_FFT_PLUS || field == PHX_FFT_MINUS) {
            const int q = field == PHX_FFT_MINUS ? 1 : 0;
            if (q >= comps) fail(PHX_ERR_INVALID_ARG, "fft_minus needs TE/TM mode");
            if (!keep_spectrum || !spectrum[q].p) fail(PHX_ERR_INVALID_ARG, "the spectrum is kept after phx_set_spectrum_output(h, 1)");
            const long long n2 = 2LL * N_r * N_c;
            if (count != n2) fail(PHX_ERR_INVALID_ARG, "expected " + std::to_string(n2) + " values");
            std::vector<T> tmp((size_t)n2);
            PHX_CUDA(cudaMemcpyAsync(tmp.data(), spectrum[q].p, sizeof(T) * (size_t)n2, cudaMemcpyDeviceToHost, stream));
            PHX_CUDA(cudaStreamSynchronize(stream));
            for (long long i = 0; i < n2; ++i) {
                if (dtype == PHX_F64)
                    static_cast<double*>(host)[i] = (double)tmp[i];
                else
                    static_cast<float*>(host)[i] = (float)tmp[i];
            }
            return;
        }
        FieldRef f = field_ref(field, group);
        const long long N = (long long)N_r * N_c;
        const long long want = f.complex ? 2 * N : N;
        if (count != want) fail(PHX_ERR_INVALID_ARG, "expected " + std::to_string(want) + " values");
        const size_t esz = f.complex ? sizeof(C) : sizeof(T);
        const char* src = reinterpret_cast<const char*>(f.buf->p) + esz * (G * pitch + G + (long long)f.plane_index * plane);
        if ((dtype == PHX_F64) == (sizeof(T) == 8)) {
            PHX_CUDA(cudaMemcpy2DAsync(host, esz * N_c, src, esz * pitch, esz * N_c, N_r, cudaMemcpyDeviceToHost, stream));
            PHX_CUDA(cudaStreamSynchronize(stream));
            return;
        }
        std::vector<T> tmp((size_t)want);
        PHX_CUDA(cudaMemcpy2DAsync(tmp.data(), esz * N_c, src, esz * pitch, esz * N_c, N_r, cudaMemcpyDeviceToHost, stream));
        PHX_CUDA(cudaStreamSynchronize(stream));
        if (dtype == PHX_F64) {
            double* o = static_cast<double*>(host);
            for (long long i = 0; i < want; ++i) o[i] = (double)tmp[i];
        } else {
            float* o = static_cast<float*>(host);
            for (long long i = 0; i < want; ++i) o[i] = (float)tmp[i];
        }
    }

    void field_ptr(int field, int group, void** ptr, int64_t* pp) override {
        FieldRef f = field_ref(field, group);
        const size_t esz = f.complex ? sizeof(C) : sizeof(T);
        *ptr = reinterpret_cast<char*>(f.buf->p) + esz * (G * pitch + G + (long long)f.plane_index * plane);
        if (pp) *pp = pitch;
    }

    // The reference plans (N_c, N_r) on the full N_r x N_c matrix
    // (solver_fft.cu:35-48).  Square grids transform the halo-padded state
    // plane in place (advanced layout: rows of `pitch` elements), with no
    // copies in or out; other shapes reinterpret the row-major matrix as N_c
    // rows of N_r, which only a contiguous copy can express.
    bool fft_in_place = false;
    // phx_set_spectrum_output: the k-space field of the last filter time
    bool keep_spectrum = false;
    DevBuf spectrum[2];
    void set_spectrum_output(bool enable) override {
        keep_spectrum = enable;
        if (have_plan) {
            PHX_CUDA(cudaStreamSynchronize(stream));
            cufftDestroy(plan);
            have_plan = false;
        }
        if (enable || have_mask[0] || have_mask[1]) ensure_fft();
        if (enable)
            for (int q = 0; q < comps; ++q)
                if (!spectrum[q].p) {
                    spectrum[q].alloc(sizeof(C) * (size_t)N_r * N_c, stream);
                    PHX_CUDA(cudaMemsetAsync(spectrum[q].p, 0, sizeof(C) * (size_t)N_r * N_c, stream));
                }
    }
    void ensure_fft() {
        if (have_plan) return;
        // the spectrum is kept from the contiguous transform, whose plan has the
        // reference's (N_c, N_r) dimensions
        fft_in_place = N_r == N_c && !keep_spectrum && !std::getenv("PHX_FFT_CONTIGUOUS");
        if (fft_in_place) {
            int n[2] = {N_r, N_c};
            int embed[2] = {(int)rows, (int)pitch};
            PHX_CUFFT(cufftPlanMany(&plan, 2, n, embed, 1, (int)plane, embed, 1, (int)plane,
                                    sizeof(T) == 4 ? CUFFT_C2C : CUFFT_Z2Z, 1));
        } else {
            fft_x.alloc(sizeof(C) * (size_t)N_r * N_c, stream);
            PHX_CUFFT(cufftPlan2d(&plan, N_c, N_r, sizeof(T) == 4 ? CUFFT_C2C : CUFFT_Z2Z));
        }
        PHX_CUFFT(cufftSetStream(plan, stream));
        have_plan = true;
    }

    void get_time(double* tt, double* dd) override {
        if (tt) *tt = (double)t;
        if (dd) *dd = (double)dt;
    }
    void set_time(double tt, double dd) override {
        t = (T)tt;
        dt = (T)dd;
    }

    // ------------------------------------------------------------ stage launch
    StageParams<T> base_params(int comp) {
        StageParams<T> S;
        std::memset(&S, 0, sizeof(S));
        S.N_r = N_r;
        S.N_c = N_c;
        S.img_x = P.periodic_x;
        S.img_y = P.periodic_y;
        S.pitch = pitch;
        S.plane = plane;
        S.m2 = d.m2;
        S.odx2 = d.odx2;
        S.ody2 = d.ody2;
        S.meff = d.meff;
        S.ohb = d.ohb;
        S.ohb_gc = d.ohb * (T)P.g_c;
        S.half_gamma_c = (T)0.5 * (T)P.gamma_c;
        S.ohb_gr = d.ohb * (T)P.g_r;
        S.half_R = (T)0.5 * (T)P.R;
        S.gamma_r = (T)P.gamma_r;
        S.R = (T)P.R;
        (void)comp;
        S.n_pump = P.n_pump_groups;
        S.n_pot = P.n_potential_groups;
        S.n_pulse = P.n_pulse_groups;
        S.dt = dt;
        S.error_passes = 1;
        // stochastic terms of this iteration (noise drawn in the kernels)
        S.noise.on = P.stochastic_amplitude > 0.0;
        S.noise.key0 = (uint32_t)P.seed;
        S.noise.key1 = (uint32_t)(P.seed >> 32);
        S.noise.it_lo = (uint32_t)noise_iteration;
        S.noise.it_hi = (uint32_t)(noise_iteration >> 32);
        S.noise_amp = noise_amp;
        S.dV = d.dV;
        S.four_dV = (T)4.0 * d.dV;
        S.gamma_c = (T)P.gamma_c;
        S.noise_scale = std::sqrt((T)P.gamma_c / S.four_dV);
        S.imag = imag_time() ? 1 : 0;
        return S;
    }
    // weight sum of a stage sum's dw term: the right fold w_1 + (w_2 + (...))
    // of the weights the reference instantiates (kernel_summation.cuh:62-64)
    static T right_fold(const T* w, int n) {
        T acc = w[n - 1];
        for (int q = n - 2; q >= 0; --q) acc = w[q] + acc;
        return acc;
    }

    // temporal amplitudes at t (amp) and t+dt (amp_next): updateKernelTime
    std::complex<T> amp_pump[kMaxGroups], next_pump[kMaxGroups];
    std::complex<T> amp_pot[kMaxGroups], next_pot[kMaxGroups];
    std::complex<T> amp_pulse[kMaxGroups], next_pulse[kMaxGroups];
    void update_kernel_time() {
        const T tn = t + dt;
        for (int g = 0; g < P.n_pulse_groups; ++g) amp_pulse[g] = temporal_value<T>(pulse_t[g], t);
        for (int g = 0; g < P.n_potential_groups; ++g) amp_pot[g] = temporal_value<T>(pot_t[g], t);
        for (int g = 0; g < P.n_pump_groups; ++g) amp_pump[g] = temporal_value<T>(pump_t[g], t);
        for (int g = 0; g < P.n_pulse_groups; ++g) next_pulse[g] = temporal_value<T>(pulse_t[g], tn);
        for (int g = 0; g < P.n_potential_groups; ++g) next_pot[g] = temporal_value<T>(pot_t[g], tn);
        for (int g = 0; g < P.n_pump_groups; ++g) {
            next_pump[g] = temporal_value<T>(pump_t[g], tn);
            if (amp_pump[g].imag() != (T)0 || next_pump[g].imag() != (T)0)
                fail(PHX_ERR_UNSUPPORTED, "complex pump temporal envelopes (iexp) would make the reservoir complex");
        }
    }
    void set_coefficients(StageParams<T>& S, T w) {
        for (int g = 0; g < P.n_pump_groups; ++g) {
            const auto c = interp<T>(amp_pump[g], next_pump[g], w);
            S.pump_c[g] = mk_host(c);
        }
        for (int g = 0; g < P.n_potential_groups; ++g) S.pot_c[g] = mk_host(interp<T>(amp_pot[g], next_pot[g], w));
        for (int g = 0; g < P.n_pulse_groups; ++g) S.pulse_c[g] = mk_host(interp<T>(amp_pulse[g], next_pulse[g], w));
    }
    static C mk_host(std::complex<T> z) {
        C c;
        c.re = z.real();
        c.im = z.imag();
        return c;
    }

    // compute rectangle of stage s (1-based) of an H-stage step: the subgrid
    // extended by H - s cells along non-periodic axes (cuda_macro.cuh:110-113)
    void region(StageParams<T>& S, int ext) {
        const int ex = P.periodic_x ? 0 : ext;
        const int ey = P.periodic_y ? 0 : ext;
        S.r0 = -ey;
        S.r1 = N_r + ey;
        int c0 = -ex, c1 = N_c + ex;
        c0 = (c0 >= 0) ? (c0 / CPT) * CPT : -((-c0 + CPT - 1) / CPT) * CPT;
        c1 = ((c1 + CPT - 1) / CPT) * CPT;
        S.c0 = c0;
        S.c1 = c1;
    }

    // Algorithmic HBM bytes of one stage launch: every plane the kernel
    // reads or writes, once per point of its rectangle.
    double stage_bytes(int KIND, bool RES, const StageParams<T>& S) const {
        const double c = sizeof(C), r = sizeof(T);
        const double st = c + (RES ? r : 0.0);  // one state (psi, n)
        const double inputs = S.n_pump * r + S.n_pot * r + S.n_pulse * c;
        double b = 0;
        switch (KIND) {
            case kRk4First: b = st + inputs + 2 * st; break;
            case kRk4Mid: b = 3 * st + inputs + 2 * st; break;
            case kRk4Last: b = 3 * st + inputs + st; break;
            case kStack: {
                const int kreads = S.nw > 1 ? S.nw - 1 : 0;
                b = st + (S.stage > 1 ? st : 0) + kreads * st + inputs + 2 * st;
                break;
            }
            case kStackFinal: b = 2 * st + (S.nw - 1) * st + inputs + st; break;
            case kStackError: b = st + (S.nw - 1) * c + inputs; break;
        }
        return b * (double)(S.r1 - S.r0) * (double)(S.c1 - S.c0);
    }
    template <int KIND, bool RES, int SH>
    void go_scalar(const StageParams<T>& S, dim3 grid) {
        stage_scalar_kernel<T, KIND, RES, kShapeRB[SH], kShapeWarps[SH]><<<grid, 32 * kShapeWarps[SH], 0, stream>>>(S);
    }
    template <int KIND, bool RES>
    void launch_kind(const StageParams<T>& S) {
        dim3 grid((unsigned)grid_x(S.c0, S.c1), (unsigned)grid_y(S.r0, S.r1));
        cudaEvent_t a = nullptr;
        prof_begin(a);
        switch (is_fused(cur_shape()) ? kDefaultShape : cur_shape()) {
            case 0: go_scalar<KIND, RES, 0>(S, grid); break;
            case 1: go_scalar<KIND, RES, 1>(S, grid); break;
            case 2: go_scalar<KIND, RES, 2>(S, grid); break;
            default: go_scalar<KIND, RES, 3>(S, grid); break;
        }
        prof_end(KIND, a, stage_bytes(KIND, RES, S));
        ++launches;
    }
    template <int KIND, int SH>
    void go_tetm(const TetmParams<T>& Q, dim3 grid) {
        stage_tetm_kernel<T, KIND, kShapeRB[SH], kShapeWarps[SH]><<<grid, 32 * kShapeWarps[SH], 0, stream>>>(Q);
    }
    // TE/TM parameters of one stage: S wired for the plus component, the
    // minus component's planes from wire(., 1)
    template <typename Wire>
    TetmParams<T> tetm_params(const StageParams<T>& S, Wire wire) {
        TetmParams<T> Q;
        std::memset(&Q, 0, sizeof(Q));
        Q.p = S;
        StageParams<T> M = S;
        wire(M, 1);
        Q.psi_in = M.psi_in, Q.n_in = M.n_in, Q.psi0 = M.psi0, Q.n0 = M.n0, Q.psi_out = M.psi_out;
        Q.n_out = M.n_out, Q.acc_psi = M.acc_psi, Q.acc_n = M.acc_n, Q.k_psi = M.k_psi, Q.k_n = M.k_n;
        Q.pump = M.pump, Q.pot = M.pot, Q.pulse = M.pulse;
        Q.ohb_meff = d.ohb * d.meff;
        Q.ohb_gpm = d.ohb * (T)P.g_pm;
        Q.ohb_dlt = d.ohb * (T)P.delta_LT;
        Q.hidd.re = (T)0.0 / d.dx / d.dy;
        Q.hidd.im = (T)0.5 / d.dx / d.dy;
        return Q;
    }

    // Launch stage KIND.  `wire(S, q)` points S at component q's planes; in
    // TE/TM mode the minus component's planes are wired the same way and
    // both polarisations run in one kernel.
    template <int KIND, typename Wire>
    void launch(StageParams<T>& S, Wire wire) {
        wire(S, 0);
        if (P.tetm) {
            TetmParams<T> Q = tetm_params(S, wire);
            dim3 grid((unsigned)grid_x(S.c0, S.c1), (unsigned)grid_y(S.r0, S.r1));
            cudaEvent_t a = nullptr;
            prof_begin(a);
            switch (is_fused(cur_shape()) ? kDefaultShape : cur_shape()) {
                case 0: go_tetm<KIND, 0>(Q, grid); break;
                case 1: go_tetm<KIND, 1>(Q, grid); break;
                case 2: go_tetm<KIND, 2>(Q, grid); break;
                default: go_tetm<KIND, 3>(Q, grid); break;
            }
            prof_end(KIND, a, 2 * stage_bytes(KIND, true, S));
            ++launches;
        } else if (P.use_reservoir) {
            launch_kind<KIND, true>(S);
        } else {
            launch_kind<KIND, false>(S);
        }
        PHX_CUDA(cudaGetLastError());
    }

    // ------------------------------------------------------------ RK4
    // Whole iteration in one launch (phx_step_fused.cuh).  Returns false when
    // this iteration needs the per-stage kernels (complex temporal
    // coefficients).
    // fused-iteration tile shapes (TW x TH points, NT threads); FP64 uses half-height tiles
    // The one-kernel iterations are launched with programmatic stream
    // serialization: the next iteration's kernel is scheduled while this one
    // drains and waits (pdl_wait, phx_device.cuh) for it to complete before
    // reading the state.  PHX_PDL=0 launches them plainly.
    static bool pdl_on() {
        static const bool on = [] {
            const char* e = std::getenv("PHX_PDL");
            return !(e && e[0] == '0');
        }();
        return on;
    }
    template <typename... KArgs, typename... Args>
    void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, Args&&... args) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = pdl_on() ? 1 : 0;
        PHX_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
    }
    template <bool RES, int TW, int TH, int NT, bool FMA>
    void go_fused_shape(const FusedParams<T>& F) {
        dim3 grid((unsigned)((N_c + TW - 1) / TW), (unsigned)((N_r + TH - 1) / TH));
        launch_pdl(rk4_fused_kernel<T, RES, TW, TH, NT, false, FMA>, grid, dim3(NT), 0, F);
    }
    // ---- TMA-fed persistent variant
    int sm_count = 0;
    std::map<const void*, int> tma_blocks;  // CTAs per SM of each TMA kernel variant
    void tensor_map(CUtensorMap* m, void* alloc_base, bool complex, int box_w_points, int box_h) {
        plane_tensor_map<T>(m, alloc_base, complex, pitch, rows, box_w_points, box_h);
    }
    // tensor maps depend on the planes and on the tile shape (box size): a
    // map encoded for another shape would expect another byte count
    struct MapPair {
        const void* psi = nullptr;
        const void* n = nullptr;
        int tw = 0, th = 0;
        CUtensorMap psi_map, n_map;
    };
    MapPair tma_maps[2];
    int tma_next = 0;
    CUtensorMap tma_pump_map, tma_pot_map;
    int tma_inputs_tw = 0, tma_inputs_th = 0;
    // tensor maps and parameters of a TMA iteration with TW x TH tiles
    template <int TW, int TH>
    void prepare_tma(TmaParams<T>& Q, const FusedParams<T>& F) {
        static_assert(TW % 4 == 0, "TMA box x alignment needs tile origins on 16-byte boundaries");
        if (!err_flag.p) err_flag.alloc(sizeof(int), stream);
        std::memset(&Q, 0, sizeof(Q));
        Q.f = F;
        // tensor maps over whole allocations (padded (0,0) = interior (-G,-G));
        // the state alternates between two planes, so two encodings are kept
        MapPair* mp = nullptr;
        for (auto& m : tma_maps)
            if (m.psi == psi[0].p && m.n == nres[0].p && m.tw == TW && m.th == TH) mp = &m;
        if (!mp) {
            mp = &tma_maps[tma_next];
            tma_next ^= 1;
            tensor_map(&mp->psi_map, reinterpret_cast<char*>(cplane(psi[0])) - sizeof(C) * (G * pitch + G), true, TW + 8,
                       TH + 8);
            tensor_map(&mp->n_map, reinterpret_cast<char*>(rplane(nres[0])) - sizeof(T) * (G * pitch + G), false, TW + 8,
                       TH + 6);
            mp->psi = psi[0].p;
            mp->n = nres[0].p;
            mp->tw = TW;
            mp->th = TH;
        }
        if (tma_inputs_tw != TW || tma_inputs_th != TH) {
            tensor_map(&tma_pump_map, pump[0].p, false, TW + 8, TH + 6);
            tensor_map(&tma_pot_map, pot[0].p, false, TW + 8, TH + 6);
            tma_inputs_tw = TW;
            tma_inputs_th = TH;
        }
        Q.psi_map = mp->psi_map;
        Q.n_map = mp->n_map;
        Q.pump_map = tma_pump_map;
        Q.pot_map = tma_pot_map;
        Q.has_pump = F.pump != nullptr;
        Q.has_pot = F.pot != nullptr;
        Q.tiles_x = (N_c + TW - 1) / TW;
        Q.err = static_cast<int*>(err_flag.p);
        Q.wait_polls = wait_polls;
        if (!sm_count) PHX_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, P.device));
    }
    template <bool RES, int TW, int TH, int NT, int MINB, bool FMA>
    void go_tma(const FusedParams<T>& F) {
        using Lay = TmaLayout<T, TW, TH>;
        auto kern = rk4_tma_kernel<T, RES, TW, TH, NT, MINB, false, FMA>;
        int& tma_blocks_per_sm = tma_blocks[reinterpret_cast<const void*>(kern)];
        if (!tma_blocks_per_sm) {
            PHX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::total));
            PHX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tma_blocks_per_sm, kern, NT, Lay::total));
            if (tma_blocks_per_sm < 1) fail(PHX_ERR_UNSUPPORTED, "TMA iteration kernel does not fit on an SM");
        }
        TmaParams<T> Q;
        prepare_tma<TW, TH>(Q, F);
        Q.n_tiles = Q.tiles_x * ((N_r + TH - 1) / TH);
        const int blocks = std::min(Q.n_tiles, tma_blocks_per_sm * sm_count);
        launch_pdl(kern, dim3(blocks), dim3(NT), Lay::total, Q);
    }
    // ---- column strips (phx_step_stream.cuh): a CTA walks down a segment of a
    // TW-wide strip, TH rows per step
    template <bool RES, int TW, int TH, int NT, int MINB, bool FMA>
    void go_stream(const FusedParams<T>& F) {
        using Lay = StreamLayout<T, TW, TH>;
        auto kern = rk4_stream_kernel<T, RES, TW, TH, NT, MINB, FMA>;
        int& blocks_per_sm = tma_blocks[reinterpret_cast<const void*>(kern)];
        if (!blocks_per_sm) {
            PHX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::total));
            PHX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, NT, Lay::total));
            if (blocks_per_sm < 1) fail(PHX_ERR_UNSUPPORTED, "column-strip iteration kernel does not fit on an SM");
        }
        if (!err_flag.p) err_flag.alloc(sizeof(int), stream);
        if (!sm_count) PHX_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, P.device));
        auto map_of = [&](const void* base, bool complex) -> const CUtensorMap& {
            const auto key = std::make_tuple(base, complex, TW + 8, TH);
            auto it = store_maps.find(key);
            if (it == store_maps.end()) {
                CUtensorMap m;
                tensor_map(&m, const_cast<void*>(base), complex, TW + 8, TH);
                it = store_maps.emplace(key, m).first;
            }
            return it->second;
        };
        StreamParams<T> Q;
        std::memset(&Q, 0, sizeof(Q));
        Q.f = F;
        Q.psi_map = map_of(psi[0].p, true);
        if (RES) Q.n_map = map_of(nres[0].p, false);
        if (F.pump) Q.pump_map = map_of(pump[0].p, false);
        if (F.pot) Q.pot_map = map_of(pot[0].p, false);
        Q.has_pump = F.pump != nullptr;
        Q.has_pot = F.pot != nullptr;
        Q.err = static_cast<int*>(err_flag.p);
        Q.wait_polls = wait_polls;
        // segments: the fewest step times, counting a prologue step per
        // segment and the waves of CTAs over the SMs
        Q.strips = (N_c + TW - 1) / TW;
        const int row_steps = (N_r + TH - 1) / TH;
        const long long slots = (long long)blocks_per_sm * sm_count;
        long long best = -1;
        for (int per = 1; per <= row_steps; ++per) {
            const int seg_steps = (row_steps + per - 1) / per;
            const int segs = (row_steps + seg_steps - 1) / seg_steps;
            const long long ctas = (long long)Q.strips * segs;
            const long long cost = ((ctas + slots - 1) / slots) * (seg_steps + 1);
            if (best < 0 || cost < best) {
                best = cost;
                Q.seg_steps = seg_steps;
                Q.n_segs = (int)ctas;
            }
        }
        const int blocks = (int)std::min<long long>(Q.n_segs, slots);
        launch_pdl(kern, dim3(blocks), dim3(NT), Lay::total, Q);
    }
    void check_err_flag() {
        if (!err_flag.p) return;
        int v = 0;
        PHX_CUDA(cudaMemcpy(&v, err_flag.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (v) {
            PHX_CUDA(cudaMemset(err_flag.p, 0, sizeof(int)));
            fail(PHX_ERR_TIMEOUT, "a bounded wait for TMA data gave up; the iteration's results are invalid");
        }
    }

    // FMA: the fused multiply-add arithmetic (phx_params.fma, FP32 only)
    template <bool RES, bool FMA = false>
    void go_fused(const FusedParams<T>& F) {
        constexpr bool f32 = sizeof(T) == 4;
        switch (cur_shape() - kFusedShape) {
            case 4: go_tma<RES, 32, f32 ? 32 : 16, 256, 1, FMA>(F); return;
            // 12 warps per CTA, two CTAs per SM: registers capped at 85
            case 5: go_tma<RES, 32, f32 ? 32 : 16, 384, 2, FMA>(F); return;
            case 6: go_tma<RES, 64, f32 ? 16 : 8, 384, 2, FMA>(F); return;
            // taller tiles, one CTA per SM: less halo recomputation per output point
            case 7: go_tma<RES, 64, f32 ? 32 : 16, 768, 1, FMA>(F); return;
            case 8: go_tma<RES, 64, f32 ? 32 : 16, 512, 1, FMA>(F); return;
            // 64 x 14: 1024^2 makes 1184 tiles, exactly four rounds of 296 CTAs
            // (64 x 16 leaves the fourth round half empty)
            case 9: go_tma<RES, 64, f32 ? 14 : 7, 384, 2, FMA>(F); return;
            // column strips: FP32 64 wide, 12 rows per step; FP64 32 wide, 8 rows
            case 10:
                if constexpr (f32)
                    go_stream<RES, 64, 12, 448, 2, FMA>(F);
                else
                    go_stream<RES, 32, 8, 160, 2, FMA>(F);
                return;
            default: break;
        }
        switch (cur_shape() - kFusedShape) {
            case 0: go_fused_shape<RES, 32, f32 ? 32 : 16, 256, FMA>(F); break;
            case 1: go_fused_shape<RES, 64, f32 ? 16 : 8, 256, FMA>(F); break;
            case 2: go_fused_shape<RES, 32, f32 ? 16 : 8, 128, FMA>(F); break;
            default:
                if constexpr (f32)
                    go_fused_shape<RES, 64, 32, 512, FMA>(F);
                else
                    go_fused_shape<RES, 32, 24, 384, FMA>(F);  // 48 KiB static shared-memory limit
                break;
        }
    }
    bool step_rk4_fused() {
        const T cw[4] = {(T)0.0, (T)0.5, (T)0.5, (T)1.0};
        FusedParams<T> F;
        std::memset(&F, 0, sizeof(F));
        for (int s = 0; s < 4; ++s) {
            if (P.n_pump_groups) {
                const auto c = interp<T>(amp_pump[0], next_pump[0], cw[s]);
                if (c.imag() != (T)0) return false;
                F.pump_c[s] = c.real();
            }
            if (P.n_potential_groups) {
                const auto c = interp<T>(amp_pot[0], next_pot[0], cw[s]);
                if (c.imag() != (T)0) return false;
                F.pot_c[s] = c.real();
            }
        }
        if (!psi_alt.p) {
            psi_alt.alloc(sizeof(C) * plane, stream);
            n_alt.alloc(sizeof(T) * plane, stream);
        }
        fused_constants<T>(F, P, d, dt, pitch);
        F.psi0 = cplane(psi[0]);
        F.n0 = rplane(nres[0]);
        F.psi1 = cplane(psi_alt);
        F.n1 = rplane(n_alt);
        F.pump = P.n_pump_groups ? rplane(pump[0]) : nullptr;
        F.pot = P.n_potential_groups ? rplane(pot[0]) : nullptr;
        cudaEvent_t a = nullptr;
        prof_begin(a);
        bool done = false;
        if constexpr (sizeof(T) == 4) {
            if (P.fma) {
                if (P.use_reservoir)
                    go_fused<true, true>(F);
                else
                    go_fused<false, true>(F);
                done = true;
            }
        }
        if (!done) {
            if (P.use_reservoir)
                go_fused<true>(F);
            else
                go_fused<false>(F);
        }
        const double pts = (double)N_r * N_c;
        const double st = sizeof(C) + (P.use_reservoir ? sizeof(T) : 0);
        prof_end(PHX_KERNEL_RK4_FUSED, a,
                 pts * (2 * st + (P.n_pump_groups ? sizeof(T) : 0) + (P.n_potential_groups ? sizeof(T) : 0)));
        ++launches;
        PHX_CUDA(cudaGetLastError());
        std::swap(psi[0].p, psi_alt.p);
        std::swap(nres[0].p, n_alt.p);
        return true;
    }

    // ---- TE/TM: the whole iteration in one kernel (phx_step_tetm_fused.cuh);
    // PHX_TETM_FUSED=0 selects the four stage kernels instead
    bool tetm_fused_set = false;
    static bool tetm_fused_on() {
        const char* e = std::getenv("PHX_TETM_FUSED");
        return !(e && e[0] == '0');
    }
    template <int TW, int TH, int NT>
    void go_tetm_fused(const TetmFusedParams<T>& F) {
        using Lay = TetmFusedLayout<T, TW, TH>;
        auto kern = rk4_tetm_fused_kernel<T, TW, TH, NT>;
        if (!tetm_fused_set) {
            PHX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::bytes));
            tetm_fused_set = true;
        }
        dim3 grid((unsigned)((N_c + TW - 1) / TW), (unsigned)((N_r + TH - 1) / TH));
        launch_pdl(kern, grid, dim3(NT), Lay::bytes, F);
    }
    void step_rk4_tetm_fused() {
        const T cw[4] = {(T)0.0, (T)0.5, (T)0.5, (T)1.0};
        const T aw[3] = {(T)0.5, (T)0.5, (T)1.0};
        const T bw[4] = {(T)(1.0 / 6.0), (T)(1.0 / 3.0), (T)(1.0 / 3.0), (T)(1.0 / 6.0)};
        TetmFusedParams<T> F;
        std::memset(&F, 0, sizeof(F));
        for (int s = 1; s <= 4; ++s) {
            // the per-stage kernels' parameters of stage s (step_rk4 below)
            StageParams<T> S = base_params(0);
            set_coefficients(S, cw[s - 1]);
            S.stage = s;
            S.b = bw[s - 1];
            if (s < 4) S.dtw = dt * aw[s - 1];
            S.w_sum = s < 4 ? aw[s - 1] : right_fold(bw, 4);
            auto wire = [this](StageParams<T>& X, int q) {
                X.pump = rplane(pump[q]);
                X.pot = rplane(pot[q]);
                X.pulse = cplane(pulse[q]);
            };
            wire(S, 0);
            F.st[s - 1] = tetm_params(S, wire);
        }
        for (int q = 0; q < 2; ++q) {
            F.psi0[q] = cplane(psi[q]);
            F.n0[q] = rplane(nres[q]);
            F.psi1[q] = cplane(sbuf_psi[q][0]);
            F.n1[q] = rplane(sbuf_n[q][0]);
        }
        cudaEvent_t a = nullptr;
        prof_begin(a);
        if constexpr (sizeof(T) == 4)
            go_tetm_fused<32, 16, 512>(F);
        else
            go_tetm_fused<32, 8, 512>(F);
        // read psi, n (both components) + pump, potential per group; write psi, n
        const double pt = 2.0 * (2.0 * sizeof(C) + 2.0 * sizeof(T)) +
                          2.0 * sizeof(T) * (P.n_pump_groups + P.n_potential_groups) + 2.0 * sizeof(C) * P.n_pulse_groups;
        prof_end(PHX_KERNEL_RK4_FUSED, a, pt * (double)N_r * N_c);
        ++launches;
        PHX_CUDA(cudaGetLastError());
        swap_state_with(0);
    }

    // ---- scalar RK4 with what rk4_tma_kernel does not take (noise, pulses,
    // several groups): one kernel per iteration as well; PHX_GENERAL_FUSED=0
    // selects the four stage kernels
    bool general_set = false;
    static bool general_fused_on() {
        const char* e = std::getenv("PHX_GENERAL_FUSED");
        return !(e && e[0] == '0');
    }
    template <bool RES, int TW, int TH, int NT>
    void go_general(const ScalarFusedParams<T>& F) {
        using Lay = ScalarFusedLayout<T, TW, TH>;
        auto kern = rk4_scalar_general_kernel<T, RES, TW, TH, NT>;
        if (!general_set) {
            PHX_CUDA(cudaFuncSetAttribute(rk4_scalar_general_kernel<T, true, TW, TH, NT>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::bytes));
            PHX_CUDA(cudaFuncSetAttribute(rk4_scalar_general_kernel<T, false, TW, TH, NT>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::bytes));
            general_set = true;
        }
        dim3 grid((unsigned)((N_c + TW - 1) / TW), (unsigned)((N_r + TH - 1) / TH));
        launch_pdl(kern, grid, dim3(NT), Lay::bytes, F);
    }
    void step_rk4_general() {
        const T cw[4] = {(T)0.0, (T)0.5, (T)0.5, (T)1.0};
        const T aw[3] = {(T)0.5, (T)0.5, (T)1.0};
        const T bw[4] = {(T)(1.0 / 6.0), (T)(1.0 / 3.0), (T)(1.0 / 3.0), (T)(1.0 / 6.0)};
        ScalarFusedParams<T> F;
        std::memset(&F, 0, sizeof(F));
        for (int s = 1; s <= 4; ++s) {
            // the per-stage kernels' parameters of stage s (step_rk4 below)
            StageParams<T> S = base_params(0);
            set_coefficients(S, cw[s - 1]);
            S.stage = s;
            S.b = bw[s - 1];
            if (s < 4) S.dtw = dt * aw[s - 1];
            S.w_sum = s < 4 ? aw[s - 1] : right_fold(bw, 4);
            S.pump = rplane(pump[0]);
            S.pot = rplane(pot[0]);
            S.pulse = cplane(pulse[0]);
            F.st[s - 1] = S;
        }
        F.psi0 = cplane(psi[0]);
        F.n0 = rplane(nres[0]);
        F.psi1 = cplane(sbuf_psi[0][0]);
        F.n1 = rplane(sbuf_n[0][0]);
        cudaEvent_t a = nullptr;
        prof_begin(a);
        constexpr bool f32 = sizeof(T) == 4;
        if (P.use_reservoir)
            go_general<true, 32, f32 ? 16 : 8, 512>(F);
        else
            go_general<false, 32, f32 ? 16 : 8, 512>(F);
        const double pt = 2.0 * (sizeof(C) + (P.use_reservoir ? sizeof(T) : 0.0)) +
                          sizeof(T) * (P.n_pump_groups + P.n_potential_groups) + sizeof(C) * P.n_pulse_groups;
        prof_end(PHX_KERNEL_RK4_FUSED, a, pt * (double)N_r * N_c);
        ++launches;
        PHX_CUDA(cudaGetLastError());
        swap_state_with(0);
    }

    void step_rk4() {
        if (P.tetm && tetm_fused_on()) {
            step_rk4_tetm_fused();
            return;
        }
        if (!P.tetm && !fused_eligible_static() && general_fused_on()) {
            step_rk4_general();
            return;
        }
        if (is_fused(cur_shape()) && step_rk4_fused()) return;
        const T cw[4] = {(T)0.0, (T)0.5, (T)0.5, (T)1.0};
        const T aw[3] = {(T)0.5, (T)0.5, (T)1.0};
        const T bw[4] = {(T)(1.0 / 6.0), (T)(1.0 / 3.0), (T)(1.0 / 3.0), (T)(1.0 / 6.0)};
        for (int s = 1; s <= 4; ++s) {
            StageParams<T> S = base_params(0);
            set_coefficients(S, cw[s - 1]);
            region(S, 4 - s);
            S.stage = s;
            S.b = bw[s - 1];
            if (s < 4) S.dtw = dt * aw[s - 1];
            // RK4 stage sums (runge_kutta.cu:78-91): (1/2), (0, 1/2), (0, 0, 1), (b1..b4)
            S.w_sum = s < 4 ? aw[s - 1] : right_fold(bw, 4);
            auto wire = [this, s](StageParams<T>& X, int q) {
                X.psi0 = cplane(psi[q]);
                X.n0 = rplane(nres[q]);
                X.psi_in = s == 1 ? cplane(psi[q]) : cplane(sbuf_psi[q][(s - 2) & 1]);
                X.n_in = s == 1 ? rplane(nres[q]) : rplane(sbuf_n[q][(s - 2) & 1]);
                X.psi_out = s == 4 ? cplane(psi[q]) : cplane(sbuf_psi[q][(s - 1) & 1]);
                X.n_out = s == 4 ? rplane(nres[q]) : rplane(sbuf_n[q][(s - 1) & 1]);
                X.acc_psi = cplane(acc_psi[q]);
                X.acc_n = rplane(acc_n[q]);
                X.pump = rplane(pump[q]);
                X.pot = rplane(pot[q]);
                X.pulse = cplane(pulse[q]);
            };
            if (s == 1)
                launch<kRk4First>(S, wire);
            else if (s < 4)
                launch<kRk4Mid>(S, wire);
            else
                launch<kRk4Last>(S, wire);
        }
    }

    // ------------------------------------------------------------ other tableaux
    // Stage s: k_s = f(Y_s) kept in the k-stack and Y_{s+1} = y0 + dt sum a_sq k_q
    // over the subgrid extended by H - s; the last stage adds dt sum b_q k_q to
    // the state in place (CALCULATE_K / INTERMEDIATE_SUM_K / FINAL_SUM_K).
    void step_tableau() {
        // a one-stage method (Newton) reads its stencil from the state, so its
        // sum goes to a stage plane that then becomes the state; so does every
        // final sum in imaginary time, whose normalisation reads the state of
        // the step's start
        const bool single = tab.S == 1;
        const bool imag = imag_time();
        const bool to_buf = single || imag;
        // reference norm: the final stage also covers the rings where its k
        // exists (H - S), as CALCULATE_K does there
        const bool ring = imag && P.norm_mode == PHX_NORM_REFERENCE;
        for (int s = 1; s <= tab.S; ++s) {
            const bool last = s == tab.S;
            StageParams<T> S = base_params(0);
            set_coefficients(S, (T)tab.c[s - 1]);
            region(S, last ? (ring ? std::max(0, H - s) : 0) : H - s);
            S.stage = s;
            S.nw = last ? tab.nb : tab.nw[s - 1];
            for (int q = 0; q < S.nw; ++q) S.w[q] = (T)(last ? tab.b[q] : tab.a[s - 1][q]);
            if (S.nw == 1) S.dtw = dt * S.w[0];
            S.w_sum = right_fold(S.w, S.nw);
            auto wire = [this, s, last, to_buf](StageParams<T>& X, int q) {
                X.psi0 = cplane(psi[q]);
                X.n0 = rplane(nres[q]);
                X.psi_in = s == 1 ? cplane(psi[q]) : cplane(sbuf_psi[q][(s - 2) & 1]);
                X.n_in = s == 1 ? rplane(nres[q]) : rplane(sbuf_n[q][(s - 2) & 1]);
                X.k_psi = cplane(k_psi[q]);
                X.k_n = rplane(k_n[q]);
                X.psi_out = last && !to_buf ? cplane(psi[q]) : cplane(sbuf_psi[q][(s - 1) & 1]);
                X.n_out = last && !to_buf ? rplane(nres[q]) : rplane(sbuf_n[q][(s - 1) & 1]);
                X.pump = rplane(pump[q]);
                X.pot = rplane(pot[q]);
                X.pulse = cplane(pulse[q]);
            };
            if (last && !ring)
                launch<kStackFinal>(S, wire);
            else
                launch<kStack>(S, wire);
        }
        if (!imag) {
            if (single) swap_state_with(0);
            return;
        }
        long long nb = kNormBlocks;
        if (ring) {
            // the halo rings of the reference's buffer after its in-place final
            // sum, from the state of the step's start and the k-stack
            RingParams<T> R;
            std::memset(&R, 0, sizeof(R));
            R.psi0 = cplane(psi[0]);
            R.k = cplane(k_psi[0]);
            R.pitch = pitch;
            R.plane = plane;
            R.N_r = N_r;
            R.N_c = N_c;
            R.periodic_x = P.periodic_x;
            R.periodic_y = P.periodic_y;
            R.H = H;
            R.S = tab.S;
            R.dt = dt;
            R.nw[tab.S - 1] = tab.nb;
            for (int q = 0; q < tab.nb; ++q) R.a[tab.S - 1][q] = (T)tab.b[q];
            R.dtw_final = dt * (T)tab.b[0];
            const StageParams<T> B = base_params(0);
            R.noise = B.noise;
            R.noise_amp = B.noise_amp;
            R.w_sum[tab.S - 1] = right_fold(R.a[tab.S - 1], tab.nb);
            R.R = B.R;
            R.gamma_c = B.gamma_c;
            R.four_dV = B.four_dV;
            R.noise_scale = B.noise_scale;
            R.n0 = nullptr;
            R.imag = 1;
            R.partials = reinterpret_cast<double*>(partials.p) + 2 * kNormBlocks;
            final_ring_kernel<T><<<kRingBlocks, 256, 0, stream>>>(R);
            ++launches;
            PHX_CUDA(cudaGetLastError());
            nb += kRingBlocks;
        }
        swap_state_with((tab.S - 1) & 1);
        imag_normalize_device(psi[0], true, nb);
    }

    // Solver::normalizeImaginaryTimePropagation (solver_normalize_imag_time.cu:12-48)
    // for one field: the interior sum (FP64 partials, plus `nb - kNormBlocks`
    // ring partials already in place), the factor on the device, and the
    // whole padded plane scaled by it
    void imag_normalize_device(DevBuf& f, bool complex_field, long long nb) {
        double* pp = reinterpret_cast<double*>(partials.p);
        if (complex_field)
            sum_abs2_kernel<T, true><<<kNormBlocks, 256, 0, stream>>>(reinterpret_cast<const T*>(cplane(f)), pitch, N_r, N_c, pp);
        else
            sum_abs2_kernel<T, false><<<kNormBlocks, 256, 0, stream>>>(rplane(f), pitch, N_r, N_c, pp);
        imag_factor_kernel<T><<<1, 1024, 0, stream>>>(pp, nb, (T)P.imag_time_amplitude, d.dV, reinterpret_cast<T*>(imag_f.p));
        scale_plane_kernel<T><<<kNormBlocks, 256, 0, stream>>>(reinterpret_cast<T*>(f.p), (complex_field ? 2 : 1) * plane,
                                                               reinterpret_cast<const T*>(imag_f.p), (T)0);
        launches += 3;
        PHX_CUDA(cudaGetLastError());
    }
    // adaptive stepping: the accepted attempt's norm is the state's norm
    void imag_normalize_host(DevBuf& f, double norm) {
        T sum = (T)norm;
        if ((double)sum < 1e-10) sum = (T)1.0;
        const T fac = std::sqrt((T)P.imag_time_amplitude / (sum * d.dV));
        scale_plane_kernel<T><<<kNormBlocks, 256, 0, stream>>>(reinterpret_cast<T*>(f.p), 2 * plane, nullptr, fac);
        ++launches;
        PHX_CUDA(cudaGetLastError());
    }

    // ------------------------------------------------------------ adaptive tableaux
    // DP45, BoSha, CashKarp, Fehlberg2/5, DP85, NSRK78 (tableaux in
    // phx_host.hpp): stages 1..S, then either the final sum in place (fixed
    // dt) or the solution sum into a stage plane, an extra stage S + 1 for
    // first-same-as-last tableaux, the error sum and the norm (FP64), and
    // Solver::adaptTimeStep on the host.
    T row_w(int m, int q) const { return (T)(m < tab.S - 1 ? tab.a[m][q] : tab.b[q]); }
    int row_n(int m) const { return m < tab.S - 1 ? tab.nw[m] : tab.nb; }
    int sol_slot() const { return (tab.S - 1) & 1; }
    long long adaptive_stages(bool adaptive, bool ref_norm = false) {
        const int S_ = tab.S;
        for (int s = 1; s <= S_; ++s) {
            StageParams<T> S = base_params(0);
            set_coefficients(S, (T)tab.c[s - 1]);
            const bool final_fixed = !adaptive && s == S_;
            region(S, final_fixed ? 0 : H - s);
            S.stage = s;
            S.nw = row_n(s - 1);
            for (int q = 0; q < S.nw; ++q) S.w[q] = row_w(s - 1, q);
            if (S.nw == 1) S.dtw = dt * S.w[0];
            S.w_sum = right_fold(S.w, S.nw);
            auto wire = [this, s, final_fixed](StageParams<T>& X, int q) {
                X.psi0 = cplane(psi[q]);
                X.n0 = rplane(nres[q]);
                X.psi_in = s == 1 ? cplane(psi[q]) : cplane(sbuf_psi[q][(s - 2) & 1]);
                X.n_in = s == 1 ? rplane(nres[q]) : rplane(sbuf_n[q][(s - 2) & 1]);
                X.k_psi = cplane(k_psi[q]);
                X.k_n = rplane(k_n[q]);
                X.psi_out = final_fixed ? cplane(psi[q]) : cplane(sbuf_psi[q][(s - 1) & 1]);
                X.n_out = final_fixed ? rplane(nres[q]) : rplane(sbuf_n[q][(s - 1) & 1]);
                X.pump = rplane(pump[q]);
                X.pot = rplane(pot[q]);
                X.pulse = cplane(pulse[q]);
            };
            if (final_fixed)
                launch<kStackFinal>(S, wire);
            else
                launch<kStack>(S, wire);
        }
        if (!adaptive) return 0;
        // error (e_1..e_E; k_{S+1} = f(solution) for first-same-as-last tableaux,
        // evaluated but unused otherwise) and the solution's norm over the interior
        StageParams<T> S = base_params(0);
        set_coefficients(S, (T)tab.c[tab.fsal ? S_ : S_ - 1]);
        region(S, 0);
        S.stage = S_ + 1;
        S.nw = tab.E;
        for (int q = 0; q < tab.E; ++q) S.w[q] = (T)tab.e[q];
        S.partials = reinterpret_cast<double*>(partials.p);
        S.error_passes = P.tetm ? 2 : 1;
        const int slot = sol_slot();
        launch<kStackError>(S, [this, slot](StageParams<T>& X, int q) {
            X.psi0 = cplane(psi[q]);
            X.n0 = rplane(nres[q]);
            X.psi_in = cplane(sbuf_psi[q][slot]);
            X.n_in = rplane(sbuf_n[q][slot]);
            X.k_psi = cplane(k_psi[q]);
            X.k_n = rplane(k_n[q]);
            X.pump = rplane(pump[q]);
            X.pot = rplane(pot[q]);
            X.pulse = cplane(pulse[q]);
        });
        long long nb = grid_x(S.c0, S.c1) * grid_y(S.r0, S.r1);
        if (ref_norm) {
            RingParams<T> R;
            std::memset(&R, 0, sizeof(R));
            R.psi0 = cplane(psi[0]);
            R.k = cplane(k_psi[0]);
            R.pitch = pitch;
            R.plane = plane;
            R.N_r = N_r;
            R.N_c = N_c;
            R.periodic_x = P.periodic_x;
            R.periodic_y = P.periodic_y;
            R.H = H;
            R.S = S_;
            R.dt = dt;
            R.dtw1 = dt * row_w(0, 0);
            for (int m = 0; m < S_; ++m) {
                R.nw[m] = row_n(m);
                for (int q = 0; q < R.nw[m]; ++q) R.a[m][q] = row_w(m, q);
            }
            R.E = tab.E;
            for (int q = 0; q < tab.E; ++q) R.e[q] = (T)tab.e[q];
            R.passes = P.tetm ? 2 : 1;
            R.imag = imag_time() ? 1 : 0;
            R.partials = reinterpret_cast<double*>(partials.p) + 2 * nb;
            {
                const StageParams<T> B = base_params(0);
                R.noise = B.noise;
                R.noise_amp = B.noise_amp;
                for (int m = 0; m < S_; ++m) R.w_sum[m] = right_fold(R.a[m], R.nw[m]);
                R.R = B.R;
                R.gamma_c = B.gamma_c;
                R.four_dV = B.four_dV;
                R.noise_scale = B.noise_scale;
                R.n0 = P.use_reservoir ? rplane(nres[0]) : nullptr;
            }
            dp45_ring_kernel<T><<<kRingBlocks, 256, 0, stream>>>(R);
            ++launches;
            PHX_CUDA(cudaGetLastError());
            nb += kRingBlocks;
        }
        return nb;
    }

    bool adapt_time_step(double err_sum, double norm_sum) {
        // Solver::adaptTimeStep (solver.cu:72-105) with the tableau's power
        const T normalization_factor = (T)norm_sum;
        const T integrated_error = (T)err_sum;
        T final_error = std::abs(integrated_error / normalization_factor);
        const T tol = (T)P.tol;
        const T lo = std::numeric_limits<T>::min();
        const T dh_arg = (T)((double)tol / 2.0 / (double)(final_error > lo ? final_error : lo));
        T dh = std::pow(dh_arg, (T)tab.power);  // std::pow<Type::real>(dh_arg, Type::real(power))
        if (std::isnan(dh)) {
            dh = (T)0.9;
            final_error = std::numeric_limits<T>::max();
        }
        if (std::isnan(final_error)) {
            dh = (T)0.9;
            final_error = std::numeric_limits<T>::max();
        }
        const T cand = dt * dh;
        T new_dt = std::min(cand, (T)P.dt_max);
        if (new_dt < (T)P.dt_min) new_dt = (T)P.dt_min;
        dt = new_dt;
        update_kernel_time();
        return final_error < tol;
    }

    // the stage plane `slot` becomes the state (and the state a stage plane);
    // rings along zero axes are zeroed again
    void swap_state_with(int slot) {
        for (int q = 0; q < comps; ++q) {
            std::swap(psi[q].p, sbuf_psi[q][slot].p);
            std::swap(nres[q].p, sbuf_n[q][slot].p);
            if (!(P.periodic_x && P.periodic_y)) {
                ring_fill_kernel<C><<<64, 256, 0, stream>>>(cplane(psi[q]), N_r, N_c, pitch, G, P.periodic_x, P.periodic_y);
                ring_fill_kernel<T><<<64, 256, 0, stream>>>(rplane(nres[q]), N_r, N_c, pitch, G, P.periodic_x, P.periodic_y);
                launches += 2;
                PHX_CUDA(cudaGetLastError());
            }
        }
    }

    // ---- DP45 attempt in one launch (phx_dp45_fused.cuh): scalar, at most one
    // pump and one potential group, no pulse, no noise, real time, real
    // temporal coefficients; PHX_DP45_FUSED=0 selects the stage kernels
    static bool dp45_fused_on() {
        const char* e = std::getenv("PHX_DP45_FUSED");
        return !(e && e[0] == '0');
    }
    bool dp45_fused_eligible() const {
        return P.iterator == PHX_ITER_DP45 && !P.tetm && !(P.stochastic_amplitude > 0.0) && !imag_time() &&
               P.n_pump_groups <= 1 && P.n_potential_groups <= 1 && P.n_pulse_groups == 0 && dp45_fused_on();
    }
    // the fused kernel reads the state over tile + 7: periodic images must be
    // 7 deep, which the stage kernels (4 deep) do not leave behind
    bool state_images_deep = false;
    // the attempt kernel writes its three sums straight into mapped host
    // memory (no device-to-host copy per attempt); -1 unknown, 0 the device
    // cannot map host memory (the sums then go through `result` and a copy)
    MappedBuf dp45_sums;
    int dp45_mapped = -1;
    bool dp45_fused_set = false;
    DevBuf dp45_ticket;  // blocks of a fused attempt that have finished (the last one resets it)
    static constexpr int kDpTW = 32, kDpTH = 16;
    // FP32: 10 warps, two CTAs per SM (two pair slots per thread: the per-stage
    // pair counts spread over fewer idle slots than with 8 warps and three);
    // FP64: one CTA per SM (196 KB of shared memory), 12 warps (210.6 us per
    // accepted step at 1024^2 against 215.5 with 8)
    static constexpr int kDpNT = sizeof(T) == 4 ? 320 : 384;
    // one attempt, which leaves (error, norm, ring 7) in `result`; returns
    // false when this attempt needs the stage kernels (complex temporal
    // coefficients)
    bool dp45_fused_attempt(bool ref_norm) {
        Dp45Params<T> Q;
        std::memset(&Q, 0, sizeof(Q));
        for (int s = 0; s < 7; ++s) {
            if (P.n_pump_groups) {
                const auto c = interp<T>(amp_pump[0], next_pump[0], (T)tab.c[s]);
                if (c.imag() != (T)0) return false;
                Q.pump_c[s] = c.real();
            }
            if (P.n_potential_groups) {
                const auto c = interp<T>(amp_pot[0], next_pot[0], (T)tab.c[s]);
                if (c.imag() != (T)0) return false;
                Q.pot_c[s] = c.real();
            }
        }
        if (!state_images_deep && (P.periodic_x || P.periodic_y)) {
            ring_fill_kernel<C><<<64, 256, 0, stream>>>(cplane(psi[0]), N_r, N_c, pitch, G, P.periodic_x, P.periodic_y);
            launches += 1;
            if (P.use_reservoir) {
                ring_fill_kernel<T><<<64, 256, 0, stream>>>(rplane(nres[0]), N_r, N_c, pitch, G, P.periodic_x,
                                                            P.periodic_y);
                launches += 1;
            }
        }
        const StageParams<T> B = base_params(0);
        Q.N_r = N_r;
        Q.N_c = N_c;
        Q.img_x = P.periodic_x;
        Q.img_y = P.periodic_y;
        Q.pitch = pitch;
        Q.psi0 = cplane(psi[0]);
        Q.n0 = rplane(nres[0]);
        Q.psi1 = cplane(sbuf_psi[0][sol_slot()]);
        Q.n1 = rplane(sbuf_n[0][sol_slot()]);
        Q.pump = P.n_pump_groups ? rplane(pump[0]) : nullptr;
        Q.pot = P.n_potential_groups ? rplane(pot[0]) : nullptr;
        Q.m2 = B.m2, Q.odx2 = B.odx2, Q.ody2 = B.ody2, Q.meff = B.meff, Q.ohb = B.ohb;
        Q.ohb_gc = B.ohb_gc, Q.half_gamma_c = B.half_gamma_c, Q.ohb_gr = B.ohb_gr, Q.half_R = B.half_R;
        Q.gamma_r = B.gamma_r, Q.R = B.R;
        for (int m = 0; m < 6; ++m)
            for (int q = 0; q < row_n(m) && q < 6; ++q) Q.w[m][q] = row_w(m, q);
        Q.dtw1 = dt * row_w(0, 0);
        Q.dt = dt;
        for (int q = 0; q < 7; ++q) Q.e[q] = (T)tab.e[q];
        Q.ring = ref_norm ? 1 : 0;
        const unsigned gx = (unsigned)((N_c + kDpTW - 1) / kDpTW), gy = (unsigned)((N_r + kDpTH - 1) / kDpTH);
        const long long nb = (long long)gx * gy;
        if (partials.bytes < sizeof(double) * 3 * (size_t)nb) partials.alloc(sizeof(double) * 3 * (size_t)nb, stream);
        if (!dp45_ticket.p) dp45_ticket.alloc(sizeof(unsigned), stream);  // zeroed; the kernel leaves it at 0
        Q.partials = reinterpret_cast<double*>(partials.p);
        Q.ticket = static_cast<unsigned*>(dp45_ticket.p);
        if (dp45_mapped < 0) {
            int can = 0;
            PHX_CUDA(cudaDeviceGetAttribute(&can, cudaDevAttrCanMapHostMemory, P.device));
            dp45_mapped = can ? 1 : 0;
            if (dp45_mapped) dp45_sums.alloc(4 * sizeof(double));
        }
        Q.result = dp45_mapped ? static_cast<double*>(dp45_sums.d) : reinterpret_cast<double*>(result.p);
        constexpr int MINB = sizeof(T) == 4 ? 2 : 1;
        using Lay = Dp45Layout<T, kDpTW, kDpTH>;
        auto kern = P.use_reservoir ? dp45_fused_kernel<T, true, kDpTW, kDpTH, kDpNT, MINB>
                                    : dp45_fused_kernel<T, false, kDpTW, kDpTH, kDpNT, MINB>;
        if (!dp45_fused_set) {
            PHX_CUDA(cudaFuncSetAttribute(dp45_fused_kernel<T, true, kDpTW, kDpTH, kDpNT, MINB>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::total));
            PHX_CUDA(cudaFuncSetAttribute(dp45_fused_kernel<T, false, kDpTW, kDpTH, kDpNT, MINB>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::total));
            dp45_fused_set = true;
        }
        cudaEvent_t a = nullptr;
        prof_begin(a);
        kern<<<dim3(gx, gy), kDpNT, Lay::total, stream>>>(Q);
        const double pt = 2.0 * (sizeof(C) + (P.use_reservoir ? sizeof(T) : 0.0)) +
                          sizeof(T) * (P.n_pump_groups + P.n_potential_groups);
        prof_end(PHX_KERNEL_DP45_FUSED, a, pt * (double)N_r * N_c);
        ++launches;
        PHX_CUDA(cudaGetLastError());
        return true;
    }

    void step_adaptive(bool adaptive, int64_t& acc, int64_t& rej) {
        if (tab.inverted) return step_inverted(adaptive, acc, rej);
        if (!adaptive) {
            adaptive_stages(false);
            state_images_deep = false;  // the final stage kernel writes images four deep
            return;
        }
        const bool ref_norm = P.norm_mode == PHX_NORM_REFERENCE;
        bool accept = false, ring7_done = false;
        int rejections = 0;
        do {
            // the fused attempt sums its norms (ring 7 included) in the same launch
            const bool fused_attempt = dp45_fused_eligible() && dp45_fused_attempt(ref_norm);
            if (!fused_attempt) {
                if (ref_norm && !ring7_done) {
                    // outer ring H of the state's halo at the start of this step -> result[2]
                    ring7_kernel<T><<<1, 1024, 0, stream>>>(cplane(psi[0]), pitch, N_r, N_c, P.periodic_x,
                                                            P.periodic_y, H, reinterpret_cast<double*>(result.p) + 2);
                    ++launches;
                    ring7_done = true;
                }
                const long long nb = adaptive_stages(true, ref_norm);
                finalize_pairs_kernel<<<1, 1024, 0, stream>>>(reinterpret_cast<double*>(partials.p), nb,
                                                              reinterpret_cast<double*>(result.p));
                ++launches;
                PHX_CUDA(cudaGetLastError());
            }
            const bool mapped = fused_attempt && dp45_mapped == 1;
            if (!mapped)
                PHX_CUDA(cudaMemcpyAsync(host_result.p, result.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, stream));
            PHX_CUDA(cudaStreamSynchronize(stream));
            const double* r = static_cast<const double*>(mapped ? dp45_sums.p : host_result.p);
            double err = r[0], nrm = r[1];
            if (ref_norm) {
                // the reference's buffer still holds, in its outermost halo ring,
                // the state of the previous accepted step (zero before the first)
                nrm += r7_prev;
                r7_cur = r[2];
            }
            accept = adapt_time_step(err, nrm);
            // a non-finite error norm is rejected with dt * 0.9 (solver.cu:90-97);
            // once dt is at dt_min no smaller step is left to try
            if (!accept && !(std::isfinite(err) && std::isfinite(nrm)) && dt <= (T)P.dt_min)
                fail(PHX_ERR_NONFINITE, "the adaptive error norm is not finite at the smallest step size dt_min "
                                        "(NaN or Inf in the state)");
            if (accept) {
                swap_state_with(sol_slot());
                state_images_deep = fused_attempt;
                r7_prev = r7_cur;
                imag_nrm = nrm;
                ++acc;
            } else {
                ++rej;
                if (++rejections > kMaxRejections)
                    fail(PHX_ERR_NONFINITE, "step size control rejected " + std::to_string(kMaxRejections) +
                                                " attempts in a row (non-finite error norm?)");
            }
        } while (!accept);
    }
    static constexpr int kMaxRejections = 100000;

    // DormandPrince85::step as the reference has it (dormand_prince.cu:182-190):
    // its fixed and variable branches are swapped.  Fixed dt: the solution goes
    // to the buffer and is dropped, the state stays as it is.  Variable dt: the
    // final sum is added to the state in place and no error is formed (the
    // error array keeps its zeros), so adaptTimeStep accepts with dt -> dt_max
    // unless the buffer's norm is zero or not finite, and the swap makes the
    // buffer -- the stage-12 input -- the state.
    void step_inverted(bool adaptive, int64_t& acc, int64_t& rej) {
        if (!adaptive) return;
        int rejections = 0;
        for (;;) {
            // stages 1 .. S-1 leave Y_S in a stage plane (k_S and the in-place sum
            // end up in the plane the swap hands back to the buffer)
            const int S_ = tab.S;
            for (int s = 1; s < S_; ++s) {
                StageParams<T> S = base_params(0);
                set_coefficients(S, (T)tab.c[s - 1]);
                region(S, H - s);
                S.stage = s;
                S.nw = row_n(s - 1);
                for (int q = 0; q < S.nw; ++q) S.w[q] = row_w(s - 1, q);
                if (S.nw == 1) S.dtw = dt * S.w[0];
                S.w_sum = right_fold(S.w, S.nw);
                launch<kStack>(S, [this, s](StageParams<T>& X, int q) {
                    X.psi0 = cplane(psi[q]);
                    X.n0 = rplane(nres[q]);
                    X.psi_in = s == 1 ? cplane(psi[q]) : cplane(sbuf_psi[q][(s - 2) & 1]);
                    X.n_in = s == 1 ? rplane(nres[q]) : rplane(sbuf_n[q][(s - 2) & 1]);
                    X.k_psi = cplane(k_psi[q]);
                    X.k_n = rplane(k_n[q]);
                    X.psi_out = cplane(sbuf_psi[q][(s - 1) & 1]);
                    X.n_out = rplane(sbuf_n[q][(s - 1) & 1]);
                    X.pump = rplane(pump[q]);
                    X.pot = rplane(pot[q]);
                    X.pulse = cplane(pulse[q]);
                });
            }
            const int slot = (S_ - 2) & 1;
            // normalization_factor = sum |buffer|^2; integrated_error = 0
            FieldRef f{&sbuf_psi[0][slot], true, 0, 0};
            const double nrm = plane_norm(f);
            const bool ok = adapt_time_step(0.0, nrm);
            if (ok) {
                swap_state_with(slot);
                ++acc;
                return;
            }
            ++rej;
            if (++rejections > kMaxRejections) fail(PHX_ERR_NONFINITE, "DP85 buffer norm is zero or not finite");
        }
    }
    double plane_norm(const FieldRef& f) {
        const int blocks = 296;
        sum_abs2_kernel<T, true><<<blocks, 256, 0, stream>>>(reinterpret_cast<const T*>(cplane(*f.buf)), pitch, N_r, N_c,
                                                             reinterpret_cast<double*>(partials.p));
        finalize_pairs_kernel<<<1, 1024, 0, stream>>>(reinterpret_cast<double*>(partials.p), blocks,
                                                      reinterpret_cast<double*>(result.p));
        launches += 2;
        PHX_CUDA(cudaGetLastError());
        PHX_CUDA(cudaMemcpyAsync(host_result.p, result.p, sizeof(double), cudaMemcpyDeviceToHost, stream));
        PHX_CUDA(cudaStreamSynchronize(stream));
        return static_cast<const double*>(host_result.p)[0];
    }

    // ------------------------------------------------------------ SSFM
    // SSFM::step (split_step_fourier_method.cu:24-72): four unnormalised
    // transforms per iteration on contiguous copies of psi, with the
    // reference's (N_c, N_r) plan; kernels in phx_ssfm.cuh.
    DevBuf ssfm_w[2], ssfm_f[2];
    cufftHandle ssfm_plan = 0;
    bool have_ssfm_plan = false;
    void ssfm_fft(C* in, C* out, int dir) {
        if constexpr (sizeof(T) == 4) {
            PHX_CUFFT(cufftExecC2C(ssfm_plan, reinterpret_cast<cufftComplex*>(in), reinterpret_cast<cufftComplex*>(out), dir));
        } else {
            PHX_CUFFT(cufftExecZ2Z(ssfm_plan, reinterpret_cast<cufftDoubleComplex*>(in), reinterpret_cast<cufftDoubleComplex*>(out),
                                   dir));
        }
    }
    void step_ssfm() {
        const long long N = (long long)N_r * N_c;
        if (!have_ssfm_plan) {
            for (int q = 0; q < comps; ++q) {
                ssfm_w[q].alloc(sizeof(C) * N, stream);
                ssfm_f[q].alloc(sizeof(C) * N, stream);
            }
            PHX_CUFFT(cufftPlan2d(&ssfm_plan, N_c, N_r, sizeof(T) == 4 ? CUFFT_C2C : CUFFT_Z2Z));
            PHX_CUFFT(cufftSetStream(ssfm_plan, stream));
            have_ssfm_plan = true;
        }
        SsfmParams<T> S;
        std::memset(&S, 0, sizeof(S));
        S.N_r = N_r, S.N_c = N_c, S.pitch = pitch, S.tetm = P.tetm, S.res = P.use_reservoir;
        S.hbs = (T)P.h_bar_s, S.meff = (T)P.m_eff, S.Lx = (T)P.L_x, S.Ly = (T)P.L_y, S.dt = dt, S.N2 = (T)(unsigned)N;
        S.g_c = (T)P.g_c, S.g_r = (T)P.g_r, S.R = (T)P.R, S.gamma_c = (T)P.gamma_c, S.gamma_r = (T)P.gamma_r;
        S.g_pm = (T)P.g_pm, S.ohb = d.ohb, S.dV = d.dV;
        S.n_pump = P.n_pump_groups, S.n_pot = P.n_potential_groups, S.n_pulse = P.n_pulse_groups;
        S.plane = plane;
        for (int q = 0; q < comps; ++q) {
            S.pump[q] = rplane(pump[q]);
            S.pot[q] = rplane(pot[q]);
            S.pulse[q] = cplane(pulse[q]);
        }
        // the envelopes' amplitudes at t (amp, not interpolated)
        for (int g = 0; g < P.n_pump_groups; ++g) S.amp_pump[g] = mk_host(amp_pump[g]);
        for (int g = 0; g < P.n_potential_groups; ++g) S.amp_pot[g] = mk_host(amp_pot[g]);
        for (int g = 0; g < P.n_pulse_groups; ++g) S.amp_pulse[g] = mk_host(amp_pulse[g]);
        const StageParams<T> B = base_params(0);
        S.noise = B.noise;
        S.noise_amp = B.noise_amp;
        S.periodic_x = P.periodic_x, S.periodic_y = P.periodic_y;
        const int blocks = (int)std::min<long long>((N + 255) / 256, 148 * 16);
        C* w[2] = {reinterpret_cast<C*>(ssfm_w[0].p), comps > 1 ? reinterpret_cast<C*>(ssfm_w[1].p) : nullptr};
        C* f[2] = {reinterpret_cast<C*>(ssfm_f[0].p), comps > 1 ? reinterpret_cast<C*>(ssfm_f[1].p) : nullptr};
        cudaEvent_t a = nullptr;
        prof_begin(a);
        for (int q = 0; q < comps; ++q)
            gather_interior_kernel<T><<<blocks, 256, 0, stream>>>(cplane(psi[q]), pitch, N_r, N_c, w[q]);
        for (int half = 0; half < 2; ++half) {
            for (int q = 0; q < comps; ++q) {
                ssfm_fft(w[q], f[q], CUFFT_FORWARD);
                ssfm_linear_kernel<T><<<blocks, 256, 0, stream>>>(S, f[q], w[q]);
                ssfm_fft(w[q], f[q], CUFFT_INVERSE);
            }
            if (half == 1) break;
            T* rvm = comps > 1 ? rplane(nres[1]) : nullptr;
            T* brvm = comps > 1 ? rplane(sbuf_n[1][0]) : nullptr;
            ssfm_nonlinear_kernel<T><<<blocks, 256, 0, stream>>>(S, f[0], f[1], rplane(nres[0]), rvm, w[0], w[1],
                                                                 rplane(sbuf_n[0][0]), brvm);
        }
        ssfm_independent_kernel<T><<<blocks, 256, 0, stream>>>(S, f[0], f[1], rplane(nres[0]), rplane(sbuf_n[0][0]),
                                                               comps > 1 ? rplane(sbuf_n[1][0]) : nullptr, cplane(psi[0]),
                                                               comps > 1 ? cplane(psi[1]) : nullptr);
        prof_end(PHX_KERNEL_OTHER, a, (double)N * comps * 16 * sizeof(C));
        launches += comps * 3 + 2;
        PHX_CUDA(cudaGetLastError());
    }

    // ------------------------------------------------------------ FFT filter
    void fft_filter() {
        state_images_deep = false;  // the scatter path writes images four deep
        for (int q = 0; q < comps; ++q) {
            if (!have_mask[q] && !keep_spectrum) continue;
            const long long N = (long long)N_r * N_c;
            const int blocks = (int)std::min<long long>((N + 255) / 256, 148 * 16);
            cudaEvent_t a = nullptr;
            prof_begin(a);
            if (keep_spectrum) {
                // applyFFTFilter with its fft_plus buffer kept: transform, mask / N
                // where a mask is set, keep, and back only where it was masked
                ensure_fft();
                gather_interior_kernel<T><<<blocks, 256, 0, stream>>>(cplane(psi[q]), pitch, N_r, N_c, reinterpret_cast<C*>(fft_x.p));
                exec_fft(CUFFT_FORWARD);
                if (have_mask[q])
                    mask_kernel<T><<<blocks, 256, 0, stream>>>(reinterpret_cast<C*>(fft_x.p), reinterpret_cast<const T*>(mask[q].p), N);
                PHX_CUDA(cudaMemcpyAsync(spectrum[q].p, fft_x.p, sizeof(C) * (size_t)N, cudaMemcpyDeviceToDevice, stream));
                launches += have_mask[q] ? 2 : 1;
                if (have_mask[q]) {
                    exec_fft(CUFFT_INVERSE);
                    scatter_interior_kernel<T><<<blocks, 256, 0, stream>>>(reinterpret_cast<C*>(fft_x.p), cplane(psi[q]), pitch, N_r,
                                                                           N_c, P.periodic_x, P.periodic_y);
                    ++launches;
                }
                prof_end(PHX_KERNEL_FILTER, a, (double)N * (6 * sizeof(C) + sizeof(T)));
                PHX_CUDA(cudaGetLastError());
                continue;
            }
            if (fft_in_place) {
                // applyFFTFilter on the padded plane itself: FFT, (data / N) * mask,
                // inverse FFT, then the ring's images / zeros again
                C* base = cplane(psi[q]);
                exec_fft_on(base, CUFFT_FORWARD);
                mask_padded_kernel<T><<<blocks, 256, 0, stream>>>(base, pitch, N_r, N_c, reinterpret_cast<const T*>(mask[q].p));
                exec_fft_on(base, CUFFT_INVERSE);
                ring_fill_kernel<C><<<64, 256, 0, stream>>>(base, N_r, N_c, pitch, G, P.periodic_x, P.periodic_y);
                prof_end(PHX_KERNEL_FILTER, a, (double)N * (4 * sizeof(C) + sizeof(T)));
                launches += 2;
                PHX_CUDA(cudaGetLastError());
                continue;
            }
            gather_interior_kernel<T><<<blocks, 256, 0, stream>>>(cplane(psi[q]), pitch, N_r, N_c, reinterpret_cast<C*>(fft_x.p));
            exec_fft(CUFFT_FORWARD);
            mask_kernel<T><<<blocks, 256, 0, stream>>>(reinterpret_cast<C*>(fft_x.p), reinterpret_cast<const T*>(mask[q].p), N);
            exec_fft(CUFFT_INVERSE);
            scatter_interior_kernel<T><<<blocks, 256, 0, stream>>>(reinterpret_cast<C*>(fft_x.p), cplane(psi[q]), pitch, N_r, N_c,
                                                                   P.periodic_x, P.periodic_y);
            prof_end(PHX_KERNEL_FILTER, a, (double)N * (6 * sizeof(C) + sizeof(T)));
            launches += 3;
            PHX_CUDA(cudaGetLastError());
        }
    }
    void exec_fft_on(C* data, int dir) {
        if constexpr (sizeof(T) == 4) {
            PHX_CUFFT(cufftExecC2C(plan, reinterpret_cast<cufftComplex*>(data), reinterpret_cast<cufftComplex*>(data), dir));
        } else {
            PHX_CUFFT(cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(data), reinterpret_cast<cufftDoubleComplex*>(data),
                                   dir));
        }
    }
    void exec_fft(int dir) {
        if constexpr (sizeof(T) == 4) {
            PHX_CUFFT(cufftExecC2C(plan, reinterpret_cast<cufftComplex*>(fft_x.p), reinterpret_cast<cufftComplex*>(fft_x.p), dir));
        } else {
            PHX_CUFFT(cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(fft_x.p),
                                   reinterpret_cast<cufftDoubleComplex*>(fft_x.p), dir));
        }
    }

    // ------------------------------------------------------------ iterate
    void step(int64_t max_iterations, phx_step_info* info) override {
        const int64_t l0 = launches;
        int64_t its = 0, acc = 0, rej = 0, filt = 0;
        const T t_max = (T)P.t_max, fft_every = (T)P.fft_every;
        bool aborted = false;
        while (its < max_iterations) {
            if (t >= t_max) break;
            if (abort_requested.exchange(0)) {
                aborted = true;
                break;
            }
            if (P.stochastic_amplitude > 0.0) noise_amp = (T)P.stochastic_amplitude * std::sqrt(dt);
            update_kernel_time();
            t = t + dt;
            cudaEvent_t ta = nullptr, tb = nullptr;
            if (shape < 0) {
                ta = get_event();
                PHX_CUDA(cudaEventRecord(ta, stream));
            }
            if (P.iterator == PHX_ITER_RK4 && !imag_time()) {
                step_rk4();
            } else if (P.iterator == PHX_ITER_SSFM) {
                step_ssfm();
            } else if (tab.adaptive && !(imag_time() && !adaptive_now())) {
                step_adaptive(adaptive_now(), acc, rej);
            } else {
                step_tableau();  // imaginary time: normalised inside
            }
            if (imag_time()) {
                if (P.iterator == PHX_ITER_SSFM) {
                    // halo 0: the sums run over the grid points
                    for (int q = 0; q < comps; ++q) {
                        imag_normalize_device(psi[q], true, kNormBlocks);
                        if (P.use_reservoir) imag_normalize_device(nres[q], false, kNormBlocks);
                    }
                } else if (tab.adaptive && adaptive_now()) {
                    imag_normalize_host(psi[0], imag_nrm);
                }
            }
            if (shape < 0) tune_record(ta, tb);
            ++its;
            ++noise_iteration;
            if (t - fft_cached_t < fft_every) continue;
            fft_cached_t = t;
            if (have_mask[0] || have_mask[1] || keep_spectrum) {
                fft_filter();
                if (have_mask[0] || have_mask[1]) ++filt;
            }
        }
        // RK4 work stays queued on the stream (no host sync); DP45 synchronised
        // on every attempt already.  Reads of fields synchronise.
        PHX_CUDA(cudaGetLastError());
        if (info) {
            info->t = (double)t;
            info->dt = (double)dt;
            info->iterations = its;
            info->accepted = acc;
            info->rejected = rej;
            info->fft_filters = filt;
            info->kernel_launches = launches - l0;
            info->launch_shape = shape;
            info->reserved = 0;
        }
        if (aborted)
            fail(PHX_ERR_ABORTED, "stopped by phx_request_abort after " + std::to_string(its) +
                                      " iterations; the state is that of the last completed iteration");
    }

    // Launch-shape autotuning: the first kTuneRounds x kTuneIters x
    // (candidates) iterations of a handle run the candidate shapes round-robin,
    // kTuneIters consecutive iterations per candidate and round (results do not
    // depend on the shape: every point is computed by the same operations).
    // The first round warms up; each later round gives one sample per shape
    // (the summed device time of its iterations), and the median sample ranks
    // the shapes.  The incumbent shape is kept unless the fastest median beats
    // it by more than kTuneMargin, so that boxes whose timings differ by noise
    // pick the same shape.  The kept shape is remembered for the process:
    // a later handle of the same configuration (grid, precision, boundaries,
    // inputs, iterator, device) starts with it.  PHX_TUNE_CACHE=0 turns the
    // memory off.
    static bool tune_cache_on() {
        const char* e = std::getenv("PHX_TUNE_CACHE");
        return !(e && e[0] == '0');
    }
    using TuneKey = std::array<long long, 14>;
    static std::map<TuneKey, int>& tune_cache() {
        static std::map<TuneKey, int> m;
        return m;
    }
    static std::mutex& tune_cache_mu() {
        static std::mutex mu;
        return mu;
    }
    TuneKey tune_key() const {
        return {(long long)sizeof(T), N_r, N_c, P.use_reservoir, P.n_pump_groups, P.n_potential_groups,
                P.n_pulse_groups, P.periodic_x, P.periodic_y, P.iterator, P.tetm, P.device,
                (long long)(P.stochastic_amplitude > 0.0), (long long)imag_time()};
    }
    void tune_record(cudaEvent_t ta, cudaEvent_t tb) {
        tb = get_event();
        PHX_CUDA(cudaEventRecord(tb, stream));
        tune_ev[(tune_step / kTuneIters) % n_candidates()].push_back({ta, tb});
        ++tune_step;
        if (tune_step < kTuneRounds * kTuneIters * n_candidates()) return;
        PHX_CUDA(cudaStreamSynchronize(stream));
        double best = 1e300;
        int best_sh = incumbent();
        double inc_ms = 1e300;
        tune_medians.clear();
        for (int sh = 0; sh < n_candidates(); ++sh) {
            std::vector<double> samples;
            for (int r = 1; r < kTuneRounds; ++r) {
                double sum = 0.0;
                for (int i = 0; i < kTuneIters; ++i) {
                    const auto& pr = tune_ev[sh][(size_t)(r * kTuneIters + i)];
                    float m = 0.f;
                    PHX_CUDA(cudaEventElapsedTime(&m, pr.first, pr.second));
                    sum += m;
                }
                samples.push_back(sum / kTuneIters);
            }
            std::sort(samples.begin(), samples.end());
            const double med = samples[samples.size() / 2];
            tune_medians.push_back({first_candidate() + sh, med * 1e3});
            if (med < best) best = med, best_sh = first_candidate() + sh;
            if (first_candidate() + sh == incumbent()) inc_ms = med;
            for (auto& pr : tune_ev[sh]) {
                event_pool.push_back(pr.first);
                event_pool.push_back(pr.second);
            }
            tune_ev[sh].clear();
        }
        if (inc_ms <= best * (1.0 + kTuneMargin)) best_sh = incumbent();
        shape = best_sh;
        if (tune_cache_on()) {
            std::lock_guard<std::mutex> lk(tune_cache_mu());
            tune_cache()[tune_key()] = shape;
        }
    }

    // ------------------------------------------------------------ device-pointer field I/O
    // A contiguous N_r x N_c array in device memory, in the build precision
    // (complex fields interleaved), copied on the handle's stream; uploads
    // rebuild the plane's ring.
    void field_device(int field, int group, void* dev, int64_t count, bool upload) override {
        if (!dev) fail(PHX_ERR_INVALID_ARG, "device pointer is NULL");
        if (field == PHX_FFT_MASK_PLUS || field == PHX_FFT_MASK_MINUS) fail(PHX_ERR_UNSUPPORTED, "mask fields are host-only");
        FieldRef f = field_ref(field, group);
        const long long N = (long long)N_r * N_c;
        if (count != (f.complex ? 2 * N : N)) fail(PHX_ERR_INVALID_ARG, "count does not match the field");
        if (!upload) check_err_flag();
        const size_t esz = f.complex ? sizeof(C) : sizeof(T);
        char* base = reinterpret_cast<char*>(f.buf->p) + esz * (G * pitch + G + (long long)f.plane_index * plane);
        if (upload) {
            PHX_CUDA(cudaMemcpy2DAsync(base, esz * pitch, dev, esz * N_c, esz * N_c, N_r, cudaMemcpyDeviceToDevice, stream));
            if (f.complex)
                ring_fill_kernel<C><<<64, 256, 0, stream>>>(reinterpret_cast<C*>(base), N_r, N_c, pitch, G, P.periodic_x,
                                                            P.periodic_y);
            else
                ring_fill_kernel<T><<<64, 256, 0, stream>>>(reinterpret_cast<T*>(base), N_r, N_c, pitch, G, P.periodic_x,
                                                            P.periodic_y);
            PHX_CUDA(cudaGetLastError());
        } else {
            PHX_CUDA(cudaMemcpy2DAsync(dev, esz * N_c, base, esz * pitch, esz * N_c, N_r, cudaMemcpyDeviceToDevice, stream));
        }
    }

    // ------------------------------------------------------------ adjoint
    // Forward with checkpoints every `every` iterations, then reverse sweeps
    // segment by segment: recompute the segment's states and stage values
    // Y2..Y4 with the stage kernels (bit-identical to the forward), then run
    // the four vector-Jacobian stage kernels of phx_adjoint.cuh per
    // iteration, last to first.
    std::vector<std::unique_ptr<DevBuf>> ck_psi, ck_n;    // checkpoints (state planes)
    std::vector<std::unique_ptr<DevBuf>> sg_psi, sg_n;    // states of one segment
    std::vector<std::unique_ptr<DevBuf>> st_psi, st_n;    // Y2..Y4 of every iteration of a segment
    std::vector<std::unique_ptr<DevBuf>> sg_psi2, sg_n2, st_psi2, st_n2;  // the second set (overlapped recompute)
    DevBuf lam_psi[2], lam_n[2], yb_psi[2], yb_n[2], la_psi, la_n, pbar, vbar;
    int64_t adj_T = 0, adj_every = 0;
    T adj_dt = 0;
    bool adj_ready = false;
    // one fused launch per iteration (adj_fused_kernel); PHX_ADJOINT_STAGES=1
    // selects the four-launch path (adj_stage_kernel)
    bool adj_fused = !(std::getenv("PHX_ADJOINT_STAGES") && std::atoi(std::getenv("PHX_ADJOINT_STAGES")) == 1);
    bool adj_recompute_tma =
        !(std::getenv("PHX_ADJOINT_RECOMPUTE") && std::string(std::getenv("PHX_ADJOINT_RECOMPUTE")) == "fused");

    void adjoint_check() {
        if (P.iterator != PHX_ITER_RK4 || P.tetm) fail(PHX_ERR_UNSUPPORTED, "the adjoint covers scalar fixed-step RK4");
        if (!P.periodic_x || !P.periodic_y) fail(PHX_ERR_UNSUPPORTED, "the adjoint needs periodic boundaries on both axes");
        if (P.stochastic_amplitude > 0.0) fail(PHX_ERR_UNSUPPORTED, "the adjoint of a noisy run is not defined here");
        if (imag_time()) fail(PHX_ERR_UNSUPPORTED, "the adjoint covers real-time RK4");
        if (have_mask[0] || have_mask[1]) fail(PHX_ERR_UNSUPPORTED, "the adjoint does not cover the k-space filter");
        if (P.n_pump_groups > 1 || P.n_potential_groups > 1 || P.n_pulse_groups != 0)
            fail(PHX_ERR_UNSUPPORTED, "the adjoint takes at most one pump and one potential group and no pulse");
        for (int g = 0; g < P.n_pump_groups; ++g)
            if (pump_t[g].kind != PHX_TEMPORAL_CONSTANT) fail(PHX_ERR_UNSUPPORTED, "the adjoint needs constant envelopes");
        for (int g = 0; g < P.n_potential_groups; ++g)
            if (pot_t[g].kind != PHX_TEMPORAL_CONSTANT) fail(PHX_ERR_UNSUPPORTED, "the adjoint needs constant envelopes");
    }
    void plane_copy(DevBuf& dst, const DevBuf& src) {
        PHX_CUDA(cudaMemcpyAsync(dst.p, src.p, src.bytes, cudaMemcpyDeviceToDevice, stream));
    }
    void ensure_planes(std::vector<std::unique_ptr<DevBuf>>& v, size_t n, size_t bytes) {
        while (v.size() < n) {
            v.emplace_back(new DevBuf());
            v.back()->alloc(bytes, stream);
        }
    }
    void adjoint_forward(int64_t iterations, int64_t every) override {
        adjoint_check();
        if (iterations < 1) fail(PHX_ERR_INVALID_ARG, "iterations must be >= 1");
        if (every <= 0) every = (int64_t)std::ceil(std::sqrt((double)iterations));
        if (every > iterations) every = iterations;
        const int64_t nck = (iterations + every - 1) / every;
        const size_t cb = sizeof(C) * plane, rb = sizeof(T) * plane;
        ensure_planes(ck_psi, (size_t)nck, cb);
        if (P.use_reservoir) ensure_planes(ck_n, (size_t)nck, rb);
        adj_ready = false;
        for (int64_t k = 0; k < nck; ++k) {
            plane_copy(*ck_psi[k], psi[0]);
            if (P.use_reservoir) plane_copy(*ck_n[k], nres[0]);
            const int64_t len = std::min(every, iterations - k * every);
            phx_step_info info{};
            step(len, &info);
            if (info.iterations != len) fail(PHX_ERR_STATE, "t_max was reached inside the adjoint's forward run");
        }
        adj_T = iterations;
        adj_every = every;
        adj_dt = dt;
        adj_ready = true;
    }
    // one RK4 iteration with the stage kernels: state (yp, yn) -> (op, on),
    // stage values Y2..Y4 into (sp[0..2], sn[0..2])
    void rk4_recompute(DevBuf& yp, DevBuf* yn, DevBuf* sp[3], DevBuf* sn[3], DevBuf& op, DevBuf* on) {
        const T cw[4] = {(T)0.0, (T)0.5, (T)0.5, (T)1.0};
        const T aw[3] = {(T)0.5, (T)0.5, (T)1.0};
        const T bw[4] = {(T)(1.0 / 6.0), (T)(1.0 / 3.0), (T)(1.0 / 3.0), (T)(1.0 / 6.0)};
        for (int s = 1; s <= 4; ++s) {
            StageParams<T> S = base_params(0);
            set_coefficients(S, cw[s - 1]);
            region(S, 4 - s);
            S.stage = s;
            S.b = bw[s - 1];
            if (s < 4) S.dtw = dt * aw[s - 1];
            auto wire = [&, s](StageParams<T>& X, int) {
                X.psi0 = cplane(yp);
                X.n0 = yn ? rplane(*yn) : nullptr;
                X.psi_in = s == 1 ? cplane(yp) : cplane(*sp[s - 2]);
                X.n_in = s == 1 ? (yn ? rplane(*yn) : nullptr) : (sn[s - 2] ? rplane(*sn[s - 2]) : nullptr);
                X.psi_out = s == 4 ? cplane(op) : cplane(*sp[s - 1]);
                X.n_out = s == 4 ? (on ? rplane(*on) : nullptr) : (sn[s - 1] ? rplane(*sn[s - 1]) : nullptr);
                X.acc_psi = cplane(acc_psi[0]);
                X.acc_n = rplane(acc_n[0]);
                X.pump = rplane(pump[0]);
                X.pot = rplane(pot[0]);
                X.pulse = cplane(pulse[0]);
            };
            if (s == 1)
                launch<kRk4First>(S, wire);
            else if (s < 4)
                launch<kRk4Mid>(S, wire);
            else
                launch<kRk4Last>(S, wire);
        }
    }
    // storing variants of the non-TMA one-kernel shapes (go_fused's cases 0-3);
    // false when the tuned shape is not one of them
    template <bool RES, int TW, int TH, int NT>
    void go_fused_shape_store(const FusedParams<T>& F) {
        dim3 grid((unsigned)((N_c + TW - 1) / TW), (unsigned)((N_r + TH - 1) / TH));
        rk4_fused_kernel<T, RES, TW, TH, NT, true><<<grid, NT, 0, stream>>>(F);
    }
    template <bool RES>
    bool go_fused_store_tuned(const FusedParams<T>& F) {
        constexpr bool f32 = sizeof(T) == 4;
        if (!is_fused(cur_shape())) return false;
        switch (cur_shape() - kFusedShape) {
            case 0: go_fused_shape_store<RES, 32, f32 ? 32 : 16, 256>(F); return true;
            case 1: go_fused_shape_store<RES, 64, f32 ? 16 : 8, 256>(F); return true;
            case 2: go_fused_shape_store<RES, 32, f32 ? 16 : 8, 128>(F); return true;
            case 3:
                if constexpr (f32)
                    go_fused_shape_store<RES, 64, 32, 512>(F);
                else
                    go_fused_shape_store<RES, 32, 24, 384>(F);
                return true;
            default: return false;
        }
    }
    // The recompute's TMA iteration: the state planes change from one
    // iteration to the next; the launch's parameters carry their tensor maps.
    // (plane address, complex, box width, box height) -> encoded map
    std::map<std::tuple<const void*, bool, int, int>, CUtensorMap> store_maps;
    template <bool RES, int TW, int TH, int NT, int MINB>
    void go_tma_store(const FusedParams<T>& F, DevBuf& yp, DevBuf* yn) {
        using Lay = TmaLayout<T, TW, TH>;
        auto kern = rk4_tma_kernel<T, RES, TW, TH, NT, MINB, true>;
        int& blocks_per_sm = tma_blocks[reinterpret_cast<const void*>(kern)];
        if (!blocks_per_sm) {
            PHX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::total));
            PHX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, NT, Lay::total));
            if (blocks_per_sm < 1) fail(PHX_ERR_UNSUPPORTED, "TMA iteration kernel does not fit on an SM");
        }
        if (!err_flag.p) err_flag.alloc(sizeof(int), stream);
        if (!sm_count) PHX_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, P.device));
        // a map depends on the plane's address, on whether it is complex and
        // on the box (the tile shape); pitch and rows are fixed for the handle
        auto map_of = [&](const void* base, bool complex, int box_h) -> const CUtensorMap& {
            const auto key = std::make_tuple(base, complex, TW + 8, box_h);
            auto it = store_maps.find(key);
            if (it == store_maps.end()) {
                CUtensorMap m;
                tensor_map(&m, const_cast<void*>(base), complex, TW + 8, box_h);
                it = store_maps.emplace(key, m).first;
            }
            return it->second;
        };
        TmaParams<T> Q;
        std::memset(&Q, 0, sizeof(Q));
        Q.f = F;
        Q.psi_map = map_of(yp.p, true, TH + 8);
        if (RES) Q.n_map = map_of(yn->p, false, TH + 6);
        if (F.pump) Q.pump_map = map_of(pump[0].p, false, TH + 6);
        if (F.pot) Q.pot_map = map_of(pot[0].p, false, TH + 6);
        Q.has_pump = F.pump != nullptr;
        Q.has_pot = F.pot != nullptr;
        Q.tiles_x = (N_c + TW - 1) / TW;
        Q.n_tiles = Q.tiles_x * ((N_r + TH - 1) / TH);
        Q.err = static_cast<int*>(err_flag.p);
        Q.wait_polls = wait_polls;
        const int blocks = std::min(Q.n_tiles, blocks_per_sm * sm_count);
        // the backward's recomputes run on a second stream beside the
        // vector-Jacobian sweep: launched plainly, no CTA waits resident for a
        // predecessor while the other stream could use its slot
        kern<<<blocks, NT, Lay::total, stream>>>(Q);
    }
    // the same in one launch: the fused iteration kernel that also stores the
    // stage values (bit-identical to the stage kernels); the TMA-fed iteration
    // by default, rk4_fused_kernel with PHX_ADJOINT_RECOMPUTE=fused
    void rk4_recompute_fused(DevBuf& yp, DevBuf* yn, DevBuf* sp[3], DevBuf* sn[3], DevBuf& op, DevBuf* on) {
        const T cw[4] = {(T)0.0, (T)0.5, (T)0.5, (T)1.0};
        FusedParams<T> F;
        std::memset(&F, 0, sizeof(F));
        for (int s = 0; s < 4; ++s) {
            if (P.n_pump_groups) F.pump_c[s] = interp<T>(amp_pump[0], next_pump[0], cw[s]).real();
            if (P.n_potential_groups) F.pot_c[s] = interp<T>(amp_pot[0], next_pot[0], cw[s]).real();
        }
        fused_constants<T>(F, P, d, dt, pitch);
        F.psi0 = cplane(yp);
        F.n0 = yn ? rplane(*yn) : nullptr;
        F.psi1 = cplane(op);
        F.n1 = on ? rplane(*on) : nullptr;
        F.pump = P.n_pump_groups ? rplane(pump[0]) : nullptr;
        F.pot = P.n_potential_groups ? rplane(pot[0]) : nullptr;
        for (int s = 0; s < 3; ++s) {
            F.st_psi[s] = cplane(*sp[s]);
            F.st_n[s] = sn[s] ? rplane(*sn[s]) : nullptr;
        }
        cudaEvent_t a = nullptr;
        prof_begin(a);
        if (adj_recompute_tma) {
            // the forward's tuned one-kernel shape when it is a non-TMA one (small
            // grids, where the TMA kernel's few large CTAs leave SMs idle);
            // otherwise the TMA iteration -- FP32: 64 x 16 tiles, 12 warps, two
            // CTAs per SM; FP64: 64 x 16 tiles, 24 warps, one CTA per SM (no
            // register spills)
            const bool done = P.use_reservoir ? go_fused_store_tuned<true>(F) : go_fused_store_tuned<false>(F);
            constexpr int NT = sizeof(T) == 4 ? 384 : 768, MINB = sizeof(T) == 4 ? 2 : 1;
            if (!done && P.use_reservoir)
                go_tma_store<true, 64, 16, NT, MINB>(F, yp, yn);
            else if (!done)
                go_tma_store<false, 64, 16, NT, MINB>(F, yp, yn);
        } else {
            constexpr int TW = 32, TH = sizeof(T) == 4 ? 32 : 16;
            dim3 grid((unsigned)((N_c + TW - 1) / TW), (unsigned)((N_r + TH - 1) / TH));
            if (P.use_reservoir)
                rk4_fused_kernel<T, true, TW, TH, 256, true><<<grid, 256, 0, stream>>>(F);
            else
                rk4_fused_kernel<T, false, TW, TH, 256, true><<<grid, 256, 0, stream>>>(F);
        }
        const double st = sizeof(C) + (P.use_reservoir ? sizeof(T) : 0);
        prof_end(PHX_KERNEL_RK4_FUSED, a, (double)N_r * N_c * (5 * st + (P.n_pump_groups ? sizeof(T) : 0)));
        ++launches;
        PHX_CUDA(cudaGetLastError());
    }
    void adjoint_backward(const void* dpsi, const void* dn, void* dpsi0, void* dn0, void* dpump, void* dpot) override {
        if (!adj_ready) fail(PHX_ERR_STATE, "phx_adjoint_forward must run first");
        if (!dpsi) fail(PHX_ERR_INVALID_ARG, "dL/dpsi_T is NULL");
        adjoint_check();
        const bool res = P.use_reservoir != 0;
        const size_t cb = sizeof(C) * plane, rb = sizeof(T) * plane;
        const int64_t every = adj_every, nck = (adj_T + every - 1) / every;
        ensure_planes(sg_psi, (size_t)every + 1, cb);
        ensure_planes(st_psi, (size_t)(3 * every), cb);
        if (res) {
            ensure_planes(sg_n, (size_t)every + 1, rb);
            ensure_planes(st_n, (size_t)(3 * every), rb);
        }
        if (adj_fused && nck > 1) {
            ensure_planes(sg_psi2, (size_t)every + 1, cb);
            ensure_planes(st_psi2, (size_t)(3 * every), cb);
            if (res) {
                ensure_planes(sg_n2, (size_t)every + 1, rb);
                ensure_planes(st_n2, (size_t)(3 * every), rb);
            }
        }
        for (int b = 0; b < 2; ++b) {
            if (!lam_psi[b].p) lam_psi[b].alloc(cb, stream);
            if (!yb_psi[b].p) yb_psi[b].alloc(cb, stream);
            if (res && !lam_n[b].p) lam_n[b].alloc(rb, stream);
            if (res && !yb_n[b].p) yb_n[b].alloc(rb, stream);
        }
        if (!la_psi.p) la_psi.alloc(cb, stream);
        if (res && !la_n.p) la_n.alloc(rb, stream);
        if (!pbar.p) pbar.alloc(rb, stream);
        PHX_CUDA(cudaMemsetAsync(pbar.p, 0, rb, stream));
        if (dpot && !P.n_potential_groups) fail(PHX_ERR_INVALID_ARG, "dL/dV needs a potential group");
        const bool want_v = dpot != nullptr;
        if (want_v) {
            if (!vbar.p) vbar.alloc(rb, stream);
            PHX_CUDA(cudaMemsetAsync(vbar.p, 0, rb, stream));
        }
        // lam_T = dL/d(psi_T, n_T), with periodic images
        int cur = 0;
        unpack_interior_kernel<C><<<256, 256, 0, stream>>>(static_cast<const C*>(dpsi), cplane(lam_psi[0]), pitch, N_r, N_c);
        ring_fill_kernel<C><<<64, 256, 0, stream>>>(cplane(lam_psi[0]), N_r, N_c, pitch, G, 1, 1);
        if (res) {
            if (dn)
                unpack_interior_kernel<T><<<256, 256, 0, stream>>>(static_cast<const T*>(dn), rplane(lam_n[0]), pitch, N_r, N_c);
            else
                PHX_CUDA(cudaMemsetAsync(lam_n[0].p, 0, rb, stream));
            ring_fill_kernel<T><<<64, 256, 0, stream>>>(rplane(lam_n[0]), N_r, N_c, pitch, G, 1, 1);
        }
        PHX_CUDA(cudaGetLastError());
        const T saved_dt = dt;
        dt = adj_dt;
        DevBuf scratch_psi, scratch_n;  // the recomputed state after a segment's last iteration is not needed
        scratch_psi.alloc(cb, stream);
        if (res) scratch_n.alloc(rb, stream);
        const T bw[4] = {(T)(1.0 / 6.0), (T)(1.0 / 3.0), (T)(1.0 / 3.0), (T)(1.0 / 6.0)};
        const T aw[3] = {(T)0.5, (T)0.5, (T)1.0};
        const T cw[4] = {(T)0.0, (T)0.5, (T)0.5, (T)1.0};
        // Segment k's recompute (states and stage values) does not depend on the
        // vector-Jacobian sweep of segment k + 1.  With the fused sweep the
        // recomputes run on a second stream into the other of two plane sets,
        // overlapped with the sweep of the segment before; events order a set's
        // reuse after the sweep that read it.
        const bool overlap = adj_fused;
        struct Overlap {
            cudaStream_t s2 = nullptr;
            cudaEvent_t start = nullptr, rec_done[2] = {nullptr, nullptr}, vjp_done[2] = {nullptr, nullptr};
            ~Overlap() {
                if (s2) (void)cudaStreamSynchronize(s2);
                for (cudaEvent_t e : {start, rec_done[0], rec_done[1], vjp_done[0], vjp_done[1]})
                    if (e) (void)cudaEventDestroy(e);
                if (s2) (void)cudaStreamDestroy(s2);
            }
        } ov;
        bool vjp_used[2] = {false, false};
        if (overlap) {
            PHX_CUDA(cudaStreamCreateWithFlags(&ov.s2, cudaStreamNonBlocking));
            for (cudaEvent_t* e : {&ov.start, &ov.rec_done[0], &ov.rec_done[1], &ov.vjp_done[0], &ov.vjp_done[1]})
                PHX_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
            PHX_CUDA(cudaEventRecord(ov.start, stream));
            PHX_CUDA(cudaStreamWaitEvent(ov.s2, ov.start, 0));
        }
        auto recompute_segment = [&](int64_t k, int set) {
            auto& SGp = set ? sg_psi2 : sg_psi;
            auto& SGn = set ? sg_n2 : sg_n;
            auto& STp = set ? st_psi2 : st_psi;
            auto& STn = set ? st_n2 : st_n;
            struct StreamSwap {  // the recompute's launches go to the second stream
                cudaStream_t& a;
                cudaStream_t& b;
                bool on;
                StreamSwap(cudaStream_t& x, cudaStream_t& y, bool o) : a(x), b(y), on(o) {
                    if (on) std::swap(a, b);
                }
                ~StreamSwap() {
                    if (on) std::swap(a, b);
                }
            };
            if (overlap && vjp_used[set]) PHX_CUDA(cudaStreamWaitEvent(ov.s2, ov.vjp_done[set], 0));
            StreamSwap sw(stream, ov.s2, overlap);
            const int64_t len = std::min(every, adj_T - k * every);
            plane_copy(*SGp[0], *ck_psi[k]);
            if (res) plane_copy(*SGn[0], *ck_n[k]);
            for (int64_t j = 0; j < len; ++j) {
                DevBuf* sp[3] = {STp[3 * j].get(), STp[3 * j + 1].get(), STp[3 * j + 2].get()};
                DevBuf* sn[3] = {res ? STn[3 * j].get() : nullptr, res ? STn[3 * j + 1].get() : nullptr,
                                 res ? STn[3 * j + 2].get() : nullptr};
                DevBuf& op = j + 1 < len ? *SGp[j + 1] : scratch_psi;
                DevBuf* on = res ? (j + 1 < len ? SGn[j + 1].get() : &scratch_n) : nullptr;
                if (adj_fused)
                    rk4_recompute_fused(*SGp[j], res ? SGn[j].get() : nullptr, sp, sn, op, on);
                else
                    rk4_recompute(*SGp[j], res ? SGn[j].get() : nullptr, sp, sn, op, on);
            }
            if (overlap) PHX_CUDA(cudaEventRecord(ov.rec_done[set], stream));
        };
        if (overlap) recompute_segment(nck - 1, (int)((nck - 1) & 1));
        for (int64_t k = nck - 1; k >= 0; --k) {
            const int set = overlap ? (int)(k & 1) : 0;
            if (overlap) {
                if (k >= 1) recompute_segment(k - 1, set ^ 1);
                PHX_CUDA(cudaStreamWaitEvent(stream, ov.rec_done[set], 0));
            } else {
                recompute_segment(k, 0);
            }
            auto& SGp = set ? sg_psi2 : sg_psi;
            auto& SGn = set ? sg_n2 : sg_n;
            auto& STp = set ? st_psi2 : st_psi;
            auto& STn = set ? st_n2 : st_n;
            const int64_t len = std::min(every, adj_T - k * every);
            for (int64_t j = len - 1; j >= 0; --j) {
                if (adj_fused) {
                    AdjFusedParams<T> Q;
                    std::memset(&Q, 0, sizeof(Q));
                    Q.N_r = N_r;
                    Q.N_c = N_c;
                    Q.pitch = pitch;
                    Q.Ypsi[0] = cplane(*SGp[j]);
                    Q.Yn[0] = res ? rplane(*SGn[j]) : nullptr;
                    for (int s = 2; s <= 4; ++s) {
                        Q.Ypsi[s - 1] = cplane(*STp[3 * j + s - 2]);
                        Q.Yn[s - 1] = res ? rplane(*STn[3 * j + s - 2]) : nullptr;
                    }
                    Q.lam_psi = cplane(lam_psi[cur]);
                    Q.lam_n = res ? rplane(lam_n[cur]) : nullptr;
                    Q.out_psi = cplane(lam_psi[cur ^ 1]);
                    Q.out_n = res ? rplane(lam_n[cur ^ 1]) : nullptr;
                    Q.pot = P.n_potential_groups ? rplane(pot[0]) : nullptr;
                    Q.pbar = (res && P.n_pump_groups) ? rplane(pbar) : nullptr;
                    Q.vbar = want_v ? rplane(vbar) : nullptr;
                    for (int s = 1; s <= 4; ++s) {
                        Q.c_pot[s - 1] = P.n_potential_groups ? interp<T>(amp_pot[0], next_pot[0], cw[s - 1]).real() : (T)0;
                        Q.c_pump[s - 1] = P.n_pump_groups ? interp<T>(amp_pump[0], next_pump[0], cw[s - 1]).real() : (T)0;
                        Q.dt_b[s - 1] = adj_dt * bw[s - 1];
                        Q.a_dt[s - 1] = s < 4 ? aw[s - 1] * adj_dt : (T)0;
                    }
                    Q.A = d.ohb * d.meff;
                    Q.ohb = d.ohb;
                    Q.ohb_gc = d.ohb * (T)P.g_c;
                    Q.ohb_gr = d.ohb * (T)P.g_r;
                    Q.half_R = (T)0.5 * (T)P.R;
                    Q.half_gamma_c = (T)0.5 * (T)P.gamma_c;
                    Q.gamma_r = (T)P.gamma_r;
                    Q.R = (T)P.R;
                    Q.m2 = d.m2;
                    Q.odx2 = d.odx2;
                    Q.ody2 = d.ody2;
                    Q.res = res;
                    cudaEvent_t a = nullptr;
                    prof_begin(a);
                    auto go_adj = [&](auto tw, auto th, auto nt, auto minb) {
                        constexpr int TW = decltype(tw)::value, TH = decltype(th)::value, NT = decltype(nt)::value;
                        constexpr int MINB = decltype(minb)::value;
                        dim3 grid((unsigned)((N_c + TW - 1) / TW), (unsigned)((N_r + TH - 1) / TH));
                        adj_fused_kernel<T, TW, TH, NT, MINB><<<grid, NT, 0, stream>>>(Q);
                    };
                    using std::integral_constant;
                    if constexpr (sizeof(T) == 4)  // 64 x 16 tiles, 16 warps, two CTAs per SM
                        go_adj(integral_constant<int, 64>{}, integral_constant<int, 16>{}, integral_constant<int, 512>{},
                               integral_constant<int, 2>{});
                    else
                        go_adj(integral_constant<int, 32>{}, integral_constant<int, 16>{}, integral_constant<int, 256>{},
                               integral_constant<int, 1>{});
                    prof_end(PHX_KERNEL_OTHER, a, (double)N_r * N_c * (5.0 * sizeof(C) + 7.0 * sizeof(T)));
                    ++launches;
                    PHX_CUDA(cudaGetLastError());
                    cur ^= 1;
                    continue;
                }
                for (int s = 4; s >= 1; --s) {
                    AdjParams<T> Q;
                    std::memset(&Q, 0, sizeof(Q));
                    Q.N_r = N_r;
                    Q.N_c = N_c;
                    Q.pitch = pitch;
                    Q.Ypsi = s == 1 ? cplane(*SGp[j]) : cplane(*STp[3 * j + s - 2]);
                    Q.Yn = res ? (s == 1 ? rplane(*SGn[j]) : rplane(*STn[3 * j + s - 2])) : nullptr;
                    Q.lam_psi = cplane(lam_psi[cur]);
                    Q.lam_n = res ? rplane(lam_n[cur]) : nullptr;
                    Q.ybar_in_psi = cplane(yb_psi[(s + 1) & 1]);
                    Q.ybar_in_n = res ? rplane(yb_n[(s + 1) & 1]) : nullptr;
                    Q.ybar_out_psi = cplane(yb_psi[s & 1]);
                    Q.ybar_out_n = res ? rplane(yb_n[s & 1]) : nullptr;
                    Q.acc_in_psi = cplane(la_psi);
                    Q.acc_in_n = res ? rplane(la_n) : nullptr;
                    Q.acc_psi = s == 1 ? cplane(lam_psi[cur ^ 1]) : cplane(la_psi);
                    Q.acc_n = res ? (s == 1 ? rplane(lam_n[cur ^ 1]) : rplane(la_n)) : nullptr;
                    Q.pot = P.n_potential_groups ? rplane(pot[0]) : nullptr;
                    Q.pump = P.n_pump_groups ? rplane(pump[0]) : nullptr;
                    Q.pbar = (res && P.n_pump_groups) ? rplane(pbar) : nullptr;
                    Q.vbar = want_v ? rplane(vbar) : nullptr;
                    Q.c_pot = P.n_potential_groups ? interp<T>(amp_pot[0], next_pot[0], cw[s - 1]).real() : (T)0;
                    Q.c_pump = P.n_pump_groups ? interp<T>(amp_pump[0], next_pump[0], cw[s - 1]).real() : (T)0;
                    Q.dt_b = adj_dt * bw[s - 1];
                    Q.a_dt = s < 4 ? aw[s - 1] * adj_dt : (T)0;
                    Q.A = d.ohb * d.meff;
                    Q.ohb = d.ohb;
                    Q.ohb_gc = d.ohb * (T)P.g_c;
                    Q.ohb_gr = d.ohb * (T)P.g_r;
                    Q.half_R = (T)0.5 * (T)P.R;
                    Q.half_gamma_c = (T)0.5 * (T)P.gamma_c;
                    Q.gamma_r = (T)P.gamma_r;
                    Q.R = (T)P.R;
                    Q.m2 = d.m2;
                    Q.odx2 = d.odx2;
                    Q.ody2 = d.ody2;
                    Q.s = s;
                    Q.res = res;
                    dim3 grid((unsigned)((N_c + 31) / 32), (unsigned)((N_r + 7) / 8));
                    cudaEvent_t a = nullptr;
                    prof_begin(a);
                    adj_stage_kernel<T><<<grid, 256, 0, stream>>>(Q);
                    prof_end(PHX_KERNEL_OTHER, a, (double)N_r * N_c * (4.0 * sizeof(C) + 4.0 * sizeof(T)));
                    ++launches;
                    PHX_CUDA(cudaGetLastError());
                }
                cur ^= 1;
            }
            if (overlap) {
                PHX_CUDA(cudaEventRecord(ov.vjp_done[set], stream));
                vjp_used[set] = true;
            }
        }
        dt = saved_dt;
        if (dpsi0) pack_interior_kernel<C><<<256, 256, 0, stream>>>(cplane(lam_psi[cur]), pitch, N_r, N_c, static_cast<C*>(dpsi0));
        if (dn0 && res) pack_interior_kernel<T><<<256, 256, 0, stream>>>(rplane(lam_n[cur]), pitch, N_r, N_c, static_cast<T*>(dn0));
        if (dpump) {
            if (!(res && P.n_pump_groups)) fail(PHX_ERR_INVALID_ARG, "dL/dP needs a pump group and the reservoir");
            pack_interior_kernel<T><<<256, 256, 0, stream>>>(rplane(pbar), pitch, N_r, N_c, static_cast<T*>(dpump));
        }
        if (want_v) pack_interior_kernel<T><<<256, 256, 0, stream>>>(rplane(vbar), pitch, N_r, N_c, static_cast<T*>(dpot));
        PHX_CUDA(cudaGetLastError());
        PHX_CUDA(cudaStreamSynchronize(stream));  // scratch planes are freed on return
        check_err_flag();
    }

    double sum_abs2(int field) override {
        PHX_CUDA(cudaStreamSynchronize(stream));
        check_err_flag();
        FieldRef f = field_ref(field, 0);
        const int blocks = 296;
        if (f.complex)
            sum_abs2_kernel<T, true><<<blocks, 256, 0, stream>>>(reinterpret_cast<const T*>(cplane(*f.buf)), pitch, N_r, N_c,
                                                                 reinterpret_cast<double*>(partials.p));
        else
            sum_abs2_kernel<T, false><<<blocks, 256, 0, stream>>>(rplane(*f.buf), pitch, N_r, N_c,
                                                                  reinterpret_cast<double*>(partials.p));
        finalize_pairs_kernel<<<1, 1024, 0, stream>>>(reinterpret_cast<double*>(partials.p), blocks,
                                                      reinterpret_cast<double*>(result.p));
        launches += 2;
        PHX_CUDA(cudaGetLastError());
        PHX_CUDA(cudaMemcpyAsync(host_result.p, result.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        PHX_CUDA(cudaStreamSynchronize(stream));
        const double v = static_cast<const double*>(host_result.p)[0];
        if (!std::isfinite(v)) fail(PHX_ERR_NONFINITE, "the sum of |field|^2 is not finite: the field holds NaN or Inf");
        return v;
    }
};

}  // namespace phx

// ====================================================================== C ABI
struct phx_handle {
    std::unique_ptr<phx::EngineBase> eng;
    std::string err;
};

namespace {

phx_status guard(phx_handle* h, const std::function<void()>& f) {
    try {
        f();
        if (h) h->err.clear();
        return PHX_OK;
    } catch (const phx::Error& e) {
        if (h) h->err = e.msg;
        else phx::g_create_error = e.msg;
        return e.status;
    } catch (const std::bad_alloc&) {
        if (h) h->err = "host allocation failed";
        else phx::g_create_error = "host allocation failed";
        return PHX_ERR_OOM;
    } catch (const std::exception& e) {
        if (h) h->err = e.what();
        else phx::g_create_error = e.what();
        return PHX_ERR_INVALID_ARG;
    }
}

void validate(const phx_params& p) {
    using phx::fail;
    if (p.abi_version != PHX_ABI_VERSION) fail(PHX_ERR_INVALID_ARG, "abi_version mismatch");
    if (p.N_c < 8 || p.N_r < 8) fail(PHX_ERR_INVALID_ARG, "grid must be at least 8 x 8");
    if ((long long)p.N_c * p.N_r > (1LL << 31)) fail(PHX_ERR_INVALID_ARG, "grid too large");
    if (p.dtype != PHX_F32 && p.dtype != PHX_F64) fail(PHX_ERR_INVALID_ARG, "dtype must be PHX_F32 or PHX_F64");
    if (p.dtype == PHX_F32 && (p.N_c & 1)) fail(PHX_ERR_UNSUPPORTED, "FP32 grids need an even N_c");
    if (p.iterator < PHX_ITER_RK4 || p.iterator > PHX_ITER_SSFM) fail(PHX_ERR_INVALID_ARG, "unknown iterator");
    {
        phx::Tableau t;
        if (p.adaptive && (p.iterator == PHX_ITER_RK4 || p.iterator == PHX_ITER_SSFM || !phx::tableau_resolve(p.iterator, t) ||
                           !t.adaptive))
            fail(PHX_ERR_INVALID_ARG, "adaptive stepping needs an adaptive iterator (DP45, BoSha, CashKarp, Fehlberg2, "
                                      "Fehlberg5, DP85, NSRK78)");
    }
    if (p.norm_mode != PHX_NORM_REFERENCE && p.norm_mode != PHX_NORM_INTERIOR) fail(PHX_ERR_INVALID_ARG, "bad norm_mode");
    if (!(p.L_x > 0) || !(p.L_y > 0) || !(p.h_bar_s > 0) || !(p.m_eff > 0)) fail(PHX_ERR_INVALID_ARG, "L, h_bar_s and m_eff must be > 0");
    if (!(p.dt > 0)) fail(PHX_ERR_INVALID_ARG, "dt must be > 0");
    if (p.n_pump_groups < 0 || p.n_pump_groups > phx::kMaxGroups || p.n_potential_groups < 0 ||
        p.n_potential_groups > phx::kMaxGroups || p.n_pulse_groups < 0 || p.n_pulse_groups > phx::kMaxGroups)
        fail(PHX_ERR_INVALID_ARG, "temporal group count out of range (0..8)");
    if (p.n_pump_groups > 0 && !p.use_reservoir) fail(PHX_ERR_INVALID_ARG, "pump groups need use_reservoir");
    if (p.tetm && !p.use_reservoir) fail(PHX_ERR_UNSUPPORTED, "TE/TM mode reads the reservoir; set use_reservoir");
    if (!std::isfinite(p.imag_time_amplitude)) fail(PHX_ERR_INVALID_ARG, "imag_time_amplitude must be finite");
    if (p.imag_time_amplitude != 0.0) {
        if (p.use_reservoir && p.iterator != PHX_ITER_SSFM)
            fail(PHX_ERR_UNSUPPORTED, "imaginary time with a reservoir: the complex step makes the reservoir complex, "
                                      "which this library stores real (SSFM keeps it real and is supported)");
        if (p.iterator == PHX_ITER_DP85)
            fail(PHX_ERR_UNSUPPORTED, "imaginary time is not provided for DP85 (its reference step swaps the fixed and "
                                      "variable branches)");
    }
    if (!std::isfinite(p.stochastic_amplitude)) fail(PHX_ERR_INVALID_ARG, "stochastic_amplitude must be finite");
    if (p.fma != 0 && p.fma != 1) fail(PHX_ERR_INVALID_ARG, "fma must be 0 or 1");
    if (p.fma && p.dtype != PHX_F32) fail(PHX_ERR_UNSUPPORTED, "the fused multiply-add arithmetic is provided for FP32");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        fail(PHX_ERR_CUDA, "no CUDA device available");
    }
    if (p.device < 0 || p.device >= ndev) fail(PHX_ERR_INVALID_ARG, "device ordinal out of range");
}

}  // namespace

extern "C" {

phx_status phx_create(const phx_params* p, phx_handle** out) {
    if (!p || !out) {
        phx::g_create_error = "NULL argument";
        return PHX_ERR_INVALID_ARG;
    }
    *out = nullptr;
    std::unique_ptr<phx_handle> h(new (std::nothrow) phx_handle());
    if (!h) return PHX_ERR_OOM;
    phx_status st = guard(nullptr, [&] {
        validate(*p);
        if (p->dtype == PHX_F64)
            h->eng.reset(new phx::Engine<double>());
        else
            h->eng.reset(new phx::Engine<float>());
        h->eng->P = *p;
        h->eng->init();
    });
    if (st != PHX_OK) return st;
    *out = h.release();
    return PHX_OK;
}

phx_status phx_destroy(phx_handle* h) {
    if (!h) return PHX_OK;
    if (h->eng) {
        cudaSetDevice(h->eng->P.device);
        if (h->eng->stream) cudaStreamSynchronize(h->eng->stream);
    }
    delete h;
    return PHX_OK;
}

phx_status phx_set_field(phx_handle* h, int32_t field, int32_t group, const void* host, int64_t count, int32_t host_dtype) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] { h->eng->set_field(field, group, host, count, host_dtype); });
}

phx_status phx_get_field(phx_handle* h, int32_t field, int32_t group, void* host, int64_t count, int32_t host_dtype) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] { h->eng->get_field(field, group, host, count, host_dtype); });
}

phx_status phx_set_temporal_table(phx_handle* h, int32_t envelope, int32_t group, const double* t, const double* re,
                                  const double* im, int64_t n) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] {
        if (!t || !re || !im) phx::fail(PHX_ERR_INVALID_ARG, "NULL table");
        if (n < 2) phx::fail(PHX_ERR_INVALID_ARG, "a temporal table needs at least 2 points");
        phx::TemporalSpec s;
        s.kind = PHX_TEMPORAL_LOADED;
        s.tt.assign(t, t + n);
        s.re.assign(re, re + n);
        s.im.assign(im, im + n);
        for (int64_t i = 0; i < n; ++i) {
            if (!std::isfinite(t[i]) || !std::isfinite(re[i]) || !std::isfinite(im[i]))
                phx::fail(PHX_ERR_INVALID_ARG, "temporal table values must be finite");
            if (i > 0 && !(t[i] >= t[i - 1])) phx::fail(PHX_ERR_INVALID_ARG, "temporal table times must ascend");
        }
        auto& P = h->eng->P;
        if (envelope == PHX_ENV_PUMP) {
            if (group < 0 || group >= P.n_pump_groups) phx::fail(PHX_ERR_INVALID_ARG, "pump group out of range");
            for (int64_t i = 0; i < n; ++i)
                if (im[i] != 0.0) phx::fail(PHX_ERR_UNSUPPORTED, "complex pump tables make the reservoir complex");
            h->eng->pump_t[group] = s;
        } else if (envelope == PHX_ENV_POTENTIAL) {
            if (group < 0 || group >= P.n_potential_groups) phx::fail(PHX_ERR_INVALID_ARG, "potential group out of range");
            h->eng->pot_t[group] = s;
        } else if (envelope == PHX_ENV_PULSE) {
            if (group < 0 || group >= P.n_pulse_groups) phx::fail(PHX_ERR_INVALID_ARG, "pulse group out of range");
            h->eng->pulse_t[group] = s;
        } else {
            phx::fail(PHX_ERR_INVALID_ARG, "unknown envelope family");
        }
    });
}

phx_status phx_iterate(phx_handle* h, int32_t force_fixed_time_step, phx_step_info* info) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] {
        cudaSetDevice(h->eng->P.device);
        struct Reset {
            phx::EngineBase* e;
            ~Reset() { e->force_fixed = false; }
        } reset{h->eng.get()};
        h->eng->force_fixed = force_fixed_time_step != 0;
        h->eng->step(1, info);
    });
}

phx_status phx_set_spectrum_output(phx_handle* h, int32_t enable) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] {
        cudaSetDevice(h->eng->P.device);
        h->eng->set_spectrum_output(enable != 0);
    });
}

phx_status phx_set_temporal(phx_handle* h, int32_t envelope, int32_t group, int32_t kind, double t0, double sigma, double freq) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] {
        if (kind < PHX_TEMPORAL_CONSTANT || kind > PHX_TEMPORAL_GAUSS) phx::fail(PHX_ERR_INVALID_ARG, "unknown temporal kind");
        phx::TemporalSpec s;
        s.kind = kind;
        s.t0 = t0;
        s.sigma = sigma;
        s.freq = freq;
        auto& P = h->eng->P;
        if (envelope == PHX_ENV_PUMP) {
            if (group < 0 || group >= P.n_pump_groups) phx::fail(PHX_ERR_INVALID_ARG, "pump group out of range");
            if (kind == PHX_TEMPORAL_IEXP) phx::fail(PHX_ERR_UNSUPPORTED, "complex (iexp) pump envelopes make the reservoir complex");
            h->eng->pump_t[group] = s;
        } else if (envelope == PHX_ENV_POTENTIAL) {
            if (group < 0 || group >= P.n_potential_groups) phx::fail(PHX_ERR_INVALID_ARG, "potential group out of range");
            h->eng->pot_t[group] = s;
        } else if (envelope == PHX_ENV_PULSE) {
            if (group < 0 || group >= P.n_pulse_groups) phx::fail(PHX_ERR_INVALID_ARG, "pulse group out of range");
            h->eng->pulse_t[group] = s;
        } else {
            phx::fail(PHX_ERR_INVALID_ARG, "unknown envelope family");
        }
    });
}

phx_status phx_step(phx_handle* h, int64_t max_iterations, phx_step_info* info) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] {
        if (max_iterations < 0) phx::fail(PHX_ERR_INVALID_ARG, "max_iterations < 0");
        h->eng->step(max_iterations, info);
    });
}

phx_status phx_get_time(phx_handle* h, double* t, double* dt) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] { h->eng->get_time(t, dt); });
}

phx_status phx_set_time(phx_handle* h, double t, double dt) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] {
        if (!(dt > 0)) phx::fail(PHX_ERR_INVALID_ARG, "dt must be > 0");
        h->eng->set_time(t, dt);
    });
}

phx_status phx_sum_abs2(phx_handle* h, int32_t field, double* out) {
    if (!h || !out) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] {
        if (field != PHX_PSI_PLUS && field != PHX_PSI_MINUS && field != PHX_N_PLUS && field != PHX_N_MINUS)
            phx::fail(PHX_ERR_INVALID_ARG, "sum_abs2 takes a state field");
        *out = h->eng->sum_abs2(field);
    });
}

phx_status phx_field_device_ptr(phx_handle* h, int32_t field, int32_t group, void** dev_ptr, int64_t* row_pitch_elems) {
    if (!h || !dev_ptr) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] { h->eng->field_ptr(field, group, dev_ptr, row_pitch_elems); });
}

phx_status phx_set_field_device(phx_handle* h, int32_t field, int32_t group, const void* dev, int64_t count) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] { h->eng->field_device(field, group, const_cast<void*>(dev), count, true); });
}

phx_status phx_get_field_device(phx_handle* h, int32_t field, int32_t group, void* dev, int64_t count) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] { h->eng->field_device(field, group, dev, count, false); });
}

phx_status phx_adjoint_forward(phx_handle* h, int64_t iterations, int64_t checkpoint_every) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] { h->eng->adjoint_forward(iterations, checkpoint_every); });
}

phx_status phx_adjoint_backward(phx_handle* h, const void* dpsi_T, const void* dn_T, void* dpsi_0, void* dn_0,
                                void* dpump, void* dpotential) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] { h->eng->adjoint_backward(dpsi_T, dn_T, dpsi_0, dn_0, dpump, dpotential); });
}

phx_status phx_profile_enable(phx_handle* h, int32_t enable) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] {
        h->eng->prof_reset();
        h->eng->profiling = enable != 0;
    });
}

phx_status phx_profile_read(phx_handle* h, int32_t kind, double* total_ms, int64_t* launches, double* bytes) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] {
        if (kind < 0 || kind >= PHX_KERNEL_KINDS) phx::fail(PHX_ERR_INVALID_ARG, "unknown kernel kind");
        h->eng->prof_harvest();
        if (total_ms) *total_ms = h->eng->prof_ms[kind];
        if (launches) *launches = h->eng->prof_count[kind];
        if (bytes) *bytes = h->eng->prof_bytes[kind];
    });
}

phx_status phx_tune_read(phx_handle* h, int32_t capacity, int32_t* shapes, double* median_us, int32_t* count) {
    if (!h) return PHX_ERR_INVALID_ARG;
    return guard(h, [&] {
        if (!count || capacity < 0 || (capacity > 0 && (!shapes || !median_us))) phx::fail(PHX_ERR_INVALID_ARG, "bad arguments");
        const auto& m = h->eng->tune_medians;
        *count = (int32_t)m.size();
        for (int32_t i = 0; i < std::min<int32_t>(capacity, (int32_t)m.size()); ++i) {
            shapes[i] = m[(size_t)i].first;
            median_us[i] = m[(size_t)i].second;
        }
    });
}

phx_status phx_request_abort(phx_handle* h) {
    if (!h) return PHX_ERR_INVALID_ARG;
    h->eng->abort_requested.store(1);
    return PHX_OK;
}

phx_status phx_set_wait_limit(phx_handle* h, int32_t polls) {
    if (!h) return PHX_ERR_INVALID_ARG;
    h->eng->wait_polls = polls < 0 ? phx::kWaitPolls : polls;
    return PHX_OK;
}

phx_status phx_get_stream(phx_handle* h, void** stream) {
    if (!h || !stream) return PHX_ERR_INVALID_ARG;
    *stream = (void*)h->eng->stream;
    return PHX_OK;
}

const char* phx_last_error(const phx_handle* h) {
    if (!h) return phx::g_create_error.c_str();
    return h->err.c_str();
}

const char* phx_status_string(int32_t s) {
    switch (s) {
        case PHX_OK: return "ok";
        case PHX_ERR_INVALID_ARG: return "invalid argument";
        case PHX_ERR_OOM: return "out of memory";
        case PHX_ERR_CUDA: return "CUDA error";
        case PHX_ERR_NONFINITE: return "non-finite value";
        case PHX_ERR_ABORTED: return "aborted on request";
        case PHX_ERR_TIMEOUT: return "timeout";
        case PHX_ERR_UNSUPPORTED: return "unsupported";
        case PHX_ERR_STATE: return "invalid state";
        default: return "unknown status";
    }
}

int32_t phx_abi_version(void) { return PHX_ABI_VERSION; }

const char* phx_build_info(void) { return "phx-b200 sm_100a fused-stage RK4/DP45 (nvcc " PHX_NVCC_VERSION ")"; }

}  // extern "C"
