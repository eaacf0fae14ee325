// phx_rt.hpp -- host-side pieces shared by the single-simulation handle
// (phx_runtime.cu) and the batch (phx_batch.cu): error reporting through
// exceptions that the C ABI turns into phx_status, device and pinned
// buffers, TMA tensor maps over halo-padded planes, and the constants of
// the fused RK4 iteration.
#pragma once

#include <cstring>

#include <cuda.h>
#include <cuda_runtime.h>
#include <cufft.h>

#include <string>

#include "../../include/phx.h"
#include "phx_host.hpp"
#include "phx_step_fused.cuh"

namespace phx {

// message of the last failed call that takes no handle (this thread)
extern thread_local std::string g_create_error;

struct Error {
    phx_status status;
    std::string msg;
};

#define PHX_CUDA(call)                                                                                       \
    do {                                                                                                     \
        cudaError_t e_ = (call);                                                                             \
        if (e_ != cudaSuccess) throw Error{PHX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)
#define PHX_CUFFT(call)                                                                       \
    do {                                                                                      \
        cufftResult r_ = (call);                                                              \
        if (r_ != CUFFT_SUCCESS) throw Error{PHX_ERR_CUDA, std::string(#call) + " failed (" + \
                                             std::to_string((int)r_) + ")"};                  \
    } while (0)

[[noreturn]] inline void fail(phx_status s, const std::string& m) { throw Error{s, m}; }

// ---------------------------------------------------------------- device memory
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    void alloc(size_t n, cudaStream_t s) {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = n;
        if (n == 0) return;
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            p = nullptr;
            (void)cudaGetLastError();
            fail(PHX_ERR_OOM, "cudaMalloc(" + std::to_string(n) + " bytes): " + cudaGetErrorString(e));
        }
        PHX_CUDA(cudaMemsetAsync(p, 0, n, s));
    }
};

struct PinnedBuf {
    void* p = nullptr;
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
    void alloc(size_t n) {
        if (p) cudaFreeHost(p);
        p = nullptr;
        PHX_CUDA(cudaMallocHost(&p, n));
    }
};

// Pinned host memory mapped into the device's address space: a kernel writes
// it directly, the host reads it after synchronising the stream (no copy).
struct MappedBuf {
    void* p = nullptr;  // host address
    void* d = nullptr;  // device address
    ~MappedBuf() {
        if (p) cudaFreeHost(p);
    }
    void alloc(size_t n) {
        if (p) cudaFreeHost(p);
        p = d = nullptr;
        PHX_CUDA(cudaHostAlloc(&p, n, cudaHostAllocMapped));
        std::memset(p, 0, n);
        PHX_CUDA(cudaHostGetDevicePointer(&d, p, 0));
    }
};

// ---------------------------------------------------------------- TMA maps
// 2-D tensor map over a whole halo-padded allocation: rows x pitch points
// (2 values a point for complex planes), element T, box of box_w_points x
// box_h points.  The driver entry point is looked up once.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* f = nullptr;
        PHX_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !f) fail(PHX_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<EncodeTiledFn>(f);
    }
    return fn;
}
template <typename T>
void plane_tensor_map(CUtensorMap* m, void* alloc_base, bool complex, long long pitch, long long rows, int box_w_points,
                      int box_h) {
    const int per = complex ? 2 : 1;
    const cuuint64_t dims[2] = {(cuuint64_t)(per * pitch), (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)(per * pitch * sizeof(T))};
    const cuuint32_t box[2] = {(cuuint32_t)(per * box_w_points), (cuuint32_t)box_h};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode_tiled_fn()(m, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                                         2, alloc_base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(PHX_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

// ---------------------------------------------------------------- fused RK4
// Scalars of one fused RK4 iteration (everything but the plane pointers and
// the per-stage temporal coefficients), in the build precision, as the
// reference derives them (source/system/system.cpp:134-157) and the RK4 tableau
// (source/cuda_solver/solver/iterator/runge_kutta.cu:53-96): stage offsets
// 0, 1/2, 1/2, 1; weights 1/6, 1/3, 1/3, 1/6.
template <typename T>
void fused_constants(FusedParams<T>& F, const phx_params& P, const Derived<T>& d, T dt, long long pitch) {
    const T aw[3] = {(T)0.5, (T)0.5, (T)1.0};
    const T bw[4] = {(T)(1.0 / 6.0), (T)(1.0 / 3.0), (T)(1.0 / 3.0), (T)(1.0 / 6.0)};
    for (int s = 0; s < 4; ++s) {
        F.b[s] = bw[s];
        if (s < 3) F.dtw[s] = dt * aw[s];
    }
    F.N_r = P.N_r;
    F.N_c = P.N_c;
    F.img_x = P.periodic_x;
    F.img_y = P.periodic_y;
    F.pitch = pitch;
    F.m2 = d.m2, F.odx2 = d.odx2, F.ody2 = d.ody2, F.meff = d.meff, F.ohb = d.ohb;
    F.ohb_gc = d.ohb * (T)P.g_c;
    F.half_gamma_c = (T)0.5 * (T)P.gamma_c;
    F.ohb_gr = d.ohb * (T)P.g_r;
    F.half_R = (T)0.5 * (T)P.R;
    F.gamma_r = (T)P.gamma_r;
    F.R = (T)P.R;
    F.dt = dt;
}

}  // namespace phx
