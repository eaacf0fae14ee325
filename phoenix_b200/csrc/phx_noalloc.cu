// phx_noalloc.cu -- phx_sum_abs2_noalloc: the FP64 norm reduction for callers
// that must not allocate device memory.
//
// Some callers cannot call cudaMalloc: code that runs while another runtime
// is capturing a CUDA graph (allocation is not permitted during capture),
// hosts whose device memory is owned and budgeted by their own allocator
// (a framework memory pool, a solver that pre-allocates everything), and
// loops that cannot afford the implicit device synchronisation of
// cudaMalloc / cudaFree.  phx_sum_abs2 needs a handle, and a handle
// allocates; this entry point takes the caller's device field and device
// output and keeps its only scratch -- the per-block partial sums of the
// two-pass reduction -- in a fixed array inside this library.
//
// The array is a file-scope __device__ variable of kNoAllocBlocks doubles
// (32 KiB).  Every GPU that loads the library holds it until the
// process exits.  Each block reduces a fixed chunk of kChunk points, so
// fields of up to kNoAllocBlocks * kChunk = 16,777,216 points (4096 x 4096)
// are accepted; larger ones are rejected.  All calls share the array: calls
// whose kernels overlap on the GPU (different streams, or different host
// threads without ordering) race on it.  Every slot a call reads was written
// by the same call, so nothing needs clearing between calls.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/phx.h"

namespace phx {
// message of the last failed call without a handle (phx_last_error(NULL)),
// defined with the handle code in phx_runtime.cu
extern thread_local std::string g_create_error;
}  // namespace phx

namespace {

constexpr int kChunk = 4096;           // points reduced by one block
constexpr int kNoAllocBlocks = 4096;   // blocks, i.e. partial-sum slots
constexpr int kThreads = 256;
constexpr long long kMaxPoints = (long long)kNoAllocBlocks * kChunk;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocBlocks];

std::mutex g_setup_mutex;
constexpr int kMaxDevices = 64;
double* g_partials_addr[kMaxDevices] = {};

template <typename T, bool COMPLEX>
__global__ void __launch_bounds__(kThreads)
    chunk_abs2_kernel(const T* __restrict__ base, long long pitch, int N_c, long long n, double* __restrict__ partials) {
    const long long lo = (long long)blockIdx.x * kChunk;
    const long long hi = lo + kChunk < n ? lo + kChunk : n;
    double a = 0.0;
    for (long long i = lo + threadIdx.x; i < hi; i += kThreads) {
        const long long r = i / N_c, c = i - r * N_c;
        if (COMPLEX) {
            const T re = base[2 * (r * pitch + c)], im = base[2 * (r * pitch + c) + 1];
            a += (double)re * (double)re + (double)im * (double)im;
        } else {
            const T x = base[r * pitch + c];
            a += (double)x * (double)x;
        }
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    __shared__ double s[kThreads / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += s[w];
        partials[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(1024) finish_kernel(const double* __restrict__ partials, int nb, double* __restrict__ out) {
    __shared__ double s[32];
    double a = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) a += partials[i];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) t += s[w];
        *out = t;
    }
}

phx_status fail(phx_status s, const std::string& m) {
    phx::g_create_error = m;
    return s;
}

// Device address of the scratch array for the current device.  In host code
// g_noalloc_partials names a host-side stand-in, not device memory, so the
// address is looked up once per device with that device current.
phx_status scratch_for_current_device(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(PHX_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(PHX_ERR_UNSUPPORTED, "device ordinal beyond the supported range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p)
            return fail(PHX_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_partials_addr[dev] = static_cast<double*>(p);
    }
    *out = g_partials_addr[dev];
    return PHX_OK;
}

}  // namespace

extern "C" {

PHX_API phx_status phx_sum_abs2_noalloc(const void* field_dev, int32_t dtype, int32_t is_complex, int32_t N_r, int32_t N_c,
                                        int64_t row_pitch_elems, double* out_dev, void* stream) {
    if (!field_dev || !out_dev) return fail(PHX_ERR_INVALID_ARG, "field and output pointers must be device pointers, not NULL");
    if (dtype != PHX_F32 && dtype != PHX_F64) return fail(PHX_ERR_INVALID_ARG, "dtype must be PHX_F32 or PHX_F64");
    if (N_r <= 0 || N_c <= 0) return fail(PHX_ERR_INVALID_ARG, "grid dimensions must be positive");
    if (row_pitch_elems < N_c) return fail(PHX_ERR_INVALID_ARG, "row pitch is smaller than N_c");
    const long long n = (long long)N_r * N_c;
    if (n > kMaxPoints)
        return fail(PHX_ERR_INVALID_ARG, "field of " + std::to_string(n) + " points exceeds the no-alloc scratch limit of " +
                                             std::to_string(kMaxPoints) + " points (4096 x 4096)");
    double* partials = nullptr;
    phx_status st = scratch_for_current_device(&partials);
    if (st != PHX_OK) return st;
    const int nb = (int)((n + kChunk - 1) / kChunk);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == PHX_F32) {
        if (is_complex)
            chunk_abs2_kernel<float, true><<<nb, kThreads, 0, s>>>(static_cast<const float*>(field_dev), row_pitch_elems, N_c, n, partials);
        else
            chunk_abs2_kernel<float, false><<<nb, kThreads, 0, s>>>(static_cast<const float*>(field_dev), row_pitch_elems, N_c, n, partials);
    } else {
        if (is_complex)
            chunk_abs2_kernel<double, true><<<nb, kThreads, 0, s>>>(static_cast<const double*>(field_dev), row_pitch_elems, N_c, n, partials);
        else
            chunk_abs2_kernel<double, false><<<nb, kThreads, 0, s>>>(static_cast<const double*>(field_dev), row_pitch_elems, N_c, n, partials);
    }
    finish_kernel<<<1, 1024, 0, s>>>(partials, nb, out_dev);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(PHX_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return PHX_OK;
}

}  // extern "C"
