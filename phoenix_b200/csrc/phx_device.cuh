// Device-side arithmetic and field layout shared by the PHOENIX B200 kernels.
//
// Every real operation goes through an explicitly rounded intrinsic
// (__fadd_rn, __dmul_rn, ...), which the compiler never fuses into an FMA.
// Together with the operand order of the reference kernels this makes each
// grid-point update bit-identical to the reference's CPU build, where
// Type::complex is std::complex and products are (ac - bd) + (ad + bc) i
// (include/cuda/typedef.cuh:131-166, include/kernel/kernel_gp_compute.cuh).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace phx {

template <typename T>
struct alignas(2 * sizeof(T)) cx {
    T re, im;
};

__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float rsqrt_rn(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double rsqrt_rn(double a) { return __dsqrt_rn(a); }

template <typename T>
__device__ __forceinline__ cx<T> mk(T re, T im) {
    cx<T> z;
    z.re = re;
    z.im = im;
    return z;
}
template <typename T>
__device__ __forceinline__ cx<T> cadd(cx<T> a, cx<T> b) { return mk(radd(a.re, b.re), radd(a.im, b.im)); }
template <typename T>
__device__ __forceinline__ cx<T> csub(cx<T> a, cx<T> b) { return mk(rsub(a.re, b.re), rsub(a.im, b.im)); }
// complex * complex
template <typename T>
__device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b) {
    return mk(rsub(rmul(a.re, b.re), rmul(a.im, b.im)), radd(rmul(a.re, b.im), rmul(a.im, b.re)));
}
// real * complex (== complex * real)
template <typename T>
__device__ __forceinline__ cx<T> smul(T s, cx<T> a) { return mk(rmul(s, a.re), rmul(s, a.im)); }
// -i z
template <typename T>
__device__ __forceinline__ cx<T> mi(cx<T> z) { return mk(z.im, -z.re); }
template <typename T>
__device__ __forceinline__ T abs2(cx<T> z) { return radd(rmul(z.re, z.re), rmul(z.im, z.im)); }
// (complex(s_re, s_im) with s_im == 0) * z, as the reference computes it for
// a real-valued complex coefficient: (s*zr - 0*zi, s*zi + 0*zr) == s*z for finite z
template <typename T>
__device__ __forceinline__ cx<T> cmul_general(cx<T> s, cx<T> z) { return cmul(s, z); }

// Programmatic dependent launch (sm_90+): a kernel launched with the
// programmatic stream serialization attribute may start while the kernel
// before it in the stream drains; pdl_wait() returns once that kernel has
// completed and its writes are visible, so it comes before the first read of
// anything the previous kernel wrote (and before any write it could still
// read).  pdl_trigger() lets the next such kernel be scheduled once every CTA
// of this grid has issued it or exited.  Both do nothing in a kernel launched
// without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Grid-point storage.  Every field is a halo-padded plane: interior point
// (r, c), 0 <= r < N_r, 0 <= c < N_c, sits at base[r * pitch + c] where base
// points at interior (0, 0); rows and columns -G .. N+G-1 are addressable.
// The ring holds zeros along non-periodic axes and periodic images of the
// first/last interior row/column along periodic axes.
constexpr int kRing = 8;           // G: ring width of RK4 / DP45 handles (wider for larger halos)
constexpr int kMaxGroups = 8;      // temporal groups per envelope family
constexpr int kMaxStages = 16;  // weights of one stage sum (NSRK78: 13)

}  // namespace phx
