// Checked indices of the GO_DEBUG_BOUNDS build of the stage kernels.
//
// Built with -DGO_DEBUG_BOUNDS (build.py makes lib/libgocean_debug.so that
// way), every global load and store of the stage kernels, and the reads of
// their shared-memory rings, test the index range against the extent of the
// array or buffer.  An access outside sets GO_STATUS_BOUNDS in the stage's
// status word and is skipped: a load reads zero, a store writes nothing.  No
// assert, no trap: the kernel runs to its end and the host reads the word.
// Without the flag every test is a compile-time true and costs nothing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gocean.h"

namespace go {

#ifdef GO_DEBUG_BOUNDS
constexpr bool kCheckedIndices = true;
#else
constexpr bool kCheckedIndices = false;
#endif

// [i, i + n) inside [0, extent)?  (extent and i in elements)
__device__ __forceinline__ bool idx_ok(long long i, int n, long long extent, unsigned int* status) {
    if (!kCheckedIndices) return true;
    if (i >= 0 && i + n <= extent) return true;
    if (status) atomicOr(status, GO_STATUS_BOUNDS);
    return false;
}

__device__ __forceinline__ float ldg1(const float* p, long long i, long long extent, unsigned int* status) {
    return idx_ok(i, 1, extent, status) ? __ldg(p + i) : 0.0f;
}
// two consecutive floats at an 8-byte aligned index
__device__ __forceinline__ float2 ldg2(const float* p, long long i, long long extent, unsigned int* status) {
    return idx_ok(i, 2, extent, status) ? __ldg(reinterpret_cast<const float2*>(p + i)) : make_float2(0.0f, 0.0f);
}
__device__ __forceinline__ float ld1(const float* p, long long i, long long extent, unsigned int* status) {
    return idx_ok(i, 1, extent, status) ? p[i] : 0.0f;
}
__device__ __forceinline__ void st1(float* p, long long i, float v, long long extent, unsigned int* status) {
    if (idx_ok(i, 1, extent, status)) p[i] = v;
}
__device__ __forceinline__ void st2(float* p, long long i, float2 v, long long extent, unsigned int* status) {
    if (idx_ok(i, 2, extent, status)) *reinterpret_cast<float2*>(p + i) = v;
}

// Extents (floats) of the arrays a stage reads and writes: states of
// (ny + 4) rows, corners of (ny + 5) rows, one Coriolis value per row, per-cell
// wind of ny rows.
template <class A> __device__ __forceinline__ long long ext_in(const A& a) { return (long long)(a.k.ny + 4) * a.pin; }
template <class A> __device__ __forceinline__ long long ext_out(const A& a) { return (long long)(a.k.ny + 4) * a.pout; }
template <class A> __device__ __forceinline__ long long ext_qn(const A& a) { return (long long)(a.k.ny + 4) * a.pqn; }
template <class A> __device__ __forceinline__ long long ext_hi(const A& a) { return (long long)(a.k.ny + 5) * a.phi; }
template <class A> __device__ __forceinline__ long long ext_f(const A& a) { return (long long)(a.k.ny + 4); }
template <class A> __device__ __forceinline__ long long ext_w(const A& a) { return (long long)a.k.ny * a.pw; }

}  // namespace go
