// SELL-C-sigma sparse matrices and the memory-bound kernels of the V-cycle and PCG.
//
// Layout: the rows are cut into slices of C consecutive rows (sigma = 1: no reordering, the
// operators of a grid hierarchy have nearly equal rows). Slice s holds w_s groups of 4 entries
// per row (w_s = ceil(longest row / 4)); group k of row r of the slice is at
// slice_ptr[s] + 4 (k C + r). A thread owns a row and reads its values and columns 4 at a time
// (16-byte loads for FP32 values and the int32 columns, 32 bytes for FP64 values), and the C
// threads of a slice read consecutive addresses. Padding entries have value 0 and the row's own
// column, so they read an x entry the row reads anyway.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace femgpu {

template <class T>
struct SellView {
    int64_t n;        // rows
    int64_t nslices;  // ceil(n / C)
    int C;
    const int64_t* __restrict__ slice_ptr;  // in entries; nslices + 1
    const uint32_t* __restrict__ col;
    const T* __restrict__ val;
};

template <class T>
struct Vec4;
template <>
struct Vec4<float> {
    using type = float4;
};
template <>
struct Vec4<double> {
    using type = double4;
};

__device__ __forceinline__ double4 load4(const double* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 load4(const float* p) {
    return __ldg(reinterpret_cast<const float4*>(p));
}

// A load of a vector: read-only through the non-coherent path (the kernel never writes it), or
// COH: a load cached in L2 only (ld.global.cg), for a vector that the same kernel wrote before
// a grid- or cluster-wide barrier, which such a barrier's memory ordering covers.
template <bool COH, class T>
__device__ __forceinline__ T ldx(const T* p) {
    if constexpr (COH)
        return __ldcg(p);
    else
        return __ldg(p);
}

// (A x)_row for the thread's row in slice `s`, lane `r` of the slice. Accumulates in TA.
template <class T, class TX, class TA, bool COH = false>
__device__ __forceinline__ TA sell_row(const SellView<T>& A, int64_t s, int r,
                                       const TX* __restrict__ x) {
    int64_t b = A.slice_ptr[s], e = A.slice_ptr[s + 1];
    int64_t groups = (e - b) / (4 * A.C);
    const T* v = A.val + b + 4 * r;
    const uint32_t* c = A.col + b + 4 * r;
    TA acc = 0;
    for (int64_t k = 0; k < groups; ++k) {
        auto vv = load4(v);
        uint4 cc = __ldg(reinterpret_cast<const uint4*>(c));
        acc += (TA)vv.x * (TA)ldx<COH>(x + cc.x);
        acc += (TA)vv.y * (TA)ldx<COH>(x + cc.y);
        acc += (TA)vv.z * (TA)ldx<COH>(x + cc.z);
        acc += (TA)vv.w * (TA)ldx<COH>(x + cc.w);
        v += 4 * A.C;
        c += 4 * A.C;
    }
    return acc;
}

// Block-wide sum of up to 2 doubles, then the last block to finish sums the block partials in
// block order (a deterministic result) and calls `fin(sum0, sum1)`.
template <int THREADS, class Fin>
__device__ __forceinline__ void reduce2_finalize(double a, double b, double* partial,
                                                 unsigned* counter, Fin fin) {
    __shared__ double sa[THREADS / 32], sb[THREADS / 32];
    __shared__ bool last;
    for (int o = 16; o; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sa[w] = a;
        sb[w] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0, tb = 0;
        for (int k = 0; k < THREADS / 32; ++k) {
            ta += sa[k];
            tb += sb[k];
        }
        partial[2 * blockIdx.x] = ta;
        partial[2 * blockIdx.x + 1] = tb;
        __threadfence();
        unsigned done = atomicAdd(counter, 1u);
        last = done == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // The last block sums the partials of every block: each thread a strided subset in a
    // fixed order, then the block tree; the same order every launch.
    double ta = 0, tb = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += THREADS) {
        ta += ((volatile double*)partial)[2 * k];
        tb += ((volatile double*)partial)[2 * k + 1];
    }
    for (int o = 16; o; o >>= 1) {
        ta += __shfl_xor_sync(0xffffffffu, ta, o);
        tb += __shfl_xor_sync(0xffffffffu, tb, o);
    }
    __syncthreads();
    if (lane == 0) {
        sa[w] = ta;
        sb[w] = tb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double fa = 0, fb = 0;
        for (int k = 0; k < THREADS / 32; ++k) {
            fa += sa[k];
            fb += sb[k];
        }
        fin(fa, fb);
        *counter = 0;
    }
}

}  // namespace femgpu
