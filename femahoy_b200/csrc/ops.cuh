// The operators of a level, as seen by the kernels: SELL-C (any sparse matrix) or a symmetric
// stencil (a matrix whose entries sit at a few constant column offsets, as the operators of a
// box grid in grid order do).
//
// Stencil layout: offsets 0 = o_0 < o_1 < ... < o_{K-1}; coef[k n + i] = a(i, i + o_k), 0 where
// the matrix has no such entry. Row i is then
//   sum_k coef[k][i] x[i + o_k] + sum_{k >= 1} coef[k][i - o_k] x[i - o_k],
// the lower entries taken from the rows above (the matrix is symmetric). The columns are
// implicit: a row reads K coefficients of its own, K - 1 of earlier rows (recently read by
// other threads, so from L2) and 2K - 1 entries of x; no index is stored.
#pragma once
#include "sell.cuh"

namespace femgpu {

constexpr int MAXK = 32;

// Row numbers and offsets are 32-bit (a stencil is built only when n plus the largest offset
// fits): with 64-bit row arithmetic the products ran 2.4 times slower on B200, the extra integer
// work, not the memory, setting their time.
template <class T>
struct StencilView {
    int n;
    int K;
    int off[MAXK];
    const T* __restrict__ coef;
};

template <class T>
struct SellOp {
    SellView<T> v;
    __device__ __forceinline__ int64_t threads() const { return v.nslices * v.C; }
    __device__ __forceinline__ bool valid(int64_t g) const { return g < v.n; }
    template <class TA, class TX>
    __device__ __forceinline__ TA apply(int64_t g, const TX* __restrict__ x) const {
        return sell_row<T, TX, TA>(v, g / v.C, (int)(g % v.C), x);
    }
};

template <class T>
struct StencilOp {
    StencilView<T> v;
    __device__ __forceinline__ int64_t threads() const { return v.n; }
    __device__ __forceinline__ bool valid(int64_t) const { return true; }
    template <class TA, class TX>
    __device__ __forceinline__ TA apply(int64_t g, const TX* __restrict__ x) const {
        const int i = (int)g, n = v.n;
        const T* __restrict__ c = v.coef;
        TA acc = (TA)__ldg(c + i) * (TA)__ldg(x + i);
        for (int k = 1; k < v.K; ++k) {
            const int o = v.off[k];
            const T* __restrict__ ck = c + (size_t)k * n;
            const int j = i + o, m = i - o;
            if (j < n) acc += (TA)__ldg(ck + i) * (TA)__ldg(x + j);
            if (m >= 0) acc += (TA)__ldg(ck + m) * (TA)__ldg(x + m);
        }
        return acc;
    }
};

// The same with K known at compile time: the K own coefficients, the K - 1 coefficients of the
// rows above and the 2K - 1 entries of x are all loaded before the first product, so a thread
// has 4K - 2 independent loads in flight (the runtime-K loop issues them 4 at a time). Loads
// past either end are predicated off and count 0.
template <class T, int K>
struct StencilOpK {
    StencilView<T> v;
    __device__ __forceinline__ int64_t threads() const { return v.n; }
    __device__ __forceinline__ bool valid(int64_t) const { return true; }
    template <class TA, class TX>
    __device__ __forceinline__ TA apply(int64_t g, const TX* __restrict__ x) const {
        const int i = (int)g, n = v.n;
        const T* __restrict__ c = v.coef;
        TA acc = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int o = v.off[k];
            const T* __restrict__ ck = c + (size_t)k * n;
            const int j = i + o, m = i - o;
            TA a = (TA)__ldg(ck + i) * (j < n ? (TA)__ldg(x + j) : (TA)0);
            if (k > 0) a += (m >= 0 ? (TA)__ldg(ck + m) : (TA)0) * (m >= 0 ? (TA)__ldg(x + m) : (TA)0);
            acc += a;
        }
        return acc;
    }
};

}  // namespace femgpu
