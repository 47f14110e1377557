// The operators of a level, as seen by the kernels: SELL-C (any sparse matrix) or a symmetric
// stencil (a matrix whose entries sit at a few constant column offsets, as the operators of a
// box grid in grid order do).
//
// Stencil layout: offsets 0 = o_0 < o_1 < ... < o_{K-1}; coef[k ld + i] = a(i, i + o_k), 0 where
// the matrix has no such entry (ld >= n: each offset's array starts on a 4 KB boundary, the
// padding 0). Row i is then
//   sum_k coef[k][i] x[i + o_k] + sum_{k >= 1} coef[k][i - o_k] x[i - o_k],
// the lower entries taken from the rows above (the matrix is symmetric). The columns are
// implicit: a row reads K coefficients of its own, K - 1 of earlier rows (recently read by
// other threads, so from L2) and 2K - 1 entries of x; no index is stored.
#pragma once
#include <cuda_fp16.h>

#include "sell.cuh"

namespace femgpu {

constexpr int MAXK = 32;

// The rows of a stencil tile streamed into shared memory by the bulk-copy kernels, and the
// stride of a stencil's coefficient arrays: n rounded up to whole tiles, so that every array and
// tile starts on a 4 KB boundary and every tile is 1 full copy.
constexpr int STENCIL_TILE = 1024;
__host__ __device__ __forceinline__ int64_t stencil_ld(int64_t n) {
    return (n + STENCIL_TILE - 1) / STENCIL_TILE * STENCIL_TILE;
}

// a b + c with 1 rounding, so that every product kernel below sums in the same way whatever
// the compiler contracts.
__device__ __forceinline__ float fmadd(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmadd(double a, double b, double c) { return __fma_rn(a, b, c); }

// Row numbers and offsets are 32-bit (a stencil is built only when n plus the largest offset
// fits): with 64-bit row arithmetic the products ran 2.4 times slower on B200, the extra integer
// work, not the memory, setting their time.
template <class T>
struct StencilView {
    int n;
    int K;
    int ld;
    int off[MAXK];
    const T* __restrict__ coef;
};

// The plane frame of a box level's stencil for the marching kernels (solver.cu
// k_stencil_march): rows z P + j, T rows of a plane per block, `chunk` planes per block.
struct MarchGeom {
    int P;       // the plane stride: the first offset after the largest gap of the offsets
    int s1;      // off[0, s1) are in-plane, off[s1, K) cross-plane (P + delta, delta in [0, H])
    int H;       // the halo: the largest in-plane offset and cross-plane delta
    int planes;  // ceil(n / P)
    int chunk;   // planes per block
    int tiles;   // blocks per plane: ceil(P / T)
    int T;       // rows of a plane per block = threads per block
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

// Row i of the stencil product with K read at run time (COH: x through ldx<true>).
template <class T, class TA, class TX, bool COH = false>
__device__ __forceinline__ TA stencil_apply(const StencilView<T>& v, int i,
                                            const TX* __restrict__ x) {
    const int n = v.n;
    const T* __restrict__ c = v.coef;
    TA acc = (TA)__ldg(c + i) * (TA)ldx<COH>(x + i);
    for (int k = 1; k < v.K; ++k) {
        const int o = v.off[k];
        const T* __restrict__ ck = c + (size_t)k * v.ld;
        const int j = i + o, m = i - o;
        if (j < n) acc = fmadd((TA)__ldg(ck + i), (TA)ldx<COH>(x + j), acc);
        if (m >= 0) acc = fmadd((TA)__ldg(ck + m), (TA)ldx<COH>(x + m), acc);
    }
    return acc;
}

template <class T>
struct StencilOp {
    StencilView<T> v;
    __device__ __forceinline__ int64_t threads() const { return v.n; }
    __device__ __forceinline__ bool valid(int64_t) const { return true; }
    template <class TA, class TX>
    __device__ __forceinline__ TA apply(int64_t g, const TX* __restrict__ x) const {
        return stencil_apply<T, TA, TX>(v, (int)g, x);
    }
};

// The same products through a reference to a view held elsewhere (shared memory), so that the
// view is not copied per thread; COH: for the fused kernels, whose x they wrote themselves.
template <class T, bool COH = false>
struct StencilRefOp {
    const StencilView<T>& v;
    static constexpr bool coherent = COH;
    __device__ __forceinline__ bool valid(int64_t) const { return true; }
    template <class TA, class TX>
    __device__ __forceinline__ TA apply(int64_t g, const TX* __restrict__ x) const {
        return stencil_apply<T, TA, TX, COH>(v, (int)g, x);
    }
};

template <class T, bool COH = false>
struct SellRefOp {
    const SellView<T>& v;
    static constexpr bool coherent = COH;
    __device__ __forceinline__ bool valid(int64_t g) const { return g < v.n; }
    template <class TA, class TX>
    __device__ __forceinline__ TA apply(int64_t g, const TX* __restrict__ x) const {
        return sell_row<T, TX, TA, COH>(v, g / v.C, (int)(g % v.C), x);
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
        // The same fused multiply-adds in the same order as StencilOp: a term past either end
        // adds 0 * 0 = +0, which changes no nonzero sum, so both kernels give the same bits and
        // the autotuner's choice between them (made by timing) cannot change a result.
        TA acc = (TA)__ldg(c + i) * (TA)__ldg(x + i);
#pragma unroll
        for (int k = 1; k < K; ++k) {
            const int o = v.off[k];
            const T* __restrict__ ck = c + (size_t)k * v.ld;
            const int j = i + o, m = i - o;
            const bool up = j < n, lo = m >= 0;
            acc = fmadd(up ? (TA)__ldg(ck + i) : (TA)0, up ? (TA)__ldg(x + j) : (TA)0, acc);
            acc = fmadd(lo ? (TA)__ldg(ck + m) : (TA)0, lo ? (TA)__ldg(x + m) : (TA)0, acc);
        }
        return acc;
    }
};

// A stencil whose coefficients are stored as FP16, divided by the level's largest coefficient
// magnitude `scale` so that they lie in [-1, 1] (11 significant bits, relative error at most
// 2^-11 for magnitudes above 2^-14 of the largest). The products of the fine levels read little
// but their coefficients, so these read about 0.6 of the bytes of the FP32 stencil. Each term is
// converted to TA and accumulated with the fused multiply-adds of StencilOp, in the same order;
// the sum is multiplied by `scale` at the end. KC > 0: K known at compile time; KC = 0: K read
// from the view. Both give the same bits, so the autotuner's choice changes no result.
struct StencilViewH {
    int n;
    int K;
    int ld;
    int off[MAXK];
    const __half* __restrict__ coef;
    float scale;
};

template <int KC>
struct StencilOpH {
    StencilViewH v;
    __device__ __forceinline__ int64_t threads() const { return v.n; }
    __device__ __forceinline__ bool valid(int64_t) const { return true; }
    template <class TA, class TX>
    __device__ __forceinline__ TA apply(int64_t g, const TX* __restrict__ x) const {
        const int i = (int)g, n = v.n;
        const __half* __restrict__ c = v.coef;
        const int K = KC > 0 ? KC : v.K;
        TA acc = (TA)__half2float(__ldg(c + i)) * (TA)__ldg(x + i);
#pragma unroll
        for (int k = 1; k < (KC > 0 ? KC : MAXK); ++k) {
            if (KC == 0 && k >= K) break;
            const int o = v.off[k];
            const __half* __restrict__ ck = c + (size_t)k * v.ld;
            const int j = i + o, m = i - o;
            const bool up = j < n, lo = m >= 0;
            acc = fmadd(up ? (TA)__half2float(__ldg(ck + i)) : (TA)0,
                        up ? (TA)__ldg(x + j) : (TA)0, acc);
            acc = fmadd(lo ? (TA)__half2float(__ldg(ck + m)) : (TA)0,
                        lo ? (TA)__ldg(x + m) : (TA)0, acc);
        }
        return acc * (TA)v.scale;
    }
};

}  // namespace femgpu

