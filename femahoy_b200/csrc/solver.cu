// The device solver (see solver.cuh).
//
// Per PCG iteration (multigrid.rs:721-751) the device runs: q = A p fused with p.q and
// alpha; x += alpha p, r -= alpha q fused with r.r and the convergence test; the V-cycle;
// r.z (and z.q) fused with beta; p = z + beta p. The scalars never leave the device; the host
// reads 1 small struct per iteration to apply the reference's stopping rules. Each iteration
// is 1 CUDA graph launch.
//
// The V-cycle (multigrid.rs:151-179 with the line Gauss-Seidel replaced by Chebyshev-Jacobi):
// `degree` Chebyshev steps from x = 0 (the first needs no matrix product), the residual, the
// restriction R = P^T (a gather), the coarser cycle, the prolongation and correction, and
// `degree` Chebyshev steps. The pre- and post-smoother are the same polynomial in D^-1 A, so
// the cycle is a symmetric positive definite preconditioner in exact arithmetic. The coarsest
// level is solved by its inverse, formed on the device from a dense Cholesky factor.
#include <algorithm>
#include <cmath>
#include <atomic>
#include <chrono>
#include <cstring>
#include <deque>
#include <array>
#include <map>
#include <mutex>
#include <optional>
#include <thread>
#include <type_traits>

#include <cooperative_groups.h>

#include "assemble.cuh"
#include "solver.cuh"
#include "coarsen.cuh"
#include "offsets.cuh"
#include "symbolic.hpp"
#include "rust_format.hpp"

namespace femgpu {

constexpr int TH = 256;
// The mixed form's stencil levels read FP16 coefficients unless the options say otherwise.
constexpr bool kHalfDefault = false;

static double bits_to_double(long long v) {
    double d;
    std::memcpy(&d, &v, sizeof d);
    return d;
}

// The grid that gives 1 thread to each of `rows` rows.
static int row_blocks(int64_t rows) {
    return (int)std::max<int64_t>(1, (rows + TH - 1) / TH);
}
constexpr double PIVOT = 1e-10;  // cholesky.rs:22

// Times a phase of the setup: the host time from its start until the solver's stream has
// finished the phase's device work.
struct PhaseTimer {
    SolverImpl* solver;
    const char* name;
    cudaStream_t s;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    PhaseTimer(SolverImpl* sv, const char* nm, cudaStream_t st) : solver(sv), name(nm), s(st) {}
    PhaseTimer(const PhaseTimer&) = delete;
    PhaseTimer& operator=(const PhaseTimer&) = delete;
    ~PhaseTimer() {
        cudaStreamSynchronize(s);
        solver->phase(name, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0)
                                .count());
    }
};

// ------------------------------------------------------------------ SELL build
__global__ void k_slice_entries(const int64_t* __restrict__ ptr, int64_t n, int C, int64_t ns,
                                int64_t* __restrict__ entries) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < ns;
         s += (int64_t)gridDim.x * blockDim.x) {
        int64_t w = 0;
        for (int r = 0; r < C; ++r) {
            int64_t i = s * C + r;
            if (i < n) w = max(w, ptr[i + 1] - ptr[i]);
        }
        entries[s] = ((w + 3) / 4) * 4 * C;
    }
}

template <class T>
__global__ void k_sell_fill(const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                            const double* __restrict__ val, int64_t n, int C, int64_t ns,
                            const int64_t* __restrict__ sptr, uint32_t* __restrict__ col,
                            T* __restrict__ sval) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ns * C;
         g += (int64_t)gridDim.x * blockDim.x) {
        int64_t s = g / C;
        int r = (int)(g % C);
        int64_t b = sptr[s], width = (sptr[s + 1] - b) / C;
        int64_t len = g < n ? ptr[g + 1] - ptr[g] : 0;
        int64_t at = g < n ? ptr[g] : 0;
        uint32_t self = g < n ? (uint32_t)g : 0u;
        for (int64_t k = 0; k < width; ++k) {
            int64_t off = b + 4 * ((k / 4) * C + r) + (k % 4);
            if (k < len) {
                col[off] = idx[at + k];
                sval[off] = (T)val[at + k];
            } else {
                col[off] = self;
                sval[off] = (T)0;
            }
        }
    }
}

template <class T>
void make_sell(const DevCsr& a, int C, Sell<T>* out, cudaStream_t s) {
    out->n = a.n;
    out->C = C;
    out->nslices = (a.n + C - 1) / C;
    DevBuf<int64_t> ent(out->nslices);
    k_slice_entries<<<blocks_for(out->nslices, TH), TH, 0, s>>>(a.ptr.p, a.n, C, out->nslices,
                                                                  ent.p);
    FG_CHECK_LAUNCH();
    out->slice_ptr.alloc(out->nslices + 1);
    exclusive_scan(ent.p, out->slice_ptr.p, out->nslices, s);
    out->entries = fetch(out->slice_ptr.p + out->nslices, s);
    out->col.alloc(out->entries);
    out->val.alloc(out->entries);
    k_sell_fill<T><<<blocks_for(out->nslices * C, TH), TH, 0, s>>>(
        a.ptr.p, a.idx.p, a.val.p, a.n, C, out->nslices, out->slice_ptr.p, out->col.p,
        out->val.p);
    FG_CHECK_LAUNCH();
}
template void make_sell<double>(const DevCsr&, int, Sell<double>*, cudaStream_t);
template void make_sell<float>(const DevCsr&, int, Sell<float>*, cudaStream_t);

// The stencil of a symmetric matrix whose entries sit at a few constant offsets col - row:
// coef[k ld + i] = a(i, i + o_k) for the offsets o_k >= 0, found and filled on the device
// (offsets.cuh). Refused (false) when there are more than MAXK such offsets, or when the slots
// would hold more than 1.5 times the upper entries.
template <class T>
static bool make_stencil(const DevCsr& d, Operator<T>* out, cudaStream_t s) {
    const int64_t n = d.n;
    OffsetScan sc;
    if (!scan_offsets(d.ptr.p, d.idx.p, n, true, MAXK, nullptr, &sc, s)) return false;
    const std::vector<int64_t>& offs = sc.offs;
    if (offs.empty() || offs[0] != 0) return false;
    // 32-bit row arithmetic in the kernels: n + the largest offset must fit.
    if (n + offs.back() >= (int64_t)0x7fffffff) return false;
    // A symmetric pattern has as many entries below the diagonal as above it.
    if (d.nnz - sc.upper != sc.upper - sc.diag) return false;
    const int K = (int)offs.size();
    if ((double)K * n > 1.5 * (double)sc.upper) return false;
    const int64_t ld = stencil_ld(n);
    if (ld + offs.back() >= (int64_t)0x7fffffff) return false;
    out->coef.alloc((size_t)K * ld);
    fill_offsets<T>(d.ptr.p, d.idx.p, d.val.p, n, true, nullptr, offs, ld, out->coef.p, s);
    out->stencil = true;
    out->n = n;
    out->nnz = d.nnz;
    out->K = K;
    out->ld = ld;
    out->off.assign(offs.begin(), offs.end());
    return true;
}

template <class T>
void make_operator(const DevCsr& d, int C, bool allow, Operator<T>* out, cudaStream_t s) {
    if (allow && make_stencil<T>(d, out, s)) return;
    out->stencil = false;
    out->n = d.n;
    out->nnz = d.nnz;
    // Elasticity levels (node-major unknowns, grid order): the 3x3-block form, 40 bytes per 9
    // FP32 entries instead of 72.
    if (allow && make_bsell3_device<T>(d, &out->b3ptr, &out->b3col, &out->b3val, s)) {
        out->block3 = true;
        return;
    }
    make_sell<T>(d, C, &out->sell, s);
}
template void make_operator<double>(const DevCsr&, int, bool, Operator<double>*, cudaStream_t);
template void make_operator<float>(const DevCsr&, int, bool, Operator<float>*, cudaStream_t);

// Calls f with the kernel-side view of the operator.
// The stencils of the box-grid hierarchies have K = 8 (the finest P1 level: the 15-point Kuhn
// stencil) and K = 14 (Galerkin levels: 27 points); these get unrolled kernels.
template <class T, class F>
static void with_op(const Operator<T>& op, F&& f) {
    if constexpr (std::is_same<T, float>::value) {
        if (op.half) {
            if (op.unrolled && op.K == 8)
                f(StencilOpH<8>{op.hview()});
            else if (op.unrolled && op.K == 14)
                f(StencilOpH<14>{op.hview()});
            else
                f(StencilOpH<0>{op.hview()});
            return;
        }
    }
    if (op.block3)
        f(Block3Op<T>{op.b3view(), (int)op.n});
    else if (!op.stencil)
        f(SellOp<T>{op.sell.view()});
    else if (op.unrolled && op.K == 8)
        f(StencilOpK<T, 8>{op.sview()});
    else if (op.unrolled && op.K == 14)
        f(StencilOpK<T, 14>{op.sview()});
    else
        f(StencilOp<T>{op.sview()});
}


// ------------------------------------------------------------------ V-cycle kernels
#define GRID_STRIDE(i, n)                                                     \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); \
         i += (int64_t)gridDim.x * blockDim.x)

// Kernels over the rows of an operator give each thread 1 row, numbered in 32 bits: with a
// 64-bit grid-stride loop around the same product, the finest stencil step took 1.6 times as
// long on B200.
__device__ __forceinline__ int row_of_thread() { return (int)(blockIdx.x * blockDim.x + threadIdx.x); }

// ------------------------------------------------------------------ V-cycle rows
// The work of 1 row of each V-cycle step, shared by the separate kernels below and by the fused
// kernel of the coarse levels (k_tail), so that both give the same bits. COH: the fused kernel's
// form, whose right sides and iterates it wrote itself before a grid-wide barrier, read through
// ldx<true> (L2, coherent) instead of the read-only path.

// The first Chebyshev step from x = 0: d = c1 D^-1 b, x = d.
template <class T, bool COH = false>
__device__ __forceinline__ void cheb_first_row(int i, const T* __restrict__ b,
                                               const T* __restrict__ dinv, T c1,
                                               T* __restrict__ d, T* __restrict__ x) {
    T v = c1 * dinv[i] * (COH ? ldx<true>(b + i) : b[i]);
    d[i] = v;
    x[i] = v;
}

// The Chebyshev update of 1 row from its product ax: d' = c2 d + c1 D^-1 (b - ax), with 1
// explicit fused multiply-add, so that every kernel that smooths (1 row or 2 per thread, tiles,
// the fused coarse levels) gives the same bits whatever the compiler contracts.
template <class T>
__device__ __forceinline__ T cheb_update(T bi, T ax, T di, T dprev, T c1, T c2) {
    const T r = bi - ax;
    return fmadd(c1 * di, r, c2 * dprev);
}

// A Chebyshev step: r = b - A x_in, d = c2 d + c1 D^-1 r, x_out = x_in + d.
template <class T, class Op, bool COH = false>
__device__ __forceinline__ void cheb_step_row(const Op& A, int g, const T* __restrict__ b,
                                              const T* __restrict__ xin,
                                              const T* __restrict__ dinv, T c1, T c2,
                                              T* __restrict__ d, T* __restrict__ xout) {
    T ax = A.template apply<T>(g, xin);
    if (!A.valid(g)) return;
    const T bg = COH ? ldx<true>(b + g) : b[g];
    const T dd = cheb_update(bg, ax, dinv[g], d[g], c1, c2);
    d[g] = dd;
    xout[g] = (COH ? ldx<true>(xin + g) : xin[g]) + dd;
}

template <class T, class Op, bool COH = false>
__device__ __forceinline__ void residual_row(const Op& A, int g, const T* __restrict__ b,
                                             const T* __restrict__ x, T* __restrict__ r) {
    T ax = A.template apply<T>(g, x);
    if (A.valid(g)) r[g] = (COH ? ldx<true>(b + g) : b[g]) - ax;
}

// Row i of a CSR transfer times x (multigrid.rs:166-172, sparse.rs:212-230).
template <class T, bool COH = false>
__device__ __forceinline__ T csr_row(int i, const int64_t* __restrict__ ptr,
                                     const uint32_t* __restrict__ idx, const T* __restrict__ val,
                                     const T* __restrict__ x) {
    const int e = (int)ptr[i + 1];
    T s = 0;
    for (int k = (int)ptr[i]; k < e; ++k) s += val[k] * ldx<COH>(x + idx[k]);
    return s;
}

// Row i of a transfer in offset form times x. KC > 0: K known at compile time (8 for P, 27 for
// R), so that all of a row's weight and x loads are in flight at once; KC = 0 reads K from the
// view. The terms are fused multiply-adds in increasing offset (= column) order either way.
template <class T, int KC, bool COH = false>
__device__ __forceinline__ T offset_row(const OffsetView<T>& M, int i, const T* __restrict__ x) {
    const int b = M.base[i];
    const int K = KC > 0 ? KC : M.K;
    T s = 0;
#pragma unroll
    for (int k = 0; k < (KC > 0 ? KC : MAXK); ++k) {
        if (KC == 0 && k >= K) break;
        const int j = b + M.off[k];
        const T w = __ldg(M.w + (size_t)k * M.rows + i);
        const T v = j < M.cols ? ldx<COH>(x + j) : (T)0;
        s = fmadd(w, v, s);
    }
    return s;
}

// Row i of x = M b for the n x n matrix M stored with leading dimension ld, by 1 warp (lane
// `lane`): 4 lane-strided partial sums, then a butterfly over the warp; every lane ends with the
// sum.
template <class T>
__device__ __forceinline__ T gemv_warp_row(const T* __restrict__ M, const T* __restrict__ b,
                                           int64_t n, int64_t ld, int64_t i, int lane) {
    const T* row = M + i * ld;
    T s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    int64_t k = lane;
    for (; k + 96 < n; k += 128) {
        s0 += row[k] * __ldg(b + k);
        s1 += row[k + 32] * __ldg(b + k + 32);
        s2 += row[k + 64] * __ldg(b + k + 64);
        s3 += row[k + 96] * __ldg(b + k + 96);
    }
    for (; k < n; k += 32) s0 += row[k] * __ldg(b + k);
    T s = (s0 + s1) + (s2 + s3);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// The leading dimension of a coarsest inverse: n rounded up to 32 elements, so that every row
// starts on a 128-byte boundary. The padding columns, and the coarse right side past n, are 0.
__host__ __device__ __forceinline__ int64_t dense_ld(int64_t n) { return (n + 31) / 32 * 32; }

template <class T>
struct Vec16;
template <>
struct Vec16<float> {
    typedef float4 type;
};
template <>
struct Vec16<double> {
    typedef double2 type;
};
__device__ __forceinline__ float dot_add(float4 m, float4 x, float s) {
    s += m.x * x.x;
    s += m.y * x.y;
    s += m.z * x.z;
    s += m.w * x.w;
    return s;
}
__device__ __forceinline__ double dot_add(double2 m, double2 x, double s) {
    s += m.x * x.x;
    s += m.y * x.y;
    return s;
}


// Row i of x = M b with M at leading dimension ld = dense_ld(n) and b padded to it with zeros,
// by all TH threads of a block: thread t takes the 16-byte chunks t, t + TH, ... of the row (4 in
// flight per thread, so a row of the 4,913-row coarsest level of the box grids is read in 1 or
// 2 round trips), 4 partial sums, a butterfly over each warp, then the warps' sums in order.
// Every thread of the block must call it; thread 0 returns the sum. `red` holds TH / 32 values.
template <class T, bool COH = false>
__device__ __forceinline__ T gemv_block_row(const T* __restrict__ M, const T* __restrict__ b,
                                            int64_t ld, int64_t i, T* red) {
    typedef typename Vec16<T>::type VT;
    const VT* row = reinterpret_cast<const VT*>(M + i * ld);
    const VT* bv = reinterpret_cast<const VT*>(b);
    const int nc = (int)(ld / (int64_t)(sizeof(VT) / sizeof(T)));
    T s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    int c = threadIdx.x;
    for (; c + 3 * TH < nc; c += 4 * TH) {
        const VT m0 = __ldg(row + c), m1 = __ldg(row + c + TH), m2 = __ldg(row + c + 2 * TH),
                 m3 = __ldg(row + c + 3 * TH);
        const VT x0 = ldx<COH>(bv + c), x1 = ldx<COH>(bv + c + TH), x2 = ldx<COH>(bv + c + 2 * TH),
                 x3 = ldx<COH>(bv + c + 3 * TH);
        s0 = dot_add(m0, x0, s0);
        s1 = dot_add(m1, x1, s1);
        s2 = dot_add(m2, x2, s2);
        s3 = dot_add(m3, x3, s3);
    }
    for (; c < nc; c += TH) s0 = dot_add(__ldg(row + c), ldx<COH>(bv + c), s0);
    T s = (s0 + s1) + (s2 + s3);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    T t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < TH / 32; ++w) t += red[w];
    __syncthreads();  // `red` is free for the next row
    return t;
}

template <class T>
__global__ void k_cheb_first(int64_t n, const T* __restrict__ b, const T* __restrict__ dinv, T c1,
                             T* __restrict__ d, T* __restrict__ x, const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    const int i = row_of_thread();
    if (i >= n) return;
    cheb_first_row(i, b, dinv, c1, d, x);
}

template <class T, class Op>
__global__ void __launch_bounds__(TH)
    k_cheb_step(Op A, const T* __restrict__ b, const T* __restrict__ xin,
                const T* __restrict__ dinv, T c1, T c2, T* __restrict__ d, T* __restrict__ xout,
                const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    const int g = row_of_thread();
    if (g >= A.threads()) return;
    cheb_step_row(A, g, b, xin, dinv, c1, c2, d, xout);
}

// r = b - A x
template <class T, class Op>
__global__ void __launch_bounds__(TH)
    k_residual(Op A, const T* __restrict__ b, const T* __restrict__ x, T* __restrict__ r,
               const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    const int g = row_of_thread();
    if (g >= A.threads()) return;
    residual_row(A, g, b, x, r);
}

// ------------------------------------------------------------------ 2 rows per thread
// The compile-time-K stencil with 2 adjacent rows (i0 even, i0 + 1) per thread: the arrays read
// once per row from DRAM (each row's own coefficients, x, b, D^-1 and d) come as 8- or 16-byte
// pairs, so a thread keeps twice the streamed bytes in flight per load; the neighbours (x at
// i +- o, the coefficients of the rows above, mostly cache hits) as predicated single loads, so
// that no branch stands between the loads and all of them issue before the first product. Each
// row's sum is StencilOpK's: the same fused multiply-adds in the same order, so the bits are
// those of the 1-row kernels.
template <class T>
struct Vec2;
template <>
struct Vec2<float> {
    typedef float2 type;
};
template <>
struct Vec2<double> {
    typedef double2 type;
};
template <class T>
__device__ __forceinline__ typename Vec2<T>::type ld2(const T* p) {
    return __ldg(reinterpret_cast<const typename Vec2<T>::type*>(p));
}
template <class T>
__device__ __forceinline__ void st2(T* p, T a, T b) {
    typename Vec2<T>::type v;
    v.x = a;
    v.y = b;
    *reinterpret_cast<typename Vec2<T>::type*>(p) = v;
}

// Rows i0 (even) and i0 + 1 < n of A x (TA: the accumulation type).
template <class T, int K, class TA, class TX>
__device__ __forceinline__ void stencil_pair(const StencilView<T>& v, int i0,
                                             const TX* __restrict__ x, TA& a0, TA& a1) {
    const int n = v.n;
    const T* __restrict__ c = v.coef;
    const auto cc = ld2(c + i0);
    const auto xx = ld2(x + i0);
    a0 = (TA)cc.x * (TA)xx.x;
    a1 = (TA)cc.y * (TA)xx.y;
#pragma unroll
    for (int k = 1; k < K; ++k) {
        const int o = v.off[k];
        const T* __restrict__ ck = c + (size_t)k * v.ld;
        const auto cu = ld2(ck + i0);  // in bounds: i0 + 1 < n <= ld
        const int j0 = i0 + o, m0 = i0 - o;
        const bool u0 = j0 < n, u1 = j0 + 1 < n, l0 = m0 >= 0, l1 = m0 + 1 >= 0;
        const TX xu0 = u0 ? __ldg(x + j0) : (TX)0, xu1 = u1 ? __ldg(x + j0 + 1) : (TX)0;
        const T cl0 = l0 ? __ldg(ck + m0) : (T)0, cl1 = l1 ? __ldg(ck + m0 + 1) : (T)0;
        const TX xl0 = l0 ? __ldg(x + m0) : (TX)0, xl1 = l1 ? __ldg(x + m0 + 1) : (TX)0;
        a0 = fmadd(u0 ? (TA)cu.x : (TA)0, (TA)xu0, a0);
        a0 = fmadd((TA)cl0, (TA)xl0, a0);
        a1 = fmadd(u1 ? (TA)cu.y : (TA)0, (TA)xu1, a1);
        a1 = fmadd((TA)cl1, (TA)xl1, a1);
    }
}

// Threads of the 2-row kernels: ceil(n / 2).
inline int64_t pair_threads(int64_t n) { return (n + 1) / 2; }

template <class T, int K>
__global__ void __launch_bounds__(TH)
    k_cheb_step_pair(StencilView<T> v, const T* __restrict__ b, const T* __restrict__ xin,
                     const T* __restrict__ dinv, T c1, T c2, T* __restrict__ d,
                     T* __restrict__ xout, const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    const int i0 = 2 * row_of_thread();
    if (i0 >= v.n) return;
    if (i0 + 1 == v.n) {  // the last row of an odd n
        cheb_step_row(StencilOpK<T, K>{v}, i0, b, xin, dinv, c1, c2, d, xout);
        return;
    }
    T a0, a1;
    stencil_pair<T, K, T, T>(v, i0, xin, a0, a1);
    const auto bb = ld2(b + i0), di = ld2(dinv + i0), dp = ld2(d + i0), xi = ld2(xin + i0);
    const T d0 = cheb_update(bb.x, a0, di.x, dp.x, c1, c2);
    const T d1 = cheb_update(bb.y, a1, di.y, dp.y, c1, c2);
    st2(d + i0, d0, d1);
    st2(xout + i0, xi.x + d0, xi.y + d1);
}

template <class T, int K>
__global__ void __launch_bounds__(TH)
    k_residual_pair(StencilView<T> v, const T* __restrict__ b, const T* __restrict__ x,
                    T* __restrict__ r, const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    const int i0 = 2 * row_of_thread();
    if (i0 >= v.n) return;
    if (i0 + 1 == v.n) {
        residual_row(StencilOpK<T, K>{v}, i0, b, x, r);
        return;
    }
    T a0, a1;
    stencil_pair<T, K, T, T>(v, i0, x, a0, a1);
    const auto bb = ld2(b + i0);
    st2(r + i0, bb.x - a0, bb.y - a1);
}

// ------------------------------------------------------------------ stencil tiles by bulk copy
// The finest level's Chebyshev steps and residuals with the row-own arrays streamed into shared
// memory. Each block of 1024 threads takes tiles of STENCIL_TILE rows, 1 row per thread. One
// thread issues 1D bulk copies (cp.async.bulk into the block's own shared memory) of the tile's
// K coefficient arrays, b, and for a step D^-1 and d, completing on an mbarrier; the next tile's
// copies run while this tile computes (2 stages). The rows' x neighbours, and the coefficients of rows
// above the tile, come from L1/L2 as in StencilOpK. The arithmetic is StencilOpK's and
// cheb_step_row's / residual_row's in the same order on the same values, so the bits are those
// of the kernels it replaces. A partial last tile reads global memory directly. Every wait on an
// mbarrier has an iteration limit: on running out, the kernel sets *timeout, waits (bounded) for
// its copies in flight and returns.
constexpr int BULK_TH = STENCIL_TILE;
constexpr unsigned BULK_SPIN = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(
                     smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes,
                                          uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for phase `parity` of `bar`, at most `limit` polls: false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned limit) {
    for (unsigned k = 0; k < limit; ++k)
        if (mbar_try(bar, parity)) return true;
    return false;
}

template <int K, bool STEP>
__global__ void __launch_bounds__(BULK_TH, 2)
    k_stencil_tiles(StencilView<float> v, const float* __restrict__ b,
                    const float* __restrict__ xin, const float* __restrict__ dinv, float c1,
                    float c2, float* __restrict__ d, float* __restrict__ out,
                    const int* __restrict__ done, int* __restrict__ timeout, unsigned spin) {
    constexpr int NA = K + (STEP ? 3 : 1);  // coefficients, b (, D^-1, d)
    constexpr unsigned TILE_BYTES = STENCIL_TILE * sizeof(float);
    extern __shared__ __align__(128) float tiles[];  // [2][NA][STENCIL_TILE]
    __shared__ uint64_t bar[2];
    pdl_wait();
    if (*done) return;
    const int n = v.n;
    const int nfull = n / STENCIL_TILE;
    const int ntiles = (n + STENCIL_TILE - 1) / STENCIL_TILE;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](int t, int s) {
        float* base = tiles + (size_t)s * NA * STENCIL_TILE;
        const size_t r0 = (size_t)t * STENCIL_TILE;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect(&bar[s], NA * TILE_BYTES);
#pragma unroll
        for (int k = 0; k < K; ++k)
            bulk_copy(base + k * STENCIL_TILE, v.coef + (size_t)k * v.ld + r0, TILE_BYTES,
                      &bar[s]);
        bulk_copy(base + K * STENCIL_TILE, b + r0, TILE_BYTES, &bar[s]);
        if (STEP) {
            bulk_copy(base + (K + 1) * STENCIL_TILE, dinv + r0, TILE_BYTES, &bar[s]);
            bulk_copy(base + (K + 2) * STENCIL_TILE, d + r0, TILE_BYTES, &bar[s]);
        }
    };
    // pending[s]: stage s has copies issued and not yet waited for, completing phase parity[s].
    int t = blockIdx.x;
    if (threadIdx.x == 0 && t < nfull) issue(t, 0);
    bool pending[2] = {t < nfull, false};
    unsigned parity[2] = {0, 0};
    int j = 0;
    for (; t < ntiles; t += gridDim.x, ++j) {
        const int s = j & 1;
        const int tn = t + gridDim.x;
        if (tn < nfull) {
            if (threadIdx.x == 0) issue(tn, s ^ 1);
            pending[s ^ 1] = true;
            parity[s ^ 1] = ((j + 1) >> 1) & 1;
        }
        const int r0 = t * STENCIL_TILE;
        const int i = r0 + threadIdx.x;
        const bool full = t < nfull;
        if (full) {
            const bool ok = mbar_wait(&bar[s], (j >> 1) & 1, spin);
            if (__syncthreads_or(!ok)) {
                if (threadIdx.x == 0) atomicExch(timeout, 1);
                break;
            }
            pending[s] = false;
        }
        const float* own = tiles + (size_t)s * NA * STENCIL_TILE;
        if (i < n) {
            const int li = threadIdx.x;
            const float* __restrict__ c = v.coef;
            // StencilOpK<float, K>::apply on the same values.
            float acc = (full ? own[li] : __ldg(c + i)) * __ldg(xin + i);
#pragma unroll
            for (int k = 1; k < K; ++k) {
                const int o = v.off[k];
                const float* __restrict__ ck = c + (size_t)k * v.ld;
                const int jj = i + o, m = i - o;
                const bool up = jj < n, lo = m >= 0;
                const float cu = up ? (full ? own[k * STENCIL_TILE + li] : __ldg(ck + i)) : 0.0f;
                acc = fmadd(cu, up ? __ldg(xin + jj) : 0.0f, acc);
                const float cl =
                    lo ? ((full && m >= r0) ? own[k * STENCIL_TILE + (m - r0)] : __ldg(ck + m))
                       : 0.0f;
                acc = fmadd(cl, lo ? __ldg(xin + m) : 0.0f, acc);
            }
            const float bi = full ? own[K * STENCIL_TILE + li] : b[i];
            if (STEP) {
                const float di = full ? own[(K + 1) * STENCIL_TILE + li] : dinv[i];
                const float dd0 = full ? own[(K + 2) * STENCIL_TILE + li] : d[i];
                const float dd = cheb_update(bi, acc, di, dd0, c1, c2);  // cheb_step_row
                d[i] = dd;
                out[i] = xin[i] + dd;
            } else {
                out[i] = bi - acc;  // residual_row
            }
        }
        __syncthreads();
    }
    // After a timeout: wait, again bounded (by the full limit, whatever `spin` was), for the
    // copies still in flight into this block's shared memory before the block exits.
    if (threadIdx.x == 0)
        for (int s = 0; s < 2; ++s)
            if (pending[s]) mbar_wait(&bar[s], parity[s], BULK_SPIN);
}

// ------------------------------------------------------------------ stencil planes, marching
// The stencil product of a box level with every gather from shared memory. The sorted offsets
// of a box grid in grid order fall into 2 groups around their largest gap: in-plane offsets
// (at most about 1 row of a plane, nx + 1) and cross-plane ones P + delta, where P is the first
// offset after the gap and 0 <= delta <= H. A block takes T consecutive rows j0 + t (t < T,
// j0 + t < P) of each plane of the frame of stride P (rows z P + j) and marches z over a chunk
// of planes. Shared memory holds the windows [j0 - H, j0 + T + H) of x of the planes z - 1, z,
// z + 1 and [j0 - H, j0 + T) of the K coefficient arrays of the planes z - 1 and z, each loaded
// as a plain range of rows: a window's rows past the plane's end are the next plane's, which is
// what the product reads there, and rows outside [0, n) load as 0. Row i = z P + j0 + t reads
// the upper terms' c_k[i] from plane z's window and x[i + o] from plane z's (in-plane o) or
// z + 1's (cross-plane) x window, the lower terms' c_k[i - o] and x[i - o] from plane z's or
// z - 1's windows. The next plane's windows and rows (b, D^-1, d) are loaded into registers
// while this plane computes. Each row's sum is StencilOpK's: the same fused multiply-adds in the
// same order, and a window's 0 at a missing neighbour is the 0 of StencilOpK's predicates (the
// coefficient of a missing neighbour is 0 too), so the bits are those of the 1-row kernels.
// Exact for any level whose in-plane offsets and cross-plane distances are at most H; the host
// builds the geometry (march_geometry) only when 2 H <= T.
// Threads per block at most: 1024 for the FP32 K = 8 kernels (52-62 registers), 512 for the
// others (their next-plane registers take up to 128 without spilling).
template <class T, int K>
constexpr int MARCH_TMAX = sizeof(T) == 4 && K == 8 ? 1024 : 512;

template <class T, int K>
__host__ __device__ inline size_t march_smem(int Tn, int H) {
    return ((size_t)3 * (Tn + 2 * H) + (size_t)2 * K * (Tn + H)) * sizeof(T);
}

template <class T, int K, bool STEP>
__global__ void __launch_bounds__(MARCH_TMAX<T, K>)
    k_stencil_march(StencilView<T> v, MarchGeom g, const T* __restrict__ b,
                    const T* __restrict__ xin, const T* __restrict__ dinv, T c1, T c2,
                    T* __restrict__ d, T* __restrict__ out, const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    extern __shared__ __align__(16) unsigned char march_raw[];
    T* const X = reinterpret_cast<T*>(march_raw);
    const int Tn = blockDim.x, H = g.H, t = threadIdx.x;
    const int WX = Tn + 2 * H, WC = Tn + H;
    T* const C = X + 3 * WX;
    const int j0 = (blockIdx.x % g.tiles) * Tn;
    const int z0 = (blockIdx.x / g.tiles) * g.chunk;
    const int z1 = min(z0 + g.chunk, g.planes);
    const int64_t n = v.n, P = g.P;
    const bool own = j0 + t < P;
    // Window loads: element t and t + Tn of the window that starts at row q P + j0 - H.
    auto load_x = [&](int q, T r[2]) {
        const int64_t base = (int64_t)q * P + j0 - H;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int idx = t + e * Tn;
            const int64_t gi = base + idx;
            r[e] = (idx < WX && gi >= 0 && gi < n) ? __ldg(xin + gi) : (T)0;
        }
    };
    auto store_x = [&](int q, const T r[2]) {
        T* dst = X + ((q + 3) % 3) * WX;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int idx = t + e * Tn;
            if (idx < WX) dst[idx] = r[e];
        }
    };
    auto load_c = [&](int q, T r[K][2]) {
        const int64_t base = (int64_t)q * P + j0 - H;
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int idx = t + e * Tn;
                const int64_t gi = base + idx;
                r[k][e] = (idx < WC && gi >= 0 && gi < n)
                              ? __ldg(v.coef + (size_t)k * v.ld + gi)
                              : (T)0;
            }
    };
    auto store_c = [&](int q, const T r[K][2]) {
        T* dst = C + ((q + 2) % 2) * K * WC;
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int idx = t + e * Tn;
                if (idx < WC) dst[k * WC + idx] = r[k][e];
            }
    };
    auto load_rows = [&](int q, T& bo, T& dio, T& dpo) {
        const int64_t i = (int64_t)q * P + j0 + t;
        const bool ok = own && i < n;
        bo = ok ? __ldg(b + i) : (T)0;
        dio = STEP && ok ? __ldg(dinv + i) : (T)0;
        dpo = STEP && ok ? d[i] : (T)0;
    };
    {
        T r[2];
        load_x(z0 - 1, r);
        store_x(z0 - 1, r);
        load_x(z0, r);
        store_x(z0, r);
        load_x(z0 + 1, r);
        store_x(z0 + 1, r);
        T c[K][2];
        load_c(z0 - 1, c);
        store_c(z0 - 1, c);
        load_c(z0, c);
        store_c(z0, c);
    }
    T bo, dio, dpo;
    load_rows(z0, bo, dio, dpo);
    __syncthreads();
    for (int z = z0; z < z1; ++z) {
        const bool more = z + 1 < z1;
        T px[2], pc[K][2], nb = 0, ndi = 0, ndp = 0;
        if (more) {
            load_x(z + 2, px);
            load_c(z + 1, pc);
            load_rows(z + 1, nb, ndi, ndp);
        }
        const int64_t i = (int64_t)z * P + j0 + t;
        if (own && i < n) {
            const T* X0 = X + (z % 3) * WX + H + t;
            const T* Xm = X + ((z + 2) % 3) * WX + H + t;
            const T* Xp = X + ((z + 1) % 3) * WX + H + t;
            const T* C0 = C + (z % 2) * K * WC + H + t;
            const T* Cm = C + ((z + 1) % 2) * K * WC + H + t;
            T acc = C0[0] * X0[0];
#pragma unroll
            for (int k = 1; k < K; ++k) {
                const int o = v.off[k];
                const T cu = C0[k * WC];
                T xu, cl, xl;
                if (k < g.s1) {
                    xu = X0[o];
                    cl = C0[k * WC - o];
                    xl = X0[-o];
                } else {
                    const int dl = o - g.P;
                    xu = Xp[dl];
                    cl = Cm[k * WC - dl];
                    xl = Xm[-dl];
                }
                acc = fmadd(cu, xu, acc);
                acc = fmadd(cl, xl, acc);
            }
            if (STEP) {
                const T dd = cheb_update(bo, acc, dio, dpo, c1, c2);
                d[i] = dd;
                out[i] = X0[0] + dd;
            } else {
                out[i] = bo - acc;
            }
        }
        __syncthreads();
        if (more) {
            store_x(z + 2, px);
            store_c(z + 1, pc);
            bo = nb;
            dio = ndi;
            dpo = ndp;
        }
        __syncthreads();
    }
}

// The plane frame of a stencil level for k_stencil_march, or false (not a K = 8 or 14 stencil,
// halo too wide, or shared memory too small). The threads per block: the plane's rows split
// evenly into blocks of at most 1024 (K = 8) or 512 (K = 14) rows; the chunk of planes per block
// such that all blocks are resident at once.
template <class T, int K>
static bool march_frame(const Operator<T>& op, MarchGeom* g) {
    const std::vector<int64_t>& o = op.off;  // sorted, o[0] = 0
    int gap = 0;
    for (int k = 1; k + 1 < K; ++k)
        if (o[k + 1] - o[k] > o[gap + 1] - o[gap]) gap = k;
    const int s1 = gap + 1;
    const int64_t P = o[s1];
    const int64_t H = std::max(o[s1 - 1], o[K - 1] - P);
    const int64_t tmax = MARCH_TMAX<T, K>;
    const int64_t tiles = (P + tmax - 1) / tmax;
    const int64_t Tn = ((P + tiles - 1) / tiles + 31) / 32 * 32;
    if (P >= 0x7fffffff || 2 * H > Tn || Tn > tmax) return false;
    const size_t smem = march_smem<T, K>((int)Tn, (int)H);
    if (smem > 227 * 1024) return false;
    FG_CUDA(cudaFuncSetAttribute(k_stencil_march<T, K, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FG_CUDA(cudaFuncSetAttribute(k_stencil_march<T, K, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, dev = 0, sms = 0;
    FG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stencil_march<T, K, true>,
                                                          (int)Tn, smem));
    FG_CUDA(cudaGetDevice(&dev));
    FG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1) return false;
    const int64_t planes = (op.n + P - 1) / P;
    const int64_t chunks = std::max<int64_t>(1, std::min<int64_t>(planes, (int64_t)per_sm * sms / tiles));
    g->P = (int)P;
    g->s1 = s1;
    g->H = (int)H;
    g->planes = (int)planes;
    g->chunk = (int)((planes + chunks - 1) / chunks);
    g->tiles = (int)tiles;
    g->T = (int)Tn;
    return true;
}

template <class T>
static bool march_geometry(const Operator<T>& op, MarchGeom* g) {
    if (!op.stencil || op.half) return false;
    if (op.K == 8) return march_frame<T, 8>(op, g);
    if (op.K == 14) return march_frame<T, 14>(op, g);
    return false;
}

// A Chebyshev step (STEP) or a residual by the marching kernel.
template <class T, bool STEP>
static void launch_march(bool pdl, const Operator<T>& op, cudaStream_t s, const T* b,
                         const T* xin, const T* dinv, T c1, T c2, T* d, T* out,
                         const int* done) {
    const MarchGeom& g = op.mg;
    const int grid = g.tiles * ((g.planes + g.chunk - 1) / g.chunk);
    if (op.K == 8)
        launch_smem(pdl, k_stencil_march<T, 8, STEP>, grid, g.T, march_smem<T, 8>(g.T, g.H), s,
                    op.sview(), g, b, xin, dinv, c1, c2, d, out, done);
    else
        launch_smem(pdl, k_stencil_march<T, 14, STEP>, grid, g.T, march_smem<T, 14>(g.T, g.H),
                    s, op.sview(), g, b, xin, dinv, c1, c2, d, out, done);
}

// bc = P^T r as a gather over the rows of R = P^T (multigrid.rs:166, sparse.rs:223-230).
template <class T>
__global__ void k_restrict(int64_t nc, const int64_t* __restrict__ ptr,
                           const uint32_t* __restrict__ idx, const T* __restrict__ val,
                           const T* __restrict__ r, T* __restrict__ bc,
                           const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    const int c = row_of_thread();
    if (c >= nc) return;
    bc[c] = csr_row(c, ptr, idx, val, r);
}

// x += P e (multigrid.rs:169-172, sparse.rs:212-220)
template <class T>
__global__ void k_prolong(int64_t nf, const int64_t* __restrict__ ptr,
                          const uint32_t* __restrict__ idx, const T* __restrict__ val,
                          const T* __restrict__ e, T* __restrict__ x,
                          const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    const int i = row_of_thread();
    if (i >= nf) return;
    x[i] += csr_row(i, ptr, idx, val, e);
}

// A transfer in offset form: out = M in, or out += M in (accumulate).
template <class T, int KC>
__global__ void __launch_bounds__(TH)
    k_transfer(OffsetView<T> M, const T* __restrict__ in, T* __restrict__ out, int accumulate,
               const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    const int i = row_of_thread();
    if (i >= M.rows) return;
    const T s = offset_row<T, KC>(M, i, in);
    if (accumulate)
        out[i] += s;
    else
        out[i] = s;
}

// The restriction into the next level's right side fused with that level's first smoothing step
// from x = 0 (cheb_first_row: d = c1 D^-1 b, x = d, on the value just stored): the same bits, 1
// launch less per level.
template <class T, int KC>
__global__ void __launch_bounds__(TH)
    k_restrict_first(OffsetView<T> M, const T* __restrict__ in, T* __restrict__ out,
                     const T* __restrict__ dinv, T c1, T* __restrict__ d, T* __restrict__ x,
                     const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    const int i = row_of_thread();
    if (i >= M.rows) return;
    const T s = offset_row<T, KC>(M, i, in);
    out[i] = s;
    const T v = c1 * dinv[i] * s;
    d[i] = v;
    x[i] = v;
}

template <class T>
static void launch_transfer(const OffsetTransfer<T>& M, const T* in, T* out, int accumulate,
                            const int* done, cudaStream_t s, bool pdl) {
    const int g = row_blocks(M.rows);
    const auto v = M.view();
    if (v.K == 8)
        launch(pdl, k_transfer<T, 8>, g, TH, s, v, in, out, accumulate, done);
    else if (v.K == 27)
        launch(pdl, k_transfer<T, 27>, g, TH, s, v, in, out, accumulate, done);
    else
        launch(pdl, k_transfer<T, 0>, g, TH, s, v, in, out, accumulate, done);
}

// x = M b for the symmetric n x n matrix M (a dense inverse) at leading dimension ld: 1 warp per
// row. PADDED: ld = dense_ld(n) and b padded to it (the coarsest level of a hierarchy, whose
// right side is the hierarchy's own padded vector); else scalar loads (the direct method, and a
// hierarchy of no smoothed level, whose right side is the caller's vector).
// A launch with programmatic dependent launch (pdl) and, if `win`, an L2 access policy window.
template <class... KArgs, class... Args>
static void launch_window(bool pdl, const cudaAccessPolicyWindow* win, void (*kernel)(KArgs...),
                          int grid, int block, cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = s;
    cudaLaunchAttribute attrs[2]{};
    unsigned na = 0;
    if (pdl) {
        attrs[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attrs[na].val.programmaticStreamSerializationAllowed = 1;
        ++na;
    }
    if (win) {
        attrs[na].id = cudaLaunchAttributeAccessPolicyWindow;
        attrs[na].val.accessPolicyWindow = *win;
        ++na;
    }
    cfg.attrs = na ? attrs : nullptr;
    cfg.numAttrs = na;
    FG_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

// The same row with M in FP16 (8 values per 16-byte chunk) against FP32 b: 8 products per
// chunk, the sums in FP32, times `scale` (M's largest entry, which the FP16 copy divides out).
__device__ __forceinline__ float gemv_block_row_half(const __half* __restrict__ M,
                                                     const float* __restrict__ b, int64_t ld,
                                                     int64_t i, float scale, float* red) {
    const uint4* row = reinterpret_cast<const uint4*>(M + i * ld);
    const float4* bv = reinterpret_cast<const float4*>(b);
    const int nc = (int)(ld / 8);
    float s0 = 0.f, s1 = 0.f;
    for (int c = threadIdx.x; c < nc; c += TH) {
        const uint4 m = __ldg(row + c);
        const float4 x0 = __ldg(bv + 2 * c), x1 = __ldg(bv + 2 * c + 1);
        const __half2* h = reinterpret_cast<const __half2*>(&m);
        const float2 a = __half22float2(h[0]), bb = __half22float2(h[1]),
                     cc = __half22float2(h[2]), dd = __half22float2(h[3]);
        s0 = fmaf(a.x, x0.x, s0);
        s1 = fmaf(a.y, x0.y, s1);
        s0 = fmaf(bb.x, x0.z, s0);
        s1 = fmaf(bb.y, x0.w, s1);
        s0 = fmaf(cc.x, x1.x, s0);
        s1 = fmaf(cc.y, x1.y, s1);
        s0 = fmaf(dd.x, x1.z, s0);
        s1 = fmaf(dd.y, x1.w, s1);
    }
    float s = s0 + s1;
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    float t = 0.f;
    if (threadIdx.x == 0)
        for (int w = 0; w < TH / 32; ++w) t += red[w];
    __syncthreads();
    return t * scale;
}

__global__ void __launch_bounds__(TH)
    k_gemv_rows_half(int64_t n, int64_t ld, const __half* __restrict__ M, float scale,
                     const float* __restrict__ b, float* __restrict__ x,
                     const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    __shared__ float red[TH / 32];
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
        const float s = gemv_block_row_half(M, b, ld, i, scale, red);
        if (threadIdx.x == 0) x[i] = s;
    }
}

// FP16 copy of a padded FP64 inverse divided by `scale` (its largest entry).
__global__ void k_half_of(int64_t n, int64_t ld, const double* __restrict__ a, double scale,
                          __half* __restrict__ h) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * ld;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / ld, j = t % ld;
        h[t] = __float2half_rn(j < n ? (float)(a[i * n + j] / scale) : 0.0f);
    }
}

__global__ void k_abs_max(int64_t n, const double* __restrict__ a, unsigned long long* out) {
    double m = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(a[t]));
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    // Non-negative doubles order as their bit patterns.
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// The coarsest product x = M b (padded M and b): 1 block per row at a time.
template <class T>
__global__ void __launch_bounds__(TH)
    k_gemv_rows(int64_t n, int64_t ld, const T* __restrict__ M, const T* __restrict__ b,
                T* __restrict__ x, const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    __shared__ T red[TH / 32];
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
        const T s = gemv_block_row(M, b, ld, i, red);
        if (threadIdx.x == 0) x[i] = s;
    }
}

template <class T>
__global__ void k_gemv(int64_t n, int64_t ld, const T* __restrict__ M, const T* __restrict__ b,
                       T* __restrict__ x, const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;
    int lane = threadIdx.x & 31;
    int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = w; i < n; i += nw) {
        T s = gemv_warp_row(M, b, n, ld, i, lane);
        if (lane == 0) x[i] = s;
    }
}

// ------------------------------------------------------------------ fused coarse levels
namespace cg = cooperative_groups;

constexpr int TAIL_MAXLEVELS = 8;
static_assert(sizeof(TailLevel<float>) % sizeof(int) == 0 &&
                  sizeof(TailLevel<double>) % sizeof(int) == 0,
              "the descriptors are copied to shared memory as ints");

// 1 smoothing step of a level of the fused kernel, over all its rows.
template <class T>
__device__ __forceinline__ void tail_smooth(const TailLevel<T>& L, const T* __restrict__ b,
                                            const T* xin, T* xout, T c1, T c2, int tid,
                                            int nth) {
    if (L.stencil) {
        const StencilRefOp<T, true> A{L.sv};
        for (int i = tid; i < L.n; i += nth) cheb_step_row<T, decltype(A), true>(A, i, b, xin, L.dinv, c1, c2, L.d, xout);
    } else {
        const SellRefOp<T, true> A{L.sell};
        for (int i = tid; i < L.n; i += nth) cheb_step_row<T, decltype(A), true>(A, i, b, xin, L.dinv, c1, c2, L.d, xout);
    }
}

// The V-cycle from the first fused level down to the coarsest and back, as 1 cooperative
// kernel: the steps of the separate kernels (the same row functions, so the same bits), each
// over all rows of its level, with a grid-wide barrier between steps. On the small levels a
// step is a few microseconds of launch and drain for well under a microsecond of work; here it
// costs 1 barrier.
template <class T>
__global__ void __launch_bounds__(TH)
    k_tail(const TailLevel<T>* __restrict__ Ls, int nl, const T* __restrict__ b0,
           const T* __restrict__ inv, int64_t nco, T* __restrict__ cx,
           const int* __restrict__ done) {
    if (*done) return;  // the same value in every block: all leave, or none
    // The levels' descriptors in shared memory, read by all threads of the block.
    __shared__ TailLevel<T> sL[TAIL_MAXLEVELS];
    {
        const int words = nl * (int)(sizeof(TailLevel<T>) / sizeof(int));
        const int* src = reinterpret_cast<const int*>(Ls);
        int* dst = reinterpret_cast<int*>(sL);
        for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = src[k];
        __syncthreads();
    }
    cg::grid_group grid = cg::this_grid();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    for (int l = 0; l < nl; ++l) {
        const TailLevel<T>& L = sL[l];
        const T* b = l == 0 ? b0 : L.b;
        T* xa = L.xa;
        T* xb = L.xb;
        for (int i = tid; i < L.n; i += nth) cheb_first_row<T, true>(i, b, L.dinv, L.c1[0], L.d, xa);
        grid.sync();
        for (int k = 1; k < L.deg; ++k) {
            tail_smooth(L, b, xa, xb, L.c1[k], L.c2[k], tid, nth);
            grid.sync();
            T* t = xa;
            xa = xb;
            xb = t;
        }
        if (L.stencil) {
            const StencilRefOp<T, true> A{L.sv};
            for (int i = tid; i < L.n; i += nth) residual_row<T, decltype(A), true>(A, i, b, xa, L.r);
        } else {
            const SellRefOp<T, true> A{L.sell};
            for (int i = tid; i < L.n; i += nth) residual_row<T, decltype(A), true>(A, i, b, xa, L.r);
        }
        grid.sync();
        for (int j = tid; j < L.nc; j += nth)
            L.bc[j] = L.r_offset ? offset_row<T, 0, true>(L.Ro, j, L.r)
                                 : csr_row<T, true>(j, L.rptr, L.ridx, L.rval, L.r);
        grid.sync();
    }
    {
        __shared__ T red[TH / 32];
        const T* bc = sL[nl - 1].bc;
        for (int64_t i = blockIdx.x; i < nco; i += gridDim.x) {
            const T s = gemv_block_row<T, true>(inv, bc, dense_ld(nco), i, red);
            if (threadIdx.x == 0) cx[i] = s;
        }
        grid.sync();
    }
    const T* e = cx;
    for (int l = nl - 1; l >= 0; --l) {
        const TailLevel<T>& L = sL[l];
        const T* b = l == 0 ? b0 : L.b;
        // Where the pre-smoothing left x: after deg - 1 swaps.
        T* xa = (L.deg - 1) % 2 ? L.xb : L.xa;
        T* xb = (L.deg - 1) % 2 ? L.xa : L.xb;
        for (int i = tid; i < L.n; i += nth)
            xa[i] += L.p_offset ? offset_row<T, 0, true>(L.Po, i, e)
                                : csr_row<T, true>(i, L.pptr, L.pidx, L.pval, e);
        grid.sync();
        for (int k = 0; k < L.deg; ++k) {
            tail_smooth(L, b, xa, xb, L.c1[k], L.c2[k], tid, nth);
            grid.sync();
            T* t = xa;
            xa = xb;
            xb = t;
        }
        e = xa;
    }
}

// ------------------------------------------------------------------ small levels by cluster
// A small level's down leg (the first step, the other pre-smoothing steps, the residual and the
// restriction into the next level's right side) or up leg (the prolongation and correction, the
// post-smoothing steps) as 1 launch of 1 thread-block cluster of CL_CTAS blocks: the blocks share
// the level's rows and meet at a cluster barrier (release and acquire at cluster scope) between
// steps, which costs well under the several microseconds of a kernel boundary. The steps are the
// separate kernels' row functions, so the bits are the same; the data that the launch writes and
// reads again go through coherent loads.
constexpr int CL_TH = 1024;

template <class T, bool UP>
__global__ void __launch_bounds__(CL_TH)
    k_level_cluster(TailLevel<T> L, const T* __restrict__ e, const int* __restrict__ done) {
    pdl_wait();
    if (*done) return;  // the same value in every block
    cg::cluster_group cluster = cg::this_cluster();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    const T* b = L.b;
    if (!UP) {
        T* xa = L.xa;
        T* xb = L.xb;
        for (int i = tid; i < L.n; i += nth) cheb_first_row<T, true>(i, b, L.dinv, L.c1[0], L.d, xa);
        cluster.sync();
        for (int k = 1; k < L.deg; ++k) {
            tail_smooth(L, b, xa, xb, L.c1[k], L.c2[k], tid, nth);
            cluster.sync();
            T* t = xa;
            xa = xb;
            xb = t;
        }
        if (L.stencil) {
            const StencilRefOp<T, true> A{L.sv};
            for (int i = tid; i < L.n; i += nth) residual_row<T, decltype(A), true>(A, i, b, xa, L.r);
        } else {
            const SellRefOp<T, true> A{L.sell};
            for (int i = tid; i < L.n; i += nth) residual_row<T, decltype(A), true>(A, i, b, xa, L.r);
        }
        cluster.sync();
        for (int j = tid; j < L.nc; j += nth)
            L.bc[j] = L.r_offset ? offset_row<T, 0, true>(L.Ro, j, L.r)
                                 : csr_row<T, true>(j, L.rptr, L.ridx, L.rval, L.r);
    } else {
        // Where the pre-smoothing left x: after deg - 1 swaps.
        T* xa = (L.deg - 1) % 2 ? L.xb : L.xa;
        T* xb = (L.deg - 1) % 2 ? L.xa : L.xb;
        for (int i = tid; i < L.n; i += nth)
            xa[i] = ldx<true>(xa + i) + (L.p_offset ? offset_row<T, 0, true>(L.Po, i, e)
                                                    : csr_row<T, true>(i, L.pptr, L.pidx,
                                                                       L.pval, e));
        cluster.sync();
        for (int k = 0; k < L.deg; ++k) {
            tail_smooth(L, b, xa, xb, L.c1[k], L.c2[k], tid, nth);
            if (k + 1 < L.deg) cluster.sync();
            T* t = xa;
            xa = xb;
            xb = t;
        }
    }
}

// The largest level that takes the cluster legs: 65,536 rows over 16 blocks of 1024 threads is
// 4 rows per thread and step.
constexpr int64_t CLUSTER_MAX_ROWS = 65536;

// The blocks of 1 cluster that the device schedules for k_level_cluster: 16 (a non-portable
// size, where a GPC has room) or 8; 0 if neither.
template <class T>
static int cluster_ctas() {
    for (int ctas : {16, 8}) {
        auto* kd = k_level_cluster<T, false>;
        auto* ku = k_level_cluster<T, true>;
        if (ctas > 8) {
            if (cudaFuncSetAttribute(kd, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                    cudaSuccess ||
                cudaFuncSetAttribute(ku, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                    cudaSuccess) {
                cudaGetLastError();
                continue;
            }
        }
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(ctas);
        cfg.blockDim = dim3(CL_TH);
        cudaLaunchAttribute attr{};
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = ctas;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        int nd = 0, nu = 0;
        if (cudaOccupancyMaxActiveClusters(&nd, kd, &cfg) == cudaSuccess &&
            cudaOccupancyMaxActiveClusters(&nu, ku, &cfg) == cudaSuccess && nd > 0 && nu > 0)
            return ctas;
        cudaGetLastError();
    }
    return 0;
}

// 1 leg of a small level as 1 cluster launch (with programmatic dependent launch if pdl).
template <class T, bool UP>
static void launch_cluster(bool pdl, int ctas, const TailLevel<T>& t, const T* e,
                           const int* done, cudaStream_t s) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(CL_TH);
    cfg.stream = s;
    cudaLaunchAttribute attrs[2]{};
    attrs[0].id = cudaLaunchAttributeClusterDimension;
    attrs[0].val.clusterDim.x = ctas;
    attrs[0].val.clusterDim.y = 1;
    attrs[0].val.clusterDim.z = 1;
    unsigned na = 1;
    if (pdl) {
        attrs[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attrs[1].val.programmaticStreamSerializationAllowed = 1;
        na = 2;
    }
    cfg.attrs = attrs;
    cfg.numAttrs = na;
    FG_CUDA(cudaLaunchKernelEx(&cfg, k_level_cluster<T, UP>, t, e, done));
}

// x += t
__global__ void k_add(int64_t n, const double* __restrict__ t, double* __restrict__ x) {
    GRID_STRIDE(i, n) x[i] += t[i];
}

template <class S, class D>
__global__ void k_convert(int64_t n, const S* __restrict__ a, D* __restrict__ b) {
    GRID_STRIDE(i, n) b[i] = (D)a[i];
}

// The n x n matrix a (row-major) into b at leading dimension ld, the padding columns 0.
template <class S, class D>
__global__ void k_convert_pad(int64_t n, int64_t ld, const S* __restrict__ a, D* __restrict__ b) {
    GRID_STRIDE(k, n * ld) {
        const int64_t i = k / ld, j = k % ld;
        b[k] = j < n ? (D)a[i * n + j] : (D)0;
    }
}

// ------------------------------------------------------------------ reductions
// A sum over rows is 2 launches: each block writes its partial sums (no fence, no atomic: on
// B200 the last-block-done pattern cost 5 times the product on 8,000 blocks), then k_finish
// sums the partials in block order (a deterministic result) and applies the scalar step.
__device__ __forceinline__ void block_partial(double a, double b, double* __restrict__ partial) {
    __shared__ double sa[TH / 32], sb[TH / 32];
    for (int o = 16; o; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sa[w] = a;
        sb[w] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0, tb = 0;
        for (int k = 0; k < TH / 32; ++k) {
            ta += sa[k];
            tb += sb[k];
        }
        partial[2 * blockIdx.x] = ta;
        partial[2 * blockIdx.x + 1] = tb;
    }
}

// The threads of a finishing block: 1024, so that the ~8,000 partial pairs of the finest level
// are read about 8 per thread with all loads in flight (1 L2 round trip instead of 32).
constexpr int FIN_TH = 1024;

template <class Fin>
__global__ void __launch_bounds__(FIN_TH) k_finish(const double* __restrict__ partial,
                                                    int nblocks, Fin fin) {
    pdl_wait();
    if (fin.skip()) return;
    __shared__ double sa[FIN_TH / 32], sb[FIN_TH / 32];
    const double2* pp = reinterpret_cast<const double2*>(partial);
    double a = 0, b = 0;
#pragma unroll 8
    for (int k = threadIdx.x; k < nblocks; k += FIN_TH) {
        const double2 v = pp[k];
        a += v.x;
        b += v.y;
    }
    for (int o = 16; o; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sa[w] = a;
        sb[w] = b;
    }
    __syncthreads();
    if (w == 0) {
        // The warps' sums by a second butterfly (a fixed order: the same bits every time).
        double ta = lane < FIN_TH / 32 ? sa[lane] : 0.0, tb = lane < FIN_TH / 32 ? sb[lane] : 0.0;
        for (int o = 16; o; o >>= 1) {
            ta += __shfl_xor_sync(0xffffffffu, ta, o);
            tb += __shfl_xor_sync(0xffffffffu, tb, o);
        }
        if (lane == 0) fin(ta, tb);
    }
}

// ------------------------------------------------------------------ PCG kernels (FP64)
struct FinResidual0 {
    Scalars* sc;
    __device__ bool skip() const { return false; }
    __device__ void operator()(double bb, double rr) const {
        sc->bb = bb;
        sc->norm_b = sqrt(bb);
        sc->rr = rr;
    }
};

// r = b - A x, with b.b and r.r; also the FP32 copy of r (mixed form).
template <class Op>
__global__ void __launch_bounds__(TH)
    k_pcg_residual(Op A, const double* __restrict__ b, const double* __restrict__ x,
                   double* __restrict__ r, float* __restrict__ r32, double* __restrict__ partial) {
    pdl_wait();
    double bb = 0, rr = 0;
    const int g = row_of_thread();
    if (g < A.threads()) {
        double ax = A.template apply<double>(g, x);
        if (A.valid(g)) {
            double bi = b[g], ri = bi - ax;
            r[g] = ri;
            if (r32) r32[g] = (float)ri;
            bb = bi * bi;
            rr = ri * ri;
        }
    }
    block_partial(bb, rr, partial);
}

struct FinPq {
    Scalars* sc;
    __device__ bool skip() const { return sc->done; }
    __device__ void operator()(double pq, double) const {
        sc->pq = pq;
        sc->alpha = sc->rz / pq;
    }
};

// q = A p with the partial sums of p.q (multigrid.rs:740-741; alpha in FinPq).
template <class Op>
__global__ void __launch_bounds__(TH)
    k_pcg_spmv_pq(Op A, const double* __restrict__ p, double* __restrict__ q,
                  double* __restrict__ partial, const Scalars* __restrict__ sc) {
    pdl_wait();
    if (sc->done) return;
    double pq = 0;
    const int g = row_of_thread();
    if (g < A.threads()) {
        double ap = A.template apply<double>(g, p);
        if (A.valid(g)) {
            q[g] = ap;
            pq = p[g] * ap;
        }
    }
    block_partial(pq, 0.0, partial);
}

// The same with 2 rows per thread (stencil_pair): the block of TH threads covers 2 TH rows and
// writes the partials of 2 blocks of the 1-row kernel, each summed in that kernel's order (the
// rows of a warp by the butterfly, then the warps in order), so the result is the same bits.
template <int K>
__global__ void __launch_bounds__(TH)
    k_pcg_spmv_pq_pair(StencilView<double> v, const double* __restrict__ p,
                       double* __restrict__ q, double* __restrict__ partial,
                       const Scalars* __restrict__ sc) {
    pdl_wait();
    if (sc->done) return;
    __shared__ double prod[2 * TH];
    __shared__ double sw[2][TH / 32];
    const int i0 = 2 * row_of_thread();
    double pq0 = 0, pq1 = 0;
    if (i0 + 1 < v.n) {
        double a0, a1;
        stencil_pair<double, K, double, double>(v, i0, p, a0, a1);
        const double2 pp = ld2(p + i0);
        st2(q + i0, a0, a1);
        pq0 = pp.x * a0;
        pq1 = pp.y * a1;
    } else if (i0 < v.n) {
        const double a0 = StencilOpK<double, K>{v}.template apply<double>(i0, p);
        q[i0] = a0;
        pq0 = p[i0] * a0;
    }
    prod[2 * threadIdx.x] = pq0;
    prod[2 * threadIdx.x + 1] = pq1;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int half = 0; half < 2; ++half) {
        double a = prod[half * TH + threadIdx.x];
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) sw[half][w] = a;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        const int64_t blk = 2 * (int64_t)blockIdx.x + threadIdx.x;
        if (blk * TH < v.n) {
            double t = 0;
            for (int k = 0; k < TH / 32; ++k) t += sw[threadIdx.x][k];
            partial[2 * blk] = t;
            partial[2 * blk + 1] = 0.0;
        }
    }
}

struct FinUpdate {
    Scalars* sc;
    double tol;
    __device__ bool skip() const { return sc->done; }
    __device__ void operator()(double rr, double) const {
        sc->rr = rr;
        sc->iters += 1;
        // multigrid.rs:722-723: |r| / |b| <= tol, on the updated residual.
        if (sqrt(rr) / sc->norm_b <= tol) sc->done = 1;
    }
};

// x += alpha p, r -= alpha q (multigrid.rs:742-745), with the partial sums of r.r.
__global__ void __launch_bounds__(TH)
    k_pcg_update(int64_t n, double* __restrict__ x, double* __restrict__ r,
                 const double* __restrict__ p, const double* __restrict__ q,
                 float* __restrict__ r32, double* __restrict__ partial,
                 const Scalars* __restrict__ sc) {
    pdl_wait();
    if (sc->done) return;
    const double alpha = sc->alpha;
    double rr = 0;
    const int i = row_of_thread();
    if (i < n) {
        x[i] += alpha * p[i];
        double ri = r[i] - alpha * q[i];
        r[i] = ri;
        if (r32) r32[i] = (float)ri;
        rr = ri * ri;
    }
    block_partial(rr, 0.0, partial);
}

struct FinDots {
    Scalars* sc;
    int flexible, init;
    __device__ bool skip() const { return sc->done; }
    __device__ void operator()(double rz, double zq) const {
        if (init) {
            sc->beta = 0;
        } else if (flexible) {
            // Flexible CG (Y. Notay, Flexible conjugate gradients, SIAM J. Sci. Comput. 22 (2000)
            // 1444-1460): beta = z_new.(r_new - r_old) / rz_old = -alpha z_new.q / rz_old.
            sc->beta = -sc->alpha * zq / sc->rz;
        } else {
            sc->beta = rz / sc->rz;  // multigrid.rs:747-748
        }
        sc->rz = rz;
        sc->zq = zq;
    }
};

template <class TZ>
__global__ void __launch_bounds__(TH)
    k_pcg_dots(int64_t n, const double* __restrict__ r, const TZ* __restrict__ z,
               const double* __restrict__ q, int flexible, int init,
               double* __restrict__ partial, const Scalars* __restrict__ sc) {
    pdl_wait();
    if (sc->done) return;
    double rz = 0, zq = 0;
    const int i = row_of_thread();
    if (i < n) {
        double zi = (double)z[i];
        rz = r[i] * zi;
        if (flexible && !init) zq = zi * q[i];
    }
    block_partial(rz, zq, partial);
}

// p = z + beta p (multigrid.rs:749-751); p = z on the first call.
template <class TZ>
__global__ void k_pcg_p(int64_t n, const TZ* __restrict__ z, double* __restrict__ p,
                        const Scalars* sc, int init) {
    pdl_wait();
    if (sc->done) return;
    const double beta = sc->beta;
    const int i = row_of_thread();
    if (i >= n) return;
    p[i] = init ? (double)z[i] : (double)z[i] + beta * p[i];
}

// The end of a device-side PCG iteration: continue unless the solve converged, reached its
// iteration limit, broke down (a NaN residual) or was cancelled (multigrid.rs:721-738, in the
// same order of tests).
__global__ void k_loop_control(cudaGraphConditionalHandle h, const Scalars* sc,
                               const volatile int* cancel) {
    double rr = sc->rr;
    bool go = !sc->done && sc->iters < sc->max_iter && rr == rr && !*cancel && !sc->bulk_timeout;
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// ------------------------------------------------------------------ power iteration
struct FinTwo {
    double* out;
    __device__ bool skip() const { return false; }
    __device__ void operator()(double a, double b) const {
        out[0] = a;
        out[1] = b;
    }
};

// w = D^-1 A v; partial sums of v.Av and v.Dv (the Rayleigh quotient of D^-1 A in the D inner
// product).
template <class Op>
__global__ void __launch_bounds__(TH)
    k_power_step(Op A, const double* __restrict__ v, const double* __restrict__ dg,
                 double* __restrict__ w, double* __restrict__ partial) {
    double vav = 0, vdv = 0;
    const int g = row_of_thread();
    if (g < A.threads()) {
        double av = A.template apply<double>(g, v);
        if (A.valid(g)) {
            vav = v[g] * av;
            vdv = v[g] * dg[g] * v[g];
            w[g] = av / dg[g];
        }
    }
    block_partial(vav, vdv, partial);
}

__global__ void __launch_bounds__(TH)
    k_norm2(int64_t n, const double* __restrict__ w, double* __restrict__ partial) {
    double s = 0;
    const int i = row_of_thread();
    if (i < n) s = w[i] * w[i];
    block_partial(s, 0.0, partial);
}

__global__ void k_scale_into(int64_t n, const double* __restrict__ w, const double* __restrict__ nrm,
                             double* __restrict__ v) {
    double f = 1.0 / sqrt(nrm[0]);
    GRID_STRIDE(i, n) v[i] = w[i] * f;
}

__global__ void k_seed(int64_t n, double* __restrict__ v) {
    GRID_STRIDE(i, n) {
        uint32_t x = (uint32_t)i * 2654435761u + 12345u;
        x ^= x >> 16;
        x *= 0x7feb352dU;
        x ^= x >> 15;
        v[i] = 0.5 + (double)(x & 0xffffff) / (double)0x1000000;
    }
}

__global__ void k_diagonal(int64_t n, const int64_t* __restrict__ ptr,
                           const uint32_t* __restrict__ idx, const double* __restrict__ val,
                           double* __restrict__ dg, int* __restrict__ bad) {
    GRID_STRIDE(i, n) {
        double d = 0;
        for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
            if (idx[k] == (uint32_t)i) d = val[k];
        dg[i] = d;
        if (!(d > 0.0)) atomicExch(bad, 1);
    }
}

// ------------------------------------------------------------------ helpers
// (The dense Cholesky factor and inverse of the direct method and the coarsest level are in
// dense_factor.cu.)
void upload_csr(const HostCsr& h, DevCsr* d, cudaStream_t s) {
    d->n = h.n;
    d->nnz = h.nnz();
    d->ptr.upload(h.ptr.data(), h.n + 1, s);
    d->idx.upload(h.idx.data(), h.nnz(), s);
    d->val.upload(h.val.data(), h.nnz(), s);
}

HostCsr download_csr(const DevCsr& d, cudaStream_t s) {
    HostCsr h;
    h.n = d.n;
    h.ptr.resize(d.n + 1);
    h.idx.resize(d.nnz);
    h.val.resize(d.nnz);
    d.ptr.download(h.ptr.data(), d.n + 1, s);
    d.idx.download(h.idx.data(), d.nnz, s);
    d.val.download(h.val.data(), d.nnz, s);
    FG_CUDA(cudaStreamSynchronize(s));
    return h;
}

HostRect transpose(const HostRect& p) {
    HostRect r;
    r.rows = p.cols;
    r.cols = p.rows;
    r.ptr.assign(p.cols + 1, 0);
    for (uint32_t j : p.idx) r.ptr[j + 1] += 1;
    for (int64_t j = 0; j < p.cols; ++j) r.ptr[j + 1] += r.ptr[j];
    r.idx.resize(p.idx.size());
    r.val.resize(p.idx.size());
    std::vector<int64_t> next(r.ptr.begin(), r.ptr.end() - 1);
    for (int64_t i = 0; i < p.rows; ++i)
        for (int64_t k = p.ptr[i]; k < p.ptr[i + 1]; ++k) {
            uint32_t j = p.idx[k];
            r.idx[next[j]] = (uint32_t)i;
            r.val[next[j]] = p.val[k];
            next[j]++;
        }
    return r;
}


// The FP16 copy of a stencil's coefficients (StencilOpH): each divided by the largest
// magnitude and rounded to nearest. The FP32 coefficients stay for the fused coarse kernel.
static void make_half(Operator<float>* op, cudaStream_t s) {
    std::vector<float> c = op->coef.to_host(s);
    float m = 0.0f;
    for (float v : c) m = std::max(m, std::fabs(v));
    if (!(m > 0.0f) || !std::isfinite(m)) return;
    std::vector<__half> h(c.size());
    for (size_t k = 0; k < c.size(); ++k) h[k] = __float2half_rn(c[k] / m);
    op->hcoef.upload(h.data(), h.size(), s);
    FG_CUDA(cudaStreamSynchronize(s));
    op->hscale = m;
    op->half = true;
}

// The autotuner's choice for a stencil operator: times y = b - A x with the runtime-K and the
// compile-time-K kernels (5 launches each after 2 warm-up launches, CUDA events) and keeps the
// faster. The choice depends on the level's size and on how the L2 serves its offsets.
// ------------------------------------------------------------------ the autotuner
// The autotuner's choices per size class, kept for the process: the first operator (or solver)
// of a class is timed, and later ones of the same class take its choice without timing, so the
// solvers of one class also choose alike. A class is (what is tuned, the element size, the
// operator's kind, log2 of its rows, its entries per row).
namespace {
std::mutex g_tune_mutex;
std::map<std::array<int64_t, 5>, int> g_tune;

int64_t log2_of(int64_t n) {
    int64_t b = 0;
    while ((int64_t)1 << (b + 1) <= n) ++b;
    return b;
}

bool tune_lookup(const std::array<int64_t, 5>& key, int* value) {
    std::lock_guard<std::mutex> g(g_tune_mutex);
    auto it = g_tune.find(key);
    if (it == g_tune.end()) return false;
    *value = it->second;
    return true;
}

void tune_store(const std::array<int64_t, 5>& key, int value) {
    std::lock_guard<std::mutex> g(g_tune_mutex);
    g_tune[key] = value;
}
}  // namespace

// The best mean device time (ms) of `launch` over `rounds` rounds of 5, after `warm` launches
// (the clocks may still be rising after host work).
template <class F>
static double time_best(F&& launch, int warm, int rounds, cudaStream_t s) {
    cudaEvent_t e0, e1;
    FG_CUDA(cudaEventCreate(&e0));
    FG_CUDA(cudaEventCreate(&e1));
    for (int w = 0; w < warm; ++w) launch();
    FG_CHECK_LAUNCH();
    double best = 1e30;
    for (int round = 0; round < rounds; ++round) {
        FG_CUDA(cudaEventRecord(e0, s));
        for (int k = 0; k < 5; ++k) launch();
        FG_CUDA(cudaEventRecord(e1, s));
        FG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        FG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, (double)ms / 5);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

// A stencil level: the runtime-K or the compile-time-K product kernel (the same bits), by timing
// the residual.
template <class T>
static void tune_operator(Operator<T>* op, int force, cudaStream_t s) {
    if (!op->stencil || (op->K != 8 && op->K != 14)) return;
    if (force > 0) {
        // The kernel asked for, or the next lower one that the level can take.
        op->march = force >= 4 && march_geometry(*op, &op->mg);
        op->pair = !op->march && force >= 3 && !op->half;
        op->unrolled = force >= 2;
        return;
    }
    const std::array<int64_t, 5> key{0, (int64_t)sizeof(T), op->K, log2_of(op->n), op->half};
    int v = 0;
    if (tune_lookup(key, &v)) {
        op->unrolled = v != 0;
        op->pair = v == 2;
        op->march = v == 3 && march_geometry(*op, &op->mg);
        return;
    }
    int64_t n = op->n;
    DevBuf<T> x(n), b(n), r(n);
    x.zero(s);
    b.zero(s);
    DevBuf<int> done(1);
    done.zero(s);
    int gs = row_blocks(n);
    op->pair = false;
    for (int variant = 0; variant < 2; ++variant)
        op->probe_ms[variant] = time_best(
            [&] {
                op->unrolled = variant == 1;
                with_op(*op, [&](auto o) {
                    k_residual<T><<<gs, TH, 0, s>>>(o, b.p, x.p, r.p, done.p);
                });
            },
            variant == 0 ? 20 : 5, 3, s);
    // The 2-row kernels (FP16 coefficients have none).
    op->probe_ms[3] = 1e30;
    if (!op->half) {
        const StencilView<T> sv = op->sview();
        const int gp = row_blocks(pair_threads(n));
        op->probe_ms[3] = time_best(
            [&] {
                if (op->K == 8)
                    k_residual_pair<T, 8><<<gp, TH, 0, s>>>(sv, b.p, x.p, r.p, done.p);
                else
                    k_residual_pair<T, 14><<<gp, TH, 0, s>>>(sv, b.p, x.p, r.p, done.p);
            },
            5, 3, s);
    }
    // The plane-marching kernels.
    op->probe_ms[4] = 1e30;
    op->march = false;
    if (march_geometry(*op, &op->mg)) {
        op->probe_ms[4] = time_best(
            [&] {
                launch_march<T, false>(false, *op, s, b.p, x.p, nullptr, (T)0, (T)0, nullptr,
                                       r.p, done.p);
            },
            5, 3, s);
    }
    const double best =
        std::min({op->probe_ms[0], op->probe_ms[1], op->probe_ms[3], op->probe_ms[4]});
    op->march = op->probe_ms[4] == best;
    op->pair = !op->march && op->probe_ms[3] == best;
    op->unrolled = op->march || op->pair || op->probe_ms[1] == best;
    tune_store(key, op->march ? 3 : op->pair ? 2 : op->unrolled ? 1 : 0);
}

// A SELL level: the rows per slice (C = 16, 32 or 64; a warp reads 1 slice of 32 rows, 2 of 16,
// or half of one of 64), by timing the residual of each form.
template <class T>
static void tune_sell(const DevCsr& d, Operator<T>* op, cudaStream_t s) {
    if (op->stencil || op->block3) return;
    const int64_t per_row = op->n ? (op->nnz + op->n / 2) / op->n : 0;
    const std::array<int64_t, 5> key{1, (int64_t)sizeof(T), 0, log2_of(op->n), per_row};
    int C = 0;
    if (tune_lookup(key, &C)) {
        if (C != op->sell.C) make_sell<T>(d, C, &op->sell, s);
        return;
    }
    int64_t n = op->n;
    DevBuf<T> x(n), b(n), r(n);
    x.zero(s);
    b.zero(s);
    DevBuf<int> done(1);
    done.zero(s);
    double best = 1e30;
    int bestC = op->sell.C;
    for (int c : {16, 32, 64}) {
        Sell<T> trial;
        make_sell<T>(d, c, &trial, s);
        const SellOp<T> o{trial.view()};
        const int gs = row_blocks(trial.nslices * trial.C);
        const double ms = time_best(
            [&] { k_residual<T><<<gs, TH, 0, s>>>(o, b.p, x.p, r.p, done.p); }, 5, 3, s);
        if (ms < best) {
            best = ms;
            bestC = c;
        }
    }
    if (bestC != op->sell.C) make_sell<T>(d, bestC, &op->sell, s);
    FG_CUDA(cudaStreamSynchronize(s));
    tune_store(key, bestC);
}

// The launch of the tile kernels: persistent blocks, 2 per SM, 2 stages of NA tiles each.
template <bool STEP>
static size_t tile_smem() {
    return 2 * (size_t)(8 + (STEP ? 3 : 1)) * STENCIL_TILE * sizeof(float);
}
static int tile_grid(int64_t n) {
    int64_t tiles = (n + STENCIL_TILE - 1) / STENCIL_TILE;
    return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, 2 * NUM_SMS));
}
static void tile_attributes() {
    static bool done = false;
    if (done) return;
    FG_CUDA(cudaFuncSetAttribute(k_stencil_tiles<8, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_smem<true>()));
    FG_CUDA(cudaFuncSetAttribute(k_stencil_tiles<8, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_smem<false>()));
    done = true;
}

// Whether a finest FP32 stencil level (K = 8, large enough to fill the GPU with tiles) takes the
// tile kernels: mode 2 yes, mode 1 no, mode 0 when its residual by tiles is faster than by the
// kernel the autotuner chose (the same timing as tune_operator). A probe whose copies time out
// keeps the direct kernels.
static void tune_tiles(Operator<float>* op, int mode, cudaStream_t s) {
    op->bulk = false;
    if (mode == 1 || !op->stencil || op->half || op->K != 8) return;
    int64_t n = op->n;
    if (n < (int64_t)STENCIL_TILE * NUM_SMS) return;
    tile_attributes();
    DevBuf<float> x(n), b(n), r(n);
    x.zero(s);
    b.zero(s);
    DevBuf<int> done(1), timeout(1);
    done.zero(s);
    timeout.zero(s);
    const StencilView<float> v = op->sview();
    auto probe = [&]() {
        k_stencil_tiles<8, false><<<tile_grid(n), BULK_TH, tile_smem<false>(), s>>>(
            v, b.p, x.p, nullptr, 0.f, 0.f, nullptr, r.p, done.p, timeout.p, BULK_SPIN);
    };
    cudaEvent_t e0, e1;
    FG_CUDA(cudaEventCreate(&e0));
    FG_CUDA(cudaEventCreate(&e1));
    for (int w = 0; w < 10; ++w) probe();
    FG_CHECK_LAUNCH();
    double best = 1e30;
    for (int round = 0; round < 4; ++round) {
        FG_CUDA(cudaEventRecord(e0, s));
        for (int k = 0; k < 5; ++k) probe();
        FG_CUDA(cudaEventRecord(e1, s));
        FG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        FG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, (double)ms / 5);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    op->probe_ms[2] = best;
    if (fetch(timeout.p, s)) return;
    const double direct = op->march  ? op->probe_ms[4]
                          : op->pair   ? op->probe_ms[3]
                          : op->unrolled ? op->probe_ms[1]
                                         : op->probe_ms[0];
    op->bulk = mode == 2 || best < direct;
}

// lambda_max of D^-1 A by the power method in the D inner product (15 steps), on the device.
template <class T>
double lambda_max(const Operator<T>& A, const double* dg, cudaStream_t s,
                  DevBuf<double>& partial) {
    int64_t n = A.n;
    // out[0..1]: v.Av and v.Dv of this step; out[2..3]: |w|^2 (and an unused 0).
    DevBuf<double> v(n), w(n), out(4);
    k_seed<<<blocks_for(n, TH), TH, 0, s>>>(n, v.p);
    double lam = 0;
    for (int it = 0; it < 15; ++it) {
        const int nb = row_blocks(A.threads()), nv = row_blocks(n);
        with_op(A, [&](auto op) {
            k_power_step<<<nb, TH, 0, s>>>(op, v.p, dg, w.p, partial.p);
        });
        k_finish<<<1, FIN_TH, 0, s>>>(partial.p, nb, FinTwo{out.p});
        k_norm2<<<nv, TH, 0, s>>>(n, w.p, partial.p);
        k_finish<<<1, FIN_TH, 0, s>>>(partial.p, nv, FinTwo{out.p + 2});
        k_scale_into<<<blocks_for(n, TH), TH, 0, s>>>(n, w.p, out.p + 2, v.p);
        FG_CHECK_LAUNCH();
        if (it >= 12) {
            double h[2];
            FG_CUDA(cudaMemcpyAsync(h, out.p, 16, cudaMemcpyDeviceToHost, s));
            FG_CUDA(cudaStreamSynchronize(s));
            lam = std::max(lam, h[0] / h[1]);
        }
    }
    return lam;
}
template double lambda_max<double>(const Operator<double>&, const double*, cudaStream_t,
                                   DevBuf<double>&);
template double lambda_max<float>(const Operator<float>&, const double*, cudaStream_t,
                                  DevBuf<double>&);

void chebyshev(double lam, int degree, double lower, std::vector<double>* c1,
               std::vector<double>* c2, int kind, double upper) {
    if (!(upper > 0.0)) upper = 1.1;
    if (kind == 4) {
        // The fourth-kind Chebyshev smoother on [0, 1.1] x lambda_max of D^-1 A (J. Lottes,
        // Optimal polynomial smoothers for multigrid V-cycles, Numer. Linear Algebra Appl. 30
        // (2023) e2518): d_0 = 4 / (3 l) D^-1 r_0, d_k = (2k - 1) / (2k + 3) d_(k-1)
        // + (8k + 4) / ((2k + 3) l) D^-1 r_k.
        const double l = upper * lam;
        c1->assign(degree, 0.0);
        c2->assign(degree, 0.0);
        (*c1)[0] = 4.0 / (3.0 * l);
        for (int k = 1; k < degree; ++k) {
            (*c2)[k] = (2.0 * k - 1.0) / (2.0 * k + 3.0);
            (*c1)[k] = (8.0 * k + 4.0) / ((2.0 * k + 3.0) * l);
        }
        return;
    }
    // Y. Saad, Iterative Methods for Sparse Linear Systems, 2nd ed., SIAM 2003, algorithm 12.1,
    // on the interval [lower, 1.1] x lambda_max of D^-1 A.
    double hi = upper * lam, lo = lower * lam;
    double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
    c1->assign(degree, 0.0);
    c2->assign(degree, 0.0);
    (*c1)[0] = 1.0 / theta;
    double rho = 1.0 / sigma;
    for (int k = 1; k < degree; ++k) {
        double rn = 1.0 / (2.0 * sigma - rho);
        (*c2)[k] = rn * rho;
        (*c1)[k] = 2.0 * rn / delta;
        rho = rn;
    }
}

// ------------------------------------------------------------------ SolverImpl
SolverImpl::SolverImpl() {
    FG_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
    FG_CUDA(cudaEventCreate(&ev0_));
    FG_CUDA(cudaEventCreate(&ev1_));
    partial_.alloc(2 * 1024);
    counter_.alloc(1);
    counter_.zero(s_);
    sc_.alloc(1);
    done_zero_.alloc(1);
    done_zero_.zero(s_);
    FG_CUDA(cudaMallocHost(&h_sc_, sizeof(Scalars)));
    FG_CUDA(cudaHostAlloc(&h_cancel_, sizeof(int), cudaHostAllocMapped));
    *h_cancel_ = 0;
    FG_CUDA(cudaHostGetDevicePointer(&d_cancel_, h_cancel_, 0));
}

SolverImpl::~SolverImpl() {
    if (l2_window_) cudaCtxResetPersistingL2Cache();
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (h_sc_) cudaFreeHost(h_sc_);
    if (h_cancel_) cudaFreeHost(h_cancel_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (s_) {
        cudaStreamSynchronize(s_);
        cudaStreamDestroy(s_);
    }
}

template <class T>
size_t Hierarchy<T>::bytes() const {
    size_t b = inv.bytes() + hinv.bytes() + cb.bytes() + cx.bytes() + cb64.bytes() + cx64.bytes() +
               (sparse ? sparse->bytes() : 0);
    for (const auto& l : levels)
        b += l.A.bytes() + l.dinv.bytes() + l.pptr.bytes() + l.rptr.bytes() + l.pidx.bytes() +
             l.ridx.bytes() + l.pval.bytes() + l.rval.bytes() + l.Po.bytes() + l.Ro.bytes() +
             l.b.bytes() + l.xa.bytes() + l.xb.bytes() + l.d.bytes() + l.r.bytes();
    return b + tail.bytes();
}

size_t SolverImpl::bytes() const {
    return A64_.bytes() + op64_.bytes() + a_.ptr.bytes() + a_.idx.bytes() + a_.val.bytes() + H64_.bytes() +
           H32_.bytes() + dense_inv_.bytes() + 7 * n_ * sizeof(double) + r32_.bytes() +
           (sparse_ ? sparse_->bytes() : 0);
}

std::vector<int64_t> SolverImpl::level_sizes() const { return sizes_; }

template <class T>
static std::string describe_op(const Operator<T>& op) {
    char buf[200];
    if (op.block3) {
        std::snprintf(buf, sizeof buf, "3x3-block sell C=%d nnz=%lld", B3C, (long long)op.nnz);
    } else if (!op.stencil) {
        std::snprintf(buf, sizeof buf, "sell C=%d nnz=%lld", op.sell.C, (long long)op.nnz);
    } else {
        std::snprintf(buf, sizeof buf,
                      "stencil K=%d %s%s (probe %.1f / %.1f / %.1f / %.1f us)%s nnz=%lld", op.K,
                      op.half ? "fp16 " : "",
                      op.march  ? "marching planes"
                      : op.pair ? "unrolled, 2 rows per thread"
                      : op.unrolled ? "unrolled"
                                    : "loop",
                      op.probe_ms[0] * 1e3, op.probe_ms[1] * 1e3, op.probe_ms[3] * 1e3,
                      op.probe_ms[4] < 1e29 ? op.probe_ms[4] * 1e3 : 0.0,
                      op.bulk ? ", steps from bulk-copied tiles" : "", (long long)op.nnz);
    }
    return buf;
}

std::string SolverImpl::describe() const {
    std::string out;
    char buf[256];
    std::snprintf(buf, sizeof buf, "method=%s precision=%s n=%lld\n",
                  direct_ ? "direct" : "multigrid",
                  opt_.precision == FEMGPU_MIXED ? "mixed" : "fp64", (long long)n_);
    out += buf;
    if (sparse_) out += sparse_->describe();
    if (direct_) return out;
    out += "outer fp64: " + describe_op(op64_) + "\n";
    auto levels = [&](const auto& H, const char* t) {
        for (size_t l = 0; l < H.levels.size(); ++l) {
            const auto& L = H.levels[l];
            std::snprintf(buf, sizeof buf, "level %zu %s n=%lld lambda=%.4f degree=%zu: ", l, t,
                          (long long)L.n, L.lambda, L.c1.size());
            out += buf + describe_op(L.A);
            std::snprintf(buf, sizeof buf, "; P %s, R %s",
                          L.Po.ok ? ("offsets K=" + std::to_string(L.Po.off.size())).c_str()
                                  : "CSR",
                          L.Ro.ok ? ("offsets K=" + std::to_string(L.Ro.off.size())).c_str()
                                  : "CSR");
            out += buf;
            if (cluster_on_ && l < H.cluster.size() && H.cluster[l])
                out += "; legs as clusters of " + std::to_string(cluster_ctas_) + " blocks";
            out += "\n";
        }
        if (H.sparse)
            std::snprintf(buf, sizeof buf, "coarsest n=%lld %s", (long long)H.ncoarse,
                          H.sparse->describe().c_str());
        else
            std::snprintf(buf, sizeof buf, "coarsest n=%lld dense inverse%s\n",
                          (long long)H.ncoarse, H.hinv.p ? " (FP16)" : "");
        out += buf;
        if (H.tail_from >= 0 && tail_on_) {
            std::snprintf(buf, sizeof buf,
                          "levels %d.. and the coarsest solve: 1 cooperative kernel, %d blocks\n",
                          H.tail_from, H.tail_grid);
            out += buf;
        }
    };
    if (opt_.precision == FEMGPU_MIXED)
        levels(H32_, "fp32");
    else
        levels(H64_, "fp64");
    out += "setup seconds:";
    for (const auto& p : setup_s_) {
        std::snprintf(buf, sizeof buf, " %s %.3f;", p.first.c_str(), p.second);
        out += buf;
    }
    out += "\n";
    return out;
}

void SolverImpl::phase(const std::string& name, double seconds) {
    for (auto& p : setup_s_)
        if (p.first == name) {
            p.second += seconds;
            return;
        }
    setup_s_.emplace_back(name, seconds);
}

// The coordinates of each unknown (3 each): its grid point, or the given points.
static std::vector<double> unknown_xyz(const femgpu_unknowns& u, int64_t n) {
    std::vector<double> xyz((size_t)3 * n);
    for (int64_t k = 0; k < n; ++k)
        for (int d = 0; d < 3; ++d)
            xyz[3 * k + d] = u.kind == FEMGPU_UNKNOWNS_GRID ? u.planes[d][u.points[3 * k + d]]
                                                            : u.xyz[3 * k + d];
    return xyz;
}

void SolverImpl::create(const DevCsr& a, const femgpu_unknowns& u, int method,
                        const femgpu_crossover& c, const Options& o, const HostCells* cells) {
    opt_ = o;
    pdl_ = o.pdl != 0;
    n_ = a.n;
    // The solver's own copy of the matrix (the reference moves `a` into the Solver).
    a_.n = a.n;
    a_.nnz = a.nnz;
    a_.ptr.alloc(a.n + 1);
    a_.idx.alloc(a.nnz);
    a_.val.alloc(a.nnz);
    FG_CUDA(cudaMemcpyAsync(a_.ptr.p, a.ptr.p, a_.ptr.bytes(), cudaMemcpyDeviceToDevice, s_));
    FG_CUDA(cudaMemcpyAsync(a_.idx.p, a.idx.p, a_.idx.bytes(), cudaMemcpyDeviceToDevice, s_));
    FG_CUDA(cudaMemcpyAsync(a_.val.p, a.val.p, a_.val.bytes(), cudaMemcpyDeviceToDevice, s_));
    int C = o.sell_c ? o.sell_c : 32;
    {
        PhaseTimer t{this, "outer SELL", s_};
        make_sell<double>(a_, C, &A64_, s_);
    }
    // The block partials of the reductions: 1 block per 256 rows of the largest operator.
    partial_.alloc(2 * (size_t)row_blocks(std::max<int64_t>(a.n, A64_.nslices * A64_.C) + 64));
    x_.alloc(n_);
    r_.alloc(n_);
    p_.alloc(n_);
    q_.alloc(n_);
    b_.alloc(n_);
    t_.alloc(n_);
    // solve.rs:99-183: the choice of the method.
    bool direct;
    // The host copy of the matrix, for the host steps of the direct methods only.
    HostCsr h;
    bool have_h = false;
    auto host = [&]() -> const HostCsr& {
        if (!have_h) {
            PhaseTimer t{this, "matrix to host", s_};
            h = download_csr(a_, s_);
            have_h = true;
        }
        return h;
    };
    if (u.kind == FEMGPU_UNKNOWNS_POINTS) {
        if (method == FEMGPU_METHOD_MULTIGRID)
            throw Failure(FEMGPU_ERR_NEEDS_GRID,
                          "multigrid needs the box grid: a mesh of tetrahedra has the direct solver");
        direct = true;
    } else if (method == FEMGPU_METHOD_DIRECT) {
        direct = true;
    } else if (method == FEMGPU_METHOD_MULTIGRID) {
        direct = false;
    } else if (c.rule == 0) {
        direct = (size_t)a.n <= c.unknowns;
    } else {
        // Crossover::Flops (solve.rs:108-118, 160-172): the sparse factor's entries and flops
        // in the nested dissection order of the unknowns' points.
        PhaseTimer t{this, "symbolic analysis for the crossover (host)", s_};
        std::vector<double> xyz = unknown_xyz(u, a.n);
        uint64_t entries = 0;
        double flops = 0.0;
        factor_figures(host(), nested_dissection(host(), xyz.data()), &entries, &flops);
        direct = entries <= c.entries && (c.flat || flops <= c.flops * (double)a.n);
    }
    direct_ = direct;
    if (direct) {
        // A small system takes the dense inverse; a larger one the sparse multifrontal factor in
        // the reference's order.
        if (a.n <= DENSE_DIRECT) {
            dense_direct(host());
        } else {
            const HostCsr& hh = host();
            PhaseTimer t{this, "sparse factor (analysis on the host, fronts on the device)", s_};
            sparse_direct(hh, unknown_xyz(u, a.n));
        }
        sizes_ = {n_};
        return;
    }
    {
        PhaseTimer t{this, "outer operator and autotuner", s_};
        make_operator<double>(a_, C, opt_.format == 0, &op64_, s_);
        tune_operator(&op64_, opt_.stencil, s_);
        if (!opt_.sell_c) tune_sell(a_, &op64_, s_);
    }
    if (u.kind == FEMGPU_UNKNOWNS_GRID) {
        HostLevel lv;
        for (int d = 0; d < 3; ++d) lv.planes[d].assign(u.planes[d], u.planes[d] + u.nplanes[d]);
        lv.points.resize(n_);
        for (int64_t k = 0; k < n_; ++k)
            for (int d = 0; d < 3; ++d) lv.points[k][d] = u.points[3 * k + d];
        lv.comp.assign(u.comp, u.comp + n_);
        build_multigrid(std::move(lv), nullptr, cells);
    } else {
        // p-multigrid (pmultigrid.rs:46-98): the first coarse level is P^T A P on the corners,
        // then geometric levels on the grid of the corner points.
        HostRect p;
        p.rows = n_;
        p.cols = (int64_t)u.p_cols;
        p.ptr.assign(u.p_ptr, u.p_ptr + n_ + 1);
        p.idx.assign(u.p_idx, u.p_idx + p.ptr[n_]);
        p.val.assign(u.p_val, u.p_val + p.ptr[n_]);
        HostLevel lv = level_of_points(u.coarse_xyz, p.cols, u.coarse_comp);
        build_multigrid(std::move(lv), &p, nullptr);
    }
    if (opt_.degree == 0) {
        PhaseTimer t{this, "autotuner (smoother degree)", s_};
        tune_degree();
    }
}

void SolverImpl::apply_degree(int degree, int coarse) {
    const double lower = opt_.lower > 0 ? opt_.lower : 0.3;
    if (coarse <= 0) coarse = degree;
    for (size_t l = 0; l < H32_.levels.size(); ++l)
        chebyshev(H32_.levels[l].lambda, l == 0 ? degree : coarse, lower, &H32_.levels[l].c1,
                  &H32_.levels[l].c2, opt_.smoother, opt_.upper);
    for (size_t l = 0; l < H64_.levels.size(); ++l)
        chebyshev(H64_.levels[l].lambda, l == 0 ? degree : coarse, lower, &H64_.levels[l].c1,
                  &H64_.levels[l].c2, opt_.smoother, opt_.upper);
    // The captured loop holds the coefficients as kernel arguments.
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    exec_ = nullptr;
    graph_ = nullptr;
}

// Each candidate (the finest level's degree, the coarser levels') solves a fixed right side
// (k_seed) from x = 0 to 1e-4 twice; the second solve's device time per decade of residual
// reduction decides. (2, 2) is tried first and keeps a tie; (2, 1) smooths the latency-bound
// coarse levels once before and once after their correction.
void SolverImpl::tune_degree() {
    const bool mixed = opt_.precision == FEMGPU_MIXED;
    const size_t nlevels = mixed ? H32_.levels.size() : H64_.levels.size();
    if (nlevels == 0 || opt_.tail > 0) return;  // the fused tail holds its coefficients
    int64_t kind = -2;  // SELL
    if (mixed ? H32_.levels[0].A.stencil : H64_.levels[0].A.stencil)
        kind = mixed ? H32_.levels[0].A.K : H64_.levels[0].A.K;
    else if (mixed ? H32_.levels[0].A.block3 : H64_.levels[0].A.block3)
        kind = -1;
    const std::array<int64_t, 5> key{2, (mixed ? 4 : 8) + 100 * opt_.smoother, kind, log2_of(n_),
                                     (int64_t)nlevels};
    int degree = 22;  // 10 * (the finest level's degree) + the coarser levels'
    if (tune_lookup(key, &degree)) {
        if (degree != 22) apply_degree(degree / 10, degree % 10);
        return;
    }
    DevBuf<double> rhs(n_);
    k_seed<<<blocks_for(n_, TH), TH, 0, s_>>>(n_, rhs.p);
    FG_CHECK_LAUNCH();
    const double tol0 = tol;
    const size_t max0 = max_iter;
    tol = 1e-4;
    max_iter = 200;
    double best = 1e30;
    for (int cand : {22, 11, 33, 21}) {
        if (cand % 10 != cand / 10 && nlevels < 2) continue;
        apply_degree(cand / 10, cand % 10);
        double cost = 1e30;
        for (int rep = 0; rep < 2; ++rep) {
            FG_CUDA(cudaMemsetAsync(x_.p, 0, n_ * sizeof(double), s_));
            femgpu_stats st{};
            try {
                solve(rhs.p, x_.p, nullptr, &st);
            } catch (const Failure&) {
                st.residual = 1.0;
            }
            if (rep == 1 && st.residual > 0.0 && st.residual < 1.0)
                cost = st.seconds / -std::log10(st.residual);
            // A trial of 50 ms or more: the first solve's graph capture is a small part of it,
            // so its time decides and the second is not run.
            if (rep == 0 && st.seconds >= 0.05 && st.residual > 0.0 && st.residual < 1.0) {
                cost = st.seconds / -std::log10(st.residual);
                break;
            }
        }
        if (cost < best) {
            best = cost;
            degree = cand;
        }
    }
    tol = tol0;
    max_iter = max0;
    apply_degree(degree / 10, degree % 10);
    tune_store(key, degree);
}

void SolverImpl::sparse_direct(const HostCsr& h, const std::vector<double>& xyz) {
    sparse_ = std::make_unique<SparseFactor>();
    sparse_->factor(h, xyz.data(), s_);
    // The triangles of supernodes of 8 columns or more by products with their inverses: the
    // direct solve of a 36,300-unknown P2 beam 3.7 against 5.9 ms, of a 32^3 heat cube 6.3
    // against 9.6 ms.
    sparse_->invert_blocks(8, s_);
}

void SolverImpl::dense_direct(const HostCsr& h) {
    dense_inverse(h, &dense_inv_, s_);
}

// The offset form of a transfer when its entries sit at no more than 32 distinct offsets from
// each row's first (smallest) column, which they do for the plane coarsening of a box grid in
// grid order; else `out->ok` stays false and the transfer stays CSR. Found and filled on the
// device (offsets.cuh).
template <class T>
static void make_offset(const DevRect& M, OffsetTransfer<T>* out, cudaStream_t s) {
    out->ok = false;
    if (M.rows >= 0x7fffffff || M.cols >= 0x7fffffff || M.nnz == 0) return;
    out->base.alloc(M.rows);
    OffsetScan sc;
    if (!scan_offsets(M.ptr.p, M.idx.p, M.rows, false, MAXK, out->base.p, &sc, s)) {
        out->base.release();
        return;
    }
    out->w.alloc(sc.offs.size() * (size_t)M.rows);
    fill_offsets<T>(M.ptr.p, M.idx.p, M.val.p, M.rows, false, out->base.p, sc.offs, M.rows,
                    out->w.p, s);
    out->rows = M.rows;
    out->cols = M.cols;
    out->off.assign(sc.offs.begin(), sc.offs.end());
    out->ok = true;
}

// The descriptor of level l for the fused kernels (stencil or SELL operator, at most
// TAIL_MAXDEG smoothing steps, fewer than 2^31 rows).
template <class T>
static TailLevel<T> tail_level(const Hierarchy<T>& H, size_t l) {
    const MgLevel<T>& L = H.levels[l];
    TailLevel<T> t{};
    t.n = (int)L.n;
    t.nc = (int)L.nc;
    t.stencil = L.A.stencil ? 1 : 0;
    t.deg = (int)L.c1.size();
    if (L.A.stencil)
        t.sv = L.A.sview();
    else
        t.sell = L.A.sell.view();
    t.p_offset = L.Po.ok ? 1 : 0;
    t.r_offset = L.Ro.ok ? 1 : 0;
    if (L.Po.ok) {
        t.Po = L.Po.view();
    } else {
        t.pptr = L.pptr.p;
        t.pidx = L.pidx.p;
        t.pval = L.pval.p;
    }
    if (L.Ro.ok) {
        t.Ro = L.Ro.view();
    } else {
        t.rptr = L.rptr.p;
        t.ridx = L.ridx.p;
        t.rval = L.rval.p;
    }
    t.dinv = L.dinv.p;
    t.b = L.b.p;
    t.xa = L.xa.p;
    t.xb = L.xb.p;
    t.d = L.d.p;
    t.r = L.r.p;
    t.bc = l + 1 == H.levels.size() ? H.cb.p : H.levels[l + 1].b.p;
    for (size_t k = 0; k < L.c1.size() && k < (size_t)TAIL_MAXDEG; ++k) {
        t.c1[k] = (T)L.c1[k];
        t.c2[k] = (T)L.c2[k];
    }
    return t;
}

// The descriptors of the fused kernel for the levels from the first one of at most `tail` rows
// down (tail <= 0: none), and its grid: as many blocks as fit on the GPU at once (a cooperative
// launch needs them all resident), no more than the largest of those levels has rows for.
// Measured on the 128^3 heat cube (levels 36k, 4.9k, coarsest 729): about 7 us per step of the
// fused kernel, a grid-wide barrier included, against about 4 us per separate launch in the
// loop's CUDA graph; so it is off unless asked for.
template <class T>
static void build_tail(Hierarchy<T>* H, int tail, cudaStream_t s) {
    H->tail_from = -1;
    if (tail <= 0 || H->levels.empty() || H->sparse || H->hinv.p) return;
    const int64_t limit = tail;
    size_t from = 0;
    while (from < H->levels.size() && H->levels[from].n > limit) ++from;
    if (from == H->levels.size()) return;
    std::vector<TailLevel<T>> d;
    int64_t rows = H->ncoarse;
    if (H->levels.size() - from > (size_t)TAIL_MAXLEVELS) return;
    for (size_t l = from; l < H->levels.size(); ++l) {
        const MgLevel<T>& L = H->levels[l];
        // The fused kernel reads stencil and SELL levels; a 3x3-block level keeps separate
        // launches.
        if (L.c1.size() > (size_t)TAIL_MAXDEG || L.n >= 0x7fffffff || L.A.block3) return;
        d.push_back(tail_level(*H, l));
        rows = std::max(rows, L.n);
    }
    int per_sm = 0, dev = 0, sms = 0;
    FG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tail<T>, TH, 0));
    FG_CUDA(cudaGetDevice(&dev));
    FG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1) return;
    H->tail.upload(d.data(), d.size(), s);
    FG_CUDA(cudaStreamSynchronize(s));
    H->tail_grid =
        (int)std::max<int64_t>(1, std::min<int64_t>((rows + TH - 1) / TH, (int64_t)per_sm * sms));
    H->tail_from = (int)from;
}

template <class T>
void SolverImpl::build_levels(const std::vector<const DevCsr*>& mats, std::vector<DevRect>& ps,
                              const HostLevel& coarsest, Hierarchy<T>* H) {
    size_t L = mats.size();
    H->levels.resize(L - 1);
    int C = opt_.sell_c ? opt_.sell_c : 32;
    for (size_t l = 0; l + 1 < L; ++l) {
        MgLevel<T>& lv = H->levels[l];
        const DevCsr& d = *mats[l];
        lv.n = d.n;
        lv.nnz = d.nnz;
        {
            PhaseTimer t{this, "level operators", s_};
            make_operator<T>(d, C, opt_.format == 0, &lv.A, s_);
            if constexpr (std::is_same<T, float>::value)
                if (lv.A.stencil && (opt_.values == 2 || (opt_.values == 0 && kHalfDefault)))
                    make_half(&lv.A, s_);
        }
        {
            PhaseTimer t{this, "autotuner", s_};
            tune_operator(&lv.A, opt_.stencil, s_);
            if (!opt_.sell_c) tune_sell(d, &lv.A, s_);
            if constexpr (std::is_same<T, float>::value)
                if (l == 0) tune_tiles(&lv.A, opt_.tiles, s_);
        }
        std::optional<PhaseTimer> t_lam;
        t_lam.emplace(this, "diagonals and lambda_max", s_);
        // The diagonal and lambda_max(D^-1 A) in FP64.
        DevBuf<double> dg(lv.n);
        DevBuf<int> bad(1);
        bad.zero(s_);
        k_diagonal<<<blocks_for(lv.n, TH), TH, 0, s_>>>(lv.n, d.ptr.p, d.idx.p, d.val.p, dg.p,
                                                        bad.p);
        FG_CHECK_LAUNCH();
        if (fetch(bad.p, s_))
            throw Failure(FEMGPU_ERR_NOT_SPD,
                          "the matrix is not positive definite: it has a diagonal entry that is "
                          "not above 0");
        // The finest level's lambda_max from the exact FP64 operator; a coarser level's from
        // its own (FP32 in the mixed form, the products accumulated in FP64).
        lv.lambda = l == 0 ? lambda_max(op64_, dg.p, s_, partial_)
                           : lambda_max(lv.A, dg.p, s_, partial_);
        lv.dinv.alloc(lv.n);
        reciprocal<T>(lv.n, dg.p, lv.dinv.p, s_);
        int deg = opt_.degree > 0 ? opt_.degree : 2;
        double lower = opt_.lower > 0 ? opt_.lower : 0.3;
        chebyshev(lv.lambda, deg, lower, &lv.c1, &lv.c2, opt_.smoother, opt_.upper);
        t_lam.reset();
        PhaseTimer t_tr{this, "transfers", s_};
        // Transfers to the next level: P and R = P^T (each row's columns increasing).
        DevRect& P = ps[l];
        if (P.nnz >= 0x7fffffff || P.rows >= 0x7fffffff)
            throw Failure(FEMGPU_ERR_TOO_LARGE, "a prolongation with 2^31 entries or more");
        DevRect R;
        transpose_rect(P, &R, s_);
        lv.nc = P.cols;
        if (opt_.format == 0) {
            make_offset<T>(P, &lv.Po, s_);
            make_offset<T>(R, &lv.Ro, s_);
        }
        if (!lv.Po.ok) {
            lv.pptr = std::move(P.ptr);
            lv.pidx = std::move(P.idx);
            lv.pval.alloc(P.nnz);
            convert_values<T>(P.nnz, P.val.p, lv.pval.p, s_);
        }
        if (!lv.Ro.ok) {
            lv.rptr = std::move(R.ptr);
            lv.ridx = std::move(R.idx);
            lv.rval.alloc(R.nnz);
            convert_values<T>(R.nnz, R.val.p, lv.rval.p, s_);
        }
        lv.b.alloc(lv.n);
        lv.xa.alloc(lv.n);
        lv.xb.alloc(lv.n);
        lv.d.alloc(lv.n);
        lv.r.alloc(lv.n);
        FG_CUDA(cudaStreamSynchronize(s_));
    }
    if (mats.back()->n > DENSE_COARSEST_MAX) {
        // The coarsest level's sparse factor, in the nested dissection order of its points'
        // coordinates (multigrid.rs:124-131).
        PhaseTimer t_sparse{this, "coarsest sparse factor", s_};
        const HostCsr last = download_csr(*mats.back(), s_);
        std::vector<double> xyz(3 * (size_t)last.n);
        for (int64_t k = 0; k < last.n; ++k)
            for (int d = 0; d < 3; ++d)
                xyz[3 * k + d] = coarsest.planes[d][coarsest.points[k][d]];
        H->ncoarse = last.n;
        H->sparse = std::make_unique<SparseFactor>();
        H->sparse->factor(last, xyz.data(), s_);
        // Inside the V-cycle the large supernodes' triangles are applied by products with their
        // inverses (parallel) rather than by substitution column by column.
        H->sparse->invert_blocks(8, s_);
        H->cb.alloc(last.n);
        H->cb.zero(s_);
        H->cx.alloc(last.n);
        if (!std::is_same<T, double>::value) {
            H->cb64.alloc(last.n);
            H->cx64.alloc(last.n);
        }
        FG_CUDA(cudaStreamSynchronize(s_));
        return;
    }
    // The coarsest level: its inverse from a dense Cholesky factor on the device.
    std::optional<PhaseTimer> t_dense;
    t_dense.emplace(this, "coarsest dense inverse", s_);
    const HostCsr last = download_csr(*mats.back(), s_);
    H->ncoarse = last.n;
    DevBuf<double> inv64;
    std::vector<std::pair<const char*, double>> stages;
    dense_inverse(last, &inv64, s_, &stages);
    // Rows at leading dimension dense_ld(n), the padding 0; the right side padded with zeros.
    const int64_t ld = dense_ld(last.n);
    if (std::is_same<T, float>::value && opt_.values == 3) {
        DevBuf<unsigned long long> mx(1);
        mx.zero(s_);
        k_abs_max<<<blocks_for(last.n * last.n, TH), TH, 0, s_>>>(last.n * last.n, inv64.p, mx.p);
        const double scale = bits_to_double((long long)fetch(mx.p, s_));
        if (scale > 0.0 && std::isfinite(scale)) {
            H->hinv.alloc(last.n * ld);
            k_half_of<<<blocks_for(last.n * ld, TH), TH, 0, s_>>>(last.n, ld, inv64.p, scale,
                                                                  H->hinv.p);
            H->hscale = (float)scale;
        }
    }
    if (!H->hinv.p) {
        H->inv.alloc(last.n * ld);
        k_convert_pad<double, T><<<blocks_for(last.n * ld, TH), TH, 0, s_>>>(last.n, ld, inv64.p,
                                                                             H->inv.p);
    }
    FG_CHECK_LAUNCH();
    H->cb.alloc(ld);
    H->cb.zero(s_);
    FG_CUDA(cudaStreamSynchronize(s_));
    H->cx.alloc(last.n);
    t_dense.reset();
    for (const auto& st : stages) phase(std::string("coarsest: ") + st.first, st.second);
    build_tail(H, opt_.tail, s_);
    // The small levels whose legs run as cluster launches: a stencil or SELL operator, at most
    // CLUSTER_MAX_ROWS rows, and not the first level (its right side is the caller's).
    H->cluster.assign(H->levels.size(), 0);
    if (opt_.cluster == 1) {
        if (cluster_ctas_ == 0) cluster_ctas_ = cluster_ctas<T>();
        for (size_t l = 1; l < H->levels.size() && cluster_ctas_ > 0; ++l) {
            const MgLevel<T>& L = H->levels[l];
            H->cluster[l] = L.n <= CLUSTER_MAX_ROWS && !L.A.block3 &&
                            L.c1.size() <= (size_t)TAIL_MAXDEG;
        }
    }
    if (opt_.l2 == 1 && H->inv.p) {
        // The inverse is read once per V-cycle (96 MB in FP32 for the 4,913-row level of the
        // 128^3 box) and evicted by the finer levels' streams in between; a persisting window
        // keeps it in L2 across cycles.
        int dev = 0, maxp = 0, maxw = 0;
        FG_CUDA(cudaGetDevice(&dev));
        FG_CUDA(cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, dev));
        FG_CUDA(cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, dev));
        if (maxp > 0 && maxw > 0) {
            const size_t want = std::min<size_t>(H->inv.bytes(), (size_t)maxp);
            size_t cur = 0;
            FG_CUDA(cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize));
            if (cur < want) FG_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want));
            l2win_.base_ptr = H->inv.p;
            l2win_.num_bytes = std::min<size_t>(H->inv.bytes(), (size_t)maxw);
            l2win_.hitRatio = (float)std::min(1.0, (double)want / (double)l2win_.num_bytes);
            l2win_.hitProp = cudaAccessPropertyPersisting;
            l2win_.missProp = cudaAccessPropertyStreaming;
            l2_window_ = true;
        }
    }
}

void SolverImpl::build_multigrid(HostLevel level, const HostRect* pfirst,
                                 const HostCells* cells) {
    // multigrid.rs:84-139: coarsen until a level has at most `coarsest` unknowns, 30 levels, or
    // a coarsening keeps more than 90 % of the unknowns. The coarsening, the Galerkin products
    // and the operators of the levels are built on the device (coarsen.cu, offsets.cu), the
    // coarse unknowns numbered in grid order; with cells the coarse matrices are the
    // cell-condensed ones (each level's cells from the last, on the host).
    std::deque<DevCsr> held;  // the coarse matrices
    std::vector<const DevCsr*> mats{&a_};
    std::vector<DevRect> ps;
    int threads = host_threads();
    if (pfirst) {
        // pmultigrid.rs:47: the P1 level is the Galerkin product with the P2 -> P1 prolongation.
        PhaseTimer t{this, "Galerkin products (device)", s_};
        DevRect P;
        rect_upload(*pfirst, &P, s_);
        held.emplace_back();
        galerkin_product(P, a_, &held.back(), s_);
        mats.push_back(&held.back());
        ps.push_back(std::move(P));
    }
    size_t coarsest = (size_t)(opt_.coarsest > 0 ? opt_.coarsest : DEVICE_COARSEST);
    size_t max_levels = (size_t)(opt_.max_levels > 0 ? opt_.max_levels : 30);
    HostCells stored;  // the cells of the last coarse level
    DevGrid grid;
    grid_upload(level, &grid, s_);
    for (;;) {
        const DevCsr& a = *mats.back();
        if ((size_t)a.n <= coarsest || ps.size() >= max_levels) break;
        DevRect p;
        DevGrid coarse;
        {
            PhaseTimer t{this, "coarsening (device)", s_};
            if (!coarsen_grid(grid, a, opt_.axes, &p, &coarse, s_)) break;
            if ((size_t)coarse.n * 10 > (size_t)a.n * 9) break;
        }
        held.emplace_back();
        if (cells && !cells->empty()) {
            PhaseTimer t_c{this, "coarse matrices from the cells (host)", s_};
            HostCells nxt;
            HostCsr ac = by_cells(grid_download(grid, s_), stored.empty() ? *cells : stored,
                                  grid_download(coarse, s_), &nxt, threads);
            stored = std::move(nxt);
            upload_csr(ac, &held.back(), s_);
        } else {
            PhaseTimer t_g{this, "Galerkin products (device)", s_};
            galerkin_product(p, a, &held.back(), s_);
        }
        mats.push_back(&held.back());
        ps.push_back(std::move(p));
        grid = std::move(coarse);
    }
    // The coarsest level's points, for the order of a sparse coarsest factor.
    HostLevel last;
    if (mats.back()->n > DENSE_COARSEST_MAX) last = grid_download(grid, s_);
    sizes_.clear();
    for (const DevCsr* m : mats) sizes_.push_back(m->n);
    if (opt_.precision == FEMGPU_MIXED) {
        build_levels<float>(mats, ps, last, &H32_);
        r32_.alloc(n_);
    } else {
        build_levels<double>(mats, ps, last, &H64_);
    }
}

// A Chebyshev step and the residual of level L: by tiles when the autotuner chose them.
template <class T>
void SolverImpl::enqueue_step(MgLevel<T>& L, const T* b, const T* xin, T c1, T c2, T* xout) {
    const int* done = &sc_.p->done;
    if constexpr (std::is_same<T, float>::value) {
        if (L.A.bulk) {
            launch_smem(pdl_, k_stencil_tiles<8, true>, tile_grid(L.n), BULK_TH,
                        tile_smem<true>(), s_, L.A.sview(), b, xin, (const float*)L.dinv.p, c1,
                        c2, L.d.p, xout, done, &sc_.p->bulk_timeout, wait_limit);
            return;
        }
    }
    if (L.A.march) {
        launch_march<T, true>(pdl_, L.A, s_, b, xin, (const T*)L.dinv.p, c1, c2, L.d.p, xout,
                              done);
        return;
    }
    if (L.A.pair) {
        const int gp = row_blocks(pair_threads(L.n));
        if (L.A.K == 8)
            launch(pdl_, k_cheb_step_pair<T, 8>, gp, TH, s_, L.A.sview(), b, xin,
                   (const T*)L.dinv.p, c1, c2, L.d.p, xout, done);
        else
            launch(pdl_, k_cheb_step_pair<T, 14>, gp, TH, s_, L.A.sview(), b, xin,
                   (const T*)L.dinv.p, c1, c2, L.d.p, xout, done);
        return;
    }
    with_op(L.A, [&](auto op) {
        launch(pdl_, k_cheb_step<T, decltype(op)>, row_blocks(L.A.threads()), TH, s_, op, b,
               xin, L.dinv.p, c1, c2, L.d.p, xout, done);
    });
}

template <class T>
void SolverImpl::enqueue_residual(MgLevel<T>& L, const T* b, const T* x) {
    const int* done = &sc_.p->done;
    if constexpr (std::is_same<T, float>::value) {
        if (L.A.bulk) {
            launch_smem(pdl_, k_stencil_tiles<8, false>, tile_grid(L.n), BULK_TH,
                        tile_smem<false>(), s_, L.A.sview(), b, x, (const float*)nullptr, 0.f,
                        0.f, (float*)nullptr, L.r.p, done, &sc_.p->bulk_timeout, wait_limit);
            return;
        }
    }
    if (L.A.march) {
        launch_march<T, false>(pdl_, L.A, s_, b, x, (const T*)nullptr, (T)0, (T)0, (T*)nullptr,
                               L.r.p, done);
        return;
    }
    if (L.A.pair) {
        const int gp = row_blocks(pair_threads(L.n));
        if (L.A.K == 8)
            launch(pdl_, k_residual_pair<T, 8>, gp, TH, s_, L.A.sview(), b, x, L.r.p, done);
        else
            launch(pdl_, k_residual_pair<T, 14>, gp, TH, s_, L.A.sview(), b, x, L.r.p, done);
        return;
    }
    with_op(L.A, [&](auto op) {
        launch(pdl_, k_residual<T, decltype(op)>, row_blocks(L.A.threads()), TH, s_, op, b, x,
               L.r.p, done);
    });
}

template <class T>
const T* SolverImpl::enqueue_vcycle(Hierarchy<T>& H, size_t l, const T* b, bool started) {
    const int* done = &sc_.p->done;
    if (l == H.levels.size() && H.sparse) {
        // The sparse coarsest factor's 2 triangular solves in FP64 (the right side and the
        // solution converted in the mixed form).
        const int64_t n = H.ncoarse;
        if constexpr (std::is_same<T, double>::value) {
            H.sparse->solve(b, H.cx.p, s_);
        } else {
            k_convert<T, double><<<blocks_for(n, TH), TH, 0, s_>>>(n, b, H.cb64.p);
            H.sparse->solve(H.cb64.p, H.cx64.p, s_);
            k_convert<double, T><<<blocks_for(n, TH), TH, 0, s_>>>(n, H.cx64.p, H.cx.p);
            launches_ += 2;
        }
        FG_CHECK_LAUNCH();
        mark("coarsest sparse solve n=" + std::to_string(n));
        launches_ += H.sparse->solve_launches();
        return H.cx.p;
    }
    if (l == H.levels.size()) {
        int64_t n = H.ncoarse;
        if constexpr (std::is_same<T, float>::value)
            if (H.hinv.p) {
                launch(pdl_, k_gemv_rows_half, (int)std::min<int64_t>(n, NUM_SMS * 8), TH, s_, n,
                       dense_ld(n), (const __half*)H.hinv.p, H.hscale, b, H.cx.p, done);
                FG_CHECK_LAUNCH();
                mark("coarsest dense solve n=" + std::to_string(n) + " (FP16 inverse)");
                launches_ += 1;
                return H.cx.p;
            }
        if (b == H.cb.p)
            launch_window(pdl_, l2_window_ ? &l2win_ : nullptr, k_gemv_rows<T>,
                          (int)std::min<int64_t>(n, NUM_SMS * 8), TH, s_, n, dense_ld(n),
                          H.inv.p, b, H.cx.p, done);
        else
            launch(pdl_, k_gemv<T>, blocks_for(n * 32, TH), TH, s_, n, dense_ld(n),
                   H.inv.p, b, H.cx.p, done);
        FG_CHECK_LAUNCH();
        mark("coarsest dense solve n=" + std::to_string(n));
        launches_ += 1;
        return H.cx.p;
    }
    if ((int)l == H.tail_from && tail_on_) {
        // This level and all below it, and the coarsest solve: 1 cooperative kernel.
        const TailLevel<T>* tl = H.tail.p;
        int nl = (int)(H.levels.size() - l);
        const T* b0 = b;
        const T* inv = H.inv.p;
        int64_t nco = H.ncoarse;
        T* cx = H.cx.p;
        void* args[] = {(void*)&tl, (void*)&nl, (void*)&b0, (void*)&inv,
                        (void*)&nco, (void*)&cx, (void*)&done};
        FG_CUDA(cudaLaunchCooperativeKernel((const void*)k_tail<T>, dim3(H.tail_grid), dim3(TH),
                                            args, 0, s_));
        mark("L" + std::to_string(l) + " and below, fused, with the coarsest solve");
        launches_ += 1;
        // Where the kernel leaves this level's x: the same swaps as the separate steps below.
        MgLevel<T>& L = H.levels[l];
        T* xa = L.xa.p;
        T* xb = L.xb.p;
        for (size_t k = 1; k < 2 * L.c1.size(); ++k) std::swap(xa, xb);
        return xa;
    }
    if (cluster_on_ && l < H.cluster.size() && H.cluster[l]) {
        // The level's 2 legs, each 1 cluster launch, around the coarser levels.
        MgLevel<T>& L = H.levels[l];
        TailLevel<T> t = tail_level(H, l);
        t.b = b;
        launch_cluster<T, false>(pdl_, cluster_ctas_, t, (const T*)nullptr, done, s_);
        mark("L" + std::to_string(l) + " smoothing, residual and restriction (1 cluster)");
        const T* ec = enqueue_vcycle(H, l + 1, t.bc);
        launch_cluster<T, true>(pdl_, cluster_ctas_, t, ec, done, s_);
        mark("L" + std::to_string(l) + " prolongation and smoothing (1 cluster)");
        launches_ += 2;
        // Where the legs leave x: the separate steps' swaps.
        T* xa = L.xa.p;
        T* xb = L.xb.p;
        for (size_t k = 1; k < 2 * L.c1.size(); ++k) std::swap(xa, xb);
        return xa;
    }
    MgLevel<T>& L = H.levels[l];
    int64_t n = L.n;
    const int gb = row_blocks(n);
    T* xa = L.xa.p;
    T* xb = L.xb.p;
    int deg = (int)L.c1.size();
    std::string tag = "L" + std::to_string(l) + " ";
    if (!started) {
        launch(pdl_, k_cheb_first<T>, gb, TH, s_, n, b, L.dinv.p, (T)L.c1[0], L.d.p, xa, done);
        mark(tag + "smooth (first, no product)");
    }
    for (int k = 1; k < deg; ++k) {
        enqueue_step(L, b, xa, (T)L.c1[k], (T)L.c2[k], xb);
        mark(tag + "smooth pre");
        std::swap(xa, xb);
    }
    enqueue_residual(L, b, xa);
    mark(tag + "residual");
    T* bc = l + 1 == H.levels.size() ? H.cb.p : H.levels[l + 1].b.p;
    // The next level's first step rides on the restriction when that level smooths with
    // separate launches (not the coarsest, the fused tail or the cluster legs).
    const bool fuse_first = l + 1 < H.levels.size() && L.Ro.ok &&
                            !((int)(l + 1) == H.tail_from && tail_on_) &&
                            !(cluster_on_ && l + 1 < H.cluster.size() && H.cluster[l + 1]);
    if (fuse_first) {
        MgLevel<T>& N = H.levels[l + 1];
        const auto v = L.Ro.view();
        if (v.K == 27)
            launch(pdl_, k_restrict_first<T, 27>, row_blocks(L.nc), TH, s_, v, (const T*)L.r.p,
                   bc, (const T*)N.dinv.p, (T)N.c1[0], N.d.p, N.xa.p, done);
        else
            launch(pdl_, k_restrict_first<T, 0>, row_blocks(L.nc), TH, s_, v, (const T*)L.r.p,
                   bc, (const T*)N.dinv.p, (T)N.c1[0], N.d.p, N.xa.p, done);
    } else if (L.Ro.ok) {
        launch_transfer(L.Ro, (const T*)L.r.p, bc, 0, done, s_, pdl_);
    } else {
        launch(pdl_, k_restrict<T>, row_blocks(L.nc), TH, s_, L.nc, L.rptr.p, L.ridx.p, L.rval.p,
               L.r.p, bc, done);
    }
    FG_CHECK_LAUNCH();
    mark(tag + (fuse_first ? "restrict + L" + std::to_string(l + 1) + " first smooth"
                           : std::string("restrict")));
    launches_ += (started ? deg + 1 : deg + 2);
    const T* ec = enqueue_vcycle(H, l + 1, bc, fuse_first);
    if (L.Po.ok)
        launch_transfer(L.Po, ec, xa, 1, done, s_, pdl_);
    else
        launch(pdl_, k_prolong<T>, gb, TH, s_, n, L.pptr.p, L.pidx.p, L.pval.p, ec, xa, done);
    mark(tag + "prolong + correct");
    for (int k = 0; k < deg; ++k) {
        enqueue_step(L, b, xa, (T)L.c1[k], (T)L.c2[k], xb);
        mark(tag + "smooth post");
        std::swap(xa, xb);
    }
    FG_CHECK_LAUNCH();
    launches_ += deg + 1;
    return xa;
}

// q = A p with the partials of p.q (FP64).
void SolverImpl::enqueue_spmv_pq() {
    Scalars* sc = sc_.p;
    if (op64_.pair) {
        const int gp = row_blocks(pair_threads(n_));
        if (op64_.K == 8)
            launch(pdl_, k_pcg_spmv_pq_pair<8>, gp, TH, s_, op64_.sview(), p_.p, q_.p,
                   partial_.p, sc);
        else
            launch(pdl_, k_pcg_spmv_pq_pair<14>, gp, TH, s_, op64_.sview(), p_.p, q_.p,
                   partial_.p, sc);
    } else {
        with_op(op64_, [&](auto op) {
            launch(pdl_, k_pcg_spmv_pq<decltype(op)>, row_blocks(op64_.threads()), TH, s_, op,
                   p_.p, q_.p, partial_.p, sc);
        });
    }
}

void SolverImpl::enqueue_iteration() {
    int64_t n = n_;
    launches_ += 7;
    Scalars* sc = sc_.p;
    bool mixed = opt_.precision == FEMGPU_MIXED;
    const int nbq = row_blocks(op64_.threads()), nbn = row_blocks(n);
    enqueue_spmv_pq();
    mark("pcg q = A p, p.q partials (fp64)");
    launch(pdl_, k_finish<FinPq>, 1, FIN_TH, s_, partial_.p, nbq, FinPq{sc});
    mark("pcg alpha");
    launch(pdl_, k_pcg_update, nbn, TH, s_, n, x_.p, r_.p, p_.p, q_.p, mixed ? r32_.p : nullptr,
                                     partial_.p, sc);
    mark("pcg x, r update, r.r partials");
    launch(pdl_, k_finish<FinUpdate>, 1, FIN_TH, s_, partial_.p, nbn, FinUpdate{sc, tol});
    FG_CHECK_LAUNCH();
    mark("pcg stopping test");
    if (mixed) {
        zf_ = enqueue_vcycle<float>(H32_, 0, r32_.p);
        launch(pdl_, k_pcg_dots<float>, nbn, TH, s_, n, r_.p, zf_, q_.p, 1, 0, partial_.p, sc);
        mark("pcg r.z, z.q partials");
        launch(pdl_, k_finish<FinDots>, 1, FIN_TH, s_, partial_.p, nbn, FinDots{sc, 1, 0});
        mark("pcg beta");
        launch(pdl_, k_pcg_p<float>, nbn, TH, s_, n, zf_, p_.p, sc, 0);
        mark("pcg p = z + beta p");
    } else {
        zd_ = enqueue_vcycle<double>(H64_, 0, r_.p);
        launch(pdl_, k_pcg_dots<double>, nbn, TH, s_, n, r_.p, zd_, q_.p, 0, 0, partial_.p, sc);
        mark("pcg r.z partials");
        launch(pdl_, k_finish<FinDots>, 1, FIN_TH, s_, partial_.p, nbn, FinDots{sc, 0, 0});
        mark("pcg beta");
        launch(pdl_, k_pcg_p<double>, nbn, TH, s_, n, zd_, p_.p, sc, 0);
        mark("pcg p = z + beta p");
    }
    FG_CHECK_LAUNCH();
}

// The whole PCG loop as 1 graph: a WHILE conditional node whose body is 1 iteration followed by
// k_loop_control, so the device runs iteration after iteration with no host round trip.
void SolverImpl::build_loop_graph() {
    for (;;) {
        const size_t before = launches_;
        try {
            FG_CUDA(cudaGraphCreate(&graph_, 0));
            FG_CUDA(cudaGraphConditionalHandleCreate(&cond_, graph_, 1,
                                                     cudaGraphCondAssignDefault));
            cudaGraphNodeParams cp{};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond_;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            FG_CUDA(cudaGraphAddNode(&node, graph_, nullptr, 0, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            FG_CUDA(cudaStreamBeginCaptureToGraph(s_, body, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal));
            enqueue_iteration();
            k_loop_control<<<1, 1, 0, s_>>>(cond_, sc_.p, d_cancel_);
            FG_CUDA(cudaStreamEndCapture(s_, &body));
            FG_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
            graph_kernels_ = launches_ - before + 1;
            launches_ = before;
            return;
        } catch (const Failure&) {
            // A capture that failed (a cooperative launch that the graph did not take, for
            // one) ends here; the loop is captured again with every step its own launch.
            cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
            cudaStreamIsCapturing(s_, &st);
            if (st != cudaStreamCaptureStatusNone) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(s_, &g);
            }
            cudaGetLastError();
            if (exec_) cudaGraphExecDestroy(exec_);
            if (graph_) cudaGraphDestroy(graph_);
            exec_ = nullptr;
            graph_ = nullptr;
            launches_ = before;
            // Give up the fused coarse levels first, then the cluster legs, then the
            // programmatic launches.
            const bool clustered =
                std::count(H32_.cluster.begin(), H32_.cluster.end(), 1) +
                    std::count(H64_.cluster.begin(), H64_.cluster.end(), 1) > 0;
            if (tail_on_ && H32_.tail_from + H64_.tail_from > -2) {
                tail_on_ = false;
            } else if (cluster_on_ && clustered) {
                cluster_on_ = false;
            } else if (pdl_) {
                pdl_ = false;
            } else {
                throw;
            }
        }
    }
}

void SolverImpl::set_wait_limit(unsigned polls) {
    wait_limit = polls;
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    exec_ = nullptr;
    graph_ = nullptr;
}

void SolverImpl::run_device_loop(const volatile int* cancel) {
    int before = h_sc_->iters;
    *(volatile int*)h_cancel_ = 0;
    std::atomic<bool> stop{false};
    std::thread watcher;
    if (cancel) {
        // Mirrors the caller's flag into the mapped flag the device reads each iteration.
        watcher = std::thread([&] {
            while (!stop.load(std::memory_order_relaxed)) {
                if (*cancel) *(volatile int*)h_cancel_ = 1;
                std::this_thread::sleep_for(std::chrono::microseconds(50));
            }
        });
    }
    cudaError_t e = cudaGraphLaunch(exec_, s_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_sc_, sc_.p, sizeof(Scalars), cudaMemcpyDeviceToHost, s_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s_);
    stop.store(true);
    if (watcher.joinable()) watcher.join();
    FG_CUDA(e);
    launches_ += graph_kernels_ * (size_t)(h_sc_->iters - before);
}

// Host vectors: b and the start value go straight into the solver's own device vectors and the
// solution comes back from them, so a solve allocates nothing.
void SolverImpl::solve_host(const double* h_b, double* h_x, const volatile int* cancel,
                            femgpu_stats* st) {
    FG_CUDA(cudaMemcpyAsync(b_.p, h_b, n_ * 8, cudaMemcpyHostToDevice, s_));
    FG_CUDA(cudaMemcpyAsync(x_.p, h_x, n_ * 8, cudaMemcpyHostToDevice, s_));
    try {
        solve(b_.p, x_.p, cancel, st);
    } catch (const Failure&) {
        cudaMemcpyAsync(h_x, x_.p, n_ * 8, cudaMemcpyDeviceToHost, s_);
        cudaStreamSynchronize(s_);
        throw;
    }
    FG_CUDA(cudaMemcpyAsync(h_x, x_.p, n_ * 8, cudaMemcpyDeviceToHost, s_));
    FG_CUDA(cudaStreamSynchronize(s_));
}

void SolverImpl::solve_host_zero(const double* h_b, double* h_x, const volatile int* cancel,
                                 femgpu_stats* st) {
    FG_CUDA(cudaMemcpyAsync(b_.p, h_b, n_ * 8, cudaMemcpyHostToDevice, s_));
    FG_CUDA(cudaMemsetAsync(x_.p, 0, n_ * 8, s_));
    try {
        solve(b_.p, x_.p, cancel, st);
    } catch (const Failure&) {
        cudaMemcpyAsync(h_x, x_.p, n_ * 8, cudaMemcpyDeviceToHost, s_);
        cudaStreamSynchronize(s_);
        throw;
    }
    FG_CUDA(cudaMemcpyAsync(h_x, x_.p, n_ * 8, cudaMemcpyDeviceToHost, s_));
    FG_CUDA(cudaStreamSynchronize(s_));
}

void SolverImpl::precondition(const double* d_r, double* d_z) {
    FG_CUDA(cudaMemsetAsync(&sc_.p->done, 0, sizeof(int), s_));
    if (direct_ && sparse_) {
        sparse_->solve(d_r, d_z, s_);
    } else if (direct_) {
        k_gemv<double><<<blocks_for(n_ * 32, TH), TH, 0, s_>>>(n_, n_, dense_inv_.p, d_r, d_z,
                                                               done_zero_.p);
    } else if (opt_.precision == FEMGPU_MIXED) {
        k_convert<double, float><<<blocks_for(n_, TH), TH, 0, s_>>>(n_, d_r, r32_.p);
        const float* z = enqueue_vcycle<float>(H32_, 0, r32_.p);
        k_convert<float, double><<<blocks_for(n_, TH), TH, 0, s_>>>(n_, z, d_z);
    } else {
        const double* z = enqueue_vcycle<double>(H64_, 0, d_r);
        FG_CUDA(cudaMemcpyAsync(d_z, z, n_ * 8, cudaMemcpyDeviceToDevice, s_));
    }
    FG_CHECK_LAUNCH();
    FG_CUDA(cudaStreamSynchronize(s_));
}

void SolverImpl::solve(const double* d_b, double* d_x, const volatile int* cancel,
                       femgpu_stats* st) {
    int64_t n = n_;
    bool mixed = opt_.precision == FEMGPU_MIXED;
    FG_CUDA(cudaEventRecord(ev0_, s_));
    if (d_b != b_.p) FG_CUDA(cudaMemcpyAsync(b_.p, d_b, n * 8, cudaMemcpyDeviceToDevice, s_));
    Scalars init{};
    init.max_iter = (int)std::min<size_t>(max_iter, 0x7fffffff);
    FG_CUDA(cudaMemcpyAsync(sc_.p, &init, sizeof(Scalars), cudaMemcpyHostToDevice, s_));
    femgpu_stats out{};
    launches_ = 0;
    if (direct_) {
        // solve.rs:206-218: x = A^-1 b (with 1 step of refinement in FP64), then the true
        // residual.
        auto apply = [&](const double* rhs, double* sol) {
            if (sparse_) {
                sparse_->solve(rhs, sol, s_);
            } else {
                k_gemv<double><<<blocks_for(n * 32, TH), TH, 0, s_>>>(
                    n, n, dense_inv_.p, rhs, sol, done_zero_.p);
            }
        };
        launches_ = 8;
        apply(b_.p, x_.p);
        k_pcg_residual<<<row_blocks(A64_.nslices * A64_.C), TH, 0, s_>>>(
            SellOp<double>{A64_.view()}, b_.p, x_.p, r_.p, nullptr, partial_.p);
        k_finish<<<1, FIN_TH, 0, s_>>>(partial_.p, row_blocks(A64_.nslices * A64_.C),
                                   FinResidual0{sc_.p});
        apply(r_.p, t_.p);
        k_add<<<blocks_for(n, TH), TH, 0, s_>>>(n, t_.p, x_.p);
        FG_CHECK_LAUNCH();
        k_pcg_residual<<<row_blocks(A64_.nslices * A64_.C), TH, 0, s_>>>(
            SellOp<double>{A64_.view()}, b_.p, x_.p, r_.p, nullptr, partial_.p);
        k_finish<<<1, FIN_TH, 0, s_>>>(partial_.p, row_blocks(A64_.nslices * A64_.C),
                                   FinResidual0{sc_.p});
        FG_CHECK_LAUNCH();
        FG_CUDA(cudaMemcpyAsync(h_sc_, sc_.p, sizeof(Scalars), cudaMemcpyDeviceToHost, s_));
        if (d_x != x_.p) FG_CUDA(cudaMemcpyAsync(d_x, x_.p, n * 8, cudaMemcpyDeviceToDevice, s_));
        FG_CUDA(cudaEventRecord(ev1_, s_));
        FG_CUDA(cudaStreamSynchronize(s_));
        double bn = std::sqrt(h_sc_->bb), rn = std::sqrt(h_sc_->rr);
        out.iterations = 0;
        out.residual = bn > 0.0 ? rn / bn : rn;
        out.true_residual = out.residual;
        out.launches = launches_;
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0_, ev1_);
        out.seconds = ms * 1e-3;
        if (st) *st = out;
        return;
    }
    // multigrid.rs:692-753
    if (d_x != x_.p) FG_CUDA(cudaMemcpyAsync(x_.p, d_x, n * 8, cudaMemcpyDeviceToDevice, s_));
    with_op(op64_, [&](auto op) {
        k_pcg_residual<<<row_blocks(op64_.threads()), TH, 0, s_>>>(
            op, b_.p, x_.p, r_.p, mixed ? r32_.p : nullptr, partial_.p);
    });
    k_finish<<<1, FIN_TH, 0, s_>>>(partial_.p, row_blocks(op64_.threads()), FinResidual0{sc_.p});
    FG_CHECK_LAUNCH();
    launches_ += 5;  // this residual and its sum, r.z and its sum, and p = z  // this residual, and r.z and p = z after the first cycle
    FG_CUDA(cudaMemcpyAsync(h_sc_, sc_.p, sizeof(Scalars), cudaMemcpyDeviceToHost, s_));
    FG_CUDA(cudaStreamSynchronize(s_));
    double norm_b = h_sc_->norm_b;
    if (norm_b == 0.0) {
        FG_CUDA(cudaMemsetAsync(d_x, 0, n * 8, s_));
        FG_CUDA(cudaStreamSynchronize(s_));
        if (st) *st = out;
        return;
    }
    // z = M^-1 r, p = z, rz = r.z
    if (mixed) {
        zf_ = enqueue_vcycle<float>(H32_, 0, r32_.p);
        k_pcg_dots<float><<<row_blocks(n), TH, 0, s_>>>(n, r_.p, zf_, q_.p, 1, 1, partial_.p,
                                                        sc_.p);
        k_finish<<<1, FIN_TH, 0, s_>>>(partial_.p, row_blocks(n), FinDots{sc_.p, 1, 1});
        k_pcg_p<float><<<row_blocks(n), TH, 0, s_>>>(n, zf_, p_.p, sc_.p, 1);
    } else {
        zd_ = enqueue_vcycle<double>(H64_, 0, r_.p);
        k_pcg_dots<double><<<row_blocks(n), TH, 0, s_>>>(n, r_.p, zd_, q_.p, 0, 1, partial_.p,
                                                         sc_.p);
        k_finish<<<1, FIN_TH, 0, s_>>>(partial_.p, row_blocks(n), FinDots{sc_.p, 0, 1});
        k_pcg_p<double><<<row_blocks(n), TH, 0, s_>>>(n, zd_, p_.p, sc_.p, 1);
    }
    FG_CHECK_LAUNCH();
    if (opt_.graph && !exec_) build_loop_graph();
    int status = FEMGPU_OK;
    std::string message;
    double residual = std::sqrt(h_sc_->rr) / norm_b;
    size_t it = 0;
    int restarts = 0;
    for (;;) {
        // multigrid.rs:721-738: the residual test, then the iteration limit, then the cancel.
        if (residual <= tol) {
            // The true residual in FP64; with an FP32 preconditioner the recurrence can drift
            // from it, and then the solve restarts from x (iterative refinement).
            k_pcg_residual<<<row_blocks(A64_.nslices * A64_.C), TH, 0, s_>>>(
                SellOp<double>{A64_.view()}, b_.p, x_.p, t_.p, nullptr, partial_.p);
            k_finish<<<1, FIN_TH, 0, s_>>>(partial_.p, row_blocks(A64_.nslices * A64_.C),
                                       FinResidual0{sc_.p});
            FG_CHECK_LAUNCH();
            launches_ += 2;
            FG_CUDA(cudaMemcpyAsync(h_sc_, sc_.p, sizeof(Scalars), cudaMemcpyDeviceToHost, s_));
            FG_CUDA(cudaStreamSynchronize(s_));
            double truth = std::sqrt(h_sc_->rr) / norm_b;
            out.true_residual = truth;
            if (truth <= tol || !mixed || restarts >= 3 || it >= max_iter) break;
            ++restarts;
            FG_CUDA(cudaMemsetAsync(&sc_.p->done, 0, sizeof(int), s_));
            k_pcg_residual<<<row_blocks(A64_.nslices * A64_.C), TH, 0, s_>>>(
                SellOp<double>{A64_.view()}, b_.p, x_.p, r_.p, r32_.p, partial_.p);
            k_finish<<<1, FIN_TH, 0, s_>>>(partial_.p, row_blocks(A64_.nslices * A64_.C),
                                       FinResidual0{sc_.p});
            zf_ = enqueue_vcycle<float>(H32_, 0, r32_.p);
            k_pcg_dots<float><<<row_blocks(n), TH, 0, s_>>>(n, r_.p, zf_, q_.p, 1, 1, partial_.p,
                                                            sc_.p);
            k_finish<<<1, FIN_TH, 0, s_>>>(partial_.p, row_blocks(n), FinDots{sc_.p, 1, 1});
            k_pcg_p<float><<<row_blocks(n), TH, 0, s_>>>(n, zf_, p_.p, sc_.p, 1);
            FG_CHECK_LAUNCH();
            launches_ += 5;
            residual = truth;
            continue;
        }
        if (it == max_iter) {
            char buf[200];
            std::snprintf(buf, sizeof buf,
                          "conjugate gradients did not converge: the residual is %s after %zu "
                          "iterations",
                          rust_exp(residual, 2).c_str(), max_iter);
            status = FEMGPU_ERR_NOT_CONVERGED;
            message = buf;
            break;
        }
        if (cancel && *cancel) {
            status = FEMGPU_ERR_CANCELLED;
            message = "cancelled";
            break;
        }
        if (exec_) {
            run_device_loop(cancel);
            it = (size_t)h_sc_->iters;
        } else {
            enqueue_iteration();
            FG_CUDA(cudaMemcpyAsync(h_sc_, sc_.p, sizeof(Scalars), cudaMemcpyDeviceToHost, s_));
            FG_CUDA(cudaStreamSynchronize(s_));
            ++it;
        }
        residual = std::sqrt(h_sc_->rr) / norm_b;
        if (h_sc_->bulk_timeout) break;  // reported below, before any other outcome
        if (!(residual == residual)) {
            status = FEMGPU_ERR_NOT_CONVERGED;
            message = "conjugate gradients broke down: the residual is not a number";
            break;
        }
    }
    if (d_x != x_.p) FG_CUDA(cudaMemcpyAsync(d_x, x_.p, n * 8, cudaMemcpyDeviceToDevice, s_));
    FG_CUDA(cudaEventRecord(ev1_, s_));
    FG_CUDA(cudaStreamSynchronize(s_));
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    out.iterations = it;
    out.residual = residual;
    out.seconds = ms * 1e-3;
    out.launches = launches_;
    if (st) *st = out;
    if (!H32_.levels.empty() && H32_.levels[0].A.bulk) {
        // The Scalars were read back after the last kernel of the solve. A wait that ran out
        // leaves the iteration's vectors unfinished, so it is the outcome whatever else the
        // loop saw after it.
        if (h_sc_->bulk_timeout) {
            status = FEMGPU_ERR_TIMEOUT;
            message = "a bulk copy of a stencil tile did not complete within its wait limit";
        }
    }
    if (status != FEMGPU_OK) throw Failure(status, message);
}

void SolverImpl::mark(const std::string& label) {
    if (!trace_) return;
    cudaEvent_t e;
    FG_CUDA(cudaEventCreate(&e));
    FG_CUDA(cudaEventRecord(e, s_));
    trace_->push_back({label, e});
}

__global__ void k_fill(int64_t n, double* __restrict__ v, double value) {
    GRID_STRIDE(i, n) v[i] = value;
}

std::string SolverImpl::breakdown() {
    if (direct_)
        return sparse_ ? "direct method: sparse triangular solves and 1 refinement step\n"
                       : "direct method: 1 dense product and 1 refinement step\n";
    // Defined inputs: b = 1, x = 0, p = 1; no stopping test (tol < 0), so every kernel runs.
    k_fill<<<blocks_for(n_, TH), TH, 0, s_>>>(n_, b_.p, 1.0);
    k_fill<<<blocks_for(n_, TH), TH, 0, s_>>>(n_, x_.p, 0.0);
    k_fill<<<blocks_for(n_, TH), TH, 0, s_>>>(n_, r_.p, 1.0);
    k_fill<<<blocks_for(n_, TH), TH, 0, s_>>>(n_, p_.p, 1.0);
    if (opt_.precision == FEMGPU_MIXED)
        k_convert<double, float><<<blocks_for(n_, TH), TH, 0, s_>>>(n_, r_.p, r32_.p);
    Scalars init{};
    init.rz = 1.0;
    init.norm_b = 1.0;
    init.max_iter = 1;
    FG_CUDA(cudaMemcpyAsync(sc_.p, &init, sizeof(Scalars), cudaMemcpyHostToDevice, s_));
    double saved = tol;
    tol = -1.0;
    std::vector<std::pair<std::string, cudaEvent_t>> trace;
    std::string out;
    for (int pass = 0; pass < 3; ++pass) {  // the last of 3 warm passes is reported
        for (auto& t : trace) cudaEventDestroy(t.second);
        trace.clear();
        trace_ = &trace;
        mark("start");
        enqueue_iteration();
        trace_ = nullptr;
        FG_CUDA(cudaStreamSynchronize(s_));
    }
    tol = saved;
    double total = 0;
    char buf[200];
    for (size_t k = 1; k < trace.size(); ++k) {
        float ms = 0;
        FG_CUDA(cudaEventElapsedTime(&ms, trace[k - 1].second, trace[k].second));
        total += ms;
        std::snprintf(buf, sizeof buf, "%9.2f us  %s\n", ms * 1e3, trace[k].first.c_str());
        out += buf;
    }
    std::snprintf(buf, sizeof buf, "%9.2f us  total of 1 PCG iteration\n", total * 1e3);
    out += buf;
    for (auto& t : trace) cudaEventDestroy(t.second);
    return out;
}

// A second copy of a stencil level's operator and vectors (`kernel_time`): launched alternately
// with the level itself, each launch finds its data evicted from L2 by the other's, as in a
// solve, where the rest of the V-cycle streams between 2 uses of the finest level.
template <class T>
static bool shadow_level(const MgLevel<T>& L, MgLevel<T>* S, cudaStream_t s) {
    const Operator<T>& A = L.A;
    if (!A.stencil || A.half || A.bulk) return false;
    S->n = L.n;
    S->nnz = L.nnz;
    Operator<T>& B = S->A;
    B.stencil = true;
    B.unrolled = A.unrolled;
    B.pair = A.pair;
    B.march = A.march;
    B.mg = A.mg;
    B.n = A.n;
    B.nnz = A.nnz;
    B.K = A.K;
    B.ld = A.ld;
    B.off = A.off;
    B.coef.alloc(A.coef.count);
    FG_CUDA(cudaMemcpyAsync(B.coef.p, A.coef.p, A.coef.bytes(), cudaMemcpyDeviceToDevice, s));
    S->dinv.alloc(L.n);
    FG_CUDA(cudaMemcpyAsync(S->dinv.p, L.dinv.p, L.dinv.bytes(), cudaMemcpyDeviceToDevice, s));
    for (DevBuf<T>* v : {&S->b, &S->xa, &S->xb, &S->d}) {
        v->alloc(L.n);
        v->zero(s);
    }
    return true;
}

void SolverImpl::kernel_time(int which, int reps, double* ms, double* bytes) {
    if (reps < 1) reps = 1;
    bool mixed = opt_.precision == FEMGPU_MIXED;
    FG_CUDA(cudaMemsetAsync(&sc_.p->done, 0, sizeof(int), s_));
    // The finest level's second copy, where the level is a stencil.
    MgLevel<float> S32;
    MgLevel<double> S64;
    bool shadow = false;
    if (which == 0 && mixed && !H32_.levels.empty())
        shadow = shadow_level(H32_.levels[0], &S32, s_);
    else if (which == 0 && !mixed && !H64_.levels.empty())
        shadow = shadow_level(H64_.levels[0], &S64, s_);
    // The kernels the solve launches (the same dispatch and launch attributes), with done = 0;
    // launch k takes the level's copy k % 2.
    int k_launch = 0;
    auto launch = [&]() {
        const bool other = shadow && (k_launch++ & 1);
        if (which == 1) {
            enqueue_spmv_pq();
        } else if (mixed) {
            MgLevel<float>& L = other ? S32 : H32_.levels.at(0);
            enqueue_step(L, L.b.p, L.xa.p, 0.5f, 0.5f, L.xb.p);
        } else {
            MgLevel<double>& L = other ? S64 : H64_.levels.at(0);
            enqueue_step(L, L.b.p, L.xa.p, 0.5, 0.5, L.xb.p);
        }
    };
    if (which == 0 && (mixed ? H32_.levels.empty() : H64_.levels.empty()))
        throw Failure(FEMGPU_ERR_INVALID, "the solver has no smoothed level");
    if (which == 0) {
        // Defined inputs for the timed launches.
        if (mixed) {
            auto& L = H32_.levels[0];
            L.b.zero(s_); L.xa.zero(s_); L.d.zero(s_);
        } else {
            auto& L = H64_.levels[0];
            L.b.zero(s_); L.xa.zero(s_); L.d.zero(s_);
        }
    } else {
        p_.zero(s_);
    }
    for (int w = 0; w < 3; ++w) launch();
    FG_CHECK_LAUNCH();
    FG_CUDA(cudaEventRecord(ev0_, s_));
    for (int k = 0; k < reps; ++k) launch();
    FG_CUDA(cudaEventRecord(ev1_, s_));
    FG_CUDA(cudaEventSynchronize(ev1_));
    float t = 0;
    FG_CUDA(cudaEventElapsedTime(&t, ev0_, ev1_));
    *ms = t / reps;
    FG_CUDA(cudaStreamSynchronize(s_));  // before the copies are freed
    // A smoothing step streams the operator, x, y and 4 more vectors (b, D^-1, d read and
    // written); the PCG product the operator, p and q.
    if (which == 1) {
        *bytes = op64_.stream_bytes();
    } else if (mixed) {
        auto& L = H32_.levels[0];
        *bytes = L.A.stream_bytes() + 4.0 * (double)L.n * sizeof(float);
    } else {
        auto& L = H64_.levels[0];
        *bytes = L.A.stream_bytes() + 4.0 * (double)L.n * sizeof(double);
    }
}

}  // namespace femgpu
