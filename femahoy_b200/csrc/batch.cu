// Batched solves: many small systems of uneven sizes, each with several right sides, in 1 set
// of launches (no counterpart in the reference, whose callers solve 1 model at a time).
//
// Each system, a member, keeps the reference's own hierarchy (plane coarsening and Galerkin
// products, multigrid.rs:84-139, down to `coarsest` unknowns). Inside the batch the members are
// ordered by depth, deepest first, so that the members that have a level l form a prefix of the
// order, and those that go on below l a shorter prefix. Level l is then 1 vector over the
// members that have it: first the rows of the members that smooth at l and go on (1
// block-diagonal SELL operator, 1 launch of each smoothing kernel for all of them), then the
// rows of the members whose deepest level l is, solved by a dense inverse each. The right sides
// are interleaved, R per row (x[row * R + col]): the R threads of a row share each matrix entry,
// so 1 read of the operator serves all R solves. Every (member, right side) pair, a segment, is
// its own conjugate gradient solve with its own scalars and stopping test (multigrid.rs:692-753;
// the flexible form with the FP32 cycle); the sums of each segment are reduced over chunks of
// rows that never cross a member, in a fixed order, so a result does not depend on the timing.
// The iteration is 1 CUDA graph body under a WHILE node that runs until every segment has
// stopped. The caller's vectors are in the caller's member order; they are permuted into the
// batch's order at the start of a solve and back at the end.
#include <algorithm>
#include <atomic>
#include <memory>
#include <unordered_map>
#include <mutex>
#include <deque>
#include <condition_variable>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>
#include <type_traits>

#include "common.cuh"
#include "hierarchy.hpp"
#include "coarsen.cuh"
#include "offsets.cuh"
#include "block3.cuh"
#include "solver.cuh"
#include "rust_format.hpp"

namespace femgpu {

constexpr int BTH = 256;
constexpr int DTH = 32;   // rows of a dense tile

// ------------------------------------------------------------------ right sides in lanes
// A thread of the smoother kernels takes W = 16 bytes / sizeof(T) adjacent right sides (all R
// when fewer), loaded and stored as 16-byte vectors.
template <class T, int R>
struct Lanes {
    static constexpr int W = (int)(16 / sizeof(T)) < R ? (int)(16 / sizeof(T)) : R;
};

template <class T, int W>
__device__ __forceinline__ void load_lanes(const T* p, T (&o)[W]) {
    if constexpr ((W * sizeof(T)) % 16 == 0 && sizeof(T) == 4) {
#pragma unroll
        for (int h = 0; h < W / 4; ++h) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(p) + h);
            o[4 * h] = q.x, o[4 * h + 1] = q.y, o[4 * h + 2] = q.z, o[4 * h + 3] = q.w;
        }
    } else if constexpr ((W * sizeof(T)) % 16 == 0 && sizeof(T) == 8) {
#pragma unroll
        for (int h = 0; h < W / 2; ++h) {
            const double2 q = __ldg(reinterpret_cast<const double2*>(p) + h);
            o[2 * h] = q.x, o[2 * h + 1] = q.y;
        }
    } else {
#pragma unroll
        for (int e = 0; e < W; ++e) o[e] = __ldg(p + e);
    }
}

// Loads and stores of data that the same launch writes (no read-only path).
template <class T, int W>
__device__ __forceinline__ void read_lanes(const T* p, T (&o)[W]) {
    if constexpr ((W * sizeof(T)) % 16 == 0 && sizeof(T) == 4) {
#pragma unroll
        for (int h = 0; h < W / 4; ++h) {
            const float4 q = reinterpret_cast<const float4*>(p)[h];
            o[4 * h] = q.x, o[4 * h + 1] = q.y, o[4 * h + 2] = q.z, o[4 * h + 3] = q.w;
        }
    } else if constexpr ((W * sizeof(T)) % 16 == 0 && sizeof(T) == 8) {
#pragma unroll
        for (int h = 0; h < W / 2; ++h) {
            const double2 q = reinterpret_cast<const double2*>(p)[h];
            o[2 * h] = q.x, o[2 * h + 1] = q.y;
        }
    } else {
#pragma unroll
        for (int e = 0; e < W; ++e) o[e] = p[e];
    }
}

template <class T, int W>
__device__ __forceinline__ void write_lanes(T* p, const T (&v)[W]) {
    if constexpr ((W * sizeof(T)) % 16 == 0 && sizeof(T) == 4) {
#pragma unroll
        for (int h = 0; h < W / 4; ++h)
            reinterpret_cast<float4*>(p)[h] =
                make_float4(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
    } else if constexpr ((W * sizeof(T)) % 16 == 0 && sizeof(T) == 8) {
#pragma unroll
        for (int h = 0; h < W / 2; ++h)
            reinterpret_cast<double2*>(p)[h] = make_double2(v[2 * h], v[2 * h + 1]);
    } else {
#pragma unroll
        for (int e = 0; e < W; ++e) p[e] = v[e];
    }
}

// ------------------------------------------------------------------ operator with R columns
// (A x)[row][col] for the SELL matrix A and the column `col` of the interleaved x.
template <class T, int R>
__device__ __forceinline__ T sell_row_cols(const SellView<T>& A, int row, int col,
                                           const T* __restrict__ x) {
    const int s = row / A.C, r = row % A.C;
    const int64_t b = A.slice_ptr[s], e = A.slice_ptr[s + 1];
    const int groups = (int)((e - b) / (4 * A.C));
    const T* v = A.val + b + 4 * r;
    const uint32_t* c = A.col + b + 4 * r;
    T acc = 0;
    for (int k = 0; k < groups; ++k) {
        auto vv = load4(v);
        uint4 cc = __ldg(reinterpret_cast<const uint4*>(c));
        acc += vv.x * __ldg(x + (size_t)cc.x * R + col);
        acc += vv.y * __ldg(x + (size_t)cc.y * R + col);
        acc += vv.z * __ldg(x + (size_t)cc.z * R + col);
        acc += vv.w * __ldg(x + (size_t)cc.w * R + col);
        v += 4 * A.C;
        c += 4 * A.C;
    }
    return acc;
}

__device__ __forceinline__ int64_t elem_of_thread() {
    return blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
}

// The first Chebyshev step from x = 0: d = c1 D^-1 b, x = d.
template <class T, int R>
__global__ void k_bcheb_first(int64_t n, const T* __restrict__ b, const T* __restrict__ dinv,
                              T c1, T* __restrict__ d, T* __restrict__ x) {
    pdl_wait();
    const int64_t t = elem_of_thread();
    if (t >= n * R) return;
    T v = c1 * dinv[t / R] * b[t];
    d[t] = v;
    x[t] = v;
}

// sell_row_cols for the W right sides col .. col + W of a thread, each summed in the same order.
template <class T, int R>
__device__ __forceinline__ void sell_row_lanes(const SellView<T>& A, int row, int col,
                                               const T* __restrict__ x,
                                               T (&acc)[Lanes<T, R>::W]) {
    constexpr int W = Lanes<T, R>::W;
    const int s = row / A.C, r = row % A.C;
    const int64_t b = A.slice_ptr[s], e = A.slice_ptr[s + 1];
    const int groups = (int)((e - b) / (4 * A.C));
    const T* v = A.val + b + 4 * r;
    const uint32_t* c = A.col + b + 4 * r;
#pragma unroll
    for (int q = 0; q < W; ++q) acc[q] = 0;
    for (int k = 0; k < groups; ++k) {
        auto vv = load4(v);
        uint4 cc = __ldg(reinterpret_cast<const uint4*>(c));
        T x0[W], x1[W], x2[W], x3[W];
        load_lanes<T, W>(x + (size_t)cc.x * R + col, x0);
        load_lanes<T, W>(x + (size_t)cc.y * R + col, x1);
        load_lanes<T, W>(x + (size_t)cc.z * R + col, x2);
        load_lanes<T, W>(x + (size_t)cc.w * R + col, x3);
#pragma unroll
        for (int q = 0; q < W; ++q) {
            acc[q] += vv.x * x0[q];
            acc[q] += vv.y * x1[q];
            acc[q] += vv.z * x2[q];
            acc[q] += vv.w * x3[q];
        }
        v += 4 * A.C;
        c += 4 * A.C;
    }
}

// d = c2 d + c1 D^-1 (b - A x), x_out = x + d.
template <class T, int R>
__global__ void __launch_bounds__(BTH)
    k_bcheb_step(SellView<T> A, const T* __restrict__ b, const T* __restrict__ xin,
                 const T* __restrict__ dinv, T c1, T c2, T* __restrict__ d, T* __restrict__ xout) {
    constexpr int W = Lanes<T, R>::W, P = R / W;
    pdl_wait();
    const int64_t t = elem_of_thread();
    if (t >= A.n * P) return;
    const int row = (int)(t / P), col = (int)(t % P) * W;
    T acc[W], bb[W], dd[W], xx[W];
    sell_row_lanes<T, R>(A, row, col, xin, acc);
    const int64_t i = (int64_t)row * R + col;
    read_lanes<T, W>(b + i, bb);
    read_lanes<T, W>(d + i, dd);
    read_lanes<T, W>(xin + i, xx);
    const T di = dinv[row];
#pragma unroll
    for (int q = 0; q < W; ++q) {
        const T r = bb[q] - acc[q];
        dd[q] = c2 * dd[q] + c1 * di * r;
        xx[q] = xx[q] + dd[q];
    }
    write_lanes<T, W>(d + i, dd);
    write_lanes<T, W>(xout + i, xx);
}

template <class T, int R>
__global__ void __launch_bounds__(BTH)
    k_bresidual(SellView<T> A, const T* __restrict__ b, const T* __restrict__ x, T* __restrict__ r) {
    constexpr int W = Lanes<T, R>::W, P = R / W;
    pdl_wait();
    const int64_t t = elem_of_thread();
    if (t >= A.n * P) return;
    const int row = (int)(t / P), col = (int)(t % P) * W;
    T acc[W], bb[W];
    sell_row_lanes<T, R>(A, row, col, x, acc);
    const int64_t i = (int64_t)row * R + col;
    read_lanes<T, W>(b + i, bb);
#pragma unroll
    for (int q = 0; q < W; ++q) bb[q] = bb[q] - acc[q];
    write_lanes<T, W>(r + i, bb);
}

// ------------------------------------------------------------------ 3x3-block operators
// (A x)[3 br + a][col .. col + W) for a = 0, 1, 2 on the 3x3-block form (block3.cuh): each of
// the R / W threads of a block row takes W adjacent right sides, so that a block's column and 9
// values are loaded once per W right sides and each x block row arrives as 16-byte vectors. Each
// (row, right side) sum runs over the blocks in order, 3 terms per block, as with 1 right side
// per thread.
template <class T, int R>
__device__ __forceinline__ void bsell3_rows(const BSell3View<T>& A, int br, int col,
                                            const T* __restrict__ x,
                                            T (&acc)[3][Lanes<T, R>::W]) {
    constexpr int W = Lanes<T, R>::W;
    const int s = br / B3C, r = br % B3C;
    const int64_t b = A.slice_ptr[s], e = A.slice_ptr[s + 1];
    const int w = (int)((e - b) / B3C);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int q = 0; q < W; ++q) acc[a][q] = 0;
    // 2 blocks per pass: both columns, then both blocks' x rows and values in flight before
    // the sums, which stay in block order.
    int k = 0;
    for (; k + 1 < w; k += 2) {
        const int64_t blk = b + (int64_t)k * B3C + r;
        const uint32_t J0 = __ldg(A.col + blk), J1 = __ldg(A.col + blk + B3C);
        T xv[2][3][W], v[2][9];
#pragma unroll
        for (int h = 0; h < 3; ++h) {
            load_lanes<T, W>(x + ((size_t)3 * J0 + h) * R + col, xv[0][h]);
            load_lanes<T, W>(x + ((size_t)3 * J1 + h) * R + col, xv[1][h]);
        }
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            v[0][e] = __ldg(A.val + blk * 9 + e);
            v[1][e] = __ldg(A.val + (blk + B3C) * 9 + e);
        }
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int q = 0; q < W; ++q) {
                    acc[a][q] += v[u][3 * a] * xv[u][0][q];
                    acc[a][q] += v[u][3 * a + 1] * xv[u][1][q];
                    acc[a][q] += v[u][3 * a + 2] * xv[u][2][q];
                }
    }
    if (k < w) {
        const int64_t blk = b + (int64_t)k * B3C + r;
        const uint32_t J = __ldg(A.col + blk);
        const T* v = A.val + blk * 9;
        T x0[W], x1[W], x2[W];
        load_lanes<T, W>(x + ((size_t)3 * J) * R + col, x0);
        load_lanes<T, W>(x + ((size_t)3 * J + 1) * R + col, x1);
        load_lanes<T, W>(x + ((size_t)3 * J + 2) * R + col, x2);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const T v0 = __ldg(v + 3 * a), v1 = __ldg(v + 3 * a + 1), v2 = __ldg(v + 3 * a + 2);
#pragma unroll
            for (int q = 0; q < W; ++q) {
                acc[a][q] += v0 * x0[q];
                acc[a][q] += v1 * x1[q];
                acc[a][q] += v2 * x2[q];
            }
        }
    }
}

// The sums of bsell3_rows for 1 right side `col` (the FP64 outer iteration's kernels, whose
// dot products are formed per right side).
template <class T, int R>
__device__ __forceinline__ void bsell3_rows_col(const BSell3View<T>& A, int br, int col,
                                                const T* __restrict__ x, T* acc) {
    const int s = br / B3C, r = br % B3C;
    const int64_t b = A.slice_ptr[s], e = A.slice_ptr[s + 1];
    const int w = (int)((e - b) / B3C);
    acc[0] = acc[1] = acc[2] = 0;
    int k = 0;
    for (; k + 1 < w; k += 2) {  // 2 blocks' loads in flight, the sums in block order
        const int64_t blk = b + (int64_t)k * B3C + r;
        const uint32_t J0 = __ldg(A.col + blk), J1 = __ldg(A.col + blk + B3C);
        T xv[2][3], v[2][9];
#pragma unroll
        for (int h = 0; h < 3; ++h) {
            xv[0][h] = __ldg(x + ((size_t)3 * J0 + h) * R + col);
            xv[1][h] = __ldg(x + ((size_t)3 * J1 + h) * R + col);
        }
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            v[0][e] = __ldg(A.val + blk * 9 + e);
            v[1][e] = __ldg(A.val + (blk + B3C) * 9 + e);
        }
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                acc[a] += v[u][3 * a] * xv[u][0];
                acc[a] += v[u][3 * a + 1] * xv[u][1];
                acc[a] += v[u][3 * a + 2] * xv[u][2];
            }
    }
    if (k < w) {
        const int64_t blk = b + (int64_t)k * B3C + r;
        const uint32_t J = __ldg(A.col + blk);
        const T* v = A.val + blk * 9;
        const T x0 = __ldg(x + ((size_t)3 * J) * R + col);
        const T x1 = __ldg(x + ((size_t)3 * J + 1) * R + col);
        const T x2 = __ldg(x + ((size_t)3 * J + 2) * R + col);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            acc[a] += __ldg(v + 3 * a) * x0;
            acc[a] += __ldg(v + 3 * a + 1) * x1;
            acc[a] += __ldg(v + 3 * a + 2) * x2;
        }
    }
}

// The Chebyshev step of k_bcheb_step on a 3x3-block operator.
template <class T, int R>
__global__ void __launch_bounds__(BTH)
    k_bcheb_step3(BSell3View<T> A, const T* __restrict__ b, const T* __restrict__ xin,
                  const T* __restrict__ dinv, T c1, T c2, T* __restrict__ d,
                  T* __restrict__ xout) {
    constexpr int W = Lanes<T, R>::W, P = R / W;
    pdl_wait();
    const int64_t t = elem_of_thread();
    if (t >= A.nb * P) return;
    const int br = (int)(t / P), col = (int)(t % P) * W;
    T acc[3][W];
    bsell3_rows<T, R>(A, br, col, xin, acc);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int64_t row = 3 * (int64_t)br + a, i = row * R + col;
        T bb[W], dd[W], xx[W];
        read_lanes<T, W>(b + i, bb);
        read_lanes<T, W>(d + i, dd);
        read_lanes<T, W>(xin + i, xx);
        const T di = dinv[row];
#pragma unroll
        for (int q = 0; q < W; ++q) {
            const T r = bb[q] - acc[a][q];
            dd[q] = c2 * dd[q] + c1 * di * r;
            xx[q] = xx[q] + dd[q];
        }
        write_lanes<T, W>(d + i, dd);
        write_lanes<T, W>(xout + i, xx);
    }
}

template <class T, int R>
__global__ void __launch_bounds__(BTH)
    k_bresidual3(BSell3View<T> A, const T* __restrict__ b, const T* __restrict__ x,
                 T* __restrict__ r) {
    constexpr int W = Lanes<T, R>::W, P = R / W;
    pdl_wait();
    const int64_t t = elem_of_thread();
    if (t >= A.nb * P) return;
    const int br = (int)(t / P), col = (int)(t % P) * W;
    T acc[3][W];
    bsell3_rows<T, R>(A, br, col, x, acc);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int64_t i = (3 * (int64_t)br + a) * R + col;
        T bb[W];
        read_lanes<T, W>(b + i, bb);
#pragma unroll
        for (int q = 0; q < W; ++q) bb[q] = bb[q] - acc[a][q];
        write_lanes<T, W>(r + i, bb);
    }
}

// out = M in (accumulate: out += M in) for a CSR transfer M, R columns.
template <class T, int R>
__global__ void k_bgather(int64_t rows, const int64_t* __restrict__ ptr,
                          const uint32_t* __restrict__ idx, const T* __restrict__ val,
                          const T* __restrict__ in, T* __restrict__ out, int accumulate) {
    pdl_wait();
    const int64_t t = elem_of_thread();
    if (t >= rows * R) return;
    const int64_t row = t / R;
    const int col = (int)(t % R);
    T s = 0;
    for (int64_t k = ptr[row]; k < ptr[row + 1]; ++k)
        s += val[k] * __ldg(in + (size_t)idx[k] * R + col);
    if (accumulate)
        out[t] += s;
    else
        out[t] = s;
}

// The members whose deepest level this is: out = M in for each, M its inverse, stored in tiles
// of DTH = 32 rows, each tile by column (the 32 entries of column j of the tile contiguous). A
// block takes 1 tile; its DW warps split the columns j into DW contiguous ranges. A warp takes
// its columns 32 at a time: lane q brings the R right-side values of column j + q into the
// warp's shared buffer (the next 32 already loading into registers while this 32 is used), then
// lane i (row i of the tile) adds M[i][j] times the buffered values, the loads of M 8 columns
// ahead. The DW partial sums are added in warp order through shared memory.
constexpr int DW = 8;

template <class T, int R>
struct DenseChunk {
    static constexpr int V = R % 4 == 0 ? R / 4 : R;  // loads of a row: 4-vectors, or scalars
    typename std::conditional<R % 4 == 0, typename Vec4<T>::type, T>::type v[V];
    __device__ __forceinline__ void load(const T* __restrict__ row, bool ok) {
#pragma unroll
        for (int k = 0; k < V; ++k) {
            if constexpr (R % 4 == 0) {
                if (ok) {
                    v[k] = load4(row + 4 * k);
                } else {
                    v[k].x = v[k].y = v[k].z = v[k].w = 0;
                }
            } else {
                v[k] = ok ? __ldg(row + k) : (T)0;
            }
        }
    }
    __device__ __forceinline__ void store(T* dst) const {
#pragma unroll
        for (int k = 0; k < V; ++k) {
            if constexpr (R % 4 == 0) {
                dst[4 * k] = v[k].x;
                dst[4 * k + 1] = v[k].y;
                dst[4 * k + 2] = v[k].z;
                dst[4 * k + 3] = v[k].w;
            } else {
                dst[k] = v[k];
            }
        }
    }
};

template <class T, int R>
__global__ void __launch_bounds__(32 * DW)
    k_bdense(const int2* __restrict__ tiles, const int64_t* __restrict__ off,
             const int64_t* __restrict__ ioff, const T* __restrict__ inv,
             const T* __restrict__ in, T* __restrict__ out) {
    pdl_wait();
    // Per warp a buffer of 32 right-side rows; reused at the end for the partial sums.
    constexpr int STAGE = DW * 32 * R, PART = DW * DTH * (R + 1);
    __shared__ T smem[STAGE > PART ? STAGE : PART];
    const int2 tl = tiles[blockIdx.x];
    const int64_t r0 = off[tl.x], m = off[tl.x + 1] - r0;
    const T* __restrict__ Mt = inv + ioff[tl.x] + (int64_t)tl.y * m;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool row_ok = tl.y + lane < m;
    const int64_t j0 = m * w / DW, j1 = m * (w + 1) / DW;
    T* buf = smem + w * 32 * R;
    T acc[R];
#pragma unroll
    for (int c = 0; c < R; ++c) acc[c] = 0;
    DenseChunk<T, R> next;
    next.load(in + (r0 + j0 + lane) * R, j0 + lane < j1);
    for (int64_t jc = j0; jc < j1; jc += 32) {
        __syncwarp();
        next.store(buf + lane * R);
        __syncwarp();
        if (jc + 32 < j1) next.load(in + (r0 + jc + 32 + lane) * R, jc + 32 + lane < j1);
        const int nj = (int)min((int64_t)32, j1 - jc);
        if (row_ok) {
            int q = 0;
            for (; q + 8 <= nj; q += 8) {
                T mv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) mv[u] = __ldg(Mt + 32 * (jc + q + u) + lane);
#pragma unroll
                for (int u = 0; u < 8; ++u)
#pragma unroll
                    for (int c = 0; c < R; ++c) acc[c] += mv[u] * buf[(q + u) * R + c];
            }
            for (; q < nj; ++q) {
                const T mv = __ldg(Mt + 32 * (jc + q) + lane);
#pragma unroll
                for (int c = 0; c < R; ++c) acc[c] += mv * buf[q * R + c];
            }
        }
    }
    __syncthreads();
    T* part = smem;  // [DW][DTH][R + 1]
#pragma unroll
    for (int c = 0; c < R; ++c) part[(w * DTH + lane) * (R + 1) + c] = acc[c];
    __syncthreads();
    for (int t = threadIdx.x; t < DTH * R; t += 32 * DW) {
        const int row = t / R, c = t % R;
        if (tl.y + row < m) {
            T sum = 0;
#pragma unroll
            for (int q = 0; q < DW; ++q) sum += part[(q * DTH + row) * (R + 1) + c];
            out[(r0 + tl.y + row) * R + c] = sum;
        }
    }
}

// out[row] = in[map[row]] (gather) or out[map[row]] = in[row] (scatter), R columns: the
// caller's member order to the batch's and back.
template <int R>
__global__ void k_bpermute(int64_t n, const int* __restrict__ map, const double* __restrict__ in,
                           double* __restrict__ out, int scatter) {
    const int64_t t = elem_of_thread();
    if (t >= n * R) return;
    const int64_t row = t / R;
    const int col = (int)(t % R);
    const int64_t other = (int64_t)map[row] * R + col;
    if (scatter)
        out[other] = in[t];
    else
        out[t] = in[other];
}

// The phases of a streamed segment (continuous batching, femgpu_stream_*): a free slot; a right
// side admitted this iteration (x = 0, r = b; the iteration's product and update leave them, the
// cycle and the dots start the recurrence with p = z); running PCG; its true residual being formed
// (q = A x, r = b - A x) once the recurrence has stopped; finished, its x waiting to be delivered.
enum { PH_FREE = 0, PH_FRESH = 1, PH_RUN = 2, PH_VERIFY = 3, PH_DONE = 4 };

// ------------------------------------------------------------------ PCG over segments
// A block of the PCG kernels takes 1 chunk: rows [row0, row1) of member `sys`. Thread t takes
// column t % R and rows row0 + t / R, row0 + t / R + BTH / R, ...
struct Chunk {
    int sys;
    int row0, row1;
};

// The per-segment scalars (arrays of B R; segment s = member s / R, right side s % R).
struct BatchScalars {
    double *bb, *rr, *rz, *pq, *alpha, *beta, *truth;
    int *done, *iters, *status;  // status: 0 running or converged, 1 iteration limit, 2 NaN
};

// The per-column sums of a block (2 values each), to partial[(chunk R + col) 2 + {0, 1}], each
// in a fixed order.
template <int R>
__device__ __forceinline__ void chunk_partial(double a, double b, double* __restrict__ partial) {
    __shared__ double sa[BTH], sb[BTH];
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    if (threadIdx.x < R) {
        double ta = 0, tb = 0;
        for (int k = threadIdx.x; k < BTH; k += R) {
            ta += sa[k];
            tb += sb[k];
        }
        partial[((int64_t)blockIdx.x * R + threadIdx.x) * 2] = ta;
        partial[((int64_t)blockIdx.x * R + threadIdx.x) * 2 + 1] = tb;
    }
}

// r = b - A x with the sums b.b and r.r (the exact FP64 operator); r and its FP32 copy are
// written when their pointers are set.
template <int R>
__global__ void __launch_bounds__(BTH)
    k_bpcg_residual(SellView<double> A, const Chunk* __restrict__ chunks,
                    const double* __restrict__ b, const double* __restrict__ x,
                    double* __restrict__ r, float* __restrict__ r32,
                    double* __restrict__ partial) {
    pdl_wait();
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    double bb = 0, rr = 0;
    for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R) {
        const int64_t t = (int64_t)row * R + col;
        double ri = b[t] - sell_row_cols<double, R>(A, row, col, x);
        if (r) r[t] = ri;
        if (r32) r32[t] = (float)ri;
        bb += b[t] * b[t];
        rr += ri * ri;
    }
    chunk_partial<R>(bb, rr, partial);
}

// q = A p with the sums p.q (multigrid.rs:740-741).
template <int R>
__global__ void __launch_bounds__(BTH)
    k_bpcg_spmv(SellView<double> A, const Chunk* __restrict__ chunks, const double* __restrict__ p,
                double* __restrict__ q, const int* __restrict__ done,
                double* __restrict__ partial, const int* __restrict__ phase,
                const double* __restrict__ xv) {
    pdl_wait();
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    const int seg = ch.sys * R + col;
    // A streamed segment being verified takes q = A x (its true residual follows).
    const double* __restrict__ v = (phase && phase[seg] == PH_VERIFY) ? xv : p;
    double pq = 0;
    if (!done[seg])
        for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R) {
            const int64_t t = (int64_t)row * R + col;
            double ap = sell_row_cols<double, R>(A, row, col, v);
            q[t] = ap;
            pq += v[t] * ap;
        }
    chunk_partial<R>(pq, 0.0, partial);
}

// k_bpcg_residual and k_bpcg_spmv on the 3x3-block form of the exact operator: a chunk's rows
// are whole nodes (multiples of 3), and a thread takes block rows of 1 column.
template <int R>
__global__ void __launch_bounds__(BTH)
    k_bpcg_residual3(BSell3View<double> A, const Chunk* __restrict__ chunks,
                     const double* __restrict__ b, const double* __restrict__ x,
                     double* __restrict__ r, float* __restrict__ r32,
                     double* __restrict__ partial) {
    pdl_wait();
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    double bb = 0, rr = 0;
    for (int br = ch.row0 / 3 + threadIdx.x / R; br < ch.row1 / 3; br += BTH / R) {
        double acc[3];
        bsell3_rows_col<double, R>(A, br, col, x, acc);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int64_t t = (3 * (int64_t)br + a) * R + col;
            const double ri = b[t] - acc[a];
            if (r) r[t] = ri;
            if (r32) r32[t] = (float)ri;
            bb += b[t] * b[t];
            rr += ri * ri;
        }
    }
    chunk_partial<R>(bb, rr, partial);
}

template <int R>
__global__ void __launch_bounds__(BTH)
    k_bpcg_spmv3(BSell3View<double> A, const Chunk* __restrict__ chunks,
                 const double* __restrict__ p, double* __restrict__ q,
                 const int* __restrict__ done, double* __restrict__ partial,
                 const int* __restrict__ phase, const double* __restrict__ xv) {
    pdl_wait();
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    const int seg = ch.sys * R + col;
    const double* __restrict__ v = (phase && phase[seg] == PH_VERIFY) ? xv : p;
    double pq = 0;
    if (!done[seg])
        for (int br = ch.row0 / 3 + threadIdx.x / R; br < ch.row1 / 3; br += BTH / R) {
            double acc[3];
            bsell3_rows_col<double, R>(A, br, col, v, acc);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int64_t t = (3 * (int64_t)br + a) * R + col;
                q[t] = acc[a];
                pq += v[t] * acc[a];
            }
        }
    chunk_partial<R>(pq, 0.0, partial);
}

// x += alpha p, r -= alpha q (multigrid.rs:742-745) with the sums r.r.
template <int R>
__global__ void __launch_bounds__(BTH)
    k_bpcg_update(const Chunk* __restrict__ chunks, double* __restrict__ x,
                  double* __restrict__ r, const double* __restrict__ p,
                  const double* __restrict__ q, float* __restrict__ r32, BatchScalars sc,
                  double* __restrict__ partial, const int* __restrict__ phase,
                  const double* __restrict__ b) {
    pdl_wait();
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    const int seg = ch.sys * R + col;
    double rr = 0;
    if (phase && phase[seg] == PH_VERIFY) {
        // A streamed segment being verified: r = b - A x (q holds A x), x unchanged.
        for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R) {
            const int64_t t = (int64_t)row * R + col;
            const double ri = b[t] - q[t];
            r[t] = ri;
            if (r32) r32[t] = (float)ri;
            rr += ri * ri;
        }
    } else if (!sc.done[seg]) {
        const double alpha = sc.alpha[seg];
        for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R) {
            const int64_t t = (int64_t)row * R + col;
            x[t] += alpha * p[t];
            double ri = r[t] - alpha * q[t];
            r[t] = ri;
            if (r32) r32[t] = (float)ri;
            rr += ri * ri;
        }
    }
    chunk_partial<R>(rr, 0.0, partial);
}

// The sums r.z and (flexible form, after the first) z.q.
template <int R, class TZ>
__global__ void __launch_bounds__(BTH)
    k_bpcg_dots(const Chunk* __restrict__ chunks, const double* __restrict__ r,
                const TZ* __restrict__ z, const double* __restrict__ q, int flexible, int init,
                const int* __restrict__ done, double* __restrict__ partial) {
    pdl_wait();
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    double rz = 0, zq = 0;
    if (!done[ch.sys * R + col])
        for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R) {
            const int64_t t = (int64_t)row * R + col;
            double zi = (double)z[t];
            rz += r[t] * zi;
            if (flexible && !init) zq += zi * q[t];
        }
    chunk_partial<R>(rz, zq, partial);
}

// p = z + beta p (multigrid.rs:749), p = z on the first.
template <int R, class TZ>
__global__ void k_bpcg_p(const Chunk* __restrict__ chunks, const TZ* __restrict__ z,
                         double* __restrict__ p, BatchScalars sc, int init) {
    pdl_wait();
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    const int seg = ch.sys * R + col;
    if (sc.done[seg]) return;
    const double beta = sc.beta[seg];
    for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R) {
        const int64_t t = (int64_t)row * R + col;
        p[t] = init ? (double)z[t] : (double)z[t] + beta * p[t];
    }
}

// x = 0 for the segments whose right side is 0 (multigrid.rs:704-711).
template <int R>
__global__ void k_bzero_empty(const Chunk* __restrict__ chunks, const double* __restrict__ bb,
                              double* __restrict__ x) {
    pdl_wait();
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    if (bb[ch.sys * R + col] != 0.0) return;
    for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R)
        x[(int64_t)row * R + col] = 0.0;
}

enum FinishKind { FIN_START = 0, FIN_PQ = 1, FIN_UPDATE = 2, FIN_DOTS = 3, FIN_TRUTH = 4,
                  FIN_RESTART = 5, FIN_SPQ = 6, FIN_SUPDATE = 7, FIN_SDOTS = 8 };

// The per-segment state of streaming (null in a plain batch solve).
struct StreamState {
    int* phase;
    int* restarts;
    int* fresh;  // 1: the next dots start the recurrence (beta = 0)
};

// 1 block per member: the sums of each of its R segments over the member's chunks (a fixed
// tree), then the segment's scalars. FIN_START: the first residual (stop at once if
// |r| <= tol |b| or b = 0, multigrid.rs:704-723); FIN_PQ: alpha; FIN_UPDATE: the stopping test
// and the iteration limit (multigrid.rs:721-733); FIN_DOTS: beta; FIN_TRUTH: the true residual
// |b - A x| / |b|; FIN_RESTART: the segments whose true residual drifted above tol run again
// from x (iterative refinement).
template <int R>
__global__ void __launch_bounds__(BTH)
    k_bfinish(int kind, const int* __restrict__ cstart, const double* __restrict__ partial,
              BatchScalars sc, double tol, int max_iter, int flexible, int init,
              StreamState ss, double true_tol) {
    pdl_wait();
    __shared__ double sa[BTH], sb[BTH];
    const int sys = blockIdx.x;
    const int col = threadIdx.x % R, lane = threadIdx.x / R;
    double a = 0, b = 0;
    for (int c = cstart[sys] + lane; c < cstart[sys + 1]; c += BTH / R) {
        a += partial[((int64_t)c * R + col) * 2];
        b += partial[((int64_t)c * R + col) * 2 + 1];
    }
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int st = (BTH / R) / 2; st > 0; st >>= 1) {
        if (lane < st) {
            sa[threadIdx.x] += sa[threadIdx.x + st * R];
            sb[threadIdx.x] += sb[threadIdx.x + st * R];
        }
        __syncthreads();
    }
    if (threadIdx.x >= R) return;
    a = sa[threadIdx.x];
    b = sb[threadIdx.x];
    const int s = sys * R + col;
    if (kind >= FIN_SPQ) {
        // Streaming: each segment by its phase.
        const int ph = ss.phase[s];
        if (kind == FIN_SPQ) {
            if (ph == PH_RUN) {
                sc.pq[s] = a;
                sc.alpha[s] = sc.rz[s] / a;
            } else if (ph == PH_FRESH) {
                sc.alpha[s] = 0.0;  // x and r stay 0 and b
            }
        } else if (kind == FIN_SUPDATE) {
            if (ph == PH_FRESH) {
                // r = b: the start of multigrid.rs:704-723 from x = 0.
                sc.bb[s] = a;
                sc.rr[s] = a;
                sc.iters[s] = 0;
                sc.status[s] = 0;
                sc.truth[s] = 0.0;
                ss.restarts[s] = 0;
                if (a == 0.0) {
                    ss.phase[s] = PH_DONE;  // b = 0 gives x = 0
                    sc.done[s] = 1;
                } else if (max_iter <= 0) {
                    sc.status[s] = 1;
                    ss.phase[s] = PH_VERIFY;
                } else {
                    ss.phase[s] = PH_RUN;
                    ss.fresh[s] = 1;
                }
            } else if (ph == PH_RUN) {
                sc.rr[s] = a;
                sc.iters[s] += 1;
                if (!(a == a)) {
                    sc.status[s] = 2;
                    ss.phase[s] = PH_DONE;
                    sc.done[s] = 1;
                } else if (sqrt(a) / sqrt(sc.bb[s]) <= tol) {
                    ss.phase[s] = PH_VERIFY;
                } else if (sc.iters[s] >= max_iter) {
                    sc.status[s] = 1;
                    ss.phase[s] = PH_VERIFY;
                }
            } else if (ph == PH_VERIFY) {
                // The true residual; a mixed form's recurrence that drifted above tol runs
                // again from x, at most 3 times (as the plain batch's FIN_RESTART).
                sc.truth[s] = sqrt(a) / sqrt(sc.bb[s]);
                if (flexible && sc.status[s] == 0 && sc.truth[s] > true_tol &&
                    ss.restarts[s] < 3 && sc.iters[s] < max_iter) {
                    ss.restarts[s] += 1;
                    sc.rr[s] = a;
                    ss.phase[s] = PH_RUN;
                    ss.fresh[s] = 1;
                } else {
                    ss.phase[s] = PH_DONE;
                    sc.done[s] = 1;
                }
            }
        } else if (ph == PH_RUN) {  // FIN_SDOTS
            if (ss.fresh[s]) {
                sc.beta[s] = 0;
                ss.fresh[s] = 0;
            } else if (flexible) {
                sc.beta[s] = -sc.alpha[s] * b / sc.rz[s];
            } else {
                sc.beta[s] = a / sc.rz[s];
            }
            sc.rz[s] = a;
        }
        return;
    }
    switch (kind) {
        case FIN_START:
            sc.bb[s] = a;
            sc.rr[s] = b;
            sc.iters[s] = 0;
            sc.status[s] = 0;
            sc.truth[s] = 0;
            if (a == 0.0 || sqrt(b) / sqrt(a) <= tol) {
                sc.done[s] = 1;
            } else if (max_iter <= 0) {
                sc.done[s] = 1;
                sc.status[s] = 1;
            } else {
                sc.done[s] = 0;
            }
            return;
        case FIN_TRUTH:
            sc.truth[s] = sc.bb[s] > 0.0 ? sqrt(b) / sqrt(sc.bb[s]) : 0.0;
            return;
        case FIN_RESTART:
            if (sc.done[s] && sc.status[s] == 0 && sc.bb[s] > 0.0 && sc.truth[s] > tol &&
                sc.iters[s] < max_iter) {
                sc.rr[s] = b;
                sc.done[s] = 0;
            }
            return;
        default:
            break;
    }
    if (sc.done[s]) return;
    if (kind == FIN_PQ) {
        sc.pq[s] = a;
        sc.alpha[s] = sc.rz[s] / a;
    } else if (kind == FIN_UPDATE) {
        sc.rr[s] = a;
        sc.iters[s] += 1;
        if (!(a == a)) {
            sc.done[s] = 1;
            sc.status[s] = 2;
        } else if (sqrt(a) / sqrt(sc.bb[s]) <= tol) {
            sc.done[s] = 1;
        } else if (sc.iters[s] >= max_iter) {
            sc.done[s] = 1;
            sc.status[s] = 1;
        }
    } else {
        if (init)
            sc.beta[s] = 0;
        else if (flexible)
            sc.beta[s] = -sc.alpha[s] * b / sc.rz[s];  // flexible CG: -alpha z.q / r.z_old
        else
            sc.beta[s] = a / sc.rz[s];  // multigrid.rs:747-748
        sc.rz[s] = a;
    }
}

// Continue while a segment runs, unless the caller cancelled; counts the iterations.
__global__ void k_bloop_control(cudaGraphConditionalHandle h, const int* __restrict__ done,
                                int nseg, const volatile int* cancel, int* __restrict__ loops) {
    __shared__ int running;
    if (threadIdx.x == 0) running = 0;
    __syncthreads();
    int mine = 0;
    for (int s = threadIdx.x; s < nseg; s += blockDim.x)
        if (!done[s]) mine = 1;
    if (mine) atomicOr(&running, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        *loops += 1;
        cudaGraphSetConditional(h, (running && !*cancel) ? 1u : 0u);
    }
}

// ------------------------------------------------------------------ continuous batching
// The host side of a streamed segment lives in pinned, mapped host memory: the host writes a
// request's right side into the segment's staging slot and then a new generation number into
// req[s]; the device copies it in at the start of an iteration, and when the segment is done it
// writes x into the segment's output slot, its figures into stat[s], and the generation into
// served[s] (after a system-wide fence), which the host polls.
struct StreamStat {
    double residual, truth;
    int iterations, status;
};

struct StreamHost {
    const volatile unsigned long long* req;  // generation of the request in each slot
    volatile unsigned long long* served;     // generation served
    const double* in;                        // staging: member k, slot c at boff[k] R + c m_k
    double* out;
    StreamStat* stat;
    const volatile int* stop;
};

// 1 thread per segment: a free slot with a new generation takes its request (phase FRESH).
__global__ void k_sadmit(int nseg, StreamHost h, unsigned long long* __restrict__ seen,
                         int* __restrict__ phase, int* __restrict__ done,
                         int* __restrict__ admit) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
        int a = 0;
        if (phase[s] == PH_FREE) {
            const unsigned long long g = h.req[s];
            if (g != seen[s]) {
                seen[s] = g;
                phase[s] = PH_FRESH;
                done[s] = 0;
                a = 1;
            }
        }
        admit[s] = a;
    }
}

// The admitted segments' vectors: b and r from the staging slot, x = p = q = 0.
template <int R>
__global__ void __launch_bounds__(BTH)
    k_sadmit_copy(const Chunk* __restrict__ chunks, const int64_t* __restrict__ boff,
                  const int* __restrict__ admit, StreamHost h, double* __restrict__ b,
                  double* __restrict__ r, float* __restrict__ r32, double* __restrict__ x,
                  double* __restrict__ p, double* __restrict__ q) {
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    if (!admit[ch.sys * R + col]) return;
    __threadfence_system();
    const int64_t b0 = boff[ch.sys], m = boff[ch.sys + 1] - b0;
    const double* in = h.in + b0 * R + col * m;
    for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R) {
        const int64_t t = (int64_t)row * R + col;
        const double v = in[row - b0];
        b[t] = v;
        r[t] = v;
        if (r32) r32[t] = (float)v;
        x[t] = 0.0;
        p[t] = 0.0;
        q[t] = 0.0;
    }
}

// The finished segments' x to their output slots.
template <int R>
__global__ void __launch_bounds__(BTH)
    k_sdeliver_copy(const Chunk* __restrict__ chunks, const int64_t* __restrict__ boff,
                    const int* __restrict__ phase, StreamHost h, const double* __restrict__ x) {
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    if (phase[ch.sys * R + col] != PH_DONE) return;
    const int64_t b0 = boff[ch.sys], m = boff[ch.sys + 1] - b0;
    double* out = h.out + b0 * R + col * m;
    for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R)
        out[row - b0] = x[(int64_t)row * R + col];
    __threadfence_system();
}

// Then their figures and generations, and the slots are free again.
__global__ void k_sdeliver(int nseg, StreamHost h, const unsigned long long* __restrict__ seen,
                           int* __restrict__ phase, BatchScalars sc) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
        if (phase[s] != PH_DONE) continue;
        StreamStat st;
        st.residual = sc.bb[s] > 0.0 ? sqrt(sc.rr[s]) / sqrt(sc.bb[s]) : 0.0;
        st.truth = sc.bb[s] > 0.0 ? sc.truth[s] : 0.0;
        st.iterations = sc.iters[s];
        st.status = sc.status[s];
        h.stat[s] = st;
        __threadfence_system();
        h.served[s] = seen[s];
        phase[s] = PH_FREE;
    }
}

// Continue while a segment is busy or a request waits for a free slot, unless stopped.
__global__ void k_sloop_control(cudaGraphConditionalHandle hc, int nseg, StreamHost h,
                                const unsigned long long* __restrict__ seen,
                                const int* __restrict__ phase, int* __restrict__ loops,
                                unsigned long long* __restrict__ served_iterations) {
    __shared__ int busy;
    if (threadIdx.x == 0) busy = 0;
    __syncthreads();
    int mine = 0;
    for (int s = threadIdx.x; s < nseg; s += blockDim.x)
        if (phase[s] != PH_FREE || h.req[s] != seen[s]) mine = 1;
    if (mine) atomicOr(&busy, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        *loops += 1;
        cudaGraphSetConditional(hc, (busy && !*h.stop) ? 1u : 0u);
    }
    // The segments that this iteration served (running or being verified): the packing.
    int active = 0;
    for (int s = threadIdx.x; s < nseg; s += blockDim.x)
        active += phase[s] == PH_RUN || phase[s] == PH_VERIFY;
    for (int o = 16; o; o >>= 1) active += __shfl_xor_sync(0xffffffffu, active, o);
    if ((threadIdx.x & 31) == 0 && active) atomicAdd(served_iterations, (unsigned long long)active);
}

// A member's FP64 inverse h (m x m, row-major) made exactly symmetric and stored in row tiles
// of DTH rows, each tile by column (k_bdense's layout), in T.
template <class T>
__global__ void k_tile_inverse(int64_t m, const double* __restrict__ h, T* __restrict__ t) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m * m;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / m, c = e % m;
        t[(r / DTH) * DTH * m + c * DTH + r % DTH] = (T)(0.5 * (h[r * m + c] + h[c * m + r]));
    }
}

// ------------------------------------------------------------------ the batch
// A member's levels on the device: its matrices (the first the caller's, the coarser ones held
// in `owned`, whose elements keep their addresses) and its prolongations.
struct SystemHierarchy {
    std::deque<DevCsr> owned;
    std::vector<const DevCsr*> mats;
    std::vector<DevRect> ps;
};

// Level l: rows [0, ns) of the members that smooth here and go on to level l + 1, then rows
// [ns, n) of the members whose deepest level this is.
template <class T>
struct BatchLevel {
    int64_t n = 0, ns = 0, nc = 0;  // rows, smoothed rows, rows of the next level
    Sell<T> A;                       // ns rows (when the level has no 3x3-block form)
    bool block3 = false;             // the 3x3-block form A3 instead of A
    DevBuf<int64_t> b3ptr;
    DevBuf<uint32_t> b3col;
    DevBuf<T> b3val;
    BSell3View<T> view3() const { return {ns / 3, b3ptr.p, b3col.p, b3val.p}; }
    DevBuf<T> dinv;                  // ns
    DevBuf<int64_t> pptr, rptr;      // P: ns x nc, R = P^T: nc x ns
    DevBuf<uint32_t> pidx, ridx;
    DevBuf<T> pval, rval;
    DevBuf<T> b, xa, xb;             // n R
    DevBuf<T> d, r;                  // ns R
    std::vector<double> c1, c2;
    double lambda = 0;
    int ndense = 0, ntiles = 0;
    DevBuf<int64_t> doff, dioff;     // ndense + 1: first row (in the level), first inverse entry
    DevBuf<int2> tiles;              // (dense member, first row of the tile)
    DevBuf<T> inv;
};

class BatchImpl {
   public:
    BatchImpl();
    ~BatchImpl();
    void create(const std::vector<const DevCsr*>& a, const std::vector<const femgpu_unknowns*>& u,
                int nrhs, const Options& o);
    void solve_device(const double* d_b, double* d_x, const volatile int* cancel,
                      femgpu_batch_stats* st);
    void solve_host(const double* h_b, double* h_x, const volatile int* cancel,
                    femgpu_batch_stats* st);
    void set_max_iter(int m) { max_iter_ = m; }
    // Per segment in the caller's member order.
    void segments(size_t* iterations, double* truth, double* residual, int* status) const;
    const std::vector<int64_t>& offsets() const { return offsets_; }
    std::vector<int64_t> level_sizes() const { return sizes_; }
    // "setup seconds: phase s; ..." of the batch's creation.
    std::string describe() const;
    size_t bytes() const;
    cudaStream_t stream() const { return s_; }
    // The mean device time (ms) of 1 launch of the finest level's Chebyshev step over all
    // right sides, and its algorithmic bytes.
    void kernel_time(int reps, double* ms, double* bytes);
    double tol = 1e-10;  // PCG_TOL, solve.rs:42

    // Continuous batching (femgpu_stream_*). stream_open allocates the mapped queue and captures
    // the streamed loop; stream_launch starts it on the batch's stream (it runs until no slot is
    // busy and no request waits); stream_idle tells whether that launch has ended.
    void stream_open();
    void stream_launch();
    bool stream_idle();
    void stream_stop();
    int slots() const { return R_; }
    int members() const { return B_; }
    int64_t member_rows(int member) const { return offsets_[member + 1] - offsets_[member]; }
    // The segment of (caller's member, slot) and the offset of its staging slot.
    int segment(int member, int slot) const { return position_[member] * R_ + slot; }
    int64_t slot_offset(int member, int slot) const {
        return boff_[position_[member]] * R_ + slot * member_rows(member);
    }
    volatile unsigned long long* h_req() { return h_req_; }
    volatile unsigned long long* h_served() { return h_served_; }
    double* h_in() { return h_in_; }
    double* h_out() { return h_out_; }
    const StreamStat* h_stat() { return h_stat_; }
    size_t stream_loops();
    size_t stream_served_iterations();
    bool streaming() const;

   private:
    template <int R>
    void build_stream_graph();
    DevBuf<int> phase_, restarts_seg_, fresh_, admit_;
    DevBuf<unsigned long long> seen_, served_its_;
    DevBuf<int64_t> boffd_;
    std::vector<int64_t> boff_;   // the batch order's row offsets
    std::vector<int> position_;   // caller's member -> batch position
    unsigned long long *h_req_ = nullptr, *h_served_ = nullptr;
    double *h_in_ = nullptr, *h_out_ = nullptr;
    StreamStat* h_stat_ = nullptr;
    int* h_stop_ = nullptr;
    StreamHost dh_{};  // the device's view of the mapped arrays
    cudaGraph_t sgraph_ = nullptr;
    cudaGraphExec_t sexec_ = nullptr;
    cudaGraphConditionalHandle scond_ = 0;
    cudaEvent_t sev_ = nullptr;
    bool slaunched_ = false;
    template <class T>
    void build_levels(std::vector<SystemHierarchy>& H, std::vector<BatchLevel<T>>* levels);
    template <class T, int R>
    const T* vcycle(std::vector<BatchLevel<T>>& Ls, size_t l, const T* b);
    template <int R>
    void finish(int kind, int init);
    template <int R>
    void precondition_and_dots(int init, bool stream);
    template <int R>
    void iteration(bool stream);
    template <int R>
    void run(const volatile int* cancel);
    template <int R>
    void residual(double* r, float* r32);
    void permute(const double* in, double* out, int scatter);
    void solve_loaded(const volatile int* cancel, femgpu_batch_stats* st);
    void launch_loop(const volatile int* cancel);
    bool any_running();
    void collect(femgpu_batch_stats* st);
    BatchScalars scalars() {
        return BatchScalars{bb_.p, rr_.p, rz_.p, pq_.p, alpha_.p, beta_.p, truth_.p,
                            done_.p, iters_.p, status_.p};
    }
    const Chunk* chunks() const { return reinterpret_cast<const Chunk*>(chunks_.p); }

    cudaStream_t s_ = nullptr;
    Options opt_;
    int B_ = 0, R_ = 1, nchunks_ = 0, max_iter_ = 500, graph_max_iter_ = -1;
    int64_t n_ = 0;
    std::vector<int64_t> offsets_, sizes_;  // the caller's member order
    // The creation's phases (host seconds until each phase's device work finished).
    std::vector<std::pair<std::string, double>> setup_s_;
    std::chrono::steady_clock::time_point phase_t0_;
    void phase_end(const char* name) {
        FG_CUDA(cudaStreamSynchronize(s_));
        const auto t = std::chrono::steady_clock::now();
        const double sec = std::chrono::duration<double>(t - phase_t0_).count();
        phase_t0_ = t;
        for (auto& ph : setup_s_)
            if (ph.first == name) {
                ph.second += sec;
                return;
            }
        setup_s_.emplace_back(name, sec);
    }
    std::vector<int> order_;                // batch position -> caller's member
    DevBuf<int> map_;                       // batch row -> caller's row
    Sell<double> A64_;  // the block-diagonal finest matrix (batch order), exactly
    bool fine3_ = false;  // ... in 3x3-block form instead (every member elastic)
    DevBuf<int64_t> f3ptr_;
    DevBuf<uint32_t> f3col_;
    DevBuf<double> f3val_;
    BSell3View<double> fine3() const { return {n_ / 3, f3ptr_.p, f3col_.p, f3val_.p}; }
    std::vector<BatchLevel<float>> L32_;
    std::vector<BatchLevel<double>> L64_;
    DevBuf<char> chunks_;
    DevBuf<int> cstart_;
    DevBuf<double> partial_;
    DevBuf<double> bb_, rr_, rz_, pq_, alpha_, beta_, truth_;
    DevBuf<int> done_, iters_, status_, loops_;
    DevBuf<double> x_, r_, p_, q_, b_, stage_;
    DevBuf<float> r32_;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaGraphConditionalHandle cond_ = 0;
    int* h_cancel_ = nullptr;  // pinned and mapped: the device reads it each iteration
    int* d_cancel_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    size_t launches_ = 0, graph_kernels_ = 0;
    int restarts_ = 0;
    double graph_tol_ = -1;  // tol and max_iter are arguments of the graph's kernels
};

namespace {

// A part of a block-diagonal combination: its CSR arrays on the device, its size, and where its
// rows, entries and columns start in the combination.
struct CombinePart {
    const int64_t* ptr;
    const uint32_t* idx;
    const double* val;
    int64_t rows, row0, nnz0, col0;
};

// The combination's row pointers (the part is blockIdx.y) and its entries, each part's columns
// shifted by the columns before it.
__global__ void k_combine_ptr(const CombinePart* __restrict__ parts, int64_t* __restrict__ ptr) {
    const CombinePart c = parts[blockIdx.y];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < c.rows;
         i += (int64_t)gridDim.x * blockDim.x)
        ptr[c.row0 + i + 1] = c.nnz0 + c.ptr[i + 1];
}

__global__ void k_combine_entries(const CombinePart* __restrict__ parts, uint32_t* __restrict__ idx,
                                  double* __restrict__ val) {
    const CombinePart c = parts[blockIdx.y];
    const int64_t nnz = c.ptr[c.rows];
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x) {
        idx[c.nnz0 + e] = (uint32_t)(c.idx[e] + c.col0);
        val[c.nnz0 + e] = c.val[e];
    }
}

// The block-diagonal matrix of `count` parts (rows, columns, nnz each, and their device arrays).
void combine_parts(const std::vector<CombinePart>& host, int64_t rows, int64_t nnz, int64_t maxr,
                   int64_t maxnnz, int64_t* out_ptr, uint32_t* out_idx, double* out_val,
                   cudaStream_t s) {
    if (host.empty()) return;
    if (host.size() > 65535) throw Failure(FEMGPU_ERR_TOO_LARGE, "more than 65535 members");
    DevBuf<CombinePart> d;
    d.upload(host.data(), host.size(), s);
    FG_CUDA(cudaMemsetAsync(out_ptr, 0, sizeof(int64_t), s));
    const unsigned ny = (unsigned)host.size();
    k_combine_ptr<<<dim3((unsigned)blocks_for(std::max<int64_t>(maxr, 1), BTH, 64), ny), BTH, 0,
                    s>>>(d.p, out_ptr);
    k_combine_entries<<<dim3((unsigned)blocks_for(std::max<int64_t>(maxnnz, 1), BTH, 256), ny),
                        BTH, 0, s>>>(d.p, out_idx, out_val);
    FG_CHECK_LAUNCH();
    FG_CUDA(cudaStreamSynchronize(s));  // the part table is freed on return
    (void)rows;
    (void)nnz;
}

// The block-diagonal matrix of the members' matrices, on the device.
void combine(const std::vector<const DevCsr*>& parts, DevCsr* out, cudaStream_t s) {
    std::vector<CombinePart> h;
    int64_t n = 0, nnz = 0, maxr = 0, maxnnz = 0;
    for (auto* a : parts) {
        h.push_back({a->ptr.p, a->idx.p, a->val.p, a->n, n, nnz, n});
        n += a->n;
        nnz += a->nnz;
        maxr = std::max(maxr, a->n);
        maxnnz = std::max(maxnnz, a->nnz);
    }
    if (n >= 0x7fffffff) throw Failure(FEMGPU_ERR_TOO_LARGE, "a batch of 2^31 unknowns or more");
    out->n = n;
    out->nnz = nnz;
    out->ptr.alloc(n + 1);
    out->idx.alloc(std::max<int64_t>(nnz, 1));
    out->val.alloc(std::max<int64_t>(nnz, 1));
    combine_parts(h, n, nnz, maxr, maxnnz, out->ptr.p, out->idx.p, out->val.p, s);
}

// The block-diagonal transfer of the members' transfers, on the device.
void combine_rect(const std::vector<const DevRect*>& parts, DevRect* out, cudaStream_t s) {
    std::vector<CombinePart> h;
    int64_t rows = 0, cols = 0, nnz = 0, maxr = 0, maxnnz = 0;
    for (auto* p : parts) {
        h.push_back({p->ptr.p, p->idx.p, p->val.p, p->rows, rows, nnz, cols});
        rows += p->rows;
        cols += p->cols;
        nnz += p->nnz;
        maxr = std::max(maxr, p->rows);
        maxnnz = std::max(maxnnz, p->nnz);
    }
    out->rows = rows;
    out->cols = cols;
    out->nnz = nnz;
    out->ptr.alloc(rows + 1);
    out->idx.alloc(std::max<int64_t>(nnz, 1));
    out->val.alloc(std::max<int64_t>(nnz, 1));
    combine_parts(h, rows, nnz, maxr, maxnnz, out->ptr.p, out->idx.p, out->val.p, s);
}

// The diagonal of a device CSR; *bad is set when an entry is not above 0.
__global__ void k_batch_diagonal(int64_t n, const int64_t* __restrict__ ptr,
                                 const uint32_t* __restrict__ idx, const double* __restrict__ val,
                                 double* __restrict__ dg, int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
            if ((int64_t)idx[k] == i) d = val[k];
        dg[i] = d;
        if (!(d > 0.0)) *bad = 1;
    }
}

}  // namespace

BatchImpl::BatchImpl() {
    FG_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
    FG_CUDA(cudaEventCreate(&ev0_));
    FG_CUDA(cudaEventCreate(&ev1_));
    FG_CUDA(cudaHostAlloc(&h_cancel_, sizeof(int), cudaHostAllocMapped));
    *h_cancel_ = 0;
    FG_CUDA(cudaHostGetDevicePointer(&d_cancel_, h_cancel_, 0));
}

BatchImpl::~BatchImpl() {
    if (h_stop_) *(volatile int*)h_stop_ = 1;
    if (s_) cudaStreamSynchronize(s_);
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (sexec_) cudaGraphExecDestroy(sexec_);
    if (sgraph_) cudaGraphDestroy(sgraph_);
    if (sev_) cudaEventDestroy(sev_);
    for (void* h : {(void*)h_req_, (void*)h_served_, (void*)h_in_, (void*)h_out_, (void*)h_stat_,
                    (void*)h_stop_})
        if (h) cudaFreeHost(h);
    if (h_cancel_) cudaFreeHost(h_cancel_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (s_) cudaStreamDestroy(s_);
}

void BatchImpl::create(const std::vector<const DevCsr*>& a,
                       const std::vector<const femgpu_unknowns*>& u, int nrhs, const Options& o) {
    if (nrhs != 1 && nrhs != 4 && nrhs != 16)
        throw Failure(FEMGPU_ERR_INVALID, "a batch takes 1, 4 or 16 right sides per system");
    opt_ = o;
    R_ = nrhs;
    B_ = (int)a.size();
    if (B_ < 1) throw Failure(FEMGPU_ERR_INVALID, "an empty batch");
    setup_s_.clear();
    phase_t0_ = std::chrono::steady_clock::now();
    // Each member's hierarchy on the device (multigrid.rs:84-139), the members shared among the
    // host threads, each with its own stream.
    for (int b = 0; b < B_; ++b)
        if (a[b]->n < 1) throw Failure(FEMGPU_ERR_INVALID, "an empty system");
    std::vector<SystemHierarchy> H(B_);
    // 1024 by default: the thin members (plates 1 cell thick) converge slowly under plane
    // coarsening, and a dense deepest level of up to 1024 unknowns per member cuts the most
    // iterations of a batch of 10x1x1 to 80x8x8-cell cantilevers from 66 to 20 at 1e-8, for
    // 4 MB of FP32 inverse per member read once per cycle for all right sides.
    const size_t coarsest = (size_t)(o.coarsest > 0 ? o.coarsest : 1024);
    const size_t max_levels = (size_t)(o.max_levels > 0 ? o.max_levels : 30);
    std::vector<std::string> errors(B_);
    std::vector<int> codes(B_, FEMGPU_OK);
    auto build = [&](int b, cudaStream_t st) {
        try {
            const femgpu_unknowns& uu = *u[b];
            const int64_t n = a[b]->n;
            HostLevel lv;
            for (int d = 0; d < 3; ++d)
                lv.planes[d].assign(uu.planes[d], uu.planes[d] + uu.nplanes[d]);
            lv.points.resize(n);
            for (int64_t k = 0; k < n; ++k)
                for (int d = 0; d < 3; ++d) lv.points[k][d] = uu.points[3 * k + d];
            lv.comp.assign(uu.comp, uu.comp + n);
            H[b].mats.push_back(a[b]);
            // The member's coarsening and Galerkin products on the device (coarsen.cu), the
            // coarse unknowns in grid order (z, y, x, component): the 3 unknowns of a node are
            // consecutive, which the 3x3-block operators need.
            DevGrid grid;
            grid_upload(lv, &grid, st);
            for (;;) {
                const DevCsr& m = *H[b].mats.back();
                if ((size_t)m.n <= coarsest || H[b].ps.size() >= max_levels) break;
                DevRect p;
                DevGrid coarse;
                if (!coarsen_grid(grid, m, 7, &p, &coarse, st)) break;
                if ((size_t)coarse.n * 10 > (size_t)m.n * 9) break;
                H[b].owned.emplace_back();
                galerkin_product(p, m, &H[b].owned.back(), st);
                H[b].mats.push_back(&H[b].owned.back());
                H[b].ps.push_back(std::move(p));
                grid = std::move(coarse);
            }
            FG_CUDA(cudaStreamSynchronize(st));
            if (H[b].mats.back()->n > 4096)
                throw Failure(FEMGPU_ERR_TOO_LARGE,
                              "the deepest level has more than 4096 unknowns: the grid does not "
                              "coarsen");
        } catch (const Failure& e) {
            codes[b] = e.code;
            errors[b] = e.what();
        } catch (const std::exception& e) {
            codes[b] = FEMGPU_ERR_INVALID;
            errors[b] = e.what();
        }
    };
    const int threads = std::max(1, std::min(host_threads(), B_));
    std::vector<std::thread> pool;
    int device = 0;
    FG_CUDA(cudaGetDevice(&device));
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            cudaStream_t st = nullptr;
            if (cudaSetDevice(device) != cudaSuccess ||
                cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
                for (int b = t; b < B_; b += threads) {
                    codes[b] = FEMGPU_ERR_CUDA;
                    errors[b] = "cudaStreamCreate failed";
                }
                return;
            }
            for (int b = t; b < B_; b += threads) build(b, st);
            cudaStreamDestroy(st);
        });
    for (auto& th : pool) th.join();
    for (int b = 0; b < B_; ++b)
        if (codes[b] != FEMGPU_OK)
            throw Failure(codes[b], "system " + std::to_string(b) + ": " + errors[b]);
    phase_end("members' coarsening and Galerkin products (device, host threads)");
    // The caller's row offsets, then the batch order: deepest first (stable).
    offsets_.assign(B_ + 1, 0);
    for (int b = 0; b < B_; ++b) offsets_[b + 1] = offsets_[b] + H[b].mats[0]->n;
    n_ = offsets_[B_];
    if (n_ * R_ >= 0x7fffffff)
        throw Failure(FEMGPU_ERR_TOO_LARGE, "a batch of 2^31 values or more per vector");
    order_.resize(B_);
    std::iota(order_.begin(), order_.end(), 0);
    std::stable_sort(order_.begin(), order_.end(),
                     [&](int x, int y) { return H[x].mats.size() > H[y].mats.size(); });
    std::vector<SystemHierarchy> Hs(B_);
    for (int k = 0; k < B_; ++k) Hs[k] = std::move(H[order_[k]]);
    std::vector<int> map(n_);
    std::vector<int64_t> boff(B_ + 1, 0);  // the batch order's row offsets
    for (int k = 0; k < B_; ++k) {
        const int64_t m = Hs[k].mats[0]->n;
        boff[k + 1] = boff[k] + m;
        for (int64_t i = 0; i < m; ++i) map[boff[k] + i] = (int)(offsets_[order_[k]] + i);
    }
    map_.upload(map.data(), map.size(), s_);
    boff_ = boff;
    position_.assign(B_, 0);
    for (int k = 0; k < B_; ++k) position_[order_[k]] = k;
    // The exact finest operator (FP64) of the PCG loop and the true residual.
    {
        std::vector<const DevCsr*> parts;
        for (auto& h : Hs) parts.push_back(h.mats[0]);
        DevCsr f;
        combine(parts, &f, s_);
        if (opt_.format == 0 && make_bsell3_device<double>(f, &f3ptr_, &f3col_, &f3val_, s_))
            fine3_ = true;
        else
            make_sell<double>(f, 32, &A64_, s_);
        FG_CUDA(cudaStreamSynchronize(s_));
    }
    phase_end("finest operator (device combination, 3x3 blocks)");
    // The chunks of the PCG kernels: rows of 1 member each; up to 4 rows per thread, or 2 block
    // rows (6 rows) per thread with the 3x3-block operator, whose chunks hold whole nodes.
    const int chunk_rows = fine3_ ? 3 * 2 * (BTH / R_) : 4 * BTH / R_;
    std::vector<Chunk> ch;
    std::vector<int> cstart(B_ + 1, 0);
    for (int k = 0; k < B_; ++k) {
        cstart[k] = (int)ch.size();
        for (int64_t r = boff[k]; r < boff[k + 1]; r += chunk_rows)
            ch.push_back({k, (int)r, (int)std::min<int64_t>(r + chunk_rows, boff[k + 1])});
    }
    cstart[B_] = (int)ch.size();
    nchunks_ = (int)ch.size();
    chunks_.alloc(ch.size() * sizeof(Chunk));
    FG_CUDA(cudaMemcpyAsync(chunks_.p, ch.data(), ch.size() * sizeof(Chunk),
                            cudaMemcpyHostToDevice, s_));
    cstart_.upload(cstart.data(), cstart.size(), s_);
    // The block sums: of the chunks (R columns, 2 values) and of the power iteration.
    partial_.alloc(std::max(2 * (size_t)nchunks_ * R_, 2 * (size_t)(n_ / BTH + 64)));
    if (opt_.precision == FEMGPU_MIXED)
        build_levels<float>(Hs, &L32_);
    else
        build_levels<double>(Hs, &L64_);
    const size_t S = (size_t)B_ * R_;
    for (auto* v : {&bb_, &rr_, &rz_, &pq_, &alpha_, &beta_, &truth_}) v->alloc(S);
    for (auto* v : {&done_, &iters_, &status_}) v->alloc(S);
    loops_.alloc(1);
    for (auto* v : {&x_, &r_, &p_, &q_, &b_, &stage_}) v->alloc((size_t)n_ * R_);
    if (opt_.precision == FEMGPU_MIXED) r32_.alloc((size_t)n_ * R_);
    FG_CUDA(cudaStreamSynchronize(s_));
    phase_end("vectors");
}

std::string BatchImpl::describe() const {
    std::string out = "setup seconds:";
    char buf[128];
    for (const auto& ph : setup_s_) {
        std::snprintf(buf, sizeof buf, " %s %.3f;", ph.first.c_str(), ph.second);
        out += buf;
    }
    return out + "\n";
}

template <class T>
void BatchImpl::build_levels(std::vector<SystemHierarchy>& H, std::vector<BatchLevel<T>>* levels) {
    const size_t depth = H[0].mats.size();  // the deepest member comes first
    levels->resize(depth);
    const int deg = opt_.degree > 0 ? opt_.degree : 2;
    const double lower = opt_.lower > 0 ? opt_.lower : 0.3;
    sizes_.clear();
    for (size_t l = 0; l < depth; ++l) {
        BatchLevel<T>& L = (*levels)[l];
        // Members [0, S) smooth at l and go on; [S, K) end at l (the order is by depth).
        int K = 0, S = 0;
        while (K < B_ && H[K].mats.size() > l) ++K;
        while (S < K && H[S].mats.size() > l + 1) ++S;
        for (int k = 0; k < K; ++k) L.n += H[k].mats[l]->n;
        for (int k = 0; k < S; ++k) L.ns += H[k].mats[l]->n;
        sizes_.push_back(L.n);
        if (S > 0) {
            std::vector<const DevCsr*> mats;
            std::vector<const DevRect*> ps;
            for (int k = 0; k < S; ++k) {
                mats.push_back(H[k].mats[l]);
                ps.push_back(&H[k].ps[l]);
            }
            DevCsr d;
            combine(mats, &d, s_);
            if (opt_.format == 0 && make_bsell3_device<T>(d, &L.b3ptr, &L.b3col, &L.b3val, s_))
                L.block3 = true;
            else
                make_sell<T>(d, 32, &L.A, s_);
            // The diagonal, and lambda_max of the block-diagonal D^-1 A: the largest of the
            // members'.
            DevBuf<double> ddg(d.n);
            DevBuf<int> bad(1);
            bad.zero(s_);
            k_batch_diagonal<<<blocks_for(d.n, BTH), BTH, 0, s_>>>(d.n, d.ptr.p, d.idx.p, d.val.p,
                                                                   ddg.p, bad.p);
            FG_CHECK_LAUNCH();
            if (fetch(bad.p, s_))
                throw Failure(FEMGPU_ERR_NOT_SPD,
                              "the matrix is not positive definite: it has a diagonal entry "
                              "that is not above 0");
            Operator<double> op;
            op.n = d.n;
            op.nnz = d.nnz;
            make_sell<double>(d, 32, &op.sell, s_);
            L.lambda = lambda_max(op, ddg.p, s_, partial_);
            chebyshev(L.lambda, deg, lower, &L.c1, &L.c2, opt_.smoother);
            L.dinv.alloc(d.n);
            reciprocal<T>(d.n, ddg.p, L.dinv.p, s_);
            DevRect P, Rt;
            combine_rect(ps, &P, s_);
            transpose_rect(P, &Rt, s_);
            L.nc = P.cols;
            L.pptr = std::move(P.ptr);
            L.pidx = std::move(P.idx);
            L.pval.alloc(std::max<int64_t>(P.nnz, 1));
            convert_values<T>(P.nnz, P.val.p, L.pval.p, s_);
            L.rptr = std::move(Rt.ptr);
            L.ridx = std::move(Rt.idx);
            L.rval.alloc(std::max<int64_t>(Rt.nnz, 1));
            convert_values<T>(Rt.nnz, Rt.val.p, L.rval.p, s_);
            L.d.alloc((size_t)L.ns * R_);
            L.r.alloc((size_t)L.ns * R_);
            FG_CUDA(cudaStreamSynchronize(s_));
            phase_end("smoothed levels (device combination, lambda_max, transfers)");
        }
        // The members that end here: a dense inverse each, from a dense Cholesky factor on the
        // device, made exactly symmetric, stored in tiles of DTH rows (k_bdense's layout).
        L.ndense = K - S;
        if (L.ndense > 0) {
            std::vector<int64_t> off(L.ndense + 1), ioff(L.ndense + 1, 0);
            std::vector<int2> tiles;
            off[0] = L.ns;
            for (int j = 0; j < L.ndense; ++j) {
                const int64_t m = H[S + j].mats[l]->n;
                off[j + 1] = off[j] + m;
                // Row tiles of DTH rows (the last padded with zero rows), each stored by column.
                ioff[j + 1] = ioff[j] + (m + DTH - 1) / DTH * DTH * m;
                for (int64_t t = 0; t < m; t += DTH) tiles.push_back({j, (int)t});
            }
            L.ntiles = (int)tiles.size();
            L.inv.alloc(ioff[L.ndense]);
            L.inv.zero(s_);  // the padding rows of each member's last tile
            FG_CUDA(cudaStreamSynchronize(s_));
            // The members' inverses in groups (their square work buffers within a budget), each
            // step of a group 1 launch for all its members (dense_inverse_batch), then each
            // inverse tiled into its place of L.inv.
            constexpr int64_t kGroupEntries = (int64_t)48 << 20;  // 384 MB per square buffer
            DenseBatchWork work;
            DevBuf<double> inv64;
            for (int j0 = 0; j0 < L.ndense;) {
                int j1 = j0;
                int64_t entries = 0;
                while (j1 < L.ndense) {
                    const int64_t m = off[j1 + 1] - off[j1];
                    if (j1 > j0 && entries + m * m > kGroupEntries) break;
                    entries += m * m;
                    ++j1;
                }
                if (inv64.count < (size_t)entries) inv64.alloc(entries);
                std::vector<const DevCsr*> mats;
                std::vector<double*> outs;
                int64_t at = 0;
                for (int j = j0; j < j1; ++j) {
                    const int64_t m = off[j + 1] - off[j];
                    mats.push_back(H[S + j].mats[l]);
                    outs.push_back(inv64.p + at);
                    at += m * m;
                }
                std::string text;
                const int bad = dense_inverse_batch(mats, outs, &work, s_, &text);
                if (bad >= 0)
                    throw Failure(FEMGPU_ERR_NOT_SPD,
                                  "system " + std::to_string(order_[S + j0 + bad]) + ": " + text);
                for (int j = j0; j < j1; ++j) {
                    const int64_t m = off[j + 1] - off[j];
                    k_tile_inverse<T><<<blocks_for(m * m, BTH), BTH, 0, s_>>>(
                        m, outs[j - j0], L.inv.p + ioff[j]);
                }
                FG_CHECK_LAUNCH();
                FG_CUDA(cudaStreamSynchronize(s_));
                j0 = j1;
            }
            L.doff.upload(off.data(), off.size(), s_);
            L.dioff.upload(ioff.data(), ioff.size(), s_);
            L.tiles.upload(tiles.data(), tiles.size(), s_);
            phase_end("deepest levels' dense inverses (device, batched)");
        }
        for (auto* v : {&L.b, &L.xa, &L.xb}) v->alloc((size_t)L.n * R_);
        FG_CUDA(cudaStreamSynchronize(s_));
    }
}

// ------------------------------------------------------------------ the cycle and the loop
// The V-cycle from level l on the right sides b; returns where the correction is.
template <class T, int R>
const T* BatchImpl::vcycle(std::vector<BatchLevel<T>>& Ls, size_t l, const T* b) {
    BatchLevel<T>& L = Ls[l];
    T* xa = L.xa.p;
    T* xb = L.xb.p;
    if (L.ns > 0) {
        const int g = (int)((L.ns * R + BTH - 1) / BTH);
        const int deg = (int)L.c1.size();
        launch(true, k_bcheb_first<T, R>, g, BTH, s_, L.ns, b, L.dinv.p, (T)L.c1[0], L.d.p, xa);
        const int g3 = (int)((L.ns / 3 * (R / Lanes<T, R>::W) + BTH - 1) / BTH);
        const int gs = (int)((L.ns * (R / Lanes<T, R>::W) + BTH - 1) / BTH);
        auto step = [&](const T* xin, T* xout, int k) {
            if (L.block3)
                launch(true, k_bcheb_step3<T, R>, g3, BTH, s_, L.view3(), b, xin, L.dinv.p,
                       (T)L.c1[k], (T)L.c2[k], L.d.p, xout);
            else
                launch(true, k_bcheb_step<T, R>, gs, BTH, s_, L.A.view(), b, xin, L.dinv.p,
                       (T)L.c1[k], (T)L.c2[k], L.d.p, xout);
        };
        for (int k = 1; k < deg; ++k) {
            step(xa, xb, k);
            std::swap(xa, xb);
        }
        if (L.block3)
            launch(true, k_bresidual3<T, R>, g3, BTH, s_, L.view3(), b, xa, L.r.p);
        else
            launch(true, k_bresidual<T, R>, gs, BTH, s_, L.A.view(), b, xa, L.r.p);
        T* bc = Ls[l + 1].b.p;
        const int gc = (int)((L.nc * R + BTH - 1) / BTH);
        launch(true, k_bgather<T, R>, gc, BTH, s_, L.nc, L.rptr.p, L.ridx.p, L.rval.p, L.r.p, bc, 0);
        FG_CHECK_LAUNCH();
        launches_ += deg + 2;
        const T* ec = vcycle<T, R>(Ls, l + 1, bc);
        launch(true, k_bgather<T, R>, g, BTH, s_, L.ns, L.pptr.p, L.pidx.p, L.pval.p, ec, xa, 1);
        for (int k = 0; k < deg; ++k) {
            step(xa, xb, k);
            std::swap(xa, xb);
        }
        FG_CHECK_LAUNCH();
        launches_ += deg + 1;
    }
    if (L.ndense > 0) {
        launch(true, k_bdense<T, R>, L.ntiles, 32 * DW, s_, L.tiles.p, L.doff.p, L.dioff.p,
               L.inv.p, b, xa);
        FG_CHECK_LAUNCH();
        launches_ += 1;
    }
    return xa;
}

// The recurrence's stopping target. The mixed form promises the true FP64 residual at tol, and a
// segment whose recurrence stops just under tol may sit a rounding drift (a few parts in 1000)
// above it and need a restart, which re-runs the whole batch's cycle for a few segments; the
// recurrence of the mixed form therefore stops at 0.98 tol. The FP64 form stops at tol on the
// recurrence as the reference does (multigrid.rs:721-723).
template <int R>
void BatchImpl::finish(int kind, int init) {
    const bool mixed = opt_.precision == FEMGPU_MIXED;
    const double target = (mixed && kind != FIN_RESTART) ? 0.98 * tol : tol;
    launch(true, k_bfinish<R>, B_, BTH, s_, kind, cstart_.p, partial_.p, scalars(), target,
           max_iter_, (int)mixed, init, StreamState{phase_.p, restarts_seg_.p, fresh_.p}, tol);
    FG_CHECK_LAUNCH();
    launches_ += 1;
}

// z = M^-1 r, the sums r.z (and z.q), beta, p.
template <int R>
void BatchImpl::precondition_and_dots(int init, bool stream) {
    const bool mixed = opt_.precision == FEMGPU_MIXED;
    if (mixed) {
        const float* z = vcycle<float, R>(L32_, 0, r32_.p);
        launch(true, k_bpcg_dots<R, float>, nchunks_, BTH, s_, chunks(), r_.p, z, q_.p, 1, init,
               done_.p, partial_.p);
        finish<R>(stream ? FIN_SDOTS : FIN_DOTS, init);
        launch(true, k_bpcg_p<R, float>, nchunks_, BTH, s_, chunks(), z, p_.p, scalars(), init);
    } else {
        const double* z = vcycle<double, R>(L64_, 0, r_.p);
        launch(true, k_bpcg_dots<R, double>, nchunks_, BTH, s_, chunks(), r_.p, z, q_.p, 0, init,
               done_.p, partial_.p);
        finish<R>(stream ? FIN_SDOTS : FIN_DOTS, init);
        launch(true, k_bpcg_p<R, double>, nchunks_, BTH, s_, chunks(), z, p_.p, scalars(), init);
    }
    FG_CHECK_LAUNCH();
    launches_ += 2;
}

// 1 PCG iteration of every running segment (multigrid.rs:739-750).
template <int R>
void BatchImpl::iteration(bool stream) {
    const bool mixed = opt_.precision == FEMGPU_MIXED;
    const int* ph = stream ? phase_.p : nullptr;
    const double* xv = x_.p;
    const double* bv = b_.p;
    if (fine3_)
        launch(true, k_bpcg_spmv3<R>, nchunks_, BTH, s_, fine3(), chunks(), p_.p, q_.p, done_.p,
               partial_.p, ph, xv);
    else
        launch(true, k_bpcg_spmv<R>, nchunks_, BTH, s_, A64_.view(), chunks(), p_.p, q_.p,
               done_.p, partial_.p, ph, xv);
    finish<R>(stream ? FIN_SPQ : FIN_PQ, 0);
    launch(true, k_bpcg_update<R>, nchunks_, BTH, s_, chunks(), x_.p, r_.p, p_.p, q_.p,
           mixed ? r32_.p : nullptr, scalars(), partial_.p, ph, bv);
    finish<R>(stream ? FIN_SUPDATE : FIN_UPDATE, 0);
    FG_CHECK_LAUNCH();
    launches_ += 2;
    precondition_and_dots<R>(0, stream);
}

bool BatchImpl::any_running() {
    std::vector<int> d(B_ * R_);
    done_.download(d.data(), d.size(), s_);
    FG_CUDA(cudaStreamSynchronize(s_));
    for (int v : d)
        if (!v) return true;
    return false;
}

// Runs the loop graph until every segment has stopped or the caller's flag is set; a watcher
// thread mirrors the caller's flag into the mapped flag that the device reads each iteration.
void BatchImpl::launch_loop(const volatile int* cancel) {
    *(volatile int*)h_cancel_ = 0;
    std::atomic<bool> stop{false};
    std::thread watcher;
    if (cancel) {
        watcher = std::thread([&] {
            while (!stop.load(std::memory_order_relaxed)) {
                if (*cancel) *(volatile int*)h_cancel_ = 1;
                std::this_thread::sleep_for(std::chrono::microseconds(50));
            }
        });
    }
    cudaError_t e = cudaGraphLaunch(exec_, s_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s_);
    stop.store(true);
    if (watcher.joinable()) watcher.join();
    FG_CUDA(e);
}

// r = b - A x with the FP64 exact operator and its sums (b.b, r.r) per chunk.
template <int R>
void BatchImpl::residual(double* r, float* r32) {
    if (fine3_)
        launch(true, k_bpcg_residual3<R>, nchunks_, BTH, s_, fine3(), chunks(), b_.p, x_.p, r,
               r32, partial_.p);
    else
        launch(true, k_bpcg_residual<R>, nchunks_, BTH, s_, A64_.view(), chunks(), b_.p, x_.p, r,
               r32, partial_.p);
    FG_CHECK_LAUNCH();
}

template <int R>
void BatchImpl::run(const volatile int* cancel) {
    const bool mixed = opt_.precision == FEMGPU_MIXED;
    restarts_ = 0;
    if (!exec_) {
        const size_t before = launches_;
        FG_CUDA(cudaGraphCreate(&graph_, 0));
        FG_CUDA(cudaGraphConditionalHandleCreate(&cond_, graph_, 1, cudaGraphCondAssignDefault));
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
        iteration<R>(false);
        k_bloop_control<<<1, BTH, 0, s_>>>(cond_, done_.p, B_ * R, d_cancel_, loops_.p);
        FG_CUDA(cudaStreamEndCapture(s_, &body));
        FG_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
        graph_kernels_ = launches_ - before + 1;
        graph_max_iter_ = max_iter_;
        graph_tol_ = tol;
        launches_ = before;
    }
    FG_CUDA(cudaMemsetAsync(loops_.p, 0, sizeof(int), s_));
    // r = b - A x and the first test (multigrid.rs:692-723), x = 0 where b = 0, then
    // z = M^-1 r, p = z.
    residual<R>(r_.p, mixed ? r32_.p : nullptr);
    finish<R>(FIN_START, 0);
    k_bzero_empty<R><<<nchunks_, BTH, 0, s_>>>(chunks(), bb_.p, x_.p);
    FG_CHECK_LAUNCH();
    launches_ += 2;
    precondition_and_dots<R>(1, false);
    for (;;) {
        if (any_running()) launch_loop(cancel);
        if (cancel && *cancel) return;
        // The true residual of each segment in FP64. With the FP32 cycle the recurrence can
        // drift from it; the segments that drifted above tol run again from x (at most 3 times).
        residual<R>(mixed ? r_.p : nullptr, mixed ? r32_.p : nullptr);
        finish<R>(FIN_TRUTH, 0);
        launches_ += 1;
        if (!mixed || restarts_ >= 3) break;
        finish<R>(FIN_RESTART, 0);
        if (!any_running()) break;
        ++restarts_;
        precondition_and_dots<R>(1, false);
    }
}

// ------------------------------------------------------------------ continuous batching
template <int R>
void BatchImpl::build_stream_graph() {
    const bool mixed = opt_.precision == FEMGPU_MIXED;
    const int S = B_ * R;
    const size_t before = launches_;
    FG_CUDA(cudaGraphCreate(&sgraph_, 0));
    FG_CUDA(cudaGraphConditionalHandleCreate(&scond_, sgraph_, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = scond_;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    FG_CUDA(cudaGraphAddNode(&node, sgraph_, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    FG_CUDA(cudaStreamBeginCaptureToGraph(s_, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
    k_sadmit<<<(S + BTH - 1) / BTH, BTH, 0, s_>>>(S, dh_, seen_.p, phase_.p, done_.p, admit_.p);
    k_sadmit_copy<R><<<nchunks_, BTH, 0, s_>>>(chunks(), boffd_.p, admit_.p, dh_, b_.p, r_.p,
                                               mixed ? r32_.p : nullptr, x_.p, p_.p, q_.p);
    iteration<R>(true);
    k_sdeliver_copy<R><<<nchunks_, BTH, 0, s_>>>(chunks(), boffd_.p, phase_.p, dh_, x_.p);
    k_sdeliver<<<(S + BTH - 1) / BTH, BTH, 0, s_>>>(S, dh_, seen_.p, phase_.p, scalars());
    k_sloop_control<<<1, BTH, 0, s_>>>(scond_, S, dh_, seen_.p, phase_.p, loops_.p,
                                       served_its_.p);
    FG_CUDA(cudaStreamEndCapture(s_, &body));
    FG_CUDA(cudaGraphInstantiate(&sexec_, sgraph_, 0));
    launches_ = before;
}

void BatchImpl::stream_open() {
    if (sexec_) return;
    const size_t S = (size_t)B_ * R_, vals = (size_t)n_ * R_;
    phase_.alloc(S);
    restarts_seg_.alloc(S);
    fresh_.alloc(S);
    admit_.alloc(S);
    seen_.alloc(S);
    served_its_.alloc(1);
    served_its_.zero(s_);
    loops_.zero(s_);  // the stream's loop iterations, counted from its opening
    phase_.zero(s_);
    restarts_seg_.zero(s_);
    fresh_.zero(s_);
    admit_.zero(s_);
    seen_.zero(s_);
    boffd_.upload(boff_.data(), boff_.size(), s_);
    // Every slot starts free and finished (done), its vectors 0.
    std::vector<int> ones(S, 1);
    done_.upload(ones.data(), S, s_);
    for (auto* v : {&x_, &r_, &p_, &q_, &b_}) v->zero(s_);
    if (r32_.p) r32_.zero(s_);
    FG_CUDA(cudaHostAlloc(&h_req_, S * sizeof(unsigned long long), cudaHostAllocMapped));
    FG_CUDA(cudaHostAlloc(&h_served_, S * sizeof(unsigned long long), cudaHostAllocMapped));
    FG_CUDA(cudaHostAlloc(&h_in_, vals * sizeof(double), cudaHostAllocMapped));
    FG_CUDA(cudaHostAlloc(&h_out_, vals * sizeof(double), cudaHostAllocMapped));
    FG_CUDA(cudaHostAlloc(&h_stat_, S * sizeof(StreamStat), cudaHostAllocMapped));
    FG_CUDA(cudaHostAlloc(&h_stop_, sizeof(int), cudaHostAllocMapped));
    std::memset(h_req_, 0, S * sizeof(unsigned long long));
    std::memset(h_served_, 0, S * sizeof(unsigned long long));
    std::memset(h_stat_, 0, S * sizeof(StreamStat));
    *h_stop_ = 0;
    unsigned long long *dreq, *dserved;
    double *din, *dout;
    StreamStat* dstat;
    int* dstop;
    FG_CUDA(cudaHostGetDevicePointer(&dreq, h_req_, 0));
    FG_CUDA(cudaHostGetDevicePointer(&dserved, h_served_, 0));
    FG_CUDA(cudaHostGetDevicePointer(&din, h_in_, 0));
    FG_CUDA(cudaHostGetDevicePointer(&dout, h_out_, 0));
    FG_CUDA(cudaHostGetDevicePointer(&dstat, h_stat_, 0));
    FG_CUDA(cudaHostGetDevicePointer(&dstop, h_stop_, 0));
    dh_ = StreamHost{dreq, dserved, din, dout, dstat, dstop};
    FG_CUDA(cudaEventCreateWithFlags(&sev_, cudaEventDisableTiming));
    if (R_ == 16)
        build_stream_graph<16>();
    else if (R_ == 4)
        build_stream_graph<4>();
    else
        build_stream_graph<1>();
    FG_CUDA(cudaStreamSynchronize(s_));
}

void BatchImpl::stream_launch() {
    FG_CUDA(cudaGraphLaunch(sexec_, s_));
    FG_CUDA(cudaEventRecord(sev_, s_));
    slaunched_ = true;
}

bool BatchImpl::stream_idle() {
    if (!slaunched_) return true;
    const cudaError_t e = cudaEventQuery(sev_);
    if (e == cudaErrorNotReady) return false;
    FG_CUDA(e);
    slaunched_ = false;
    return true;
}

void BatchImpl::stream_stop() {
    if (h_stop_) *(volatile int*)h_stop_ = 1;
    FG_CUDA(cudaStreamSynchronize(s_));
    slaunched_ = false;
}

size_t BatchImpl::stream_loops() { return (size_t)fetch(loops_.p, s_); }
size_t BatchImpl::stream_served_iterations() { return (size_t)fetch(served_its_.p, s_); }
bool BatchImpl::streaming() const { return sexec_ != nullptr; }

void BatchImpl::permute(const double* in, double* out, int scatter) {
    const int64_t e = n_ * R_;
    const int g = (int)((e + BTH - 1) / BTH);
    if (R_ == 16)
        k_bpermute<16><<<g, BTH, 0, s_>>>(n_, map_.p, in, out, scatter);
    else if (R_ == 4)
        k_bpermute<4><<<g, BTH, 0, s_>>>(n_, map_.p, in, out, scatter);
    else
        k_bpermute<1><<<g, BTH, 0, s_>>>(n_, map_.p, in, out, scatter);
    FG_CHECK_LAUNCH();
    launches_ += 1;
}

// The solve on b_ and x_ (the batch's order), already loaded.
void BatchImpl::solve_loaded(const volatile int* cancel, femgpu_batch_stats* st) {
    if (R_ == 16)
        run<16>(cancel);
    else if (R_ == 4)
        run<4>(cancel);
    else
        run<1>(cancel);
}

void BatchImpl::solve_device(const double* d_b, double* d_x, const volatile int* cancel,
                             femgpu_batch_stats* st) {
    if (streaming())
        throw Failure(FEMGPU_ERR_INVALID, "the batch serves a stream: solve through the stream");
    if (exec_ && (max_iter_ != graph_max_iter_ || tol != graph_tol_)) {
        cudaGraphExecDestroy(exec_);
        cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
    }
    launches_ = 0;
    FG_CUDA(cudaEventRecord(ev0_, s_));
    permute(d_b, b_.p, 0);
    permute(d_x, x_.p, 0);
    solve_loaded(cancel, st);
    permute(x_.p, d_x, 1);
    FG_CUDA(cudaEventRecord(ev1_, s_));
    FG_CUDA(cudaStreamSynchronize(s_));
    if (cancel && *cancel) throw Failure(FEMGPU_ERR_CANCELLED, "cancelled");
    collect(st);
}

// Host vectors go through the batch's own staging vector, so a solve allocates nothing.
void BatchImpl::solve_host(const double* h_b, double* h_x, const volatile int* cancel,
                           femgpu_batch_stats* st) {
    if (streaming())
        throw Failure(FEMGPU_ERR_INVALID, "the batch serves a stream: solve through the stream");
    const size_t bytes = (size_t)n_ * R_ * sizeof(double);
    if (exec_ && (max_iter_ != graph_max_iter_ || tol != graph_tol_)) {
        cudaGraphExecDestroy(exec_);
        cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
    }
    launches_ = 0;
    FG_CUDA(cudaEventRecord(ev0_, s_));
    FG_CUDA(cudaMemcpyAsync(stage_.p, h_b, bytes, cudaMemcpyHostToDevice, s_));
    permute(stage_.p, b_.p, 0);
    FG_CUDA(cudaMemcpyAsync(stage_.p, h_x, bytes, cudaMemcpyHostToDevice, s_));
    permute(stage_.p, x_.p, 0);
    solve_loaded(cancel, st);
    permute(x_.p, stage_.p, 1);
    FG_CUDA(cudaMemcpyAsync(h_x, stage_.p, bytes, cudaMemcpyDeviceToHost, s_));
    FG_CUDA(cudaEventRecord(ev1_, s_));
    FG_CUDA(cudaStreamSynchronize(s_));
    if (cancel && *cancel) throw Failure(FEMGPU_ERR_CANCELLED, "cancelled");
    collect(st);
}

void BatchImpl::segments(size_t* iterations, double* truth, double* residual,
                         int* status) const {
    const int S = B_ * R_;
    std::vector<int> it(S), stt(S);
    std::vector<double> tr(S), rr(S), bb(S);
    iters_.download(it.data(), S, s_);
    status_.download(stt.data(), S, s_);
    truth_.download(tr.data(), S, s_);
    rr_.download(rr.data(), S, s_);
    bb_.download(bb.data(), S, s_);
    FG_CUDA(cudaStreamSynchronize(s_));
    for (int k = 0; k < B_; ++k)
        for (int c = 0; c < R_; ++c) {
            const int s = k * R_ + c;           // the batch's segment
            const int o = order_[k] * R_ + c;   // the caller's
            if (iterations) iterations[o] = (size_t)it[s];
            if (truth) truth[o] = tr[s];
            if (residual) residual[o] = bb[s] > 0 ? std::sqrt(rr[s]) / std::sqrt(bb[s]) : 0.0;
            if (status) status[o] = stt[s];
        }
}

void BatchImpl::collect(femgpu_batch_stats* st) {
    const int S = B_ * R_;
    std::vector<size_t> it(S);
    std::vector<double> tr(S), res(S);
    std::vector<int> stt(S);
    segments(it.data(), tr.data(), res.data(), stt.data());  // the caller's order
    const int loops = fetch(loops_.p, s_);
    femgpu_batch_stats out{};
    size_t total = 0;
    int first_bad = -1;
    for (int s = 0; s < S; ++s) {
        out.max_iterations = std::max(out.max_iterations, it[s]);
        total += it[s];
        out.max_residual = std::max(out.max_residual, res[s]);
        out.max_true_residual = std::max(out.max_true_residual, tr[s]);
        if (stt[s]) {
            out.not_converged += 1;
            if (first_bad < 0) first_bad = s;
        }
    }
    out.mean_iterations = (double)total / S;
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    out.seconds = ms * 1e-3;
    out.launches = launches_ + graph_kernels_ * (size_t)loops;
    out.restarts = (size_t)restarts_;
    if (st) *st = out;
    if (first_bad >= 0) {
        char buf[240];
        const int s = first_bad;
        if (stt[s] == 2)
            std::snprintf(buf, sizeof buf,
                          "system %d, right side %d: conjugate gradients broke down: the residual "
                          "is not a number",
                          s / R_, s % R_);
        else
            std::snprintf(buf, sizeof buf,
                          "system %d, right side %d: conjugate gradients did not converge: the "
                          "residual is %s after %zu iterations",
                          s / R_, s % R_, rust_exp(res[s], 2).c_str(), it[s]);
        throw Failure(FEMGPU_ERR_NOT_CONVERGED, buf);
    }
}

void BatchImpl::kernel_time(int reps, double* ms, double* bytes) {
    const bool mixed = opt_.precision == FEMGPU_MIXED;
    const int64_t ns = mixed ? L32_[0].ns : L64_[0].ns;
    if (ns == 0) throw Failure(FEMGPU_ERR_INVALID, "no member smooths at the finest level");
    reps = std::max(1, reps);
    auto go = [&](auto& L, auto r) {
        using T = typename std::remove_reference<decltype(*L.dinv.p)>::type;
        constexpr int R = decltype(r)::value;
        const int g = (int)((L.ns * (R / Lanes<T, R>::W) + BTH - 1) / BTH);
        const int g3 = (int)((L.ns / 3 * (R / Lanes<T, R>::W) + BTH - 1) / BTH);
        for (int k = 0; k < reps + 5; ++k) {
            if (k == 5) FG_CUDA(cudaEventRecord(ev0_, s_));
            if (L.block3)
                k_bcheb_step3<T, R><<<g3, BTH, 0, s_>>>(L.view3(), L.b.p, L.xa.p, L.dinv.p,
                                                         (T)0.5, (T)0.5, L.d.p, L.xb.p);
            else
                k_bcheb_step<T, R><<<g, BTH, 0, s_>>>(L.A.view(), L.b.p, L.xa.p, L.dinv.p,
                                                      (T)0.5, (T)0.5, L.d.p, L.xb.p);
        }
        FG_CHECK_LAUNCH();
        FG_CUDA(cudaEventRecord(ev1_, s_));
        FG_CUDA(cudaEventSynchronize(ev1_));
        float t = 0;
        FG_CUDA(cudaEventElapsedTime(&t, ev0_, ev1_));
        *ms = t / reps;
        // Each value and index of the level once, and per right side b, x, d (read), d and
        // x_out (written) and the row's D^-1.
        const double mat = L.block3 ? (double)L.b3col.bytes() + (double)L.b3val.bytes()
                                    : (double)L.A.bytes() - (double)L.A.slice_ptr.bytes();
        *bytes = mat + (double)L.ns * sizeof(T) * (5.0 * R + 1.0);
    };
    auto pick = [&](auto& L) {
        FG_CUDA(cudaMemsetAsync(L.xa.p, 0, L.xa.bytes(), s_));
        FG_CUDA(cudaMemsetAsync(L.b.p, 0, L.b.bytes(), s_));
        FG_CUDA(cudaMemsetAsync(L.d.p, 0, L.d.bytes(), s_));
        if (R_ == 16)
            go(L, std::integral_constant<int, 16>());
        else if (R_ == 4)
            go(L, std::integral_constant<int, 4>());
        else
            go(L, std::integral_constant<int, 1>());
    };
    if (mixed)
        pick(L32_[0]);
    else
        pick(L64_[0]);
}

size_t BatchImpl::bytes() const {
    size_t b = A64_.bytes() + f3ptr_.bytes() + f3col_.bytes() + f3val_.bytes() +
               partial_.bytes() + chunks_.bytes() + cstart_.bytes() + map_.bytes();
    auto levels = [&](const auto& Ls) {
        for (const auto& L : Ls)
            b += L.A.bytes() + L.b3ptr.bytes() + L.b3col.bytes() + L.b3val.bytes() +
                 L.dinv.bytes() + L.pptr.bytes() + L.rptr.bytes() + L.pidx.bytes() +
                 L.ridx.bytes() + L.pval.bytes() + L.rval.bytes() + L.b.bytes() + L.xa.bytes() +
                 L.xb.bytes() + L.d.bytes() + L.r.bytes() + L.doff.bytes() + L.dioff.bytes() +
                 L.tiles.bytes() + L.inv.bytes();
    };
    levels(L32_);
    levels(L64_);
    b += x_.bytes() + r_.bytes() + p_.bytes() + q_.bytes() + b_.bytes() + stage_.bytes() +
         r32_.bytes();
    return b;
}

}  // namespace femgpu

// ------------------------------------------------------------------ C ABI
struct femgpu_batch {
    femgpu::BatchImpl impl;
};

// The host side of continuous batching: requests wait in a queue per system until one of its
// slots is free, then go into the mapped staging slot and the device loop admits them at its
// next iteration. 1 worker thread publishes requests, starts the device loop when a slot is busy
// and it is not running, and collects the finished slots.
struct femgpu_stream {
    femgpu_batch* batch = nullptr;
    int device = 0;
    std::mutex m;
    std::condition_variable cv;
    struct Ticket {
        int member = 0;
        std::vector<double> rhs, x;
        femgpu::StreamStat stat{};
        std::chrono::steady_clock::time_point t0, t1;
        bool done = false;
    };
    std::unordered_map<uint64_t, Ticket> tickets;
    uint64_t next = 1;
    std::vector<std::deque<uint64_t>> queue;  // per system
    std::vector<uint64_t> slot_ticket;        // per segment, 0 when free
    std::vector<unsigned long long> gen;      // per segment, the last generation published
    std::thread worker;
    bool quit = false;
    std::string failure;

    void run() {
        using namespace femgpu;
        BatchImpl& b = batch->impl;
        cudaSetDevice(device);
        const int R = b.slots(), B = b.members();
        std::unique_lock<std::mutex> lk(m);
        for (;;) {
            bool progress = false, busy = false;
            for (int k = 0; k < B; ++k)
                for (int c = 0; c < R; ++c) {
                    const int sg = b.segment(k, c);
                    const uint64_t t = slot_ticket[sg];
                    if (!t) continue;
                    if (b.h_served()[sg] != gen[sg]) {
                        busy = true;
                        continue;
                    }
                    // Finished: its x and figures from the mapped output slot.
                    std::atomic_thread_fence(std::memory_order_acquire);
                    Ticket& tk = tickets[t];
                    const double* out = b.h_out() + b.slot_offset(k, c);
                    tk.x.assign(out, out + b.member_rows(k));
                    tk.stat = b.h_stat()[sg];
                    tk.t1 = std::chrono::steady_clock::now();
                    tk.done = true;
                    slot_ticket[sg] = 0;
                    progress = true;
                }
            for (int k = 0; k < B; ++k)
                for (int c = 0; c < R && !queue[k].empty(); ++c) {
                    const int sg = b.segment(k, c);
                    if (slot_ticket[sg]) continue;
                    const uint64_t t = queue[k].front();
                    queue[k].pop_front();
                    Ticket& tk = tickets[t];
                    std::memcpy(b.h_in() + b.slot_offset(k, c), tk.rhs.data(),
                                tk.rhs.size() * sizeof(double));
                    std::atomic_thread_fence(std::memory_order_release);
                    gen[sg] += 1;
                    b.h_req()[sg] = gen[sg];
                    slot_ticket[sg] = t;
                    busy = true;
                    progress = true;
                }
            if (progress) cv.notify_all();
            try {
                if (busy && b.stream_idle()) b.stream_launch();
            } catch (const std::exception& e) {
                failure = e.what();
                cv.notify_all();
                return;
            }
            if (quit && !busy) return;
            if (busy)
                cv.wait_for(lk, std::chrono::microseconds(20));
            else
                cv.wait(lk);
        }
    }
};

using namespace femgpu;

template <class F>
static int batch_guarded(F f) {
    try {
        f();
        return FEMGPU_OK;
    } catch (const Failure& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("out of host memory");
        return FEMGPU_ERR_TOO_LARGE;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return FEMGPU_ERR_INVALID;
    }
}

extern "C" {

int femgpu_batch_new(int count, const femgpu_csr* const* a, const femgpu_unknowns* u, int nrhs,
                     const femgpu_options* options, femgpu_batch** out) {
    return batch_guarded([&] {
        if (!a || !u || !out || count < 1) throw Failure(FEMGPU_ERR_INVALID, "null argument");
        std::vector<const DevCsr*> mats;
        std::vector<const femgpu_unknowns*> us;
        for (int b = 0; b < count; ++b) {
            if (!a[b]) throw Failure(FEMGPU_ERR_INVALID, "a null matrix");
            if (u[b].kind != FEMGPU_UNKNOWNS_GRID || !u[b].points || !u[b].comp)
                throw Failure(FEMGPU_ERR_NEEDS_GRID,
                              "multigrid needs the box grid: a batch takes grid unknowns");
            if (u[b].nplanes[0] < 1 || u[b].nplanes[1] < 1 || u[b].nplanes[2] < 1)
                throw Failure(FEMGPU_ERR_INVALID, "a grid without planes");
            mats.push_back(&a[b]->m);
            us.push_back(&u[b]);
        }
        Options o;
        o.format = 0;
        o.coarsest = 0;
        if (options) {
            o.precision = options->precision;
            o.format = options->format;
            o.degree = options->degree;
            o.lower = options->lower;
            o.coarsest = options->coarsest;
            o.max_levels = options->max_levels;
        }
        o.smoother = options && options->smoother ? options->smoother : 4;
        if (o.smoother != 1 && o.smoother != 4)
            throw Failure(FEMGPU_ERR_INVALID,
                          "smoother is 1 (the first-kind Chebyshev polynomial) or 0 or 4 (the "
                          "fourth kind)");
        auto* bt = new femgpu_batch;
        try {
            bt->impl.create(mats, us, nrhs, o);
        } catch (...) {
            delete bt;
            throw;
        }
        *out = bt;
    });
}

int femgpu_batch_set_tol(femgpu_batch* b, double tol) {
    return batch_guarded([&] {
        if (!b || !(tol >= 0)) throw Failure(FEMGPU_ERR_INVALID, "a tolerance must be 0 or more");
        b->impl.tol = tol;
    });
}

int femgpu_batch_set_max_iter(femgpu_batch* b, size_t max_iter) {
    return batch_guarded([&] {
        if (!b) throw Failure(FEMGPU_ERR_INVALID, "null batch");
        b->impl.set_max_iter((int)std::min<size_t>(max_iter, 0x7fffffff));
    });
}

int femgpu_batch_systems(const femgpu_batch* b, size_t* offsets) {
    if (!b) return 0;
    const auto& o = b->impl.offsets();
    if (offsets)
        for (size_t k = 0; k < o.size(); ++k) offsets[k] = (size_t)o[k];
    return (int)o.size() - 1;
}

int femgpu_batch_describe(const femgpu_batch* b, char* buf, size_t len) {
    if (!b || !buf || len == 0) return FEMGPU_ERR_INVALID;
    const std::string d = b->impl.describe();
    std::snprintf(buf, len, "%s", d.c_str());
    return FEMGPU_OK;
}

int femgpu_batch_levels(const femgpu_batch* b, size_t* sizes) {
    if (!b) return 0;
    auto v = b->impl.level_sizes();
    if (sizes)
        for (size_t k = 0; k < v.size(); ++k) sizes[k] = (size_t)v[k];
    return (int)v.size();
}

int femgpu_batch_solve(femgpu_batch* b, const double* rhs, double* x, const volatile int* cancel,
                       femgpu_batch_stats* stats) {
    return batch_guarded([&] {
        if (!b || !rhs || !x) throw Failure(FEMGPU_ERR_INVALID, "null argument");
        b->impl.solve_host(rhs, x, cancel, stats);
    });
}

int femgpu_batch_solve_device(femgpu_batch* b, const double* rhs, double* x,
                              const volatile int* cancel, femgpu_batch_stats* stats) {
    return batch_guarded([&] {
        if (!b || !rhs || !x) throw Failure(FEMGPU_ERR_INVALID, "null argument");
        b->impl.solve_device(rhs, x, cancel, stats);
    });
}

int femgpu_batch_segments(const femgpu_batch* b, size_t* iterations, double* true_residual,
                          double* residual, int* status) {
    return batch_guarded([&] {
        if (!b) throw Failure(FEMGPU_ERR_INVALID, "null batch");
        b->impl.segments(iterations, true_residual, residual, status);
    });
}

int femgpu_batch_kernel_time(femgpu_batch* b, int reps, double* ms, double* bytes) {
    return batch_guarded([&] {
        if (!b || !ms || !bytes) throw Failure(FEMGPU_ERR_INVALID, "null argument");
        b->impl.kernel_time(reps, ms, bytes);
    });
}

size_t femgpu_batch_bytes(const femgpu_batch* b) { return b ? b->impl.bytes() : 0; }

void* femgpu_batch_stream(const femgpu_batch* b) {
    return b ? (void*)b->impl.stream() : nullptr;
}

void femgpu_batch_free(femgpu_batch* b) { delete b; }

int femgpu_stream_new(femgpu_batch* b, femgpu_stream** out) {
    return batch_guarded([&] {
        if (!b || !out) throw Failure(FEMGPU_ERR_INVALID, "null argument");
        if (b->impl.streaming()) throw Failure(FEMGPU_ERR_INVALID, "the batch serves a stream already");
        b->impl.stream_open();
        auto st = std::make_unique<femgpu_stream>();
        st->batch = b;
        FG_CUDA(cudaGetDevice(&st->device));
        const int S = b->impl.members() * b->impl.slots();
        st->queue.resize(b->impl.members());
        st->slot_ticket.assign(S, 0);
        st->gen.assign(S, 0);
        femgpu_stream* raw = st.get();
        st->worker = std::thread([raw] { raw->run(); });
        *out = st.release();
    });
}

int femgpu_stream_submit(femgpu_stream* s, int system, const double* rhs, uint64_t* ticket) {
    return batch_guarded([&] {
        if (!s || !rhs || !ticket) throw Failure(FEMGPU_ERR_INVALID, "null argument");
        BatchImpl& b = s->batch->impl;
        if (system < 0 || system >= b.members())
            throw Failure(FEMGPU_ERR_INVALID, "no such system in the batch");
        std::lock_guard<std::mutex> lk(s->m);
        if (!s->failure.empty()) throw Failure(FEMGPU_ERR_CUDA, s->failure);
        const uint64_t t = s->next++;
        femgpu_stream::Ticket& tk = s->tickets[t];
        tk.member = system;
        tk.rhs.assign(rhs, rhs + b.member_rows(system));
        tk.t0 = std::chrono::steady_clock::now();
        s->queue[system].push_back(t);
        *ticket = t;
        s->cv.notify_all();
    });
}

int femgpu_stream_wait(femgpu_stream* s, uint64_t ticket, double* x,
                       femgpu_stream_result* result) {
    return batch_guarded([&] {
        if (!s || !x) throw Failure(FEMGPU_ERR_INVALID, "null argument");
        std::unique_lock<std::mutex> lk(s->m);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) throw Failure(FEMGPU_ERR_INVALID, "no such ticket");
        s->cv.wait(lk, [&] { return it->second.done || !s->failure.empty(); });
        if (!it->second.done) throw Failure(FEMGPU_ERR_CUDA, s->failure);
        femgpu_stream::Ticket tk = std::move(it->second);
        s->tickets.erase(it);
        lk.unlock();
        std::memcpy(x, tk.x.data(), tk.x.size() * sizeof(double));
        if (result) {
            result->iterations = (size_t)tk.stat.iterations;
            result->residual = tk.stat.residual;
            result->true_residual = tk.stat.truth;
            result->status = tk.stat.status;
            result->latency_s = std::chrono::duration<double>(tk.t1 - tk.t0).count();
        }
        if (tk.stat.status == 2)
            throw Failure(FEMGPU_ERR_NOT_CONVERGED,
                          "conjugate gradients broke down: the residual is not a number");
        if (tk.stat.status == 1) {
            char buf[200];
            std::snprintf(buf, sizeof buf,
                          "conjugate gradients did not converge: the residual is %s after %d "
                          "iterations",
                          rust_exp(tk.stat.residual, 2).c_str(), tk.stat.iterations);
            throw Failure(FEMGPU_ERR_NOT_CONVERGED, buf);
        }
    });
}

int femgpu_stream_counts(femgpu_stream* s, size_t* loops, size_t* served_iterations) {
    return batch_guarded([&] {
        if (!s) throw Failure(FEMGPU_ERR_INVALID, "null stream");
        std::lock_guard<std::mutex> lk(s->m);
        if (loops) *loops = s->batch->impl.stream_loops();
        if (served_iterations) *served_iterations = s->batch->impl.stream_served_iterations();
    });
}

void femgpu_stream_free(femgpu_stream* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->quit = true;
        s->cv.notify_all();
    }
    // Requests still running end with the loop: the device stops at its next iteration.
    try {
        s->batch->impl.stream_stop();
    } catch (...) {
    }
    {
        std::lock_guard<std::mutex> lk(s->m);
        for (auto& t : s->slot_ticket) t = 0;
        s->failure = s->failure.empty() ? "the stream was freed" : s->failure;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    delete s;
}

}  // extern "C"
