// 3x3-block operators of elasticity: the 3 rows of a node have the same columns, which come in
// node triples. Stored as SELL over block rows: slices of B3C block rows, each block row padded
// to its slice's width; a block is 9 values (row-major) and 1 block column; padding blocks are 0
// and point at the block row itself, so that they read x the row reads anyway. Per block 40 bytes
// in FP32 (36 of values, 4 of index) against 72 for the same 9 entries in scalar SELL.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>

#include "hierarchy.hpp"
#include "sell.cuh"

namespace femgpu {

constexpr int B3C = 32;

template <class T>
struct BSell3View {
    int64_t nb;                             // block rows
    const int64_t* __restrict__ slice_ptr;  // in blocks; nslices + 1
    const uint32_t* __restrict__ col;       // block column per block
    const T* __restrict__ val;              // 9 per block
};

// The operator of 1 row per thread on the 3x3-block form: row g is row g % 3 of block row g / 3;
// the 3 threads of a block row read its blocks' column and each its 3 values of the block.
template <class T>
struct Block3Op {
    BSell3View<T> v;
    int n;  // rows = 3 nb
    __device__ __forceinline__ int64_t threads() const {
        return 3 * ((v.nb + B3C - 1) / B3C) * B3C;
    }
    __device__ __forceinline__ bool valid(int64_t g) const { return g < n; }
    template <class TA, class TX>
    __device__ __forceinline__ TA apply(int64_t g, const TX* __restrict__ x) const {
        const int I = (int)(g / 3), a = (int)(g % 3);
        if (I >= v.nb) return (TA)0;
        const int s = I / B3C, r = I % B3C;
        const int64_t b = v.slice_ptr[s], e = v.slice_ptr[s + 1];
        const int w = (int)((e - b) / B3C);
        TA acc = 0;
        for (int k = 0; k < w; ++k) {
            const int64_t blk = b + (int64_t)k * B3C + r;
            const int64_t J3 = 3 * (int64_t)__ldg(v.col + blk);
            const T* vv = v.val + blk * 9 + 3 * a;
            acc += (TA)__ldg(vv) * (TA)__ldg(x + J3);
            acc += (TA)__ldg(vv + 1) * (TA)__ldg(x + J3 + 1);
            acc += (TA)__ldg(vv + 2) * (TA)__ldg(x + J3 + 2);
        }
        return acc;
    }
};

// Runs f(lo, hi) over [0, n) split among the host threads.
template <class F>
inline void parallel_ranges(int64_t n, F&& f) {
    const int64_t t = std::max<int64_t>(1, std::min<int64_t>(host_threads(), n / 4096));
    if (t == 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (int64_t k = 0; k < t; ++k) pool.emplace_back([&, k] { f(n * k / t, n * (k + 1) / t); });
    for (auto& th : pool) th.join();
}

// The 3x3-block SELL form of `a`, if every node's 3 rows have the same columns and the columns
// come in aligned triples; false (and nothing built) otherwise. The block rows are checked and
// filled on all host threads.
template <class T>
inline bool make_bsell3(const HostCsr& a, std::vector<int64_t>* sptr, std::vector<uint32_t>* cols,
                        std::vector<T>* vals) {
    if (a.n % 3 != 0 || a.n / 3 >= 0x7fffffff) return false;
    const int64_t nb = a.n / 3;
    std::vector<int> width(nb);
    std::atomic<bool> ok{true};
    parallel_ranges(nb, [&](int64_t lo, int64_t hi) {
        for (int64_t I = lo; I < hi && ok.load(std::memory_order_relaxed); ++I) {
            const int64_t r0 = 3 * I;
            const int64_t len = a.ptr[r0 + 1] - a.ptr[r0];
            bool good = len % 3 == 0;
            for (int q = 1; q < 3 && good; ++q) {
                if (a.ptr[r0 + q + 1] - a.ptr[r0 + q] != len) good = false;
                for (int64_t k = 0; k < len && good; ++k)
                    if (a.idx[a.ptr[r0 + q] + k] != a.idx[a.ptr[r0] + k]) good = false;
            }
            for (int64_t k = 0; k < len && good; k += 3) {
                const uint32_t c = a.idx[a.ptr[r0] + k];
                if (c % 3 != 0 || a.idx[a.ptr[r0] + k + 1] != c + 1 ||
                    a.idx[a.ptr[r0] + k + 2] != c + 2)
                    good = false;
            }
            if (!good) ok.store(false);
            width[I] = (int)(len / 3);
        }
    });
    if (!ok.load()) return false;
    const int64_t nslices = (nb + B3C - 1) / B3C;
    sptr->assign(nslices + 1, 0);
    for (int64_t sl = 0; sl < nslices; ++sl) {
        int w = 0;
        for (int64_t I = sl * B3C; I < std::min(nb, (sl + 1) * B3C); ++I) w = std::max(w, width[I]);
        (*sptr)[sl + 1] = (*sptr)[sl] + (int64_t)w * B3C;
    }
    cols->assign((*sptr)[nslices], 0);
    vals->assign((size_t)(*sptr)[nslices] * 9, (T)0);
    parallel_ranges(nb, [&](int64_t lo, int64_t hi) {
        for (int64_t I = lo; I < hi; ++I) {
            const int64_t sl = I / B3C, r = I % B3C, base = (*sptr)[sl];
            const int w = (int)(((*sptr)[sl + 1] - base) / B3C);
            for (int k = 0; k < w; ++k) {
                const int64_t blk = base + (int64_t)k * B3C + r;
                if (k < width[I]) {
                    const int64_t e = a.ptr[3 * I] + 3 * k;
                    (*cols)[blk] = a.idx[e] / 3;
                    for (int q = 0; q < 3; ++q)
                        for (int c = 0; c < 3; ++c)
                            (*vals)[(size_t)blk * 9 + 3 * q + c] =
                                (T)a.val[a.ptr[3 * I + q] + 3 * k + c];
                } else {
                    (*cols)[blk] = (uint32_t)I;  // padding: value 0, the block row's own x
                }
            }
        }
    });
    return true;
}

}  // namespace femgpu
