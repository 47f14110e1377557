// The rectangular matrix of the reference (sparse.rs:196-293 Rect: y = P x, y = P^T x, the
// Galerkin product P^T A P) and Csr::diagonal (sparse.rs:88-93) on the device. Built with
// -fmad=false: each product sums a row in the reference's order with separate roundings, so
// P x and P^T x are the reference's bit for bit (P^T x as the rows of the transpose, whose
// entries come in increasing row of P, the order in which the reference adds into y).
#include <algorithm>

#include "coarsen.cuh"
#include "common.cuh"
#include "femgpu.h"
#include "solver.cuh"

struct femgpu_rect {
    femgpu::DevRect p;
    femgpu::DevRect t;  // the transpose, made on first use
    bool has_t = false;
};

namespace femgpu {
namespace {

constexpr int RT = 256;

__global__ void k_rect_mul(int64_t rows, const int64_t* __restrict__ ptr,
                           const uint32_t* __restrict__ idx, const double* __restrict__ val,
                           const double* __restrict__ x, double* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows;
         i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) s += val[k] * x[idx[k]];
        y[i] = s;
    }
}

__global__ void k_diag_of(int64_t n, const int64_t* __restrict__ ptr,
                          const uint32_t* __restrict__ idx, const double* __restrict__ val,
                          double* __restrict__ d) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        // The row's columns increase: a binary search, as Csr::find (sparse.rs:78-86).
        int64_t lo = ptr[i], hi = ptr[i + 1];
        double v = 0.0;
        while (lo < hi) {
            const int64_t mid = (lo + hi) / 2;
            if ((int64_t)idx[mid] < i)
                lo = mid + 1;
            else
                hi = mid;
        }
        if (lo < ptr[i + 1] && (int64_t)idx[lo] == i) v = val[lo];
        d[i] = v;
    }
}

template <class F>
int guard(F f) {
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

// A stream per call, destroyed on every path.
struct CallStream {
    cudaStream_t s = nullptr;
    CallStream() { FG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~CallStream() {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
};

}  // namespace
}  // namespace femgpu

using namespace femgpu;

extern "C" {

int femgpu_rect_upload(size_t rows, size_t cols, const int64_t* ptr, const uint32_t* idx,
                       const double* val, femgpu_rect** out) {
    return guard([&] {
        if (!out || !ptr) throw Failure(FEMGPU_ERR_INVALID, "a null argument");
        if (ptr[0] != 0) throw Failure(FEMGPU_ERR_INVALID, "the row pointers must start at 0");
        const int64_t nnz = ptr[rows];
        for (size_t i = 0; i < rows; ++i)
            if (ptr[i + 1] < ptr[i])
                throw Failure(FEMGPU_ERR_INVALID, "the row pointers must not decrease");
        if (nnz > 0 && (!idx || !val)) throw Failure(FEMGPU_ERR_INVALID, "a null argument");
        for (int64_t k = 0; k < nnz; ++k)
            if (idx[k] >= cols) throw Failure(FEMGPU_ERR_INVALID, "a column past the columns");
        CallStream cs;
        auto* h = new femgpu_rect;
        h->p.rows = (int64_t)rows;
        h->p.cols = (int64_t)cols;
        h->p.nnz = nnz;
        try {
            h->p.ptr.upload(ptr, rows + 1, cs.s);
            h->p.idx.alloc(std::max<int64_t>(nnz, 1));
            h->p.val.alloc(std::max<int64_t>(nnz, 1));
            if (nnz > 0) {
                h->p.idx.upload(idx, nnz, cs.s);
                h->p.val.upload(val, nnz, cs.s);
            }
            FG_CUDA(cudaStreamSynchronize(cs.s));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int femgpu_rect_mul(femgpu_rect* r, const double* x, double* y) {
    return guard([&] {
        if (!r || !x || !y) throw Failure(FEMGPU_ERR_INVALID, "a null argument");
        CallStream cs;
        DevBuf<double> dx, dy(std::max<int64_t>(r->p.rows, 1));
        dx.upload(x, r->p.cols, cs.s);
        k_rect_mul<<<blocks_for(r->p.rows, RT), RT, 0, cs.s>>>(r->p.rows, r->p.ptr.p, r->p.idx.p,
                                                              r->p.val.p, dx.p, dy.p);
        FG_CHECK_LAUNCH();
        dy.download(y, r->p.rows, cs.s);
        FG_CUDA(cudaStreamSynchronize(cs.s));
    });
}

int femgpu_rect_mul_transpose(femgpu_rect* r, const double* x, double* y) {
    return guard([&] {
        if (!r || !x || !y) throw Failure(FEMGPU_ERR_INVALID, "a null argument");
        CallStream cs;
        if (!r->has_t) {
            transpose_rect(r->p, &r->t, cs.s);
            r->has_t = true;
        }
        DevBuf<double> dx, dy(std::max<int64_t>(r->t.rows, 1));
        dx.upload(x, r->p.rows, cs.s);
        k_rect_mul<<<blocks_for(r->t.rows, RT), RT, 0, cs.s>>>(r->t.rows, r->t.ptr.p, r->t.idx.p,
                                                              r->t.val.p, dx.p, dy.p);
        FG_CHECK_LAUNCH();
        dy.download(y, r->t.rows, cs.s);
        FG_CUDA(cudaStreamSynchronize(cs.s));
    });
}

int femgpu_rect_galerkin(const femgpu_rect* r, const femgpu_csr* a, femgpu_csr** out) {
    return guard([&] {
        if (!r || !a || !out) throw Failure(FEMGPU_ERR_INVALID, "a null argument");
        if (r->p.rows != a->m.n)
            throw Failure(FEMGPU_ERR_INVALID, "the rows of P must be the size of the matrix");
        CallStream cs;
        auto* h = new femgpu_csr;
        try {
            galerkin_product(r->p, a->m, &h->m, cs.s);
            FG_CUDA(cudaStreamSynchronize(cs.s));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

void femgpu_rect_free(femgpu_rect* r) { delete r; }

int femgpu_csr_diagonal(const femgpu_csr* a, double* d) {
    return guard([&] {
        if (!a || !d) throw Failure(FEMGPU_ERR_INVALID, "a null argument");
        CallStream cs;
        DevBuf<double> dd(std::max<int64_t>(a->m.n, 1));
        k_diag_of<<<blocks_for(a->m.n, RT), RT, 0, cs.s>>>(a->m.n, a->m.ptr.p, a->m.idx.p,
                                                          a->m.val.p, dd.p);
        FG_CHECK_LAUNCH();
        dd.download(d, a->m.n, cs.s);
        FG_CUDA(cudaStreamSynchronize(cs.s));
    });
}

}  // extern "C"
