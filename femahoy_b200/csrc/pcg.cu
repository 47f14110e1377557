// multigrid::pcg (multigrid.rs:692-753) with the caller's preconditioner: the public PCG of the
// reference, for callers that precondition with something of their own (a host function, or a
// device function on the library's stream). The vectors stay on the device; each iteration is
// the product A p (csr_mul, each row summed in column order as Csr::mul), the dot products (fixed
// blocks summed in a fixed order: reproducible, not the reference's sequential order), the
// updates, and the preconditioner. The scalars alpha and beta are formed on the host from the
// dot products, in the reference's order of operations, and the stopping test is the
// reference's: |r| / |b| <= tol before each step, the iteration limit, then the cancel flag.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "assemble.cuh"
#include "common.cuh"
#include "femgpu.h"
#include "rust_format.hpp"
#include "solver.cuh"

namespace femgpu {
namespace {

constexpr int PT = 256;
constexpr int PBLOCKS = 4 * NUM_SMS;  // the dot products' partial sums

// partial[blockIdx.x] = sum over the block's grid-stride rows of u v (a fixed tree).
__global__ void __launch_bounds__(PT)
    k_dot_partial(int64_t n, const double* __restrict__ u, const double* __restrict__ v,
                  double* __restrict__ partial) {
    __shared__ double sh[PT];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)PT + threadIdx.x; i < n; i += (int64_t)gridDim.x * PT)
        s += u[i] * v[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = PT / 2; w > 0; w /= 2) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// out[k] = the sum of partial[k * PBLOCKS .. (k + 1) * PBLOCKS) in a fixed tree, for k < count.
__global__ void __launch_bounds__(PT) k_dot_finish(const double* __restrict__ partial,
                                                   double* __restrict__ out) {
    __shared__ double sh[PT];
    const double* p = partial + (int64_t)blockIdx.x * PBLOCKS;
    double s = 0.0;
    for (int i = threadIdx.x; i < PBLOCKS; i += PT) s += p[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = PT / 2; w > 0; w /= 2) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

__global__ void k_sub_from(int64_t n, const double* __restrict__ b, double* __restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        r[i] = b[i] - r[i];
}

// x += alpha p, r -= alpha q (multigrid.rs:742-745).
__global__ void k_update(int64_t n, double alpha, const double* __restrict__ p,
                         const double* __restrict__ q, double* __restrict__ x,
                         double* __restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
    }
}

// p = z + beta p (multigrid.rs:750-752).
__global__ void k_direction(int64_t n, double beta, const double* __restrict__ z,
                            double* __restrict__ p) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// The preconditioner the caller gave: a host function (r and z through host buffers), a device
// function (device pointers and the stream), or none (z = r).
struct Preconditioner {
    femgpu_precondition_fn host = nullptr;
    femgpu_precondition_device_fn device = nullptr;
    void* ctx = nullptr;
    std::vector<double> hr, hz;
    void apply(const double* r, double* z, int64_t n, cudaStream_t s) {
        if (device) {
            // r is complete when the preconditioner starts, so that it may work on a stream of
            // its own (a solver's V-cycle) as well as on `s`.
            FG_CUDA(cudaStreamSynchronize(s));
            device(r, z, (size_t)n, (void*)s, ctx);
            FG_CHECK_LAUNCH();
        } else if (host) {
            hr.resize(n);
            hz.assign(n, 0.0);
            FG_CUDA(cudaMemcpyAsync(hr.data(), r, n * sizeof(double), cudaMemcpyDeviceToHost, s));
            FG_CUDA(cudaStreamSynchronize(s));
            host(hr.data(), hz.data(), (size_t)n, ctx);
            FG_CUDA(cudaMemcpyAsync(z, hz.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
        } else {
            FG_CUDA(cudaMemcpyAsync(z, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        }
    }
};

// The dot products u_k . v_k (k < count) into host values, 1 synchronization.
void dots(int64_t n, const double* const* u, const double* const* v, int count, double* out,
          DevBuf<double>& partial, DevBuf<double>& sums, cudaStream_t s) {
    for (int k = 0; k < count; ++k)
        k_dot_partial<<<PBLOCKS, PT, 0, s>>>(n, u[k], v[k], partial.p + (int64_t)k * PBLOCKS);
    k_dot_finish<<<count, PT, 0, s>>>(partial.p, sums.p);
    FG_CHECK_LAUNCH();
    FG_CUDA(cudaMemcpyAsync(out, sums.p, count * sizeof(double), cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
}

// multigrid.rs:692-753 on device vectors b and x (x: the start value, then the solution).
void pcg_device(const DevCsr& a, const double* b, double* x, Preconditioner& pre, double tol,
                size_t max_iter, const volatile int* cancel, femgpu_convergence* out,
                cudaStream_t s) {
    const int64_t n = a.n;
    DevBuf<double> partial(3 * PBLOCKS), sums(3);
    DevBuf<double> r(n), z(n), p(n), q(n);
    const unsigned g = (unsigned)blocks_for(n, PT);
    double h[3];
    {
        const double* u[1] = {b};
        dots(n, u, u, 1, h, partial, sums, s);
    }
    const double norm_b = std::sqrt(h[0]);
    if (norm_b == 0.0) {
        FG_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
        FG_CUDA(cudaStreamSynchronize(s));
        out->iterations = 0;
        out->residual = 0.0;
        return;
    }
    csr_mul(a, x, r.p, s);
    k_sub_from<<<g, PT, 0, s>>>(n, b, r.p);
    pre.apply(r.p, z.p, n, s);
    FG_CUDA(cudaMemcpyAsync(p.p, z.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    {
        const double* u[2] = {r.p, r.p};
        const double* v[2] = {z.p, r.p};
        dots(n, u, v, 2, h, partial, sums, s);
    }
    double rz = h[0], rr = h[1];
    for (size_t it = 0; it <= max_iter; ++it) {
        const double residual = std::sqrt(rr) / norm_b;
        if (residual <= tol) {
            out->iterations = it;
            out->residual = residual;
            return;
        }
        if (it == max_iter) {
            char buf[200];
            std::snprintf(buf, sizeof buf,
                          "conjugate gradients did not converge: the residual is %s after %zu "
                          "iterations",
                          rust_exp(residual, 2).c_str(), max_iter);
            throw Failure(FEMGPU_ERR_NOT_CONVERGED, buf);
        }
        if (cancel && *cancel) throw Failure(FEMGPU_ERR_CANCELLED, "cancelled");
        csr_mul(a, p.p, q.p, s);
        {
            const double* u[1] = {p.p};
            const double* v[1] = {q.p};
            dots(n, u, v, 1, h, partial, sums, s);
        }
        const double alpha = rz / h[0];
        k_update<<<g, PT, 0, s>>>(n, alpha, p.p, q.p, x, r.p);
        pre.apply(r.p, z.p, n, s);
        {
            const double* u[2] = {r.p, r.p};
            const double* v[2] = {z.p, r.p};
            dots(n, u, v, 2, h, partial, sums, s);
        }
        const double rz_new = h[0];
        rr = h[1];
        const double beta = rz_new / rz;
        rz = rz_new;
        k_direction<<<g, PT, 0, s>>>(n, beta, z.p, p.p);
        FG_CHECK_LAUNCH();
    }
    throw Failure(FEMGPU_ERR_INVALID, "the loop returns");
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

}  // namespace
}  // namespace femgpu

using namespace femgpu;

extern "C" {

int femgpu_pcg(const femgpu_csr* a, const double* b, double* x, femgpu_precondition_fn precondition,
               void* ctx, double tol, size_t max_iter, const volatile int* cancel,
               femgpu_convergence* out) {
    return guard([&] {
        if (!a || !b || !x || !out) throw Failure(FEMGPU_ERR_INVALID, "a null argument");
        cudaStream_t s = nullptr;
        FG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            const int64_t n = a->m.n;
            DevBuf<double> db, dx;
            db.upload(b, n, s);
            dx.upload(x, n, s);
            Preconditioner pre;
            pre.host = precondition;
            pre.ctx = ctx;
            femgpu_convergence c{};
            std::exception_ptr failed;
            try {
                pcg_device(a->m, db.p, dx.p, pre, tol, max_iter, cancel, &c, s);
            } catch (...) {
                failed = std::current_exception();
            }
            // x holds the last iterate also when the solve failed, as the reference's.
            dx.download(x, n, s);
            FG_CUDA(cudaStreamSynchronize(s));
            if (failed) std::rethrow_exception(failed);
            *out = c;
        } catch (...) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
    });
}

int femgpu_pcg_device(const femgpu_csr* a, const double* b, double* x,
                      femgpu_precondition_device_fn precondition, void* ctx, double tol,
                      size_t max_iter, const volatile int* cancel, void* stream,
                      femgpu_convergence* out) {
    return guard([&] {
        if (!a || !b || !x || !out) throw Failure(FEMGPU_ERR_INVALID, "a null argument");
        Preconditioner pre;
        pre.device = precondition;
        pre.ctx = ctx;
        pcg_device(a->m, b, x, pre, tol, max_iter, cancel, out, (cudaStream_t)stream);
    });
}

}  // extern "C"
