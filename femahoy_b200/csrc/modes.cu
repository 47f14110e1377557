// The modes of an elastic model on the device: the lowest eigenpairs of K x = lambda M x by
// shift-invert subspace iteration with Rayleigh-Ritz (eigen.rs:81-177), as modes.rs:180-216
// calls it. K - shift M is formed once on the device and handed to this library's solver (the
// dense factor or PCG with multigrid), which stays resident for all the solves. The p subspace
// vectors, their images under M and under (K - shift M)^-1 M, and the projections all stay on
// the device; only the p x p projected matrices come back for the convergence test, and go down
// again to the dense Rayleigh-Ritz step on the device (dense_eigen.cu), whose rotation stays there.
//
// Built with -fmad=false: K - shift M and the rotation X = Q^T X_bar keep the reference's
// separate roundings. The projections are sums over n in a fixed order that is not the
// reference's sequential one, so they agree to rounding.
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "assemble.cuh"
#include "common.cuh"
#include "solver.cuh"

namespace femgpu {
void dense_generalized_device(const double* k, const double* m, int n, double* values,
                              double* q, cudaStream_t s);
}

namespace femgpu {

constexpr int MT = 256;
constexpr double EIGEN_TOL = 1e-6;    // eigen.rs:34
constexpr int EIGEN_MAX_ITER = 120;   // eigen.rs:40
constexpr double MODES_SHIFT = 1e-8;  // modes.rs:93
constexpr int GRAM_ROWS = 32;         // rows of a gram tile in shared memory
constexpr int GRAM_MAXP = 128;        // the most subspace vectors (count <= 64)

// a = K - shift M on the common pattern (modes.rs:192-195: v -= shift * w).
__global__ void k_shifted(int64_t nnz, const double* __restrict__ k, const double* __restrict__ m,
                          double shift, double* __restrict__ a) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x)
        a[e] = k[e] - shift * m[e];
}

// 1 when the two matrices' patterns differ.
__global__ void k_same_pattern(int64_t n, int64_t nnz, const int64_t* __restrict__ pa,
                               const uint32_t* __restrict__ ia, const int64_t* __restrict__ pb,
                               const uint32_t* __restrict__ ib, int* __restrict__ differ) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n;
         i += (int64_t)gridDim.x * blockDim.x)
        if (pa[i] != pb[i]) atomicExch(differ, 1);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x)
        if (ia[e] != ib[e]) atomicExch(differ, 1);
}

// x = b / mu (the start value of a solve after the first iteration, eigen.rs:122-125), or 0.
__global__ void k_start(int64_t n, const double* __restrict__ x, double mu,
                        double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = mu == 0.0 ? 0.0 : x[i] / mu;
}

// G[i][j] = sum_r A[i][r] B[j][r] for the p vectors of A and of B (each row-major p x n), per
// block over its tiles of GRAM_ROWS rows: the tile's columns of A and B in shared memory, each
// thread a set of (i, j) pairs. partial[block][p * p]; k_gram_total sums the blocks in order.
__global__ void __launch_bounds__(MT)
    k_gram(int p, int64_t n, const double* __restrict__ A, const double* __restrict__ B,
           double* __restrict__ partial) {
    extern __shared__ double sh[];  // A tile [p][GRAM_ROWS], B tile [p][GRAM_ROWS]
    double* sa = sh;
    double* sb = sh + (size_t)p * GRAM_ROWS;
    const int pairs = p * p;
    double acc[GRAM_MAXP * GRAM_MAXP / MT];
    const int mine = (pairs + MT - 1) / MT;
    for (int k = 0; k < mine; ++k) acc[k] = 0.0;
    const int64_t tiles = (n + GRAM_ROWS - 1) / GRAM_ROWS;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int64_t r0 = t * GRAM_ROWS;
        for (int e = threadIdx.x; e < p * GRAM_ROWS; e += MT) {
            const int v = e / GRAM_ROWS, c = e % GRAM_ROWS;
            const int64_t r = r0 + c;
            sa[e] = r < n ? A[(int64_t)v * n + r] : 0.0;
            sb[e] = r < n ? B[(int64_t)v * n + r] : 0.0;
        }
        __syncthreads();
        for (int k = 0; k < mine; ++k) {
            const int q = threadIdx.x + k * MT;
            if (q < pairs) {
                const double* ra = sa + (q / p) * GRAM_ROWS;
                const double* rb = sb + (q % p) * GRAM_ROWS;
                double s = acc[k];
                for (int c = 0; c < GRAM_ROWS; ++c) s += ra[c] * rb[c];
                acc[k] = s;
            }
        }
        __syncthreads();
    }
    for (int k = 0; k < mine; ++k) {
        const int q = threadIdx.x + k * MT;
        if (q < pairs) partial[(int64_t)blockIdx.x * pairs + q] = acc[k];
    }
}

__global__ void k_gram_total(int pairs, int nblocks, const double* __restrict__ partial,
                             double* __restrict__ out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= pairs) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[(int64_t)b * pairs + q];
    out[q] = s;
}

// X[j][r] = sum_i Q[i][j] Xbar[i][r] in increasing i (eigen.rs:160-167).
__global__ void k_rotate(int p, int64_t n, const double* __restrict__ q,
                         const double* __restrict__ bar, double* __restrict__ x) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)p * n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / n);
        const int64_t r = e % n;
        double v = 0.0;
        for (int i = 0; i < p; ++i) v += q[i * p + j] * bar[(int64_t)i * n + r];
        x[e] = v;
    }
}

}  // namespace femgpu

using namespace femgpu;

namespace {
template <class F>
int modes_guarded(F f) {
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

void need(bool ok, const char* what) {
    if (!ok) throw Failure(FEMGPU_ERR_INVALID, what);
}

std::vector<double> diagonal(const DevCsr& a, cudaStream_t s) {
    std::vector<int64_t> ptr(a.n + 1);
    std::vector<uint32_t> idx(a.nnz);
    std::vector<double> val(a.nnz);
    a.ptr.download(ptr.data(), a.n + 1, s);
    a.idx.download(idx.data(), a.nnz, s);
    a.val.download(val.data(), a.nnz, s);
    FG_CUDA(cudaStreamSynchronize(s));
    std::vector<double> d(a.n, 0.0);
    for (int64_t i = 0; i < a.n; ++i)
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e)
            if (idx[e] == (uint32_t)i) d[i] = val[e];
    return d;
}
}  // namespace

extern "C" {

int femgpu_dense_generalized(const double* k, const double* m, size_t n, double* values,
                             double* q) {
    return modes_guarded([&] {
        need(k && m && values && q && n > 0 && n <= 1024, "invalid dense eigenproblem");
        cudaStream_t s = nullptr;
        FG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            DevBuf<double> dk, dm, dv(n), dq(n * n);
            dk.upload(k, n * n, s);
            dm.upload(m, n * n, s);
            dense_generalized_device(dk.p, dm.p, (int)n, dv.p, dq.p, s);
            dv.download(values, n, s);
            dq.download(q, n * n, s);
            FG_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
    });
}

static int modes_impl(const femgpu_csr* k, const femgpu_csr* m, size_t count, double shift,
                      const femgpu_unknowns* unknowns, int method,
                      const femgpu_crossover* crossover, const femgpu_options* options,
                      const femgpu_cells* cells, const volatile int* cancel, double* values,
                      double* vectors, femgpu_modes_stats* stats);

int femgpu_modes(const femgpu_csr* k, const femgpu_csr* m, size_t count, double shift,
                 const femgpu_unknowns* unknowns, int method, const femgpu_crossover* crossover,
                 const femgpu_options* options, const volatile int* cancel, double* values,
                 double* vectors, femgpu_modes_stats* stats) {
    return modes_impl(k, m, count, shift, unknowns, method, crossover, options, nullptr, cancel,
                      values, vectors, stats);
}

int femgpu_modes_cells(const femgpu_csr* k, const femgpu_csr* m, size_t count, double shift,
                       const femgpu_unknowns* unknowns, int method,
                       const femgpu_crossover* crossover, const femgpu_options* options,
                       const femgpu_cells* cells, const volatile int* cancel, double* values,
                       double* vectors, femgpu_modes_stats* stats) {
    return modes_impl(k, m, count, shift, unknowns, method, crossover, options, cells, cancel,
                      values, vectors, stats);
}

static int modes_impl(const femgpu_csr* k, const femgpu_csr* m, size_t count, double shift,
                      const femgpu_unknowns* unknowns, int method,
                      const femgpu_crossover* crossover, const femgpu_options* options,
                      const femgpu_cells* cells, const volatile int* cancel, double* values,
                      double* vectors, femgpu_modes_stats* stats) {
    return modes_guarded([&] {
        need(k && m && unknowns && values, "null argument");
        const int64_t n = k->m.n;
        need(m->m.n == n && m->m.nnz == k->m.nnz, "K and M must have the same pattern");
        if (count == 0 || (int64_t)count > n)
            throw Failure(FEMGPU_ERR_INVALID,
                          "the model has " + std::to_string(n) + " unknowns, so it has 1 to " +
                              std::to_string(n) + " modes, not " + std::to_string(count));
        // eigen.rs:48-50
        const int p = (int)std::min<int64_t>(std::max<int64_t>(2 * count, count + 8), n);
        if (p > GRAM_MAXP)
            throw Failure(FEMGPU_ERR_TOO_LARGE, "at most 64 modes (128 subspace vectors)");
        const double bytes = 4.0 * p * (double)n * 8.0;
        if (3.0 * p * (double)n * 8.0 > 2e9)  // eigen.rs:54-64, MAX_BYTES
            throw Failure(FEMGPU_ERR_TOO_LARGE,
                          std::to_string(count) + " modes of " + std::to_string(n) +
                              " unknowns need more than 2 GB for the subspace vectors");
        (void)bytes;
        cudaStream_t s = nullptr;
        const int64_t nnz = k->m.nnz;
        {
            DevBuf<int> differ(1);
            differ.zero(s);
            k_same_pattern<<<blocks_for(nnz, MT), MT, 0, s>>>(n, nnz, k->m.ptr.p, k->m.idx.p,
                                                               m->m.ptr.p, m->m.idx.p, differ.p);
            FG_CHECK_LAUNCH();
            need(fetch(differ.p, s) == 0, "K and M must have the same pattern");
        }
        // modes.rs:186-191: shift = -SHIFT times the mean of K_ii / M_ii (NaN: that default).
        std::vector<double> md = diagonal(m->m, s);
        if (std::isnan(shift)) {
            std::vector<double> kd = diagonal(k->m, s);
            double sum = -0.0;
            for (int64_t i = 0; i < n; ++i) sum += kd[i] / md[i];
            shift = -MODES_SHIFT * (sum / (double)n);
        }
        femgpu_csr a;
        a.m.n = n;
        a.m.nnz = nnz;
        a.m.ptr.alloc(n + 1);
        a.m.idx.alloc(nnz);
        a.m.val.alloc(nnz);
        FG_CUDA(cudaMemcpyAsync(a.m.ptr.p, k->m.ptr.p, (n + 1) * 8, cudaMemcpyDeviceToDevice, s));
        FG_CUDA(cudaMemcpyAsync(a.m.idx.p, k->m.idx.p, nnz * 4, cudaMemcpyDeviceToDevice, s));
        k_shifted<<<blocks_for(nnz, MT), MT, 0, s>>>(nnz, k->m.val.p, m->m.val.p, shift,
                                                     a.m.val.p);
        FG_CHECK_LAUNCH();
        FG_CUDA(cudaStreamSynchronize(s));
        femgpu_crossover c{0, 16384, 0.0, 0, 0};
        if (crossover) c = *crossover;
        femgpu_solver* solver = nullptr;
        // modes.rs:394-404: each cell's matrix of K - shift M (v -= shift * w), for the coarse
        // matrices from the cells.
        std::vector<double> shifted;
        femgpu_cells sc{};
        if (cells && cells->count) {
            need(cells->matrices && cells->mass && cells->nclass > 0,
                 "the cells of a modes solve need their stiffness and mass matrices");
            shifted.resize(576 * cells->nclass);
            for (size_t i = 0; i < shifted.size(); ++i)
                shifted[i] = cells->matrices[i] - shift * cells->mass[i];
            sc = *cells;
            sc.matrices = shifted.data();
        }
        int rc = femgpu_solver_new_cells(&a, unknowns, method, &c, options,
                                         sc.count ? &sc : nullptr, &solver);
        if (rc != FEMGPU_OK) {
            char buf[1024];
            femgpu_last_error(buf, sizeof buf);
            throw Failure(rc, buf);
        }
        std::unique_ptr<femgpu_solver, void (*)(femgpu_solver*)> own(solver, femgpu_solver_free);
        SolverImpl& sv = solver->impl;
        s = sv.stream();
        // eigen.rs:96-113: the start vectors, the diagonal of M then xorshift values.
        std::vector<double> x0((size_t)p * n);
        std::copy(md.begin(), md.end(), x0.begin());
        uint64_t seed = 0x9e3779b97f4a7c15ull;
        for (size_t e = (size_t)n; e < x0.size(); ++e) {
            seed ^= seed << 13;
            seed ^= seed >> 7;
            seed ^= seed << 17;
            x0[e] = (double)(seed >> 11) / (double)(1ull << 53) - 0.5;
        }
        DevBuf<double> X, Y, B, MB, q, partial, gram;
        X.upload(x0.data(), x0.size(), s);
        Y.alloc((size_t)p * n);
        B.alloc((size_t)p * n);
        MB.alloc((size_t)p * n);
        q.alloc((size_t)p * p);
        const int gb = 2 * NUM_SMS;
        partial.alloc((size_t)gb * p * p);
        gram.alloc((size_t)p * p);
        const size_t gram_smem = 2 * (size_t)p * GRAM_ROWS * sizeof(double);
        if (gram_smem > 48 * 1024)
            FG_CUDA(cudaFuncSetAttribute(k_gram, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)gram_smem));
        auto gram_of = [&](const double* A, const double* Bv, std::vector<double>* out) {
            k_gram<<<gb, MT, gram_smem, s>>>(p, n, A, Bv, partial.p);
            k_gram_total<<<(p * p + MT - 1) / MT, MT, 0, s>>>(p * p, gb, partial.p, gram.p);
            FG_CHECK_LAUNCH();
            out->resize((size_t)p * p);
            gram.download(out->data(), (size_t)p * p, s);
            FG_CUDA(cudaStreamSynchronize(s));
        };
        std::vector<double> mu, kr((size_t)p * p), mr((size_t)p * p), g1, g2, vals(p);
        DevBuf<double> dkr((size_t)p * p), dmr((size_t)p * p), dvals(p);
        femgpu_modes_stats st{};
        st.shift = shift;
        for (int iteration = 1; iteration <= EIGEN_MAX_ITER; ++iteration) {
            if (cancel && *cancel) throw Failure(FEMGPU_ERR_CANCELLED, "cancelled");
            for (int j = 0; j < p; ++j) {
                double* yj = Y.p + (size_t)j * n;
                double* bj = B.p + (size_t)j * n;
                csr_mul(m->m, X.p + (size_t)j * n, yj, s);
                k_start<<<blocks_for(n, MT), MT, 0, s>>>(n, X.p + (size_t)j * n,
                                                         mu.empty() ? 0.0 : mu[j], bj);
                FG_CHECK_LAUNCH();
                femgpu_stats ss{};
                sv.solve(yj, bj, cancel, &ss);
                st.solves += 1;
                st.pcg_iterations += ss.iterations;
                st.seconds += ss.seconds;
                csr_mul(m->m, bj, MB.p + (size_t)j * n, s);
            }
            // K_r = 0.5 (X_bar^T Y + its transpose), M_r = X_bar^T M X_bar (upper triangle).
            gram_of(B.p, Y.p, &g1);
            gram_of(B.p, MB.p, &g2);
            for (int i = 0; i < p; ++i)
                for (int j = i; j < p; ++j) {
                    const double kv = 0.5 * (g1[(size_t)i * p + j] + g1[(size_t)j * p + i]);
                    kr[(size_t)i * p + j] = kr[(size_t)j * p + i] = kv;
                    const double mv = g2[(size_t)i * p + j];
                    mr[(size_t)i * p + j] = mr[(size_t)j * p + i] = mv;
                }
            bool converged = iteration > 1;
            for (size_t i = 0; converged && i < count; ++i) {
                const double ka = kr[i * p + i], mb = mr[i * p + i];
                converged = std::sqrt(std::max(1.0 - ka * ka / mb, 0.0)) <= EIGEN_TOL;
            }
            // The Rayleigh-Ritz problem on the device (dense_eigen.cu); its vectors stay there.
            dkr.upload(kr.data(), (size_t)p * p, s);
            dmr.upload(mr.data(), (size_t)p * p, s);
            dense_generalized_device(dkr.p, dmr.p, p, dvals.p, q.p, s);
            dvals.download(vals.data(), p, s);
            FG_CUDA(cudaStreamSynchronize(s));
            mu = vals;
            k_rotate<<<blocks_for((int64_t)p * n, MT), MT, 0, s>>>(p, n, q.p, B.p, X.p);
            FG_CHECK_LAUNCH();
            st.iterations = (size_t)iteration;
            if (converged) {
                for (size_t j = 0; j < count; ++j) values[j] = mu[j] + shift;
                if (vectors) X.download(vectors, count * (size_t)n, s);
                FG_CUDA(cudaStreamSynchronize(s));
                if (stats) *stats = st;
                return;
            }
        }
        if (stats) *stats = st;
        throw Failure(FEMGPU_ERR_NOT_CONVERGED,
                      "the subspace iteration did not converge in 120 iterations: ask for fewer "
                      "modes");
    });
}

}  // extern "C"
