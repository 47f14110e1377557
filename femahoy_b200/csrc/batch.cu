// Batched solves: many small systems of uneven sizes, each with several right sides, in 1 set
// of launches (no counterpart in the reference, whose callers solve 1 model at a time).
//
// The systems are combined level by level into block-diagonal operators: each system keeps the
// reference's own hierarchy (plane coarsening and Galerkin products, multigrid.rs:84-139, down
// to `coarsest` unknowns), the shallower hierarchies are padded with identity transfers to a
// common depth, and the deepest level is solved by a dense inverse per system. So 1 launch of
// each V-cycle kernel covers every system. The right sides are interleaved, R per row
// (x[row * R + col]): the R threads of a row share each matrix entry, so 1 read of the
// operator serves all R solves. Every (system, right side) pair, a segment, is its own
// conjugate gradient solve with its own scalars and stopping test (multigrid.rs:692-753; the
// flexible form with the FP32 cycle); the sums of each segment are reduced over chunks of rows
// that never cross a system, in a fixed order, so a result does not depend on the timing. The
// iteration is 1 CUDA graph body under a WHILE node that runs until every segment has stopped.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>

#include "common.cuh"
#include "hierarchy.hpp"
#include "solver.cuh"

namespace femgpu {

constexpr int BTH = 256;

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
    const int64_t t = elem_of_thread();
    if (t >= n * R) return;
    T v = c1 * dinv[t / R] * b[t];
    d[t] = v;
    x[t] = v;
}

// d = c2 d + c1 D^-1 (b - A x), x_out = x + d.
template <class T, int R>
__global__ void __launch_bounds__(BTH)
    k_bcheb_step(SellView<T> A, const T* __restrict__ b, const T* __restrict__ xin,
                 const T* __restrict__ dinv, T c1, T c2, T* __restrict__ d, T* __restrict__ xout) {
    const int64_t t = elem_of_thread();
    if (t >= A.n * R) return;
    const int row = (int)(t / R), col = (int)(t % R);
    T r = b[t] - sell_row_cols<T, R>(A, row, col, xin);
    T dd = c2 * d[t] + c1 * dinv[row] * r;
    d[t] = dd;
    xout[t] = xin[t] + dd;
}

template <class T, int R>
__global__ void __launch_bounds__(BTH)
    k_bresidual(SellView<T> A, const T* __restrict__ b, const T* __restrict__ x, T* __restrict__ r) {
    const int64_t t = elem_of_thread();
    if (t >= A.n * R) return;
    r[t] = b[t] - sell_row_cols<T, R>(A, (int)(t / R), (int)(t % R), x);
}

// out = M in (accumulate: out += M in) for a CSR transfer M, R columns.
template <class T, int R>
__global__ void k_bgather(int64_t rows, const int64_t* __restrict__ ptr,
                          const uint32_t* __restrict__ idx, const T* __restrict__ val,
                          const T* __restrict__ in, T* __restrict__ out, int accumulate) {
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

// The deepest level: out = inv_b in for the rows of system b (1 block per system).
template <class T, int R>
__global__ void k_bdense(const int64_t* __restrict__ off, const int64_t* __restrict__ ioff,
                         const T* __restrict__ inv, const T* __restrict__ in, T* __restrict__ out) {
    const int b = blockIdx.x;
    const int64_t r0 = off[b], m = off[b + 1] - r0;
    const T* M = inv + ioff[b];
    for (int64_t t = threadIdx.x; t < m * R; t += blockDim.x) {
        const int64_t i = t / R;
        const int col = (int)(t % R);
        T s = 0;
        for (int64_t j = 0; j < m; ++j) s += M[i * m + j] * in[(r0 + j) * R + col];
        out[(r0 + i) * R + col] = s;
    }
}

// ------------------------------------------------------------------ PCG over segments
// A block of the PCG kernels takes 1 chunk: rows [row0, row1) of system `sys`. Thread t takes
// column t % R and rows row0 + t / R, row0 + t / R + BTH / R, ...
struct Chunk {
    int sys;
    int row0, row1;
};

// The per-segment scalars (arrays of B R; segment s = system s / R, right side s % R).
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
                double* __restrict__ partial) {
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    double pq = 0;
    if (!done[ch.sys * R + col])
        for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R) {
            const int64_t t = (int64_t)row * R + col;
            double ap = sell_row_cols<double, R>(A, row, col, p);
            q[t] = ap;
            pq += p[t] * ap;
        }
    chunk_partial<R>(pq, 0.0, partial);
}

// x += alpha p, r -= alpha q (multigrid.rs:742-745) with the sums r.r.
template <int R>
__global__ void __launch_bounds__(BTH)
    k_bpcg_update(const Chunk* __restrict__ chunks, double* __restrict__ x,
                  double* __restrict__ r, const double* __restrict__ p,
                  const double* __restrict__ q, float* __restrict__ r32, BatchScalars sc,
                  double* __restrict__ partial) {
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    const int seg = ch.sys * R + col;
    double rr = 0;
    if (!sc.done[seg]) {
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
    const Chunk ch = chunks[blockIdx.x];
    const int col = threadIdx.x % R;
    if (bb[ch.sys * R + col] != 0.0) return;
    for (int row = ch.row0 + threadIdx.x / R; row < ch.row1; row += BTH / R)
        x[(int64_t)row * R + col] = 0.0;
}

enum FinishKind { FIN_START = 0, FIN_PQ = 1, FIN_UPDATE = 2, FIN_DOTS = 3, FIN_TRUTH = 4,
                  FIN_RESTART = 5 };

// The sums of each segment over the chunks of its system (in chunk order), then its scalars.
// FIN_START: the first residual (stop at once if |r| <= tol |b| or b = 0, multigrid.rs:
// 704-723); FIN_PQ: alpha; FIN_UPDATE: the stopping test and the iteration limit (multigrid.rs:
// 721-733); FIN_DOTS: beta; FIN_TRUTH: the true residual |b - A x| / |b|; FIN_RESTART: the
// segments whose true residual drifted above tol run again from x (iterative refinement).
template <int R>
__global__ void k_bfinish(int kind, int nseg, const int* __restrict__ cstart,
                          const double* __restrict__ partial, BatchScalars sc, double tol,
                          int max_iter, int flexible, int init) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int sys = s / R, col = s % R;
    double a = 0, b = 0;
    for (int c = cstart[sys]; c < cstart[sys + 1]; ++c) {
        a += partial[((int64_t)c * R + col) * 2];
        b += partial[((int64_t)c * R + col) * 2 + 1];
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

// ------------------------------------------------------------------ the batch
struct SystemHierarchy {
    std::vector<HostCsr> mats;
    std::vector<HostRect> ps;
};

template <class T>
struct BatchLevel {
    int64_t n = 0, nc = 0;
    Sell<T> A;
    DevBuf<T> dinv;
    DevBuf<int64_t> pptr, rptr;
    DevBuf<uint32_t> pidx, ridx;
    DevBuf<T> pval, rval;
    DevBuf<T> b, xa, xb, d, r;
    std::vector<double> c1, c2;
    double lambda = 0;
};

template <class T>
struct BatchCoarse {
    int64_t n = 0;
    DevBuf<int64_t> off, ioff;
    DevBuf<T> inv, b, x;
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
    void segments(size_t* iterations, double* truth, double* residual, int* status) const;
    const std::vector<int64_t>& offsets() const { return offsets_; }
    std::vector<int64_t> level_sizes() const { return sizes_; }
    size_t bytes() const;
    cudaStream_t stream() const { return s_; }
    double tol = 1e-10;  // PCG_TOL, solve.rs:42

   private:
    template <class T>
    void build_levels(std::vector<SystemHierarchy>& H, size_t depth,
                      std::vector<BatchLevel<T>>* levels, BatchCoarse<T>* coarse);
    template <class T, int R>
    const T* vcycle(std::vector<BatchLevel<T>>& Ls, BatchCoarse<T>& Cc, size_t l, const T* b);
    template <int R>
    void finish(int kind, int init);
    template <int R>
    void precondition_and_dots(int init);
    template <int R>
    void iteration();
    template <int R>
    void run(const volatile int* cancel);
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
    std::vector<int64_t> offsets_, sizes_;
    Sell<double> A64_;  // the block-diagonal finest matrix, exactly
    std::vector<BatchLevel<float>> L32_;
    std::vector<BatchLevel<double>> L64_;
    BatchCoarse<float> C32_;
    BatchCoarse<double> C64_;
    DevBuf<char> chunks_;
    DevBuf<int> cstart_;
    DevBuf<double> partial_;
    DevBuf<double> bb_, rr_, rz_, pq_, alpha_, beta_, truth_;
    DevBuf<int> done_, iters_, status_, loops_;
    DevBuf<double> x_, r_, p_, q_, b_;
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

HostRect identity(int64_t n) {
    HostRect p;
    p.rows = p.cols = n;
    p.ptr.resize(n + 1);
    p.idx.resize(n);
    p.val.assign(n, 1.0);
    for (int64_t i = 0; i <= n; ++i) p.ptr[i] = i;
    for (int64_t i = 0; i < n; ++i) p.idx[i] = (uint32_t)i;
    return p;
}

// The block-diagonal matrix of the systems' matrices.
HostCsr combine(const std::vector<const HostCsr*>& parts) {
    HostCsr out;
    int64_t n = 0, nnz = 0;
    for (auto* a : parts) {
        n += a->n;
        nnz += a->nnz();
    }
    if (n >= 0x7fffffff) throw Failure(FEMGPU_ERR_TOO_LARGE, "a batch of 2^31 unknowns or more");
    out.n = n;
    out.ptr.reserve(n + 1);
    out.idx.reserve(nnz);
    out.val.reserve(nnz);
    out.ptr.push_back(0);
    int64_t off = 0;
    for (auto* a : parts) {
        for (int64_t i = 0; i < a->n; ++i) {
            for (int64_t k = a->ptr[i]; k < a->ptr[i + 1]; ++k) {
                out.idx.push_back((uint32_t)(a->idx[k] + off));
                out.val.push_back(a->val[k]);
            }
            out.ptr.push_back((int64_t)out.idx.size());
        }
        off += a->n;
    }
    return out;
}

// The block-diagonal transfer of the systems' transfers.
HostRect combine_rect(const std::vector<const HostRect*>& parts) {
    HostRect out;
    for (auto* p : parts) {
        out.rows += p->rows;
        out.cols += p->cols;
    }
    out.ptr.reserve(out.rows + 1);
    out.ptr.push_back(0);
    int64_t off = 0;
    for (auto* p : parts) {
        for (int64_t i = 0; i < p->rows; ++i) {
            for (int64_t k = p->ptr[i]; k < p->ptr[i + 1]; ++k) {
                out.idx.push_back((uint32_t)(p->idx[k] + off));
                out.val.push_back(p->val[k]);
            }
            out.ptr.push_back((int64_t)out.idx.size());
        }
        off += p->cols;
    }
    return out;
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
    if (s_) cudaStreamSynchronize(s_);
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
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
    // Each system's hierarchy on the host (multigrid.rs:84-139), the systems shared among the
    // host threads.
    std::vector<HostCsr> fine(B_);
    for (int b = 0; b < B_; ++b) {
        if (a[b]->n < 1) throw Failure(FEMGPU_ERR_INVALID, "an empty system");
        fine[b] = download_csr(*a[b], s_);
    }
    std::vector<SystemHierarchy> H(B_);
    // 1024 by default: the thin members (plates 1 cell thick) converge slowly under plane
    // coarsening, and a dense deepest level of up to 1024 unknowns per member cuts the most
    // iterations of a batch of 10x1x1 to 80x8x8-cell cantilevers from 66 to 20 at 1e-8, for
    // 4 MB of FP32 inverse per member read once per cycle for all right sides.
    const size_t coarsest = (size_t)(o.coarsest > 0 ? o.coarsest : 1024);
    const size_t max_levels = (size_t)(o.max_levels > 0 ? o.max_levels : 30);
    std::vector<std::string> errors(B_);
    std::vector<int> codes(B_, FEMGPU_OK);
    auto build = [&](int b) {
        try {
            const femgpu_unknowns& uu = *u[b];
            const int64_t n = fine[b].n;
            HostLevel lv;
            for (int d = 0; d < 3; ++d)
                lv.planes[d].assign(uu.planes[d], uu.planes[d] + uu.nplanes[d]);
            lv.points.resize(n);
            for (int64_t k = 0; k < n; ++k)
                for (int d = 0; d < 3; ++d) lv.points[k][d] = uu.points[3 * k + d];
            lv.comp.assign(uu.comp, uu.comp + n);
            H[b].mats.push_back(std::move(fine[b]));
            for (;;) {
                const HostCsr& m = H[b].mats.back();
                if ((size_t)m.n <= coarsest || H[b].ps.size() >= max_levels) break;
                HostRect p;
                HostLevel coarse;
                if (!coarsen(lv, m, &p, &coarse)) break;
                if (coarse.points.size() * 10 > (size_t)m.n * 9) break;
                HostCsr ac = galerkin(p, m, 1);
                H[b].mats.push_back(std::move(ac));
                H[b].ps.push_back(std::move(p));
                lv = std::move(coarse);
            }
            if (H[b].mats.back().n > 4096)
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
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            for (int b = t; b < B_; b += threads) build(b);
        });
    for (auto& th : pool) th.join();
    for (int b = 0; b < B_; ++b)
        if (codes[b] != FEMGPU_OK)
            throw Failure(codes[b], "system " + std::to_string(b) + ": " + errors[b]);
    // Pad to the common depth: a level past a system's own repeats its deepest matrix, with the
    // identity as the transfer.
    size_t depth = 0;
    for (auto& h : H) depth = std::max(depth, h.mats.size());
    for (auto& h : H)
        while (h.mats.size() < depth) {
            HostCsr last = h.mats.back();
            h.ps.push_back(identity(last.n));
            h.mats.push_back(std::move(last));
        }
    offsets_.assign(B_ + 1, 0);
    for (int b = 0; b < B_; ++b) offsets_[b + 1] = offsets_[b] + H[b].mats[0].n;
    n_ = offsets_[B_];
    if (n_ * R_ >= 0x7fffffff)
        throw Failure(FEMGPU_ERR_TOO_LARGE, "a batch of 2^31 values or more per vector");
    // The exact finest operator (FP64) of the PCG loop and the true residual.
    {
        std::vector<const HostCsr*> parts;
        for (auto& h : H) parts.push_back(&h.mats[0]);
        HostCsr f = combine(parts);
        DevCsr d;
        upload_csr(f, &d, s_);
        make_sell<double>(d, 32, &A64_, s_);
        FG_CUDA(cudaStreamSynchronize(s_));
    }
    sizes_.clear();
    for (size_t l = 0; l < depth; ++l) {
        int64_t s = 0;
        for (auto& h : H) s += h.mats[l].n;
        sizes_.push_back(s);
    }
    // The chunks of the PCG kernels: up to 4 rows per thread, rows of 1 system each.
    const int chunk_rows = 4 * BTH / R_;
    std::vector<Chunk> ch;
    std::vector<int> cstart(B_ + 1, 0);
    for (int b = 0; b < B_; ++b) {
        cstart[b] = (int)ch.size();
        for (int64_t r = offsets_[b]; r < offsets_[b + 1]; r += chunk_rows)
            ch.push_back({b, (int)r, (int)std::min<int64_t>(r + chunk_rows, offsets_[b + 1])});
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
        build_levels<float>(H, depth, &L32_, &C32_);
    else
        build_levels<double>(H, depth, &L64_, &C64_);
    const size_t S = (size_t)B_ * R_;
    for (auto* v : {&bb_, &rr_, &rz_, &pq_, &alpha_, &beta_, &truth_}) v->alloc(S);
    for (auto* v : {&done_, &iters_, &status_}) v->alloc(S);
    loops_.alloc(1);
    for (auto* v : {&x_, &r_, &p_, &q_, &b_}) v->alloc((size_t)n_ * R_);
    if (opt_.precision == FEMGPU_MIXED) r32_.alloc((size_t)n_ * R_);
    FG_CUDA(cudaStreamSynchronize(s_));
}

template <class T>
void BatchImpl::build_levels(std::vector<SystemHierarchy>& H, size_t depth,
                             std::vector<BatchLevel<T>>* levels, BatchCoarse<T>* coarse) {
    levels->resize(depth - 1);
    const int deg = opt_.degree > 0 ? opt_.degree : 2;
    const double lower = opt_.lower > 0 ? opt_.lower : 0.3;
    for (size_t l = 0; l + 1 < depth; ++l) {
        BatchLevel<T>& L = (*levels)[l];
        std::vector<const HostCsr*> mats;
        std::vector<const HostRect*> ps;
        for (auto& h : H) {
            mats.push_back(&h.mats[l]);
            ps.push_back(&h.ps[l]);
        }
        HostCsr A = combine(mats);
        HostRect P = combine_rect(ps);
        L.n = A.n;
        DevCsr d;
        upload_csr(A, &d, s_);
        make_sell<T>(d, 32, &L.A, s_);
        // The diagonal, and lambda_max of the block-diagonal D^-1 A: the largest of the
        // systems'.
        std::vector<double> dg(A.n, 0.0), inv(A.n);
        for (int64_t i = 0; i < A.n; ++i)
            for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                if ((int64_t)A.idx[k] == i) dg[i] = A.val[k];
        for (int64_t i = 0; i < A.n; ++i) {
            if (!(dg[i] > 0.0))
                throw Failure(FEMGPU_ERR_NOT_SPD,
                              "the matrix is not positive definite: it has a diagonal entry that "
                              "is not above 0");
            inv[i] = 1.0 / dg[i];
        }
        Operator<double> op;
        op.n = A.n;
        op.nnz = A.nnz();
        make_sell<double>(d, 32, &op.sell, s_);
        DevBuf<double> ddg;
        ddg.upload(dg.data(), A.n, s_);
        L.lambda = lambda_max(op, ddg.p, s_, partial_);
        chebyshev(L.lambda, deg, lower, &L.c1, &L.c2);
        std::vector<T> tv(inv.begin(), inv.end());
        L.dinv.upload(tv.data(), tv.size(), s_);
        HostRect Rt = transpose(P);
        L.nc = P.cols;
        L.pptr.upload(P.ptr.data(), P.rows + 1, s_);
        L.pidx.upload(P.idx.data(), P.idx.size(), s_);
        std::vector<T> pv(P.val.begin(), P.val.end()), rv(Rt.val.begin(), Rt.val.end());
        L.pval.upload(pv.data(), pv.size(), s_);
        L.rptr.upload(Rt.ptr.data(), Rt.rows + 1, s_);
        L.ridx.upload(Rt.idx.data(), Rt.idx.size(), s_);
        L.rval.upload(rv.data(), rv.size(), s_);
        for (auto* v : {&L.b, &L.xa, &L.xb, &L.d, &L.r}) v->alloc((size_t)A.n * R_);
        FG_CUDA(cudaStreamSynchronize(s_));
    }
    // The deepest level: a dense inverse per system, from a dense Cholesky factor on the device.
    std::vector<int64_t> off(B_ + 1, 0), ioff(B_ + 1, 0);
    for (int b = 0; b < B_; ++b) {
        const int64_t m = H[b].mats[depth - 1].n;
        off[b + 1] = off[b] + m;
        ioff[b + 1] = ioff[b] + m * m;
    }
    coarse->n = off[B_];
    coarse->inv.alloc(ioff[B_]);
    for (int b = 0; b < B_; ++b) {
        DevBuf<double> inv64;
        dense_inverse(H[b].mats[depth - 1], &inv64, s_);
        const int64_t mm = ioff[b + 1] - ioff[b];
        std::vector<double> h(mm);
        inv64.download(h.data(), mm, s_);
        FG_CUDA(cudaStreamSynchronize(s_));
        std::vector<T> t(h.begin(), h.end());
        FG_CUDA(cudaMemcpyAsync(coarse->inv.p + ioff[b], t.data(), mm * sizeof(T),
                                cudaMemcpyHostToDevice, s_));
        FG_CUDA(cudaStreamSynchronize(s_));
    }
    coarse->off.upload(off.data(), off.size(), s_);
    coarse->ioff.upload(ioff.data(), ioff.size(), s_);
    coarse->b.alloc((size_t)coarse->n * R_);
    coarse->x.alloc((size_t)coarse->n * R_);
    FG_CUDA(cudaStreamSynchronize(s_));
}

// ------------------------------------------------------------------ the cycle and the loop
// The V-cycle from level l on the right sides b; returns where the correction is.
template <class T, int R>
const T* BatchImpl::vcycle(std::vector<BatchLevel<T>>& Ls, BatchCoarse<T>& Cc, size_t l,
                           const T* b) {
    if (l == Ls.size()) {
        k_bdense<T, R><<<B_, BTH, 0, s_>>>(Cc.off.p, Cc.ioff.p, Cc.inv.p, b, Cc.x.p);
        FG_CHECK_LAUNCH();
        launches_ += 1;
        return Cc.x.p;
    }
    BatchLevel<T>& L = Ls[l];
    const int g = (int)((L.n * R + BTH - 1) / BTH);
    T* xa = L.xa.p;
    T* xb = L.xb.p;
    const int deg = (int)L.c1.size();
    k_bcheb_first<T, R><<<g, BTH, 0, s_>>>(L.n, b, L.dinv.p, (T)L.c1[0], L.d.p, xa);
    for (int k = 1; k < deg; ++k) {
        k_bcheb_step<T, R><<<g, BTH, 0, s_>>>(L.A.view(), b, xa, L.dinv.p, (T)L.c1[k],
                                              (T)L.c2[k], L.d.p, xb);
        std::swap(xa, xb);
    }
    k_bresidual<T, R><<<g, BTH, 0, s_>>>(L.A.view(), b, xa, L.r.p);
    T* bc = l + 1 == Ls.size() ? Cc.b.p : Ls[l + 1].b.p;
    const int gc = (int)((L.nc * R + BTH - 1) / BTH);
    k_bgather<T, R><<<gc, BTH, 0, s_>>>(L.nc, L.rptr.p, L.ridx.p, L.rval.p, L.r.p, bc, 0);
    FG_CHECK_LAUNCH();
    launches_ += deg + 2;
    const T* ec = vcycle<T, R>(Ls, Cc, l + 1, bc);
    k_bgather<T, R><<<g, BTH, 0, s_>>>(L.n, L.pptr.p, L.pidx.p, L.pval.p, ec, xa, 1);
    for (int k = 0; k < deg; ++k) {
        k_bcheb_step<T, R><<<g, BTH, 0, s_>>>(L.A.view(), b, xa, L.dinv.p, (T)L.c1[k],
                                              (T)L.c2[k], L.d.p, xb);
        std::swap(xa, xb);
    }
    FG_CHECK_LAUNCH();
    launches_ += deg + 1;
    return xa;
}

template <int R>
void BatchImpl::finish(int kind, int init) {
    const int S = B_ * R;
    k_bfinish<R><<<(S + 127) / 128, 128, 0, s_>>>(kind, S, cstart_.p, partial_.p, scalars(), tol,
                                                  max_iter_, opt_.precision == FEMGPU_MIXED, init);
    FG_CHECK_LAUNCH();
    launches_ += 1;
}

// z = M^-1 r, the sums r.z (and z.q), beta, p.
template <int R>
void BatchImpl::precondition_and_dots(int init) {
    const bool mixed = opt_.precision == FEMGPU_MIXED;
    if (mixed) {
        const float* z = vcycle<float, R>(L32_, C32_, 0, r32_.p);
        k_bpcg_dots<R, float><<<nchunks_, BTH, 0, s_>>>(chunks(), r_.p, z, q_.p, 1, init,
                                                        done_.p, partial_.p);
        finish<R>(FIN_DOTS, init);
        k_bpcg_p<R, float><<<nchunks_, BTH, 0, s_>>>(chunks(), z, p_.p, scalars(), init);
    } else {
        const double* z = vcycle<double, R>(L64_, C64_, 0, r_.p);
        k_bpcg_dots<R, double><<<nchunks_, BTH, 0, s_>>>(chunks(), r_.p, z, q_.p, 0, init,
                                                         done_.p, partial_.p);
        finish<R>(FIN_DOTS, init);
        k_bpcg_p<R, double><<<nchunks_, BTH, 0, s_>>>(chunks(), z, p_.p, scalars(), init);
    }
    FG_CHECK_LAUNCH();
    launches_ += 2;
}

// 1 PCG iteration of every running segment (multigrid.rs:739-750).
template <int R>
void BatchImpl::iteration() {
    const bool mixed = opt_.precision == FEMGPU_MIXED;
    k_bpcg_spmv<R><<<nchunks_, BTH, 0, s_>>>(A64_.view(), chunks(), p_.p, q_.p, done_.p,
                                             partial_.p);
    finish<R>(FIN_PQ, 0);
    k_bpcg_update<R><<<nchunks_, BTH, 0, s_>>>(chunks(), x_.p, r_.p, p_.p, q_.p,
                                               mixed ? r32_.p : nullptr, scalars(), partial_.p);
    finish<R>(FIN_UPDATE, 0);
    FG_CHECK_LAUNCH();
    launches_ += 2;
    precondition_and_dots<R>(0);
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

template <int R>
void BatchImpl::run(const volatile int* cancel) {
    const bool mixed = opt_.precision == FEMGPU_MIXED;
    launches_ = 0;
    restarts_ = 0;
    if (!exec_) {
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
        iteration<R>();
        k_bloop_control<<<1, BTH, 0, s_>>>(cond_, done_.p, B_ * R, d_cancel_, loops_.p);
        FG_CUDA(cudaStreamEndCapture(s_, &body));
        FG_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
        graph_kernels_ = launches_ + 1;
        graph_max_iter_ = max_iter_;
        graph_tol_ = tol;
        launches_ = 0;
    }
    FG_CUDA(cudaMemsetAsync(loops_.p, 0, sizeof(int), s_));
    // r = b - A x and the first test (multigrid.rs:692-723), x = 0 where b = 0, then
    // z = M^-1 r, p = z.
    k_bpcg_residual<R><<<nchunks_, BTH, 0, s_>>>(A64_.view(), chunks(), b_.p, x_.p, r_.p,
                                                 mixed ? r32_.p : nullptr, partial_.p);
    finish<R>(FIN_START, 0);
    k_bzero_empty<R><<<nchunks_, BTH, 0, s_>>>(chunks(), bb_.p, x_.p);
    FG_CHECK_LAUNCH();
    launches_ += 2;
    precondition_and_dots<R>(1);
    for (;;) {
        if (any_running()) launch_loop(cancel);
        if (cancel && *cancel) return;
        // The true residual of each segment in FP64. With the FP32 cycle the recurrence can
        // drift from it; the segments that drifted above tol run again from x (at most 3 times).
        k_bpcg_residual<R><<<nchunks_, BTH, 0, s_>>>(A64_.view(), chunks(), b_.p, x_.p,
                                                     mixed ? r_.p : nullptr,
                                                     mixed ? r32_.p : nullptr, partial_.p);
        finish<R>(FIN_TRUTH, 0);
        launches_ += 1;
        if (!mixed || restarts_ >= 3) break;
        finish<R>(FIN_RESTART, 0);
        if (!any_running()) break;
        ++restarts_;
        precondition_and_dots<R>(1);
    }
}

void BatchImpl::solve_device(const double* d_b, double* d_x, const volatile int* cancel,
                             femgpu_batch_stats* st) {
    if (exec_ && (max_iter_ != graph_max_iter_ || tol != graph_tol_)) {
        cudaGraphExecDestroy(exec_);
        cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
    }
    const size_t bytes = (size_t)n_ * R_ * sizeof(double);
    FG_CUDA(cudaEventRecord(ev0_, s_));
    if (d_b != b_.p) FG_CUDA(cudaMemcpyAsync(b_.p, d_b, bytes, cudaMemcpyDeviceToDevice, s_));
    if (d_x != x_.p) FG_CUDA(cudaMemcpyAsync(x_.p, d_x, bytes, cudaMemcpyDeviceToDevice, s_));
    if (R_ == 16)
        run<16>(cancel);
    else if (R_ == 4)
        run<4>(cancel);
    else
        run<1>(cancel);
    if (d_x != x_.p) FG_CUDA(cudaMemcpyAsync(d_x, x_.p, bytes, cudaMemcpyDeviceToDevice, s_));
    FG_CUDA(cudaEventRecord(ev1_, s_));
    FG_CUDA(cudaStreamSynchronize(s_));
    if (cancel && *cancel) throw Failure(FEMGPU_ERR_CANCELLED, "cancelled");
    collect(st);
}

void BatchImpl::solve_host(const double* h_b, double* h_x, const volatile int* cancel,
                           femgpu_batch_stats* st) {
    const size_t bytes = (size_t)n_ * R_ * sizeof(double);
    FG_CUDA(cudaMemcpyAsync(b_.p, h_b, bytes, cudaMemcpyHostToDevice, s_));
    FG_CUDA(cudaMemcpyAsync(x_.p, h_x, bytes, cudaMemcpyHostToDevice, s_));
    try {
        solve_device(b_.p, x_.p, cancel, st);
    } catch (const Failure&) {
        cudaMemcpyAsync(h_x, x_.p, bytes, cudaMemcpyDeviceToHost, s_);
        cudaStreamSynchronize(s_);
        throw;
    }
    FG_CUDA(cudaMemcpyAsync(h_x, x_.p, bytes, cudaMemcpyDeviceToHost, s_));
    FG_CUDA(cudaStreamSynchronize(s_));
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
    for (int s = 0; s < S; ++s) {
        if (iterations) iterations[s] = (size_t)it[s];
        if (truth) truth[s] = tr[s];
        if (residual) residual[s] = bb[s] > 0 ? std::sqrt(rr[s]) / std::sqrt(bb[s]) : 0.0;
        if (status) status[s] = stt[s];
    }
}

void BatchImpl::collect(femgpu_batch_stats* st) {
    const int S = B_ * R_;
    std::vector<size_t> it(S);
    std::vector<double> tr(S), res(S);
    std::vector<int> stt(S);
    segments(it.data(), tr.data(), res.data(), stt.data());
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
                          "residual is %.2e after %zu iterations",
                          s / R_, s % R_, res[s], it[s]);
        throw Failure(FEMGPU_ERR_NOT_CONVERGED, buf);
    }
}

size_t BatchImpl::bytes() const {
    size_t b = A64_.bytes() + partial_.bytes() + chunks_.bytes() + cstart_.bytes();
    auto levels = [&](const auto& Ls, const auto& C) {
        for (const auto& L : Ls)
            b += L.A.bytes() + L.dinv.bytes() + L.pptr.bytes() + L.rptr.bytes() + L.pidx.bytes() +
                 L.ridx.bytes() + L.pval.bytes() + L.rval.bytes() + L.b.bytes() + L.xa.bytes() +
                 L.xb.bytes() + L.d.bytes() + L.r.bytes();
        b += C.off.bytes() + C.ioff.bytes() + C.inv.bytes() + C.b.bytes() + C.x.bytes();
    };
    levels(L32_, C32_);
    levels(L64_, C64_);
    b += x_.bytes() + r_.bytes() + p_.bytes() + q_.bytes() + b_.bytes() + r32_.bytes();
    return b;
}

}  // namespace femgpu

// ------------------------------------------------------------------ C ABI
struct femgpu_batch {
    femgpu::BatchImpl impl;
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
        o.format = 1;
        o.coarsest = 0;
        if (options) {
            o.precision = options->precision;
            o.degree = options->degree;
            o.lower = options->lower;
            o.coarsest = options->coarsest;
            o.max_levels = options->max_levels;
        }
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

size_t femgpu_batch_bytes(const femgpu_batch* b) { return b ? b->impl.bytes() : 0; }

void* femgpu_batch_stream(const femgpu_batch* b) {
    return b ? (void*)b->impl.stream() : nullptr;
}

void femgpu_batch_free(femgpu_batch* b) { delete b; }

}  // extern "C"
