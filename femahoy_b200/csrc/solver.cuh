// The solver of a matrix on the device: the reference's `Solver` (solve.rs:58-250) with a
// dense Cholesky for the direct method and for the coarsest level, and PCG with a geometric or
// p-multigrid V-cycle of Chebyshev-Jacobi smoothing.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "block3.cuh"
#include "coarsen.cuh"
#include "dense_factor.cuh"
#include "hierarchy.hpp"
#include "ops.cuh"
#include "sell.cuh"
#include "sparse_direct.cuh"

namespace femgpu {

template <class T>
struct Sell {
    int64_t n = 0, nslices = 0, entries = 0;
    int C = 32;
    DevBuf<int64_t> slice_ptr;
    DevBuf<uint32_t> col;
    DevBuf<T> val;
    SellView<T> view() const { return {n, nslices, C, slice_ptr.p, col.p, val.p}; }
    size_t bytes() const { return slice_ptr.bytes() + col.bytes() + val.bytes(); }
};

// A SELL-C matrix of `a` with values converted to T.
template <class T>
void make_sell(const DevCsr& a, int C, Sell<T>* out, cudaStream_t s);

// The operator of a level: a symmetric stencil when the level's entries sit at a few constant
// column offsets (the operators of a box grid in grid order), else SELL-C.
template <class T>
struct Operator {
    bool stencil = false;
    bool block3 = false;  // the 3x3-block form (elasticity), else SELL-C, when not a stencil
    bool unrolled = false;  // the compile-time-K kernel (K = 8 or 14), chosen by timing
    bool half = false;      // the stencil's products read its FP16 copy (hcoef, hscale)
    bool bulk = false;      // its smoothing steps and residuals stream tiles by bulk copies
    bool pair = false;      // the compile-time-K kernels with 2 rows per thread, chosen by timing
    bool march = false;     // the plane-marching kernels (gathers from shared memory), by timing
    MarchGeom mg{};
    // The timed product: runtime K, compile-time K, tiles, 2 rows per thread, marching planes.
    double probe_ms[5] = {0, 0, 0, 0, 0};
    int64_t n = 0, nnz = 0;
    Sell<T> sell;
    int K = 0;
    int64_t ld = 0;  // the stride of each offset's coefficient array (stencil_ld(n))
    std::vector<int64_t> off;
    DevBuf<T> coef;
    DevBuf<__half> hcoef;
    float hscale = 1.0f;
    DevBuf<int64_t> b3ptr;
    DevBuf<uint32_t> b3col;
    DevBuf<T> b3val;
    BSell3View<T> b3view() const { return {n / 3, b3ptr.p, b3col.p, b3val.p}; }
    int64_t threads() const {
        if (stencil) return n;
        if (block3) return 3 * ((n / 3 + B3C - 1) / B3C) * B3C;
        return sell.nslices * sell.C;
    }
    StencilView<T> sview() const {
        StencilView<T> v{};
        v.n = (int)n;
        v.K = K;
        v.ld = (int)ld;
        for (int k = 0; k < K; ++k) v.off[k] = (int)off[k];
        v.coef = coef.p;
        return v;
    }
    StencilViewH hview() const {
        StencilViewH v{};
        v.n = (int)n;
        v.K = K;
        v.ld = (int)ld;
        for (int k = 0; k < K; ++k) v.off[k] = (int)off[k];
        v.coef = hcoef.p;
        v.scale = hscale;
        return v;
    }
    size_t bytes() const {
        return sell.bytes() + coef.bytes() + hcoef.bytes() + b3ptr.bytes() + b3col.bytes() +
               b3val.bytes();
    }
    // The bytes one product reads and writes, each value once: the stored coefficients (and
    // indices), x and y.
    double stream_bytes() const {
        if (stencil) return (double)K * n * (half ? 2 : sizeof(T)) + 2.0 * n * sizeof(T);
        if (block3) return (double)nnz / 9 * (9 * sizeof(T) + 4) + 2.0 * n * sizeof(T);
        return (double)nnz * (sizeof(T) + 4) + 2.0 * n * sizeof(T);
    }
};

// The operator of the device matrix `d`, built on the device: a stencil if `allow` and the
// offsets fit, else (if `allow`) the 3x3-block form where the pattern is node triples, else
// SELL-C.
template <class T>
void make_operator(const DevCsr& d, int C, bool allow, Operator<T>* out, cudaStream_t s);

// Setup helpers shared by the solvers (solver.cu).
void upload_csr(const HostCsr& h, DevCsr* d, cudaStream_t s);
HostCsr download_csr(const DevCsr& d, cudaStream_t s);
HostRect transpose(const HostRect& p);
template <class T>
double lambda_max(const Operator<T>& A, const double* dg, cudaStream_t s,
                  DevBuf<double>& partial);
// kind 1: the first-kind Chebyshev polynomial on [lower, upper] lambda; 4: the fourth kind on
// [0, upper] lambda (upper 0: 1.1).
void chebyshev(double lam, int degree, double lower, std::vector<double>* c1,
               std::vector<double>* c2, int kind = 1, double upper = 1.1);

// The scalars of a PCG solve, in device memory.
struct Scalars {
    double bb, rr, rz, pq, alpha, beta, zq, norm_b;
    int done, iters, status, max_iter;
    int bulk_timeout;  // a bulk-copy wait of the stencil tile kernels ran out of its limit
};

// A transfer (P or R = P^T) of a box grid in grid order: the entries of row i sit at K
// constant offsets from the row's first column, y[i] = sum_k w[k][i] x[base[i] + off[k]], with
// w = 0 where the row has no entry (at most 8 offsets for P, the corners of a coarse cell, and
// 27 for R). The weights are read coalesced and no column index is stored.
template <class T>
struct OffsetView {
    int rows, cols, K;
    int off[32];
    const int* __restrict__ base;
    const T* __restrict__ w;
};

template <class T>
struct OffsetTransfer {
    bool ok = false;
    int64_t rows = 0, cols = 0;
    std::vector<int> off;
    DevBuf<int> base;
    DevBuf<T> w;
    OffsetView<T> view() const {
        OffsetView<T> v{};
        v.rows = (int)rows;
        v.cols = (int)cols;
        v.K = (int)off.size();
        for (size_t k = 0; k < off.size(); ++k) v.off[k] = off[k];
        v.base = base.p;
        v.w = w.p;
        return v;
    }
    size_t bytes() const { return base.bytes() + w.bytes(); }
};

template <class T>
struct MgLevel {
    int64_t n = 0, nnz = 0;
    Operator<T> A;
    DevBuf<T> dinv;
    // The prolongation P from the next level, and R = P^T (gather form of the restriction):
    // in offset form where they fit (Po, Ro), else CSR.
    int64_t nc = 0;
    OffsetTransfer<T> Po, Ro;
    DevBuf<int64_t> pptr, rptr;
    DevBuf<uint32_t> pidx, ridx;
    DevBuf<T> pval, rval;
    DevBuf<T> b, xa, xb, d, r;
    std::vector<double> c1, c2;
    double lambda = 0;
};

// 1 level of the fused kernel of the coarse levels (k_tail): its operator (a stencil read with
// the runtime-K product, or SELL), smoother, transfers and vectors.
constexpr int TAIL_MAXDEG = 8;
template <class T>
struct TailLevel {
    int n, nc, stencil, deg, p_offset, r_offset;
    StencilView<T> sv;
    SellView<T> sell;
    OffsetView<T> Po, Ro;
    const int64_t *pptr, *rptr;
    const uint32_t *pidx, *ridx;
    const T *pval, *rval;
    const T* dinv;
    const T* b;  // the level's right side (the first level's comes as an argument)
    T *xa, *xb, *d, *r, *bc;
    T c1[TAIL_MAXDEG], c2[TAIL_MAXDEG];
};

template <class T>
struct Hierarchy {
    std::vector<MgLevel<T>> levels;  // all but the coarsest
    int64_t ncoarse = 0;
    DevBuf<T> inv;  // the inverse of the coarsest matrix, n x n (symmetric)
    // The mixed form's FP16 copy of the inverse (values 3), divided by its largest entry.
    DevBuf<__half> hinv;
    float hscale = 1.0f;
    DevBuf<T> cb, cx;
    // A coarsest level above DENSE_COARSEST_MAX unknowns (a grid that stops coarsening, e.g. the
    // layers of an extruded footprint): its sparse multifrontal factor, as the reference's
    // coarsest solve (multigrid.rs:130-131), applied in FP64.
    std::unique_ptr<SparseFactor> sparse;
    DevBuf<double> cb64, cx64;
    // The levels from `tail_from` down, and the coarsest solve, run as 1 cooperative kernel
    // (-1: none) of `tail_grid` blocks.
    int tail_from = -1, tail_grid = 0;
    std::vector<char> cluster;  // per level: its legs run as cluster launches
    DevBuf<TailLevel<T>> tail;
    size_t bytes() const;
};

// The largest level that the dense coarse solve takes by default. The reference stops
// coarsening at 3000 unknowns (multigrid.rs:94, COARSEST) and factors that level sparsely; a
// dense inverse of up to 5000 unknowns (100 MB in FP32) is applied by 1 matrix-vector product
// on the device, and on the 128^3 heat cube the level of 4,913 rows taken whole saves 2 coarser
// levels' kernels and 1 PCG iteration (9 instead of 10, 3.28 instead of 3.50 ms).
constexpr int DEVICE_COARSEST = 5000;
// The direct method's dense inverse takes systems of up to this many unknowns; larger ones the
// sparse multifrontal factor.
constexpr int64_t DENSE_DIRECT = 4096;
// The largest coarsest level that takes the dense inverse; a larger one (a grid that does not
// coarsen further) takes the sparse factor.
constexpr int64_t DENSE_COARSEST_MAX = 16384;

struct Options {
    int precision = FEMGPU_FP64;
    int degree = 0;
    double lower = 0;
    int sell_c = 0;
    int format = 0;  // 0: stencil where possible, else SELL; 1: SELL only
    int coarsest = DEVICE_COARSEST;
    int max_levels = 30;
    bool graph = true;
    int tail = 0;  // levels of at most this many rows run fused (<= 0: none)
    int pdl = 1;   // programmatic dependent launch between the iteration's kernels
    int values = 0;  // mixed form's stencil levels: 0 default, 1 FP32, 2 FP16 coefficients
    int tiles = 0;   // finest FP32 stencil steps by bulk-copied tiles: 0 tuned, 1 off, 2 on
    int axes = 7;    // the axes that the coarsening halves (bits x, y, z)
    int stencil = 0; // stencil kernel: 0 tuned, 1 runtime K, 2 compile-time K, 3 2 rows, 4 march
    int l2 = 0;      // 1: the coarsest inverse persisting in L2
    int smoother = 4;  // the Chebyshev polynomial's kind: 1 first, 4 fourth
    int cluster = 0;   // 1: small levels' legs as 1 cluster launch each; 0: a launch per step
    double upper = 0;  // the Chebyshev interval's upper end over lambda_max (0: 1.1)
};

class SolverImpl {
   public:
    SolverImpl();
    ~SolverImpl();
    // solve.rs:92-183
    // `cells` (may be null): the cells of a box-grid displacement model, whose coarse matrices
    // then come from the cells (multigrid.rs:107-119).
    void create(const DevCsr& a, const femgpu_unknowns& u, int method, const femgpu_crossover& c,
                const Options& o, const HostCells* cells = nullptr);
    // solve.rs:199-250 on device vectors
    void solve(const double* d_b, double* d_x, const volatile int* cancel, femgpu_stats* st);
    void solve_host(const double* h_b, double* h_x, const volatile int* cancel, femgpu_stats* st);
    // The same from x = 0: x is written only (no host-to-device copy of a start value).
    void solve_host_zero(const double* h_b, double* h_x, const volatile int* cancel,
                         femgpu_stats* st);
    void precondition(const double* d_r, double* d_z);
    int method() const { return direct_ ? FEMGPU_METHOD_DIRECT : FEMGPU_METHOD_MULTIGRID; }
    std::vector<int64_t> level_sizes() const;
    // A text description of the levels: size, format, K, kernel choice, lambda_max.
    std::string describe() const;
    // The device time of each kernel of 1 PCG iteration (kernels launched one by one, a CUDA
    // event after each), as text.
    std::string breakdown();
    size_t bytes() const;
    // The mean device time (ms) of 1 launch of a kernel of the solve, and its algorithmic bytes.
    void kernel_time(int which, int reps, double* ms, double* bytes);
    size_t max_iter = 500;  // PCG_MAX_ITER, solve.rs:43
    double tol = 1e-10;     // PCG_TOL, solve.rs:42
    // The polls of each bulk-copy wait of the stencil tile kernels before they report a
    // timeout (FEMGPU_ERR_TIMEOUT); the default is far above any copy's latency.
    unsigned wait_limit = 1u << 22;
    // Sets wait_limit; the captured PCG loop holds the old value, so it is captured again.
    void set_wait_limit(unsigned polls);
    cudaStream_t stream() const { return s_; }
    // Adds `seconds` to the setup phase `name`.
    void phase(const std::string& name, double seconds);

   private:
    void build_multigrid(HostLevel level, const HostRect* pfirst, const HostCells* cells);
    template <class T>
    void build_levels(const std::vector<const DevCsr*>& mats, std::vector<DevRect>& ps,
                      const HostLevel& coarsest, Hierarchy<T>* H);
    template <class T>
    // `started`: the level's first smoothing step was done by the finer level's restriction.
    const T* enqueue_vcycle(Hierarchy<T>& H, size_t l, const T* b, bool started = false);
    template <class T>
    void enqueue_step(MgLevel<T>& L, const T* b, const T* xin, T c1, T c2, T* xout);
    template <class T>
    void enqueue_residual(MgLevel<T>& L, const T* b, const T* x);
    void enqueue_iteration();
    void enqueue_spmv_pq();
    void build_loop_graph();
    // Runs PCG iterations on the device until convergence, max_iter, a NaN or a cancel.
    void run_device_loop(const volatile int* cancel);
    void run_init(const double* d_b);
    void dense_direct(const HostCsr& a);
    // The Chebyshev degree of every level (1, 2 or 3) by timed trial solves, per size class.
    void tune_degree();
    // The Chebyshev degree of the finest level and of the coarser ones (0: the same).
    void apply_degree(int degree, int coarse = 0);
    void sparse_direct(const HostCsr& a, const std::vector<double>& xyz);

    cudaStream_t s_ = nullptr;
    Options opt_;
    bool direct_ = false;
    // The persisting L2 window of the coarsest inverse's product (option l2), if any.
    bool l2_window_ = false;
    cudaAccessPolicyWindow l2win_{};
    int64_t n_ = 0;
    Sell<double> A64_;          // the matrix exactly (the true residual, the direct method)
    Operator<double> op64_;     // the FP64 operator of PCG
    DevCsr a_;  // the matrix, FP64 CSR
    Hierarchy<double> H64_;
    Hierarchy<float> H32_;
    DevBuf<double> dense_inv_;  // the direct method: A^-1
    std::unique_ptr<SparseFactor> sparse_;  // the direct method above DENSE_DIRECT unknowns
    DevBuf<double> x_, r_, p_, q_, b_, z64_, t_;
    DevBuf<float> r32_;
    const double* zd_ = nullptr;  // where the V-cycle leaves z (FP64 form)
    const float* zf_ = nullptr;   // (mixed form)
    DevBuf<double> partial_;
    DevBuf<unsigned> counter_;
    DevBuf<Scalars> sc_;
    Scalars* h_sc_ = nullptr;
    DevBuf<int> done_zero_;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaGraphConditionalHandle cond_ = 0;
    int* h_cancel_ = nullptr;  // pinned and mapped: the device reads it each iteration
    int* d_cancel_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    std::vector<int64_t> sizes_;
    // While breakdown() runs: the label and the event recorded after each kernel.
    std::vector<std::pair<std::string, cudaEvent_t>>* trace_ = nullptr;
    void mark(const std::string& label);
    bool tail_on_ = true;      // the fused coarse levels (off if a graph would not take them)
    bool cluster_on_ = true;   // the small levels by cluster (off if a graph would not take them)
    int cluster_ctas_ = 0;     // blocks of 1 cluster (16 or 8; 0: none can be scheduled)
    bool pdl_ = true;          // programmatic dependent launch of the iteration's kernels
    // Seconds of each phase of the setup, in the order first met (reported by describe()).
    std::vector<std::pair<std::string, double>> setup_s_;
    size_t launches_ = 0;      // kernels enqueued by the current solve
    size_t graph_kernels_ = 0; // kernels of 1 iteration graph
};

}  // namespace femgpu

// The handles of include/femgpu.h.
struct femgpu_csr {
    femgpu::DevCsr m;
};

struct femgpu_solver {
    femgpu::SolverImpl impl;
};
