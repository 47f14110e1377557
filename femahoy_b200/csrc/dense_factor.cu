// Dense Cholesky factors and inverses on the FP64 tensor cores (dense_factor.cuh).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <vector>

#include "dense_factor.cuh"
#include "rust_format.hpp"

namespace femgpu {
namespace {

constexpr double PIVOT = 1e-10;  // cholesky.rs:22
constexpr int PANEL = 32;
constexpr int TILE = 64;
constexpr int TH = 256;

// Panel [p0, p0 + kb) of the column-major m x m matrix F: the diagonal block factored in shared
// memory (each pivot tested against PIVOT times its column's diagonal of A), then the panel's
// rows below solved against it (L21 = A21 L11^-T); 1 block.
__device__ __forceinline__ void panel_body(double* __restrict__ F, int64_t m, int64_t p0, int kb,
                                           const double* __restrict__ diag0, int64_t col0,
                                           unsigned long long* __restrict__ status) {
    __shared__ double D[PANEL][PANEL + 1];
    __shared__ int stop;
    for (int t = threadIdx.x; t < PANEL * PANEL; t += blockDim.x) {
        const int i = t % PANEL, j = t / PANEL;
        D[i][j] = (i < kb && j < kb) ? F[(p0 + i) + (p0 + j) * m] : 0.0;
    }
    if (threadIdx.x == 0) stop = 0;
    __syncthreads();
    for (int j = 0; j < kb; ++j) {
        if (threadIdx.x == 0) {
            const double d = D[j][j];
            if (!(d > PIVOT * fabs(diag0[p0 + j]))) {
                atomicMin(status, (unsigned long long)(col0 + p0 + j));
                stop = 1;
            } else {
                D[j][j] = sqrt(d);
            }
        }
        __syncthreads();
        if (stop) return;
        if (threadIdx.x > j && threadIdx.x < kb) D[threadIdx.x][j] /= D[j][j];
        __syncthreads();
        for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
            const int i = t % kb, c = t / kb;
            if (c > j && i >= c) D[i][c] -= D[i][j] * D[c][j];
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
        const int i = t % kb, j = t / kb;
        if (i >= j) F[(p0 + i) + (p0 + j) * m] = D[i][j];
    }
}

__global__ void __launch_bounds__(TH)
    k_panel(double* __restrict__ F, int64_t m, int64_t p0, int kb,
            const double* __restrict__ diag0, int64_t col0,
            unsigned long long* __restrict__ status) {
    panel_body(F, m, p0, kb, diag0, col0, status);
}

// The 32 x 32 lower triangle of the factored diagonal block of panel p0 (kb columns) in shared
// memory, padded with the identity past kb, so that the unrolled solves below need no branch.
__device__ __forceinline__ void load_panel_triangle(const double* __restrict__ F, int64_t m,
                                                    int64_t p0, int kb,
                                                    double (*D)[PANEL + 1]) {
    for (int t = threadIdx.x; t < PANEL * PANEL; t += blockDim.x) {
        const int i = t % PANEL, j = t / PANEL;
        double v = 0.0;
        if (i < kb && j < kb && i >= j)
            v = F[(p0 + i) + (p0 + j) * m];
        else if (i == j)
            v = 1.0;
        D[i][j] = v;
    }
}

// The panel's rows below its diagonal block: L21 = A21 L11^-T, 1 thread per row, the row's 32
// values in registers (all loads in flight at once), the sums in column order.
constexpr int ROWS_TH = 128;
__device__ __forceinline__ void panel_rows_body(double* __restrict__ F, int64_t m, int64_t p0,
                                                int kb, int64_t tile) {
    __shared__ double D[PANEL][PANEL + 1];
    load_panel_triangle(F, m, p0, kb, D);
    __syncthreads();
    const int64_t r = p0 + kb + tile * (int64_t)ROWS_TH + threadIdx.x;
    if (r >= m) return;
    double x[PANEL];
#pragma unroll
    for (int j = 0; j < PANEL; ++j) x[j] = j < kb ? F[r + (p0 + j) * m] : 0.0;
#pragma unroll
    for (int j = 0; j < PANEL; ++j) {
        double v = x[j];
#pragma unroll
        for (int q = 0; q < j; ++q) v -= x[q] * D[j][q];
        x[j] = v / D[j][j];
    }
#pragma unroll
    for (int j = 0; j < PANEL; ++j)
        if (j < kb) F[r + (p0 + j) * m] = x[j];
}

__global__ void __launch_bounds__(ROWS_TH)
    k_panel_rows(double* __restrict__ F, int64_t m, int64_t p0, int kb) {
    panel_rows_body(F, m, p0, kb, blockIdx.x);
}

// D = A B + D on the FP64 tensor cores: A 8 x 4 (row), B 4 x 8 (column), D 8 x 8; lane l holds
// A[l / 4][l % 4], B[l % 4][l / 4] and D[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// The 64 x 64 product of As (64 rows x 32 k) and Bs^T (Bs: 64 columns x 32 k) added into acc:
// warp w takes rows 8w..8w+7, 8 tiles of 8 columns.
__device__ __forceinline__ void tile_product(const double (*As)[PANEL + 1],
                                             const double (*Bs)[PANEL + 1], double acc[8][2]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int kk = 0; kk < PANEL; kk += 4) {
        const double a = As[warp * 8 + g][kk + q];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) dmma(acc[nt][0], acc[nt][1], a, Bs[nt * 8 + g][kk + q]);
    }
}

// The trailing update F[t0:m, t0:m] -= L21 L21^T (lower triangle), L21 = F[t0:m, p0:p0+kb],
// kb <= 32: 1 block per 64 x 64 tile on or below the diagonal.
__device__ __forceinline__ void syrk_body(double* __restrict__ F, int64_t m, int64_t t0,
                                          int64_t p0, int kb, int64_t b) {
    __shared__ double As[TILE][PANEL + 1], Bs[TILE][PANEL + 1];
    int64_t bi = (int64_t)((sqrt(8.0 * (double)b + 1.0) - 1.0) / 2.0);
    while ((bi + 1) * (bi + 2) / 2 <= b) ++bi;
    while (bi * (bi + 1) / 2 > b) --bi;
    const int64_t bj = b - bi * (bi + 1) / 2;
    const int64_t r0 = t0 + bi * TILE, c0 = t0 + bj * TILE;
    for (int t = threadIdx.x; t < TILE * PANEL; t += blockDim.x) {
        const int r = t % TILE, k = t / TILE;
        As[r][k] = (r0 + r < m && k < kb) ? F[(r0 + r) + (p0 + k) * m] : 0.0;
        Bs[r][k] = (c0 + r < m && k < kb) ? F[(c0 + r) + (p0 + k) * m] : 0.0;
    }
    __syncthreads();
    double acc[8][2] = {};
    tile_product(As, Bs, acc);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r = r0 + warp * 8 + (lane >> 2);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int64_t c = c0 + nt * 8 + 2 * (lane & 3) + i;
            if (r < m && c < m && r >= c) F[r + c * m] -= acc[nt][i];
        }
}

__global__ void __launch_bounds__(TH)
    k_syrk_update(double* __restrict__ F, int64_t m, int64_t t0, int64_t p0, int kb) {
    syrk_body(F, m, t0, p0, kb, blockIdx.x);
}

// C -= A B for an M x N block C (column-major, ldc), A M x kb (lda), B kb x N (ldb), kb <= 32:
// 1 block per 64 x 64 tile of C.
__device__ __forceinline__ void gemm_sub_body(double* __restrict__ C, int64_t ldc,
                                              const double* __restrict__ A, int64_t lda,
                                              const double* __restrict__ B, int64_t ldb,
                                              int64_t M, int64_t N, int kb, int64_t bx,
                                              int64_t by) {
    __shared__ double As[TILE][PANEL + 1], Bs[TILE][PANEL + 1];
    const int64_t r0 = bx * TILE, c0 = by * TILE;
    for (int t = threadIdx.x; t < TILE * PANEL; t += blockDim.x) {
        const int r = t % TILE, k = t / TILE;
        As[r][k] = (r0 + r < M && k < kb) ? A[(r0 + r) + k * lda] : 0.0;
        const int kk = t % PANEL, c = t / PANEL;
        Bs[c][kk] = (c0 + c < N && kk < kb) ? B[kk + (c0 + c) * ldb] : 0.0;
    }
    __syncthreads();
    double acc[8][2] = {};
    tile_product(As, Bs, acc);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r = r0 + warp * 8 + (lane >> 2);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int64_t c = c0 + nt * 8 + 2 * (lane & 3) + i;
            if (r < M && c < N) C[r + c * ldc] -= acc[nt][i];
        }
}

__global__ void __launch_bounds__(TH)
    k_gemm_sub(double* __restrict__ C, int64_t ldc, const double* __restrict__ A, int64_t lda,
               const double* __restrict__ B, int64_t ldb, int64_t M, int64_t N, int kb) {
    gemm_sub_body(C, ldc, A, lda, B, ldb, M, N, kb, blockIdx.x, blockIdx.y);
}

// Rows [b0, b0 + kb) of W for its columns 0..ncols: W_b = L_bb^-1 W_b (the block's triangle in
// shared memory), 1 thread per column, the column's 32 values in registers.
__device__ __forceinline__ void trsm_rows_body(double* __restrict__ W,
                                               const double* __restrict__ L, int64_t n,
                                               int64_t b0, int kb, int64_t ncols, int64_t tile) {
    __shared__ double D[PANEL][PANEL + 1];
    load_panel_triangle(L, n, b0, kb, D);
    __syncthreads();
    const int64_t c = tile * (int64_t)ROWS_TH + threadIdx.x;
    if (c >= ncols) return;
    double y[PANEL];
#pragma unroll
    for (int i = 0; i < PANEL; ++i) y[i] = i < kb ? W[(b0 + i) + c * n] : 0.0;
#pragma unroll
    for (int i = 0; i < PANEL; ++i) {
        double v = y[i];
#pragma unroll
        for (int j = 0; j < i; ++j) v -= D[i][j] * y[j];
        y[i] = v / D[i][i];
    }
#pragma unroll
    for (int i = 0; i < PANEL; ++i)
        if (i < kb) W[(b0 + i) + c * n] = y[i];
}

__global__ void __launch_bounds__(ROWS_TH)
    k_trsm_rows(double* __restrict__ W, const double* __restrict__ L, int64_t n, int64_t b0,
                int kb, int64_t ncols) {
    trsm_rows_body(W, L, n, b0, kb, ncols, blockIdx.x);
}

// X = W^T W (W lower triangular, column-major n x n): 1 block per 64 x 64 tile on or below the
// diagonal, the sum over k from the tile's first row (W[k][i] = 0 for k < i), both halves of X
// written.
__device__ __forceinline__ void gram_lower_body(const double* __restrict__ W, int64_t n,
                                                double* __restrict__ X, int64_t b) {
    __shared__ double As[TILE][PANEL + 1], Bs[TILE][PANEL + 1];
    int64_t bi = (int64_t)((sqrt(8.0 * (double)b + 1.0) - 1.0) / 2.0);
    while ((bi + 1) * (bi + 2) / 2 <= b) ++bi;
    while (bi * (bi + 1) / 2 > b) --bi;
    const int64_t bj = b - bi * (bi + 1) / 2;
    const int64_t i0 = bi * TILE, j0 = bj * TILE;
    double acc[8][2] = {};
    for (int64_t k0 = i0; k0 < n; k0 += PANEL) {
        __syncthreads();
        for (int t = threadIdx.x; t < TILE * PANEL; t += blockDim.x) {
            const int kk = t % PANEL, c = t / PANEL;
            const bool kin = k0 + kk < n;
            As[c][kk] = (kin && i0 + c < n) ? W[(k0 + kk) + (i0 + c) * n] : 0.0;
            Bs[c][kk] = (kin && j0 + c < n) ? W[(k0 + kk) + (j0 + c) * n] : 0.0;
        }
        __syncthreads();
        tile_product(As, Bs, acc);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t i = i0 + warp * 8 + (lane >> 2);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t j = j0 + nt * 8 + 2 * (lane & 3) + h;
            if (i < n && j < n && i >= j) {
                X[i + j * n] = acc[nt][h];
                X[j + i * n] = acc[nt][h];
            }
        }
}

__global__ void __launch_bounds__(TH)
    k_gram_lower(const double* __restrict__ W, int64_t n, double* __restrict__ X) {
    gram_lower_body(W, n, X, blockIdx.x);
}

// The dense lower triangle of a host CSR's device copy, and its diagonal.
__global__ void k_scatter_dense(int64_t n, const int64_t* __restrict__ ptr,
                                const uint32_t* __restrict__ idx, const double* __restrict__ val,
                                double* __restrict__ M, double* __restrict__ diag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) {
            const int64_t j = idx[e];
            if (j == i) d = val[e];
            if (j >= i) M[j + i * n] = val[e];  // column i, row j (symmetric)
        }
        diag[i] = d;
    }
}

__global__ void k_identity(int64_t n, double* __restrict__ W) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * n;
         t += (int64_t)gridDim.x * blockDim.x)
        W[t] = (t % n == t / n) ? 1.0 : 0.0;
}

// ---------------------------------------------------------------- many systems at once
// The same steps for a set of systems: the system is blockIdx.z, and a block past its system's
// size returns at once, so that each step is 1 launch for all of them.

__global__ void k_scatter_dense_b(const DenseMember* __restrict__ M) {
    const DenseMember d = M[blockIdx.z];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < d.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double g = 0.0;
        for (int64_t e = d.ptr[i]; e < d.ptr[i + 1]; ++e) {
            const int64_t j = d.idx[e];
            if (j == i) g = d.val[e];
            if (j >= i) d.L[j + i * d.n] = d.val[e];
        }
        d.diag[i] = g;
    }
}

__global__ void __launch_bounds__(TH) k_panel_b(const DenseMember* __restrict__ M, int64_t p0) {
    const DenseMember d = M[blockIdx.z];
    if (p0 >= d.n) return;
    panel_body(d.L, d.n, p0, (int)min((int64_t)PANEL, d.n - p0), d.diag, 0, d.status);
}

__global__ void __launch_bounds__(ROWS_TH)
    k_panel_rows_b(const DenseMember* __restrict__ M, int64_t p0) {
    const DenseMember d = M[blockIdx.z];
    if (p0 >= d.n) return;
    const int kb = (int)min((int64_t)PANEL, d.n - p0);
    if (p0 + kb + (int64_t)blockIdx.x * ROWS_TH >= d.n) return;
    panel_rows_body(d.L, d.n, p0, kb, blockIdx.x);
}

__global__ void __launch_bounds__(TH) k_syrk_update_b(const DenseMember* __restrict__ M, int64_t p0) {
    const DenseMember d = M[blockIdx.z];
    if (p0 >= d.n) return;
    const int kb = (int)min((int64_t)PANEL, d.n - p0);
    const int64_t t0 = p0 + kb;
    if (t0 >= d.n) return;
    const int64_t T = (d.n - t0 + TILE - 1) / TILE;
    if ((int64_t)blockIdx.x >= T * (T + 1) / 2) return;
    syrk_body(d.L, d.n, t0, p0, kb, blockIdx.x);
}

__global__ void k_identity_b(const DenseMember* __restrict__ M) {
    const DenseMember d = M[blockIdx.z];
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < d.n * d.n;
         t += (int64_t)gridDim.x * blockDim.x)
        d.W[t] = (t % d.n == t / d.n) ? 1.0 : 0.0;
}

__global__ void __launch_bounds__(ROWS_TH)
    k_trsm_rows_b(const DenseMember* __restrict__ M, int64_t b0) {
    const DenseMember d = M[blockIdx.z];
    if (b0 >= d.n) return;
    const int kb = (int)min((int64_t)PANEL, d.n - b0);
    const int64_t ncols = b0 + kb;
    if ((int64_t)blockIdx.x * ROWS_TH >= ncols) return;
    trsm_rows_body(d.W, d.L, d.n, b0, kb, ncols, blockIdx.x);
}

__global__ void __launch_bounds__(TH) k_gemm_sub_b(const DenseMember* __restrict__ M, int64_t b0) {
    const DenseMember d = M[blockIdx.z];
    if (b0 >= d.n) return;
    const int kb = (int)min((int64_t)PANEL, d.n - b0);
    const int64_t rows = d.n - b0 - kb, ncols = b0 + kb;
    if ((int64_t)blockIdx.x * TILE >= rows || (int64_t)blockIdx.y * TILE >= ncols) return;
    const int64_t n = d.n;
    gemm_sub_body(d.W + b0 + kb, n, d.L + (b0 + kb) + b0 * n, n, d.W + b0, n, rows, ncols, kb,
                  blockIdx.x, blockIdx.y);
}

__global__ void __launch_bounds__(TH) k_gram_lower_b(const DenseMember* __restrict__ M) {
    const DenseMember d = M[blockIdx.z];
    const int64_t T = (d.n + TILE - 1) / TILE;
    if ((int64_t)blockIdx.x >= T * (T + 1) / 2) return;
    gram_lower_body(d.W, d.n, d.inv, blockIdx.x);
}

}  // namespace

int dense_inverse_batch(const std::vector<const DevCsr*>& a, const std::vector<double*>& inv,
                        DenseBatchWork* w, cudaStream_t s, std::string* text) {
    const int count = (int)a.size();
    if (count == 0) return -1;
    if (count > 65535) throw Failure(FEMGPU_ERR_TOO_LARGE, "more than 65535 dense systems at once");
    // The systems' square buffers end to end.
    std::vector<int64_t> sq_at(count), n_at(count);
    int64_t nsq = 0, nrows = 0, nmax = 0;
    for (int j = 0; j < count; ++j) {
        const int64_t n = a[j]->n;
        sq_at[j] = nsq;
        n_at[j] = nrows;
        nsq += n * n;
        nrows += n;
        nmax = std::max<int64_t>(nmax, n);
    }
    auto fit = [](auto& b, size_t c) {
        if (b.count < c) b.alloc(c);
    };
    fit(w->L, nsq);
    fit(w->W, nsq);
    fit(w->diag, nrows);
    fit(w->status, count);
    fit(w->members, count);
    std::vector<DenseMember> dm(count);
    for (int j = 0; j < count; ++j)
        dm[j] = DenseMember{a[j]->ptr.p,       a[j]->idx.p,      a[j]->val.p,
                            w->L.p + sq_at[j], w->W.p + sq_at[j], inv[j],
                            w->diag.p + n_at[j], w->status.p + j, a[j]->n};
    w->members.upload(dm.data(), count, s);
    const DenseMember* M = w->members.p;
    FG_CUDA(cudaMemsetAsync(w->L.p, 0, (size_t)nsq * sizeof(double), s));
    FG_CUDA(cudaMemsetAsync(w->status.p, 0xff, (size_t)count * sizeof(unsigned long long), s));
    const unsigned z = (unsigned)count;
    k_scatter_dense_b<<<dim3((unsigned)blocks_for(nmax, TH), 1, z), TH, 0, s>>>(M);
    for (int64_t p0 = 0; p0 < nmax; p0 += PANEL) {
        k_panel_b<<<dim3(1, 1, z), TH, 0, s>>>(M, p0);
        const int64_t t0 = std::min(nmax, p0 + PANEL);
        if (t0 < nmax) {
            k_panel_rows_b<<<dim3((unsigned)((nmax - t0 + ROWS_TH - 1) / ROWS_TH), 1, z), ROWS_TH,
                             0, s>>>(M, p0);
            const int64_t T = (nmax - t0 + TILE - 1) / TILE;
            k_syrk_update_b<<<dim3((unsigned)(T * (T + 1) / 2), 1, z), TH, 0, s>>>(M, p0);
        }
    }
    FG_CHECK_LAUNCH();
    std::vector<unsigned long long> bad(count);
    FG_CUDA(cudaMemcpyAsync(bad.data(), w->status.p, count * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    for (int j = 0; j < count; ++j)
        if (bad[j] != ~0ull) {
            const double d = fetch(w->diag.p + n_at[j] + (int64_t)bad[j], s);
            char buf[320];
            std::snprintf(buf, sizeof buf,
                          "the matrix is not positive definite: the pivot of column %llu is 0 or "
                          "less to the precision of the arithmetic (its diagonal is %s)",
                          bad[j], rust_exp_shortest(d).c_str());
            *text = buf;
            return j;
        }
    k_identity_b<<<dim3((unsigned)blocks_for(nmax * nmax, TH), 1, z), TH, 0, s>>>(M);
    for (int64_t b0 = 0; b0 < nmax; b0 += PANEL) {
        const int64_t ncols = std::min(nmax, b0 + PANEL);
        k_trsm_rows_b<<<dim3((unsigned)((ncols + ROWS_TH - 1) / ROWS_TH), 1, z), ROWS_TH, 0, s>>>(
            M, b0);
        const int64_t rows = nmax - ncols;
        if (rows > 0)
            k_gemm_sub_b<<<dim3((unsigned)((rows + TILE - 1) / TILE),
                                (unsigned)((ncols + TILE - 1) / TILE), z),
                           TH, 0, s>>>(M, b0);
    }
    const int64_t T = (nmax + TILE - 1) / TILE;
    k_gram_lower_b<<<dim3((unsigned)(T * (T + 1) / 2), 1, z), TH, 0, s>>>(M);
    FG_CHECK_LAUNCH();
    return -1;
}

void triangular_inverse_batch(const std::vector<int64_t>& n, const std::vector<double*>& L,
                              const std::vector<double*>& W, DenseBatchWork* w, cudaStream_t s) {
    const int count = (int)n.size();
    if (count == 0) return;
    if (count > 65535) throw Failure(FEMGPU_ERR_TOO_LARGE, "more than 65535 triangles at once");
    int64_t nmax = 0;
    std::vector<DenseMember> dm(count);
    for (int j = 0; j < count; ++j) {
        dm[j] = DenseMember{nullptr, nullptr, nullptr, L[j], W[j], nullptr, nullptr, nullptr, n[j]};
        nmax = std::max(nmax, n[j]);
    }
    if (w->members.count < (size_t)count) w->members.alloc(count);
    w->members.upload(dm.data(), count, s);
    const DenseMember* M = w->members.p;
    const unsigned z = (unsigned)count;
    k_identity_b<<<dim3((unsigned)blocks_for(nmax * nmax, TH), 1, z), TH, 0, s>>>(M);
    for (int64_t b0 = 0; b0 < nmax; b0 += PANEL) {
        const int64_t ncols = std::min(nmax, b0 + PANEL);
        k_trsm_rows_b<<<dim3((unsigned)((ncols + ROWS_TH - 1) / ROWS_TH), 1, z), ROWS_TH, 0, s>>>(
            M, b0);
        const int64_t rows = nmax - ncols;
        if (rows > 0)
            k_gemm_sub_b<<<dim3((unsigned)((rows + TILE - 1) / TILE),
                                (unsigned)((ncols + TILE - 1) / TILE), z),
                           TH, 0, s>>>(M, b0);
    }
    FG_CHECK_LAUNCH();
    FG_CUDA(cudaStreamSynchronize(s));  // the member table is the caller's until here
}

void dense_partial_cholesky(double* F, int64_t m, int64_t k, const double* diag0, int64_t col0,
                            unsigned long long* status, cudaStream_t s) {
    for (int64_t p0 = 0; p0 < k; p0 += PANEL) {
        const int kb = (int)std::min<int64_t>(PANEL, k - p0);
        k_panel<<<1, TH, 0, s>>>(F, m, p0, kb, diag0, col0, status);
        const int64_t t0 = p0 + kb;
        if (t0 < m)
            k_panel_rows<<<(unsigned)((m - t0 + ROWS_TH - 1) / ROWS_TH), ROWS_TH, 0, s>>>(F, m, p0,
                                                                                      kb);
        if (t0 < m) {
            const int64_t T = (m - t0 + TILE - 1) / TILE;
            k_syrk_update<<<(unsigned)(T * (T + 1) / 2), TH, 0, s>>>(F, m, t0, p0, kb);
        }
    }
    FG_CHECK_LAUNCH();
}

void dense_inverse(const HostCsr& a, double* inv, DenseWork* w, cudaStream_t s,
                   std::vector<std::pair<const char*, double>>* stages) {
    const int64_t n = a.n;
    auto t0 = std::chrono::steady_clock::now();
    auto stage = [&](const char* name) {
        if (!stages) return;
        FG_CUDA(cudaStreamSynchronize(s));
        const auto t1 = std::chrono::steady_clock::now();
        stages->emplace_back(name, std::chrono::duration<double>(t1 - t0).count());
        t0 = t1;
    };
    // The work buffers grow to the largest system they have served and are kept.
    auto fit = [&](DevBuf<double>& b, size_t count) {
        if (b.count < count) b.alloc(count);
    };
    fit(w->diag, n);
    fit(w->L, n * n);
    fit(w->W, n * n);
    if (!w->status.p) w->status.alloc(1);
    double* L = w->L.p;
    double* W = w->W.p;
    stage("buffers");
    w->ptr.upload(a.ptr.data(), n + 1, s);
    w->idx.upload(a.idx.data(), a.nnz(), s);
    w->val.upload(a.val.data(), a.nnz(), s);
    FG_CUDA(cudaMemsetAsync(L, 0, (size_t)n * n * sizeof(double), s));
    k_scatter_dense<<<blocks_for(n, TH), TH, 0, s>>>(n, w->ptr.p, w->idx.p, w->val.p, L,
                                                     w->diag.p);
    FG_CUDA(cudaMemsetAsync(w->status.p, 0xff, sizeof(unsigned long long), s));
    dense_partial_cholesky(L, n, n, w->diag.p, 0, w->status.p, s);
    stage("factor");
    const unsigned long long bad = fetch(w->status.p, s);
    if (bad != ~0ull) {
        const double d = fetch(w->diag.p + bad, s);
        char buf[320];
        std::snprintf(buf, sizeof buf,
                      "the matrix is not positive definite: the pivot of column %llu is 0 or less "
                      "to the precision of the arithmetic (its diagonal is %s)",
                      bad, rust_exp_shortest(d).c_str());
        throw Failure(FEMGPU_ERR_NOT_SPD, buf);
    }
    // W = L^-1 by block rows of 32: each block's triangle solve, then the rows below updated.
    k_identity<<<blocks_for(n * n, TH), TH, 0, s>>>(n, W);
    for (int64_t b0 = 0; b0 < n; b0 += PANEL) {
        const int kb = (int)std::min<int64_t>(PANEL, n - b0);
        const int64_t ncols = b0 + kb;
        k_trsm_rows<<<(unsigned)((ncols + ROWS_TH - 1) / ROWS_TH), ROWS_TH, 0, s>>>(W, L, n, b0,
                                                                                    kb, ncols);
        const int64_t rows = n - b0 - kb;
        if (rows > 0) {
            dim3 grid((unsigned)((rows + TILE - 1) / TILE), (unsigned)((ncols + TILE - 1) / TILE));
            k_gemm_sub<<<grid, TH, 0, s>>>(W + b0 + kb, n, L + (b0 + kb) + b0 * n, n, W + b0, n,
                                           rows, ncols, kb);
        }
    }
    stage("L^-1");
    const int64_t T = (n + TILE - 1) / TILE;
    k_gram_lower<<<(unsigned)(T * (T + 1) / 2), TH, 0, s>>>(W, n, inv);
    FG_CHECK_LAUNCH();
    stage("W^T W");
}

void dense_inverse(const HostCsr& a, DevBuf<double>* inv, cudaStream_t s,
                   std::vector<std::pair<const char*, double>>* stages) {
    DenseWork w;
    inv->alloc(a.n * a.n);
    dense_inverse(a, inv->p, &w, s, stages);
    FG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace femgpu
