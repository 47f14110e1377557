// Dense Cholesky factors and inverses on the device, in FP64 on the tensor cores.
//
// The panels of a factor are 32 columns: the diagonal block is factored in shared memory by 1
// block, which then solves the panel's rows below it; the trailing matrix takes the rank-32
// update in 64 x 64 tiles of mma.sync m8n8k4 f64 products. The inverse of an SPD matrix is
// W^T W with W = L^-1, formed by a blocked forward substitution (32 rows at a time, each block's
// triangle in shared memory, the rest of the rows updated by the same tiled products) and a
// tiled product W^T W. Pivots at or below 1e-10 of their column's diagonal of A fail
// (cholesky.rs:22, 173-181): the smallest such column is recorded in `status`.
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"
#include "hierarchy.hpp"

namespace femgpu {

// Partial Cholesky of the first k columns of the column-major m x m matrix F (lower triangle):
// columns 0..k get L, the lower triangle of the trailing block the Schur complement. diag0[j]
// is column j's diagonal of A for the pivot test; a failing column j records col0 + j into
// *status (an atomic minimum; the caller sets it to ~0 first).
void dense_partial_cholesky(double* F, int64_t m, int64_t k, const double* diag0, int64_t col0,
                            unsigned long long* status, cudaStream_t s);

// The inverse of the SPD matrix `a` (host CSR, n small) on the device, FP64, n x n (symmetric,
// so row- and column-major alike). Fails with the reference's text when a pivot is not
// positive (the column in the natural order). With `stages`, the host seconds of its stages
// (buffers, factor, L^-1, W^T W), each until its device work finished.
void dense_inverse(const HostCsr& a, DevBuf<double>* inv, cudaStream_t s,
                   std::vector<std::pair<const char*, double>>* stages = nullptr);

// Work buffers of dense_inverse, kept across calls (many small systems on 1 stream allocate and
// free nothing per system, so no call waits on the whole device in cudaFree).
struct DenseWork {
    DevBuf<int64_t> ptr;
    DevBuf<uint32_t> idx;
    DevBuf<double> val, diag, L, W;
    DevBuf<unsigned long long> status;
};
// The same into `inv` (n x n, the caller's), with the buffers of `w`; returns with the work
// queued on `s` (the pivot test has synchronized `s` after the factor).
void dense_inverse(const HostCsr& a, double* inv, DenseWork* w, cudaStream_t s,
                   std::vector<std::pair<const char*, double>>* stages = nullptr);

// One system of dense_inverse_batch on the device: its CSR, its buffers and its size.
struct DenseMember {
    const int64_t* ptr;
    const uint32_t* idx;
    const double* val;
    double *L, *W, *inv, *diag;
    unsigned long long* status;
    int64_t n;
};

struct DenseBatchWork {
    DevBuf<double> diag, L, W;
    DevBuf<unsigned long long> status;
    DevBuf<DenseMember> members;
};

// The inverses of the SPD matrices a[j] (device CSR, both triangles) into inv[j] (device,
// n_j x n_j each), all systems in each launch (the system on the grid's z): as many launches as
// for the largest system alone.
// Returns -1, or the first system whose pivot failed with *text the reference's text for it.
// Returns with the inverses queued on `s`; the buffers of `w` grow to the largest set served.
int dense_inverse_batch(const std::vector<const DevCsr*>& a, const std::vector<double*>& inv,
                        DenseBatchWork* w, cudaStream_t s, std::string* text);

// W[j] = L[j]^-1 for the lower triangular n_j x n_j matrices L[j] (device, column-major, zeros
// above the diagonal), each step 1 launch for all; returns with the work finished.
void triangular_inverse_batch(const std::vector<int64_t>& n, const std::vector<double*>& L,
                              const std::vector<double*>& W, DenseBatchWork* w, cudaStream_t s);

}  // namespace femgpu
