// The sparse direct solver on the device: a multifrontal Cholesky factor P A P^T = L L^T over
// the supernodes of the host analysis (symbolic.hpp), as the reference factors its "direct"
// systems (cholesky.rs:44-167; the order of order.rs, the supernodes of symbolic.rs), and the
// two triangular solves.
//
// Layout. Each supernode s owns a dense frontal matrix F_s of m_s x m_s doubles (column-major,
// its rows R_s), kept for the solves: its first k_s columns become the columns of L, and its
// trailing block is the update matrix (Schur complement) that its parent takes. The entries of A
// are scattered into all fronts at once; then the fronts are done level by level in the
// supernode tree (height 0 = leaves), so every child is factored before its parent:
//   1. extend-add: each child's update matrix is added into its parent's front at the parent's
//      rows (relative indices found on the host), 1 launch per child rank, so the sums into a
//      parent are made in a fixed order (no atomics; the factor is reproducible bit for bit);
//   2. partial Cholesky of the k_s pivot columns: fronts of at most 128 rows in shared memory, 1
//      block each (all the level's small fronts in 1 launch); a larger front by panels of 32
//      columns (the diagonal block and the panel's rows in 1 kernel, then the trailing update
//      F22 -= L21 L21^T on the FP64 tensor cores, mma.sync m8n8k4 f64, in 64 x 64 tiles).
// A pivot at or below PIVOT = 1e-10 of the column's diagonal of A (cholesky.rs:22, 176-181) is
// recorded (the smallest column; every front with no failed descendant is still checked, so
// this is the reference's first failing column) and the factor fails with the reference's text.
// The solves run level by level too: forward, 1 block per supernode adding its children's
// contributions in order; backward from the root down.
#pragma once
#include <string>
#include <vector>

#include "common.cuh"
#include "hierarchy.hpp"
#include "symbolic.hpp"

namespace femgpu {

class SparseFactor {
   public:
    // Analyses and factors `a` (host CSR, both triangles) in the nested dissection order of the
    // unknowns' coordinates `xyz` (3 per unknown).
    void factor(const HostCsr& a, const double* xyz, cudaStream_t s);
    // x = A^-1 b, device arrays of n values (x may not alias b).
    void solve(const double* b, double* x, cudaStream_t s);
    // Keeps W = L11^-1 of the diagonal block of each supernode of at least `min_cols` columns,
    // so that the solves take its triangles by 2 products (fully parallel) instead of column by
    // column. The products round as W does, not as the substitution: on the direct solves of
    // the test systems the true residuals stay those of the substitution (4.1e-11 against
    // 4.3e-11 on a 36,300-unknown P2 beam, 1.4e-15 on a 32^3 heat cube).
    void invert_blocks(int64_t min_cols, cudaStream_t s);
    int64_t n() const { return n_; }
    // The kernels that 1 solve launches.
    size_t solve_launches() const;
    size_t bytes() const;
    std::string describe() const;
    uint64_t entries() const { return entries_; }

   private:
    int64_t n_ = 0, ns_ = 0, height_ = 0;
    uint64_t entries_ = 0;
    double flops_ = 0.0;
    size_t front_values_ = 0;
    // Per supernode (device): first column, row list, front offset, children.
    DevBuf<int64_t> perm_, first_, rows_ptr_, foff_, zoff_, child_ptr_, child_;
    DevBuf<uint32_t> rows_, relind_;
    DevBuf<int64_t> relind_off_;
    DevBuf<double> fronts_, work_, y_;
    // invert_blocks: the inverses end to end, each supernode's offset into them (-1: none), and
    // a scratch vector of n values.
    DevBuf<double> winv_, tmp_;
    DevBuf<int64_t> winv_off_;
    // The level schedule (host): the supernodes of each height, small and large fronts apart,
    // and the extend-add chunks per (height, child rank).
    std::vector<std::vector<int64_t>> small_, large_;
    std::vector<int64_t> m_, k_;  // rows and columns of each supernode (host)
    DevBuf<int64_t> small_list_, level_list_;
    std::vector<int64_t> small_at_, level_at_;  // offsets into the lists per height
    struct Chunks {
        int height, rank;
        int64_t at, count;  // into chunk_
    };
    std::vector<Chunks> chunks_;
    DevBuf<int2> chunk_;  // (child, first entry / 4096)
    std::vector<int64_t> host_first_, host_foff_;
};

}  // namespace femgpu
