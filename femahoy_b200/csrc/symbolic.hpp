// The symbolic analysis of a sparse Cholesky factor on the host, for the device's multifrontal
// factor (sparse_direct.cu) and for the figures of the reference's Crossover::Flops
// (solve.rs:108-118, 160-172): the entries of L with the diagonal and its floating point
// operations, which depend only on the fill of the elimination order.
//
// Method (the textbook one, written for this library): the elimination tree by Liu's algorithm
// with path compression; a postorder of it; the column counts by walking, for each row, its row
// subtree up the tree from the row's entries (O(entries of L)); fundamental supernodes (a column
// joins its predecessor when it is that column's only child and their counts differ by 1); the
// row pattern of each supernode from its own columns' entries and its children's patterns; and
// the height of each supernode in the supernode tree, which schedules the device's fronts level
// by level (every child before its parent).
#pragma once
#include <cstdint>
#include <vector>

#include "hierarchy.hpp"

namespace femgpu {

struct Supernodal {
    int64_t n = 0, ns = 0;
    std::vector<int64_t> perm;      // new column k -> old index (the order, postordered)
    std::vector<int64_t> iperm;     // old index -> new column
    std::vector<int64_t> first;     // ns + 1: the first new column of each supernode
    std::vector<int64_t> rows_ptr;  // ns + 1
    std::vector<uint32_t> rows;     // each supernode's rows (new indices), increasing; its own
                                    // columns first
    std::vector<int64_t> parent;    // the parent supernode, or -1
    std::vector<int> height;        // 0 for a leaf, else 1 + the largest height of a child
    uint64_t entries = 0;           // entries of L with the diagonal
    double flops = 0.0;             // sum over columns of (rows on and below the diagonal)^2
};

// The analysis of the symmetric pattern `a` (both triangles) in the order `order` (item k is the
// old index of new column k).
Supernodal analyse_factor(const HostCsr& a, const std::vector<int64_t>& order);

// Only the entries and the flops of the factor in `order` (no row patterns).
void factor_figures(const HostCsr& a, const std::vector<int64_t>& order, uint64_t* entries,
                    double* flops);

}  // namespace femgpu
