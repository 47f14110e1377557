// The compact operator forms of a level built on the device from its CSR matrix, so that the
// hierarchy's matrices never travel to the host:
//  * offset forms: a matrix whose entries sit at a few constant offsets from each row's origin
//    (the row itself for a stencil, the row's smallest column for a transfer) is stored as K
//    coefficient columns, coef[slot(o) ld + row];
//  * the 3x3-block SELL form of elasticity (block3.cuh's layout).
//
// The distinct offsets are found by 1 pass over the entries: each block keeps a table of at most
// `limit` offsets in shared memory (insertion by compare-and-swap into the first free slot, so
// that a value sits in 1 slot only and every earlier slot is taken), merged into a global table
// of the same kind; more than `limit` offsets anywhere ends the scan with a refusal.
#pragma once
#include <vector>

#include "common.cuh"

namespace femgpu {

struct OffsetScan {
    std::vector<int64_t> offs;  // sorted
    int64_t upper = 0;          // stencil: the entries with col >= row
    int64_t diag = 0;           // stencil: the entries with col == row
};

// The distinct offsets of the entries of the CSR rows [0, rows). stencil: o = col - row over the
// entries with col >= row; else o = col - base[row], base[row] the row's smallest column
// (written, 0 for an empty row). False when there are more than `limit` (<= 32) of them.
bool scan_offsets(const int64_t* ptr, const uint32_t* idx, int64_t rows, bool stencil, int limit,
                  int* base, OffsetScan* out, cudaStream_t s);

// coef[slot(o) ld + row] = (T) value for each entry (stencil: each entry with col >= row), where
// slot(o) is the position of o in `offs` (from scan_offsets); coef (K ld values) is zeroed here.
template <class T>
void fill_offsets(const int64_t* ptr, const uint32_t* idx, const double* val, int64_t rows,
                  bool stencil, const int* base, const std::vector<int64_t>& offs, int64_t ld,
                  T* coef, cudaStream_t s);

// The 3x3-block SELL form of `a` (block3.cuh): false, and nothing built, unless every node's 3
// rows have the same columns and the columns come in aligned triples.
template <class T>
bool make_bsell3_device(const DevCsr& a, DevBuf<int64_t>* sptr, DevBuf<uint32_t>* col,
                        DevBuf<T>* val, cudaStream_t s);

// dinv[i] = (T)(1 / d[i]), the reciprocal in FP64.
template <class T>
void reciprocal(int64_t n, const double* d, T* dinv, cudaStream_t s);

// b[i] = (T) a[i].
template <class T>
void convert_values(int64_t n, const double* a, T* b, cudaStream_t s);

}  // namespace femgpu
