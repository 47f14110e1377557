// The multigrid hierarchy on the device: the plane coarsening of a grid level with its
// prolongation (the rule of multigrid.rs:329-452), and the Galerkin product P^T A P (the coarse
// operator of sparse.rs:233-292) as two sparse products.
//
// Design. A grid level's unknowns carry their grid point (3 plane indices) and component. The
// coarse unknowns are numbered directly in grid order (z, y, x, component: the order in which a
// box level's entries sit at constant offsets), by sorting the keys of the coarse grid points
// that some fine row interpolates from; the reference numbers them in first-sight order, which
// is the same level up to that permutation. Each fine row forms its at most 8 tensor-product
// weights in registers (1 thread per row). The sparse products C = A B run 1 warp per row of C
// with a hash table of the row's columns in shared memory: a counting pass, a scan, and a pass
// that writes the columns increasing; every entry of C is summed in a fixed order (A's row
// order), so the coarse operators are reproducible bit for bit.
#pragma once
#include <array>
#include <vector>

#include "common.cuh"
#include "hierarchy.hpp"

namespace femgpu {

// A rectangular CSR matrix on the device (a prolongation P, or its transpose).
struct DevRect {
    int64_t rows = 0, cols = 0, nnz = 0;
    DevBuf<int64_t> ptr;
    DevBuf<uint32_t> idx;
    DevBuf<double> val;
};

// A grid level (multigrid.rs:55-59) on the device: the planes of each axis stay on the host;
// each unknown's grid point (3 plane indices, interleaved) and component are device arrays.
struct DevGrid {
    std::array<std::vector<double>, 3> planes;
    int64_t n = 0;
    int comps = 1;
    DevBuf<uint32_t> pts;
    DevBuf<uint8_t> comp;
};

// Uploads a host level; `comps` is 1 + the largest component.
void grid_upload(const HostLevel& h, DevGrid* d, cudaStream_t s);
// Downloads a device level (for the host steps that read it: the cells' coarse matrices).
HostLevel grid_download(const DevGrid& d, cudaStream_t s);

// The next coarser level of `fine`, whose matrix is `a`, and the prolongation P (fine rows, coarse
// columns, each row's columns increasing): every other plane of each axis in `axes` (bits x, y, z)
// with more than 2 planes, and the last plane; a scalar (comps 1) between 2 coarse planes takes
// the operator weights of its row's couplings to them when both are positive, a displacement the
// linear weights of the plane coordinates. False when no axis coarsens.
bool coarsen_grid(const DevGrid& fine, const DevCsr& a, int axes, DevRect* p, DevGrid* coarse,
                  cudaStream_t s);

// The transpose of a rectangular matrix (each row's columns increasing).
void transpose_rect(const DevRect& p, DevRect* t, cudaStream_t s);

// P^T A P.
void galerkin_product(const DevRect& p, const DevCsr& a, DevCsr* out, cudaStream_t s);

// Host copies.
HostRect rect_download(const DevRect& d, cudaStream_t s);
void rect_upload(const HostRect& h, DevRect* d, cudaStream_t s);

}  // namespace femgpu
