// Host setup of the multigrid hierarchy: plane coarsening with its prolongation
// (multigrid.rs:329-452), the Galerkin product P^T A P (sparse.rs:233-292) on all host threads,
// the P2 -> P1 prolongation (pmultigrid.rs:104-151), and the grid level of a set of points.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace femgpu {

struct HostCsr {
    int64_t n = 0;
    std::vector<int64_t> ptr;
    std::vector<uint32_t> idx;
    std::vector<double> val;
    int64_t nnz() const { return (int64_t)idx.size(); }
};

struct HostRect {
    int64_t rows = 0, cols = 0;
    std::vector<int64_t> ptr;
    std::vector<uint32_t> idx;
    std::vector<double> val;
};

// multigrid.rs:55-59
struct HostLevel {
    std::array<std::vector<double>, 3> planes;
    std::vector<std::array<uint32_t, 3>> points;
    std::vector<uint8_t> comp;
};

// multigrid.rs:329-452: false when no axis has more than 2 planes.
bool coarsen(const HostLevel& fine, const HostCsr& a, HostRect* p, HostLevel* coarse);

// Renumbers the coarse unknowns of `coarse` in grid order (z, then y, then x, then the
// component) and the columns of `p` with them. The Galerkin matrix of the renumbered P is the
// same matrix with its rows and columns permuted; in grid order the entries of a box level sit
// at constant offsets, which the stencil format needs.
void renumber_grid_order(HostRect* p, HostLevel* coarse);

// sparse.rs:233-292, each coarse row exactly as the reference forms it; rows shared among
// `threads` host threads.
HostCsr galerkin(const HostRect& p, const HostCsr& a, int threads);

// pmultigrid.rs:104-151
void prolongation(const double* points, int64_t npoints, int64_t corners, const uint32_t* edges,
                  int64_t nedges, const int64_t* free, int64_t nfree, HostRect* p,
                  std::vector<double>* coarse_xyz);

// The grid level of points on a rectilinear grid: the distinct coordinates of each axis are the
// planes, and each point takes the index of its coordinates. `comp` gives the component of
// each point's unknown, or, when null, the rank of the unknown among the unknowns at the same
// point (unknowns of 1 point are listed in increasing component order).
HostLevel level_of_points(const double* xyz, int64_t n, const uint8_t* comp);

int host_threads();

}  // namespace femgpu
