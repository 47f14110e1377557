// Host setup steps of the multigrid hierarchy: the coarse matrices of a box grid from its cells
// (multigrid.rs:458-681), the figures of Crossover::Flops, the P2 -> P1 prolongation
// (pmultigrid.rs:104-151) and the grid level of a set of points. The plane coarsening and the
// Galerkin products run on the device (coarsen.cuh).
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

// multigrid.rs:62-68 `Cells`: the cells of a box-grid displacement level, each by its lowest
// grid point and the class of its 24 x 24 matrix (row-major, unknown 3 n + c for corner n in
// VTK order): matrix i is table + 576 cls[i].
struct HostCells {
    std::vector<std::array<uint32_t, 3>> origin;
    std::vector<uint32_t> cls;
    std::vector<double> table;
    bool empty() const { return origin.empty(); }
};

// multigrid.rs:458-608: the coarse matrix of a displacement from its cells. Each coarse cell
// sums the energy of its fine cells for its 8 trilinear corner fields and its 9 incompatible
// modes (those that the Gram factor of the fields at the free fine unknowns keeps,
// multigrid.rs:616-652) and condenses the modes (multigrid.rs:654-681); the coarse cells are
// assembled on the unknowns of `coarse`. `next` gets the coarse cells for the next level. The
// coarse cells' matrices are formed on `threads` host threads; the fine cells of a coarse cell
// are summed in increasing order.
HostCsr by_cells(const HostLevel& fine, const HostCells& cells, const HostLevel& coarse,
                 HostCells* next, int threads);

// order.rs:19-179: the nested dissection order of the symmetric pattern `a` from the coordinates
// of each node (3 per node): item k is the old index of the new node k (order.cpp: coordinate
// bisection at the best of 5 quantile cuts per axis, the separator from the side with fewer
// coupled nodes, sets of at most 64 nodes not split; on all host threads).
std::vector<int64_t> nested_dissection(const HostCsr& a, const double* xyz);

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
