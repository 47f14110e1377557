// The 2.5D tetrahedral mesh of prism parts (prism.rs): footprints across the extrusion axis,
// meshed together in 1 quality triangle mesh (mesh2d.hpp, host), extruded through the graded
// planes of the axis (grid.rs axis_planes, host) and cut into 3 tetrahedra per prism on the
// device (extrude.cu), where the assembly reads them.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "mesh2d.hpp"

namespace femgpu {

// prism.rs:29-37 Outline: a polygon (corners in either direction) or a circle.
struct Outline {
    bool circle = false;
    std::vector<P2> corners;
    P2 centre{0.0, 0.0};
    double radius = 0.0;
};

// prism.rs:40-44 Footprint.
struct Footprint {
    Outline outline;
    std::vector<Outline> holes;
};

// grid.rs:22-35 Part: a box, or the prism of `footprint` between lo and hi on the axis.
struct Part {
    std::string name;
    size_t material = 0;
    int64_t priority = 0;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool has_footprint = false;
    Footprint footprint;
};

// grid.rs:37-46 Spacing.
struct Spacing {
    double max_cell;
    double max_growth;
    size_t min_cells;
};

// prism.rs:71-88: the corners of an outline, a circle as a polygon of segments of at most
// `max_cell`, at least 64 and a multiple of 4.
std::vector<P2> outline_corners(const Outline& o, double max_cell);

// grid.rs:413-415: 1e-9 of the length of the planes.
double plane_tol(const std::vector<double>& p);

// grid.rs:418-484: the graded planes of axis d (keys at the part faces and `extra`, cells of at
// most max_cell, min_cells through each part, neighbours within max_growth).
std::vector<double> axis_planes(const std::vector<Part>& parts, int d, const Spacing& spacing,
                                const std::vector<double>& extra);

// prism.rs:383-392 Flat: the footprints' triangle mesh, the parts covering each label (highest
// priority first), the circle of each input segment (or none) and the circles.
struct Flat {
    Mesh2 mesh;
    std::vector<std::vector<uint32_t>> covers;
    std::vector<uint32_t> segment_circle;
    std::vector<std::pair<P2, double>> circles;
};

// prism.rs:397-527 footprints.
Flat footprints(const std::vector<Part>& parts, int axis, Size2 size,
                const std::vector<double>& surface, bool periodic);

// prism.rs:144-154: the 3 tetrahedra (local corners) of a prism whose 6 corners (bottom 0 1 2,
// top 3 4 5, 3 above 0) have the global numbers g; each quadrilateral face is cut through its
// corner of smallest number (Dompierre et al. 1999).
#ifdef __CUDACC__
__host__ __device__
#endif
inline void split_prism(const uint64_t g[6], int out[3][4]) {
    // The rotations of the prism that bring each corner to corner 0 (Dompierre et al., table 2).
    const int rot[6][6] = {{0, 1, 2, 3, 4, 5}, {1, 2, 0, 4, 5, 3}, {2, 0, 1, 5, 3, 4},
                           {3, 5, 4, 0, 2, 1}, {4, 3, 5, 1, 0, 2}, {5, 4, 3, 2, 1, 0}};
    int m = 0;
    for (int k = 1; k < 6; ++k)
        if (g[k] < g[m]) m = k;
    const int* r = rot[m];
    const uint64_t a = g[r[1]] < g[r[5]] ? g[r[1]] : g[r[5]];
    const uint64_t b = g[r[2]] < g[r[4]] ? g[r[2]] : g[r[4]];
    const int first[3][4] = {{0, 1, 2, 5}, {0, 1, 5, 4}, {0, 4, 5, 3}};
    const int second[3][4] = {{0, 1, 2, 4}, {0, 4, 2, 5}, {0, 4, 5, 3}};
    const int(*t)[4] = a < b ? first : second;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) out[i][j] = r[t[i][j]];
}

}  // namespace femgpu
