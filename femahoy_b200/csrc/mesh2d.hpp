// The quality triangle mesh of a planar straight-line graph (mesh2d.rs): the footprints of the
// prism parts across the extrusion axis. Host code: Delaunay refinement inserts 1 point at a time,
// each insertion depending on the mesh that the ones before it left, so it is sequential; the
// extrusion that multiplies the mesh by the planes runs on the device (prism.cu).
//
// The steps are those of mesh2d.rs, in its order, so that the points and triangles come out the
// same: the clean (merge, split at points and crossings), insertion in x order by a visibility
// walk with Lawson flips, segment recovery by splits, region labels from the largest triangle's
// centroid, then Ruppert refinement (ratio sqrt 2, the graded size field, concentric shells, the
// small input angle rule, circumcentres that encroach split the piece instead), and for a periodic
// mesh rounds of matching the 2 sides of the bounding box.
#pragma once
#include <array>
#include <cstdint>
#include <functional>
#include <map>
#include <vector>

namespace femgpu {

using P2 = std::array<double, 2>;

constexpr uint32_t kOutside = 0xffffffffu;  // mesh2d.rs:48 OUTSIDE
constexpr double kMinAngle = 20.7;          // mesh2d.rs:56 MIN_ANGLE (degrees)

struct Size2 {
    double max_size;    // the largest edge length of a triangle (about)
    double max_growth;  // the largest size ratio of 2 triangles side by side (about), above 1
};

struct Mesh2 {
    std::vector<P2> points;
    std::vector<std::array<uint32_t, 3>> triangles;  // counterclockwise
    std::vector<uint32_t> label;
    // The kept triangle across the edge opposite each point, or 0xffffffff (hull or outside).
    std::vector<std::array<uint32_t, 3>> across;
    // The input segments that hold each edge on a segment, keyed by its 2 points (smaller first).
    std::map<std::pair<uint32_t, uint32_t>, std::vector<uint32_t>> segments;
};

// The mesh of `points` and `segments` (pairs of point indices); `classify` labels a point inside
// a region that the segments bound, or returns kOutside. Only labelled triangles are refined and
// kept. `periodic`: the 2 opposite sides of the bounding box get matching points. Errors are
// thrown as std::runtime_error with the reference's texts.
Mesh2 quality_mesh(const std::vector<P2>& points, const std::vector<std::array<uint32_t, 2>>& segs,
                   Size2 size, const std::function<uint32_t(P2)>& classify, bool periodic);

}  // namespace femgpu
