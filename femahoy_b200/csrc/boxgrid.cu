// The graded box grid of a list of parts (grid.rs:116-158 Grid::build, :292-330 assign, :234-254
// faces) and the hex mesh of its cells (heat.rs:1165-1210 number), on the device.
//
// The planes of each axis come from axis_planes (host, prism.cpp). Each cell then takes the part
// that holds its centre: 1 thread per cell replays the reference's pass over the parts in order
// (a later part takes the cell unless the holder has a higher priority; equal priorities with
// other materials are an error), and the first error in the reference's order (part, then cell)
// is the smallest key part * cells + cell, found with atomicMin. The mesh points are numbered in
// first use over the cells of the parts (cell order, VTK corner order) by the first-use keys of
// extrude.cu: an atomicMin per use and a prefix sum.
#include <algorithm>

#include "common.cuh"
#include "femgpu.h"
#include "prism.hpp"
#include "rust_format.hpp"

namespace femgpu {
namespace {

constexpr uint32_t VOID = 0xffffffffu;  // grid.rs:105
constexpr int BT = 256;

struct Dims {
    int64_t n[3];  // cells along each axis
    __host__ __device__ int64_t cells() const { return n[0] * n[1] * n[2]; }
};

// The part ranges as cell index ranges [first, end) per axis, priority and material.
struct PartRange {
    int64_t first[3], end[3];
    int64_t priority;
    uint64_t material;
};

__global__ void k_assign(Dims D, int nparts, const PartRange* pr, uint32_t* part,
                         unsigned long long* error) {
    const int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (cell >= D.cells()) return;
    const int64_t c[3] = {cell % D.n[0], (cell / D.n[0]) % D.n[1], cell / (D.n[0] * D.n[1])};
    int best = -1;
    for (int p = 0; p < nparts; ++p) {
        const PartRange& r = pr[p];
        bool in = true;
        for (int d = 0; d < 3; ++d) in = in && c[d] >= r.first[d] && c[d] < r.end[d];
        if (!in) continue;
        if (best >= 0 && pr[best].priority > r.priority) continue;
        if (best >= 0 && pr[best].priority == r.priority && pr[best].material != r.material) {
            atomicMin(error, (unsigned long long)p * (unsigned long long)D.cells() + cell);
            break;
        }
        best = p;
    }
    part[cell] = best < 0 ? VOID : (uint32_t)best;
}

// The grid point index of corner q (VTK order) of cell (i, j, k) (grid.rs:175-178, 201-214).
__device__ __forceinline__ int64_t corner_point(const Dims& D, const int64_t c[3], int q) {
    const int di = (q == 1 || q == 2 || q == 5 || q == 6), dj = (q == 2 || q == 3 || q == 6 || q == 7);
    const int dk = q >= 4;
    return (c[0] + di) + (D.n[0] + 1) * ((c[1] + dj) + (D.n[1] + 1) * (c[2] + dk));
}

__device__ __forceinline__ void cell_ijk(const Dims& D, int64_t cell, int64_t c[3]) {
    c[0] = cell % D.n[0];
    c[1] = (cell / D.n[0]) % D.n[1];
    c[2] = cell / (D.n[0] * D.n[1]);
}

__global__ void k_point_first(Dims D, const uint32_t* part, unsigned long long* first) {
    const int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (cell >= D.cells() || part[cell] == VOID) return;
    int64_t c[3];
    cell_ijk(D, cell, c);
    for (int q = 0; q < 8; ++q)
        atomicMin(&first[corner_point(D, c, q)], (unsigned long long)(cell * 8 + q));
}

__global__ void k_point_flags(Dims D, const uint32_t* part, const unsigned long long* first,
                              uint32_t* flag, uint32_t* solid) {
    const int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (cell >= D.cells()) return;
    solid[cell] = part[cell] != VOID;
    int64_t c[3];
    cell_ijk(D, cell, c);
    for (int q = 0; q < 8; ++q)
        flag[cell * 8 + q] =
            part[cell] != VOID && first[corner_point(D, c, q)] == (unsigned long long)(cell * 8 + q);
}

// The mesh points (grid point ijk and coordinates), the grid point's number, and each cell of
// a part as a mesh cell: its 8 points, its part and its grid cell; its boundary sides flagged.
__global__ void k_mesh(Dims D, const double* px, const double* py, const double* pz,
                       const uint32_t* part, const uint32_t* flag, const int64_t* pos,
                       const int64_t* rank, uint32_t* number, uint32_t* ijk, double* xyz) {
    const int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (cell >= D.cells() || part[cell] == VOID) return;
    int64_t c[3];
    cell_ijk(D, cell, c);
    for (int q = 0; q < 8; ++q) {
        if (!flag[cell * 8 + q]) continue;
        const int64_t n = pos[cell * 8 + q];
        const int64_t g[3] = {c[0] + (q == 1 || q == 2 || q == 5 || q == 6),
                              c[1] + (q == 2 || q == 3 || q == 6 || q == 7), c[2] + (q >= 4)};
        number[corner_point(D, c, q)] = (uint32_t)n;
        for (int d = 0; d < 3; ++d) ijk[3 * n + d] = (uint32_t)g[d];
        xyz[3 * n] = px[g[0]];
        xyz[3 * n + 1] = py[g[1]];
        xyz[3 * n + 2] = pz[g[2]];
    }
}

__global__ void k_cells(Dims D, const uint32_t* part, const int64_t* rank, const uint32_t* number,
                        uint32_t* cells, uint64_t* cell_of, uint32_t* mesh_part, uint32_t* side_flag) {
    const int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (cell >= D.cells()) return;
    int64_t c[3];
    cell_ijk(D, cell, c);
    for (int s = 0; s < 6; ++s) side_flag[cell * 6 + s] = 0;
    if (part[cell] == VOID) return;
    const int64_t e = rank[cell];
    for (int q = 0; q < 8; ++q) cells[8 * e + q] = number[corner_point(D, c, q)];
    cell_of[e] = (uint64_t)cell;
    mesh_part[e] = part[cell];
    // Side::ALL order: -x, +x, -y, +y, -z, +z (grid.rs:54-81); a side is a face of the model when
    // no cell of a part is beyond it (grid.rs:234-254).
    for (int s = 0; s < 6; ++s) {
        const int d = s / 2;
        const bool positive = s % 2;
        int64_t n[3] = {c[0], c[1], c[2]};
        bool outside;
        if (positive) {
            outside = n[d] + 1 >= D.n[d];
            n[d] += 1;
        } else {
            outside = n[d] == 0;
            n[d] -= 1;
        }
        if (!outside) outside = part[n[0] + D.n[0] * (n[1] + D.n[1] * n[2])] == VOID;
        side_flag[cell * 6 + s] = outside;
    }
}

__global__ void k_faces(int64_t slots, const uint32_t* side_flag, const int64_t* fpos,
                        uint64_t* face_cell, uint8_t* face_side) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= slots || !side_flag[s]) return;
    face_cell[fpos[s]] = (uint64_t)(s / 6);
    face_side[fpos[s]] = (uint8_t)(s % 6);
}

unsigned grid_of(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + BT - 1) / BT); }

}  // namespace

// grid.rs:108-114 Grid and heat.rs:1153-1162 Numbering, with the mesh also on the device.
struct BoxGrid {
    std::vector<double> planes[3];
    std::vector<uint32_t> part;       // per grid cell, VOID for none
    std::vector<double> points;       // 3 per mesh point
    std::vector<uint32_t> ijk;        // 3 per mesh point
    std::vector<uint32_t> cells;      // 8 per mesh cell (VTK order)
    std::vector<uint64_t> cell_of;    // the grid cell of each mesh cell
    std::vector<uint32_t> mesh_part;  // the part of each mesh cell
    std::vector<uint64_t> face_cell;  // the model's faces (grid.rs:234-254), in cell then side order
    std::vector<uint8_t> face_side;
    DevBuf<double> d_points;
    DevBuf<uint32_t> d_cells;
};

// The host steps first (the checks, the planes), then the stream *stream is created for the
// device steps (the caller destroys it).
void box_grid(const std::vector<Part>& parts, const Spacing& spacing,
              const std::vector<double> extra[3], size_t max_points, const std::string& refusal,
              BoxGrid* out, cudaStream_t* stream) {
    auto fail = [](const std::string& t) { throw Failure(FEMGPU_ERR_INVALID, t); };
    const char* axis[3] = {"x", "y", "z"};
    if (parts.empty()) fail("the model has no part");
    if (!(spacing.max_cell > 0.0 && std::isfinite(spacing.max_cell)))
        fail("max_cell must be a number above 0");
    if (!(spacing.max_growth > 1.0 && std::isfinite(spacing.max_growth)))
        fail("max_growth must be a number above 1");
    if (spacing.min_cells == 0) fail("min_cells must be 1 or more");
    for (const Part& p : parts)
        for (int d = 0; d < 3; ++d)
            if (!(std::isfinite(p.lo[d]) && std::isfinite(p.hi[d]) && p.lo[d] < p.hi[d]))
                fail("part " + p.name + ": its " + axis[d] +
                     " range must be 2 finite numbers, the first smaller");
    for (int d = 0; d < 3; ++d) {
        try {
            out->planes[d] = axis_planes(parts, d, spacing, extra[d]);
        } catch (const Failure&) {
            throw;
        } catch (const std::runtime_error& e) {
            fail(e.what());
        }
    }
    Dims D{{(int64_t)out->planes[0].size() - 1, (int64_t)out->planes[1].size() - 1,
            (int64_t)out->planes[2].size() - 1}};
    const int64_t ncells = D.cells();
    if ((uint64_t)(D.n[0] + 1) * (D.n[1] + 1) * (D.n[2] + 1) > 0xffffffffull)
        throw Failure(FEMGPU_ERR_TOO_LARGE, refusal);
    // Each part's cells along each axis: the planes from its lo to its hi (grid.rs:295-301).
    std::vector<PartRange> pr(parts.size());
    for (size_t k = 0; k < parts.size(); ++k) {
        for (int d = 0; d < 3; ++d) {
            const auto& pl = out->planes[d];
            const double t = plane_tol(pl);
            pr[k].first[d] = std::lower_bound(pl.begin(), pl.end(), parts[k].lo[d] - t) - pl.begin();
            pr[k].end[d] = std::lower_bound(pl.begin(), pl.end(), parts[k].hi[d] - t) - pl.begin();
        }
        pr[k].priority = parts[k].priority;
        pr[k].material = parts[k].material;
    }
    FG_CUDA(cudaStreamCreateWithFlags(stream, cudaStreamNonBlocking));
    const cudaStream_t s = *stream;
    DevBuf<PartRange> d_pr;
    d_pr.upload(pr.data(), pr.size(), s);
    DevBuf<uint32_t> part(ncells);
    DevBuf<unsigned long long> error(1);
    FG_CUDA(cudaMemsetAsync(error.p, 0xff, 8, s));
    k_assign<<<grid_of(ncells), BT, 0, s>>>(D, (int)parts.size(), d_pr.p, part.p, error.p);
    unsigned long long err = 0;
    FG_CUDA(cudaMemcpyAsync(&err, error.p, 8, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    if (err != ~0ull) {
        // The reference's first overlap: part p at cell, against the part that held it then.
        const int64_t p = (int64_t)(err / (uint64_t)ncells), cell = (int64_t)(err % (uint64_t)ncells);
        const int64_t c[3] = {cell % D.n[0], (cell / D.n[0]) % D.n[1], cell / (D.n[0] * D.n[1])};
        int best = -1;
        for (int64_t q = 0; q < p; ++q) {
            bool in = true;
            for (int d = 0; d < 3; ++d) in = in && c[d] >= pr[q].first[d] && c[d] < pr[q].end[d];
            if (in && !(best >= 0 && pr[best].priority > pr[q].priority)) best = (int)q;
        }
        double x[3];
        for (int d = 0; d < 3; ++d)
            x[d] = 0.5 * (out->planes[d][c[d]] + out->planes[d][c[d] + 1]);
        fail("parts " + parts[best].name + " and " + parts[p].name + " overlap at (" +
             rust_display(x[0]) + ", " + rust_display(x[1]) + ", " + rust_display(x[2]) +
             ") with the same priority and other materials: give the part that must hold the "
             "overlap a higher priority");
    }
    // The mesh points in first use over the cells of the parts.
    const int64_t npoints_grid = (D.n[0] + 1) * (D.n[1] + 1) * (D.n[2] + 1);
    DevBuf<unsigned long long> first(npoints_grid);
    FG_CUDA(cudaMemsetAsync(first.p, 0xff, first.bytes(), s));
    k_point_first<<<grid_of(ncells), BT, 0, s>>>(D, part.p, first.p);
    DevBuf<uint32_t> flag(8 * ncells), solid(ncells);
    k_point_flags<<<grid_of(ncells), BT, 0, s>>>(D, part.p, first.p, flag.p, solid.p);
    DevBuf<int64_t> pos(8 * ncells + 1), rank(ncells + 1);
    exclusive_scan32(flag.p, pos.p, 8 * ncells, s);
    exclusive_scan32(solid.p, rank.p, ncells, s);
    int64_t counts[2] = {0, 0};
    FG_CUDA(cudaMemcpyAsync(&counts[0], pos.p + 8 * ncells, 8, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaMemcpyAsync(&counts[1], rank.p + ncells, 8, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    const int64_t npts = counts[0], nmesh = counts[1];
    if ((size_t)npts > max_points) throw Failure(FEMGPU_ERR_TOO_LARGE, refusal);
    DevBuf<double> px, py, pz;
    px.upload(out->planes[0].data(), out->planes[0].size(), s);
    py.upload(out->planes[1].data(), out->planes[1].size(), s);
    pz.upload(out->planes[2].data(), out->planes[2].size(), s);
    DevBuf<uint32_t> number(npoints_grid), ijk(3 * std::max<int64_t>(npts, 1));
    out->d_points.alloc(3 * std::max<int64_t>(npts, 1));
    k_mesh<<<grid_of(ncells), BT, 0, s>>>(D, px.p, py.p, pz.p, part.p, flag.p, pos.p, rank.p,
                                          number.p, ijk.p, out->d_points.p);
    out->d_cells.alloc(8 * std::max<int64_t>(nmesh, 1));
    DevBuf<uint64_t> cell_of(std::max<int64_t>(nmesh, 1));
    DevBuf<uint32_t> mesh_part(std::max<int64_t>(nmesh, 1)), side_flag(6 * ncells);
    k_cells<<<grid_of(ncells), BT, 0, s>>>(D, part.p, rank.p, number.p, out->d_cells.p, cell_of.p,
                                           mesh_part.p, side_flag.p);
    DevBuf<int64_t> fpos(6 * ncells + 1);
    exclusive_scan32(side_flag.p, fpos.p, 6 * ncells, s);
    int64_t nfaces = 0;
    FG_CUDA(cudaMemcpyAsync(&nfaces, fpos.p + 6 * ncells, 8, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    DevBuf<uint64_t> face_cell(std::max<int64_t>(nfaces, 1));
    DevBuf<uint8_t> face_side(std::max<int64_t>(nfaces, 1));
    k_faces<<<grid_of(6 * ncells), BT, 0, s>>>(6 * ncells, side_flag.p, fpos.p, face_cell.p,
                                               face_side.p);
    FG_CUDA(cudaGetLastError());
    out->part.resize(ncells);
    out->points.resize(3 * npts);
    out->ijk.resize(3 * npts);
    out->cells.resize(8 * nmesh);
    out->cell_of.resize(nmesh);
    out->mesh_part.resize(nmesh);
    out->face_cell.resize(nfaces);
    out->face_side.resize(nfaces);
    part.download(out->part.data(), ncells, s);
    out->d_points.download(out->points.data(), 3 * npts, s);
    ijk.download(out->ijk.data(), 3 * npts, s);
    out->d_cells.download(out->cells.data(), 8 * nmesh, s);
    cell_of.download(out->cell_of.data(), nmesh, s);
    mesh_part.download(out->mesh_part.data(), nmesh, s);
    face_cell.download(out->face_cell.data(), nfaces, s);
    face_side.download(out->face_side.data(), nfaces, s);
    FG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace femgpu

// ------------------------------------------------------------------ C ABI
using namespace femgpu;

struct femgpu_boxgrid {
    BoxGrid g;
};

namespace {

template <class F>
int guard(F f) {
    try {
        f();
        return FEMGPU_OK;
    } catch (const Failure& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("out of host memory");
        return FEMGPU_ERR_TOO_LARGE;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return FEMGPU_ERR_INVALID;
    }
}

}  // namespace

extern "C" {

int femgpu_box_grid(const femgpu_part* parts, size_t nparts, const femgpu_spacing* spacing,
                    const double* const* extra, const size_t* nextra, size_t max_points,
                    const char* refusal, femgpu_boxgrid** out) {
    return guard([&] {
        if (!out || !spacing || (nparts && !parts))
            throw Failure(FEMGPU_ERR_INVALID, "a null argument");
        std::vector<Part> ps(nparts);
        for (size_t k = 0; k < nparts; ++k) {
            ps[k].name = parts[k].name ? parts[k].name : "";
            ps[k].material = parts[k].material;
            ps[k].priority = parts[k].priority;
            for (int d = 0; d < 3; ++d) {
                ps[k].lo[d] = parts[k].lo[d];
                ps[k].hi[d] = parts[k].hi[d];
            }
        }
        std::vector<double> ex[3];
        for (int d = 0; d < 3; ++d)
            if (extra && nextra && nextra[d]) {
                if (!extra[d]) throw Failure(FEMGPU_ERR_INVALID, "a null extra list");
                ex[d].assign(extra[d], extra[d] + nextra[d]);
            }
        const Spacing sp{spacing->max_cell, spacing->max_growth, spacing->min_cells};
        cudaStream_t s = nullptr;
        auto* h = new femgpu_boxgrid;
        try {
            box_grid(ps, sp, ex, max_points, refusal ? refusal : "", &h->g, &s);
        } catch (...) {
            if (s) {
                cudaStreamSynchronize(s);
                cudaStreamDestroy(s);
            }
            delete h;
            throw;
        }
        cudaStreamDestroy(s);
        *out = h;
    });
}

int femgpu_boxgrid_sizes(const femgpu_boxgrid* g, femgpu_boxgrid_counts* n) {
    return guard([&] {
        if (!g || !n) throw Failure(FEMGPU_ERR_INVALID, "a null argument");
        for (int d = 0; d < 3; ++d) n->planes[d] = g->g.planes[d].size();
        n->grid_cells = g->g.part.size();
        n->points = g->g.points.size() / 3;
        n->cells = g->g.cell_of.size();
        n->faces = g->g.face_cell.size();
    });
}

int femgpu_boxgrid_copy(const femgpu_boxgrid* g, double* const* planes, uint32_t* part,
                        double* points, uint32_t* ijk, uint32_t* cells, uint64_t* cell_of,
                        uint32_t* mesh_part, uint64_t* face_cell, uint8_t* face_side) {
    return guard([&] {
        if (!g) throw Failure(FEMGPU_ERR_INVALID, "a null grid");
        const BoxGrid& b = g->g;
        auto put = [](auto* dst, const auto& v) {
            if (dst) std::copy(v.begin(), v.end(), dst);
        };
        if (planes)
            for (int d = 0; d < 3; ++d) put(planes[d], b.planes[d]);
        put(part, b.part);
        put(points, b.points);
        put(ijk, b.ijk);
        put(cells, b.cells);
        put(cell_of, b.cell_of);
        put(mesh_part, b.mesh_part);
        put(face_cell, b.face_cell);
        put(face_side, b.face_side);
    });
}

int femgpu_boxgrid_device(const femgpu_boxgrid* g, const double** points, const uint32_t** cells) {
    return guard([&] {
        if (!g) throw Failure(FEMGPU_ERR_INVALID, "a null grid");
        if (points) *points = g->g.d_points.p;
        if (cells) *cells = g->g.d_cells.p;
    });
}

void femgpu_boxgrid_free(femgpu_boxgrid* g) { delete g; }

}  // extern "C"
