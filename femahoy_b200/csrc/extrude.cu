// The extrusion of the footprints' triangle mesh through the planes of the axis into tetrahedra,
// on the device (prism.rs:216-379), and the C ABI of the prism mesh.
//
// Each (triangle, layer) pair is a prism; its part comes from the label's cover list and the
// layer. The reference numbers the points in the order of first use over the prisms (triangle
// major, layer minor, corners 0-5); here every use of a point slot (plane * points + flat point)
// has a key (prism * 6 + corner), a slot's number is the rank of its smallest key among all first
// keys, found with 1 atomicMin per use and 1 prefix sum over the keys. The same scheme renumbers
// the points of the solid tetrahedra in first use over them (corners in order). A tetrahedron's
// face is on the boundary when it lies on a face of its prism whose neighbouring prism (across
// the triangle's edge in the same layer, or the layer above or below) is void or hollow: the
// mesh is conforming (each quadrilateral is cut through its corner of smallest number), so the
// neighbour holds the same triangle. Built with -fmad=false: the volume's sign is the reference's.
#include <algorithm>
#include <map>
#include <set>

#include "common.cuh"
#include "femgpu.h"
#include "prism.hpp"

namespace femgpu {
namespace {

constexpr uint32_t NONE32 = 0xffffffffu;
constexpr unsigned long long NONE64 = ~0ull;
constexpr int XT = 256;

// The tetrahedron's faces, counterclockwise from outside for a positive volume (prism.rs:296).
__constant__ int c_face[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};

struct Layers {
    const double* flat;      // 2 per flat point
    const uint32_t* tri;     // 3 per triangle
    const uint32_t* label;   // per triangle
    const uint32_t* across;  // 3 per triangle: the triangle across the edge opposite each point
    const uint32_t* part_of; // label * layers + layer: the part, or NONE
    const double* planes;
    int64_t nv, nt, layers;
    int axis;
};

__device__ __forceinline__ uint32_t prism_part(const Layers& L, int64_t q) {
    const int64_t t = q / L.layers, k = q % L.layers;
    return L.part_of[(int64_t)L.label[t] * L.layers + k];
}

// The slot (plane * nv + flat point) of corner c of prism q (bottom 0 1 2, top 3 4 5).
__device__ __forceinline__ uint64_t prism_slot(const Layers& L, int64_t q, int c) {
    const int64_t t = q / L.layers, k = q % L.layers;
    return (uint64_t)(k + c / 3) * (uint64_t)L.nv + L.tri[t * 3 + c % 3];
}

__global__ void k_first_use(Layers L, unsigned long long* first) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= L.nt * L.layers || prism_part(L, q) == NONE32) return;
    for (int c = 0; c < 6; ++c) atomicMin(&first[prism_slot(L, q, c)], (unsigned long long)(q * 6 + c));
}

__global__ void k_first_flags(Layers L, const unsigned long long* first, uint32_t* flag) {
    const int64_t key = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (key >= L.nt * L.layers * 6) return;
    const int64_t q = key / 6;
    flag[key] = prism_part(L, q) != NONE32 && first[prism_slot(L, q, (int)(key % 6))] == (uint64_t)key;
}

// The numbered points: number[slot], the point's coordinates and its flat point.
__global__ void k_points(Layers L, const uint32_t* flag, const int64_t* pos, uint32_t* number,
                         double* xyz, uint32_t* flat_of) {
    const int64_t key = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (key >= L.nt * L.layers * 6 || !flag[key]) return;
    const int64_t q = key / 6, t = q / L.layers, k = q % L.layers;
    const int c = (int)(key % 6);
    const uint32_t v = L.tri[t * 3 + c % 3];
    const int64_t n = pos[key];
    number[prism_slot(L, q, c)] = (uint32_t)n;
    double* p = xyz + 3 * n;
    p[L.axis] = L.planes[k + c / 3];
    p[(L.axis + 1) % 3] = L.flat[2 * v];
    p[(L.axis + 2) % 3] = L.flat[2 * v + 1];
    flat_of[n] = v;
}

__global__ void k_solid_flags(Layers L, uint32_t* flag) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q < L.nt * L.layers) flag[q] = prism_part(L, q) != NONE32;
}

// The signed volume with the reference's operation order (prism.rs:156-162).
__device__ double tet_volume(const double* xyz, const uint32_t* t) {
    const double* p0 = xyz + 3 * (size_t)t[0];
    double d[3][3];
    for (int k = 0; k < 3; ++k)
        for (int c = 0; c < 3; ++c) d[k][c] = __dsub_rn(xyz[3 * (size_t)t[k + 1] + c], p0[c]);
    const double(&a)[3] = d[0], (&b)[3] = d[1], (&c)[3] = d[2];
    const double x = __dmul_rn(a[0], __dsub_rn(__dmul_rn(b[1], c[2]), __dmul_rn(b[2], c[1])));
    const double y = __dmul_rn(a[1], __dsub_rn(__dmul_rn(b[0], c[2]), __dmul_rn(b[2], c[0])));
    const double z = __dmul_rn(a[2], __dsub_rn(__dmul_rn(b[0], c[1]), __dmul_rn(b[1], c[0])));
    return __ddiv_rn(__dadd_rn(__dsub_rn(x, y), z), 6.0);
}

// The 3 tetrahedra of each solid prism, in prism order, with a positive volume.
__global__ void k_tets(Layers L, const int64_t* tbase, const uint32_t* number, const double* xyz,
                       uint32_t* tets, uint32_t* part, uint32_t* prism_of) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= L.nt * L.layers) return;
    const uint32_t p = prism_part(L, q);
    if (p == NONE32) return;
    uint64_t g[6];
    uint32_t node[6];
    for (int c = 0; c < 6; ++c) {
        g[c] = prism_slot(L, q, c);
        node[c] = number[g[c]];
    }
    int local[3][4];
    split_prism(g, local);
    for (int i = 0; i < 3; ++i) {
        uint32_t t[4];
        for (int j = 0; j < 4; ++j) t[j] = node[local[i][j]];
        if (tet_volume(xyz, t) < 0.0) {
            const uint32_t s = t[2];
            t[2] = t[3];
            t[3] = s;
        }
        const int64_t e = 3 * tbase[q] + i;
        for (int j = 0; j < 4; ++j) tets[4 * e + j] = t[j];
        part[e] = p;
        prism_of[e] = (uint32_t)q;
    }
}

__global__ void k_keep_flags(int64_t ntets, const uint32_t* part, const uint8_t* hollow,
                             uint32_t* flag) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < ntets) flag[e] = !hollow[part[e]];
}

// First use of each point over the kept tetrahedra (kept index * 4 + corner).
__global__ void k_kept_first(int64_t ntets, const uint32_t* flag, const int64_t* tet_of,
                             const uint32_t* tets, unsigned long long* first) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ntets || !flag[e]) return;
    for (int j = 0; j < 4; ++j)
        atomicMin(&first[tets[4 * e + j]], (unsigned long long)(tet_of[e] * 4 + j));
}

__global__ void k_kept_point_flags(int64_t ntets, const uint32_t* flag, const int64_t* tet_of,
                                   const uint32_t* tets, const unsigned long long* first,
                                   uint32_t* pflag) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ntets || !flag[e]) return;
    for (int j = 0; j < 4; ++j) {
        const uint64_t key = (uint64_t)tet_of[e] * 4 + j;
        pflag[key] = first[tets[4 * e + j]] == key;
    }
}

__global__ void k_kept_points(int64_t npts, const unsigned long long* first, const int64_t* ppos,
                              const double* xyz, uint32_t* point_of, double* out) {
    const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (v >= npts || first[v] == NONE64) return;
    const int64_t n = ppos[first[v]];
    point_of[v] = (uint32_t)n;
    for (int c = 0; c < 3; ++c) out[3 * n + c] = xyz[3 * v + c];
}

// The kept tetrahedra in their new numbers, and each one's boundary faces sorted by their nodes
// into 4 slots (flags mark the used ones).
__global__ void k_kept_tets(Layers L, int64_t ntets, const uint32_t* flag, const int64_t* tet_of,
                            const uint32_t* tets, const uint32_t* part, const uint32_t* prism_of,
                            const uint32_t* number, const uint32_t* point_of, const uint8_t* hollow,
                            const uint32_t* flat_of, uint32_t* out_tets, uint32_t* out_part,
                            uint32_t* face_flag, uint32_t* face_rec) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ntets || !flag[e]) return;
    const int64_t j = tet_of[e];
    const uint32_t* t = tets + 4 * e;
    for (int c = 0; c < 4; ++c) out_tets[4 * j + c] = point_of[t[c]];
    out_part[j] = part[e];
    const int64_t q = prism_of[e], tri = q / L.layers, k = q % L.layers;
    uint32_t node[6];
    for (int c = 0; c < 6; ++c) node[c] = number[prism_slot(L, q, c)];
    // Up to 4 boundary faces: (new nodes, beyond, flat points).
    uint32_t rec[4][7];
    int nf = 0;
    for (int f = 0; f < 4; ++f) {
        int corner[3];
        for (int i = 0; i < 3; ++i) {
            const uint32_t v = t[c_face[f][i]];
            corner[i] = 0;
            for (int c = 0; c < 6; ++c)
                if (node[c] == v) corner[i] = c;
        }
        // Which face of the prism holds it: bottom, top, or the quadrilateral on the edge
        // opposite flat corner m.
        int64_t nq_part = -2;  // -2: inside the prism
        const bool bottom = corner[0] < 3 && corner[1] < 3 && corner[2] < 3;
        const bool top = corner[0] >= 3 && corner[1] >= 3 && corner[2] >= 3;
        if (bottom) {
            nq_part = k > 0 ? (int64_t)prism_part(L, q - 1) : -1;
        } else if (top) {
            nq_part = k + 1 < L.layers ? (int64_t)prism_part(L, q + 1) : -1;
        } else {
            for (int m = 0; m < 3; ++m) {
                const int a = corner[0] % 3, b = corner[1] % 3, c = corner[2] % 3;
                if (a != m && b != m && c != m) {
                    const uint32_t nt = L.across[tri * 3 + m];
                    nq_part = nt == NONE32 ? -1
                                           : (int64_t)L.part_of[(int64_t)L.label[nt] * L.layers + k];
                    break;
                }
            }
        }
        if (nq_part == -2) continue;
        uint32_t beyond;
        if (nq_part == -1 || nq_part == (int64_t)NONE32)
            beyond = NONE32;
        else if (hollow[nq_part])
            beyond = (uint32_t)nq_part;
        else
            continue;  // a solid tetrahedron on the other side
        uint32_t* r = rec[nf++];
        for (int i = 0; i < 3; ++i) {
            r[i] = point_of[t[c_face[f][i]]];
            r[4 + i] = flat_of[t[c_face[f][i]]];
        }
        r[3] = beyond;
    }
    // Sort by the nodes (insertion; at most 4).
    for (int a = 1; a < nf; ++a)
        for (int b = a; b > 0; --b) {
            uint32_t* x = rec[b - 1];
            uint32_t* y = rec[b];
            const bool less = y[0] != x[0] ? y[0] < x[0] : y[1] != x[1] ? y[1] < x[1] : y[2] < x[2];
            if (!less) break;
            for (int i = 0; i < 7; ++i) {
                const uint32_t s = x[i];
                x[i] = y[i];
                y[i] = s;
            }
        }
    for (int s = 0; s < 4; ++s) {
        face_flag[4 * j + s] = s < nf;
        if (s < nf)
            for (int i = 0; i < 7; ++i) face_rec[(4 * j + s) * 7 + i] = rec[s][i];
    }
}

__global__ void k_faces(int64_t slots, const uint32_t* face_flag, const int64_t* fpos,
                        const uint32_t* face_rec, uint32_t* out) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= slots || !face_flag[s]) return;
    const int64_t n = fpos[s];
    out[8 * n] = (uint32_t)(s / 4);
    for (int i = 0; i < 7; ++i) out[8 * n + 1 + i] = face_rec[7 * s + i];
}

}  // namespace

// prism.rs:117-132 TetMesh, with the points and tetrahedra also resident on the device.
struct TetMesh {
    std::vector<double> points;  // 3 per point
    std::vector<uint32_t> tets;  // 4 per tetrahedron, positive volume
    std::vector<uint32_t> part;
    std::vector<uint32_t> face_nodes, face_tet, face_beyond;
    std::vector<uint64_t> face_circle_start;  // faces + 1 offsets into face_circles
    std::vector<uint32_t> face_circles;
    std::vector<std::pair<P2, double>> circles;
    size_t triangles = 0, planes = 0;
    DevBuf<double> d_points;
    DevBuf<uint32_t> d_tets, d_part;
};

// prism.rs:185-380 mesh_hollow.
// The host steps first (footprints, planes, the parts of the layers, their errors), then the
// stream *stream is created for the device steps (the caller destroys it).
void prism_mesh(const std::vector<Part>& parts, int axis, const Spacing& spacing,
                size_t max_points, const std::string& refusal, bool periodic,
                const std::vector<uint8_t>& hollow_in, TetMesh* out, cudaStream_t* stream) {
    std::vector<uint8_t> hollow(parts.size(), 0);
    for (size_t k = 0; k < parts.size() && k < hollow_in.size(); ++k) hollow[k] = hollow_in[k] != 0;
    if (parts.empty()) throw Failure(FEMGPU_ERR_INVALID, "the model has no part");
    if (!(spacing.max_cell > 0.0 && std::isfinite(spacing.max_cell)))
        throw Failure(FEMGPU_ERR_INVALID, "max_cell must be a number above 0");
    Flat flat;
    std::vector<double> planes;
    try {
        flat = footprints(parts, axis, Size2{spacing.max_cell, spacing.max_growth},
                          std::vector<double>(parts.size(), INFINITY), periodic);
        planes = axis_planes(parts, axis, spacing, {});
    } catch (const Failure&) {
        throw;
    } catch (const std::runtime_error& e) {
        throw Failure(FEMGPU_ERR_INVALID, e.what());
    }
    const double t = plane_tol(planes);
    const int64_t layers = (int64_t)planes.size() - 1;
    // The part of each layer of each label (highest priority first), and the overlap check.
    std::vector<uint32_t> part_of(flat.covers.size() * layers, NONE32);
    for (size_t l = 0; l < flat.covers.size(); ++l) {
        const auto& list = flat.covers[l];
        for (int64_t k = 0; k < layers; ++k) {
            const double z0 = planes[k], z1 = planes[k + 1];
            auto holds = [&](const Part& p) { return p.lo[axis] <= z0 + t && p.hi[axis] >= z1 - t; };
            size_t f = 0;
            while (f < list.size() && !holds(parts[list[f]])) ++f;
            if (f == list.size()) continue;
            const Part& a = parts[list[f]];
            for (uint32_t other : list) {
                const Part& b = parts[other];
                if (other != list[f] && holds(b) && b.priority == a.priority &&
                    b.material != a.material)
                    throw Failure(FEMGPU_ERR_INVALID,
                                  "parts " + b.name + " and " + a.name +
                                      " overlap with the same priority and other materials: give "
                                      "the part that must hold the overlap a higher priority");
            }
            part_of[l * layers + k] = list[f];
        }
    }
    const Mesh2& m = flat.mesh;
    const int64_t nv = (int64_t)m.points.size(), nt = (int64_t)m.triangles.size();
    if ((uint64_t)nv * planes.size() > 0xffffffffull)
        throw Failure(FEMGPU_ERR_TOO_LARGE, "the mesh has too many points: use a larger max_cell");
    FG_CUDA(cudaStreamCreateWithFlags(stream, cudaStreamNonBlocking));
    const cudaStream_t s = *stream;
    const int64_t nq = nt * layers, slots = nv * (int64_t)planes.size();
    // The flat mesh and the tables on the device.
    DevBuf<double> d_flat, d_planes;
    DevBuf<uint32_t> d_tri, d_label, d_across, d_part_of;
    DevBuf<uint8_t> d_hollow;
    d_flat.upload(m.points.empty() ? nullptr : m.points[0].data(), 2 * nv, s);
    d_tri.upload(m.triangles.empty() ? nullptr : m.triangles[0].data(), 3 * nt, s);
    d_label.upload(m.label.data(), nt, s);
    d_across.upload(m.across.empty() ? nullptr : m.across[0].data(), 3 * nt, s);
    d_part_of.upload(part_of.data(), part_of.size(), s);
    d_planes.upload(planes.data(), planes.size(), s);
    d_hollow.upload(hollow.data(), hollow.size(), s);
    Layers L{d_flat.p, d_tri.p, d_label.p, d_across.p, d_part_of.p, d_planes.p,
             nv, nt, layers, axis};
    auto grid = [](int64_t n) { return (unsigned)std::max<int64_t>(1, (n + XT - 1) / XT); };
    // The points, numbered in first use over the prisms.
    DevBuf<unsigned long long> first(slots);
    FG_CUDA(cudaMemsetAsync(first.p, 0xff, first.bytes(), s));
    k_first_use<<<grid(nq), XT, 0, s>>>(L, first.p);
    DevBuf<uint32_t> flag(6 * nq);
    DevBuf<int64_t> pos(6 * nq + 1);
    k_first_flags<<<grid(6 * nq), XT, 0, s>>>(L, first.p, flag.p);
    exclusive_scan32(flag.p, pos.p, 6 * nq, s);
    int64_t npts = 0;
    FG_CUDA(cudaMemcpyAsync(&npts, pos.p + 6 * nq, 8, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    if ((size_t)npts > max_points) throw Failure(FEMGPU_ERR_TOO_LARGE, refusal);
    DevBuf<uint32_t> number(slots), flat_of(std::max<int64_t>(npts, 1));
    DevBuf<double> xyz(3 * std::max<int64_t>(npts, 1));
    k_points<<<grid(6 * nq), XT, 0, s>>>(L, flag.p, pos.p, number.p, xyz.p, flat_of.p);
    // The tetrahedra of the solid (non-void) prisms.
    DevBuf<uint32_t> pflag(nq);
    DevBuf<int64_t> tbase(nq + 1);
    k_solid_flags<<<grid(nq), XT, 0, s>>>(L, pflag.p);
    exclusive_scan32(pflag.p, tbase.p, nq, s);
    int64_t nprisms = 0;
    FG_CUDA(cudaMemcpyAsync(&nprisms, tbase.p + nq, 8, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    const int64_t ntets = 3 * nprisms;
    DevBuf<uint32_t> tets(4 * std::max<int64_t>(ntets, 1)), part(std::max<int64_t>(ntets, 1)),
        prism_of(std::max<int64_t>(ntets, 1));
    k_tets<<<grid(nq), XT, 0, s>>>(L, tbase.p, number.p, xyz.p, tets.p, part.p, prism_of.p);
    // The tetrahedra of parts that are not hollow, renumbered with their points.
    DevBuf<uint32_t> keep(std::max<int64_t>(ntets, 1));
    DevBuf<int64_t> tet_of(ntets + 1);
    k_keep_flags<<<grid(ntets), XT, 0, s>>>(ntets, part.p, d_hollow.p, keep.p);
    exclusive_scan32(keep.p, tet_of.p, ntets, s);
    int64_t nkept = 0;
    FG_CUDA(cudaMemcpyAsync(&nkept, tet_of.p + ntets, 8, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    if (nkept == 0) throw Failure(FEMGPU_ERR_INVALID, "the parts hold no volume");
    DevBuf<unsigned long long> first2(npts);
    FG_CUDA(cudaMemsetAsync(first2.p, 0xff, first2.bytes(), s));
    k_kept_first<<<grid(ntets), XT, 0, s>>>(ntets, keep.p, tet_of.p, tets.p, first2.p);
    DevBuf<uint32_t> kflag(4 * nkept);
    DevBuf<int64_t> kpos(4 * nkept + 1);
    kflag.zero(s);
    k_kept_point_flags<<<grid(ntets), XT, 0, s>>>(ntets, keep.p, tet_of.p, tets.p, first2.p,
                                                   kflag.p);
    exclusive_scan32(kflag.p, kpos.p, 4 * nkept, s);
    int64_t nkpts = 0;
    FG_CUDA(cudaMemcpyAsync(&nkpts, kpos.p + 4 * nkept, 8, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    DevBuf<uint32_t> point_of(npts);
    out->d_points.alloc(3 * nkpts);
    k_kept_points<<<grid(npts), XT, 0, s>>>(npts, first2.p, kpos.p, xyz.p, point_of.p,
                                            out->d_points.p);
    out->d_tets.alloc(4 * nkept);
    out->d_part.alloc(nkept);
    DevBuf<uint32_t> face_flag(4 * nkept), face_rec(28 * nkept);
    k_kept_tets<<<grid(ntets), XT, 0, s>>>(L, ntets, keep.p, tet_of.p, tets.p, part.p, prism_of.p,
                                           number.p, point_of.p, d_hollow.p, flat_of.p,
                                           out->d_tets.p, out->d_part.p, face_flag.p, face_rec.p);
    DevBuf<int64_t> fpos(4 * nkept + 1);
    exclusive_scan32(face_flag.p, fpos.p, 4 * nkept, s);
    int64_t nfaces = 0;
    FG_CUDA(cudaMemcpyAsync(&nfaces, fpos.p + 4 * nkept, 8, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    DevBuf<uint32_t> faces(8 * std::max<int64_t>(nfaces, 1));
    k_faces<<<grid(4 * nkept), XT, 0, s>>>(4 * nkept, face_flag.p, fpos.p, face_rec.p, faces.p);
    FG_CUDA(cudaGetLastError());
    // The host copy.
    out->points.resize(3 * nkpts);
    out->tets.resize(4 * nkept);
    out->part.resize(nkept);
    std::vector<uint32_t> frec(8 * nfaces);
    out->d_points.download(out->points.data(), out->points.size(), s);
    out->d_tets.download(out->tets.data(), out->tets.size(), s);
    out->d_part.download(out->part.data(), out->part.size(), s);
    faces.download(frec.data(), frec.size(), s);
    FG_CUDA(cudaStreamSynchronize(s));
    // Each face on the side of the footprints (2 distinct flat points) takes the circles of the
    // input segments under its flat edge (prism.rs:345-359).
    out->face_nodes.resize(3 * nfaces);
    out->face_tet.resize(nfaces);
    out->face_beyond.resize(nfaces);
    out->face_circle_start.assign(nfaces + 1, 0);
    out->face_circles.clear();
    for (int64_t f = 0; f < nfaces; ++f) {
        const uint32_t* r = &frec[8 * f];
        out->face_tet[f] = r[0];
        for (int i = 0; i < 3; ++i) out->face_nodes[3 * f + i] = r[1 + i];
        out->face_beyond[f] = r[4];
        std::set<uint32_t> fl{r[5], r[6], r[7]};
        if (fl.size() == 2) {
            auto it = m.segments.find({*fl.begin(), *fl.rbegin()});
            if (it != m.segments.end()) {
                std::set<uint32_t> list;
                for (uint32_t k : it->second)
                    if (flat.segment_circle[k] != NONE32) list.insert(flat.segment_circle[k]);
                out->face_circles.insert(out->face_circles.end(), list.begin(), list.end());
            }
        }
        out->face_circle_start[f + 1] = out->face_circles.size();
    }
    out->circles = flat.circles;
    out->triangles = (size_t)nt;
    out->planes = planes.size();
}

}  // namespace femgpu

// ------------------------------------------------------------------ C ABI
using namespace femgpu;

struct femgpu_tetmesh {
    TetMesh m;
};
struct femgpu_mesh2 {
    Mesh2 m;
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

void need(bool ok, const char* what) {
    if (!ok) throw Failure(FEMGPU_ERR_INVALID, what);
}

Outline outline_of(const femgpu_outline& o) {
    Outline out;
    out.circle = o.circle != 0;
    if (out.circle) {
        out.centre = {o.centre[0], o.centre[1]};
        out.radius = o.radius;
    } else {
        need(o.ncorners == 0 || o.corners, "a polygon without its corners");
        for (size_t k = 0; k < o.ncorners; ++k) out.corners.push_back({o.corners[2 * k], o.corners[2 * k + 1]});
    }
    return out;
}

std::vector<Part> parts_of(const femgpu_part* parts, size_t n) {
    need(n == 0 || parts, "a null part list");
    std::vector<Part> out(n);
    for (size_t k = 0; k < n; ++k) {
        const femgpu_part& p = parts[k];
        Part& q = out[k];
        q.name = p.name ? p.name : "";
        q.material = p.material;
        q.priority = p.priority;
        for (int d = 0; d < 3; ++d) {
            q.lo[d] = p.lo[d];
            q.hi[d] = p.hi[d];
        }
        q.has_footprint = p.has_footprint != 0;
        if (q.has_footprint) {
            q.footprint.outline = outline_of(p.outline);
            need(p.nholes == 0 || p.holes, "a null hole list");
            for (size_t h = 0; h < p.nholes; ++h) q.footprint.holes.push_back(outline_of(p.holes[h]));
        }
    }
    return out;
}

}  // namespace

extern "C" {

int femgpu_prism_mesh(const femgpu_part* parts, size_t nparts, int axis,
                      const femgpu_spacing* spacing, size_t max_points, const char* refusal,
                      int periodic, const uint8_t* hollow, size_t nhollow, femgpu_tetmesh** out) {
    return guard([&] {
        need(out && spacing, "a null argument");
        need(axis >= 0 && axis < 3, "the axis must be 0, 1 or 2");
        need(nhollow == 0 || hollow, "a null hollow list");
        const std::vector<Part> ps = parts_of(parts, nparts);
        std::vector<uint8_t> hol(hollow, hollow + nhollow);
        const Spacing sp{spacing->max_cell, spacing->max_growth, spacing->min_cells};
        cudaStream_t s = nullptr;
        auto* h = new femgpu_tetmesh;
        try {
            prism_mesh(ps, axis, sp, max_points, refusal ? refusal : "", periodic != 0, hol, &h->m,
                       &s);
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

int femgpu_tetmesh_sizes(const femgpu_tetmesh* m, femgpu_tetmesh_counts* sizes) {
    return guard([&] {
        need(m && sizes, "a null argument");
        sizes->points = m->m.points.size() / 3;
        sizes->tets = m->m.part.size();
        sizes->faces = m->m.face_tet.size();
        sizes->face_circles = m->m.face_circles.size();
        sizes->circles = m->m.circles.size();
        sizes->triangles = m->m.triangles;
        sizes->planes = m->m.planes;
    });
}

int femgpu_tetmesh_copy(const femgpu_tetmesh* m, double* points, uint32_t* tets, uint32_t* part,
                        uint32_t* face_nodes, uint32_t* face_tet, uint32_t* face_beyond,
                        uint64_t* face_circle_start, uint32_t* face_circles, double* circles) {
    return guard([&] {
        need(m, "a null mesh");
        const TetMesh& t = m->m;
        auto put = [](auto* dst, const auto& v) {
            if (dst) std::copy(v.begin(), v.end(), dst);
        };
        put(points, t.points);
        put(tets, t.tets);
        put(part, t.part);
        put(face_nodes, t.face_nodes);
        put(face_tet, t.face_tet);
        put(face_beyond, t.face_beyond);
        put(face_circle_start, t.face_circle_start);
        put(face_circles, t.face_circles);
        if (circles)
            for (size_t k = 0; k < t.circles.size(); ++k) {
                circles[3 * k] = t.circles[k].first[0];
                circles[3 * k + 1] = t.circles[k].first[1];
                circles[3 * k + 2] = t.circles[k].second;
            }
    });
}

int femgpu_tetmesh_device(const femgpu_tetmesh* m, const double** points, const uint32_t** tets,
                          const uint32_t** part) {
    return guard([&] {
        need(m, "a null mesh");
        if (points) *points = m->m.d_points.p;
        if (tets) *tets = m->m.d_tets.p;
        if (part) *part = m->m.d_part.p;
    });
}

void femgpu_tetmesh_free(femgpu_tetmesh* m) { delete m; }

int femgpu_axis_planes(const femgpu_part* parts, size_t nparts, int axis,
                       const femgpu_spacing* spacing, const double* extra, size_t nextra,
                       double* planes, size_t cap, size_t* count) {
    return guard([&] {
        need(spacing && count && axis >= 0 && axis < 3, "invalid axis_planes arguments");
        need(nparts > 0 || nextra > 0, "no part and no extra plane");
        need(nextra == 0 || extra, "a null extra list");
        const std::vector<Part> ps = parts_of(parts, nparts);
        const Spacing sp{spacing->max_cell, spacing->max_growth, spacing->min_cells};
        const std::vector<double> p = axis_planes(ps, axis, sp, std::vector<double>(extra, extra + nextra));
        *count = p.size();
        if (planes) std::copy(p.begin(), p.begin() + std::min(cap, p.size()), planes);
    });
}

int femgpu_mesh2d(const double* points, size_t npoints, const uint32_t* segments,
                  size_t nsegments, double max_size, double max_growth, int periodic,
                  femgpu_classify_fn classify, void* ctx, femgpu_mesh2** out) {
    return guard([&] {
        need(out && classify && (npoints == 0 || points) && (nsegments == 0 || segments),
             "a null argument");
        std::vector<P2> pts(npoints);
        for (size_t k = 0; k < npoints; ++k) pts[k] = {points[2 * k], points[2 * k + 1]};
        std::vector<std::array<uint32_t, 2>> segs(nsegments);
        for (size_t k = 0; k < nsegments; ++k) {
            need(segments[2 * k] < npoints && segments[2 * k + 1] < npoints,
                 "a segment end past the points");
            segs[k] = {segments[2 * k], segments[2 * k + 1]};
        }
        auto* h = new femgpu_mesh2;
        try {
            h->m = quality_mesh(pts, segs, Size2{max_size, max_growth},
                                [&](P2 p) { return classify(p.data(), ctx); }, periodic != 0);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int femgpu_mesh2_sizes(const femgpu_mesh2* m, size_t* points, size_t* triangles,
                       size_t* segment_edges, size_t* segment_origins) {
    return guard([&] {
        need(m, "a null mesh");
        if (points) *points = m->m.points.size();
        if (triangles) *triangles = m->m.triangles.size();
        if (segment_edges) *segment_edges = m->m.segments.size();
        if (segment_origins) {
            size_t n = 0;
            for (const auto& e : m->m.segments) n += e.second.size();
            *segment_origins = n;
        }
    });
}

int femgpu_mesh2_copy(const femgpu_mesh2* m, double* points, uint32_t* triangles, uint32_t* label,
                      uint32_t* across, uint32_t* edges, uint64_t* origin_start,
                      uint32_t* origins) {
    return guard([&] {
        need(m, "a null mesh");
        const Mesh2& g = m->m;
        for (size_t k = 0; k < g.points.size() && points; ++k) {
            points[2 * k] = g.points[k][0];
            points[2 * k + 1] = g.points[k][1];
        }
        for (size_t k = 0; k < g.triangles.size(); ++k)
            for (int i = 0; i < 3; ++i) {
                if (triangles) triangles[3 * k + i] = g.triangles[k][i];
                if (across) across[3 * k + i] = g.across[k][i];
            }
        if (label) std::copy(g.label.begin(), g.label.end(), label);
        size_t e = 0, o = 0;
        if (origin_start) origin_start[0] = 0;
        for (const auto& kv : g.segments) {
            if (edges) {
                edges[2 * e] = kv.first.first;
                edges[2 * e + 1] = kv.first.second;
            }
            for (uint32_t x : kv.second) {
                if (origins) origins[o] = x;
                ++o;
            }
            ++e;
            if (origin_start) origin_start[e] = o;
        }
    });
}

void femgpu_mesh2_free(femgpu_mesh2* m) { delete m; }

int femgpu_split_prism(const uint64_t* g, int32_t* out) {
    return guard([&] {
        need(g && out, "a null argument");
        int t[3][4];
        split_prism(g, t);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 4; ++j) out[4 * i + j] = t[i][j];
    });
}

}  // extern "C"
