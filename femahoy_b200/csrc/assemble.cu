// Global stiffness assembly on the device: the CSR pattern (sparse.rs:22-65), the element
// colouring, the values by row gather (bit-identical with sparse.rs:75-86) or by colour scatter,
// the quadratic mesh numbering (tet10.rs:244-272), Csr::submatrix (sparse.rs:108-135) and
// heat::reduced_rhs (heat.rs:1219-1244).
//
// Built with -fmad=false: the element arithmetic keeps the reference's separate roundings.
#include <algorithm>
#include <array>
#include <cstring>
#include <vector>

#include <cub/cub.cuh>

#include "assemble.cuh"
#include "common.cuh"
#include "elements.cuh"
#include "hex.cuh"

namespace femgpu {

// ------------------------------------------------------------------ scans (CUB)
void exclusive_scan(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) {
    // out[0..n] = exclusive sums; out[n] = total. `in` may alias nothing in `out`.
    FG_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
    if (n == 0) return;
    size_t tmp = 0;
    FG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, in, out + 1, (int)n, s));
    DevBuf<uint8_t> t(tmp);
    FG_CUDA(cub::DeviceScan::InclusiveSum(t.p, tmp, in, out + 1, (int)n, s));
}

namespace {
struct Widen {
    __host__ __device__ int64_t operator()(uint32_t v) const { return (int64_t)v; }
};
}  // namespace

void exclusive_scan32(const uint32_t* in, int64_t* out, int64_t n, cudaStream_t s) {
    FG_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
    if (n == 0) return;
    cub::TransformInputIterator<int64_t, Widen, const uint32_t*> it(in, Widen{});
    size_t tmp = 0;
    FG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, it, out + 1, (int)n, s));
    DevBuf<uint8_t> t(tmp);
    FG_CUDA(cub::DeviceScan::InclusiveSum(t.p, tmp, it, out + 1, (int)n, s));
}

// ------------------------------------------------------------------ node -> elements
__global__ void k_count_nodes(const uint32_t* __restrict__ el, int64_t total, uint32_t n,
                              uint32_t* __restrict__ count, int* __restrict__ bad) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        uint32_t v = el[t];
        if (v >= n) {
            atomicExch(bad, 1);
            continue;
        }
        atomicAdd(&count[v], 1u);
    }
}

__global__ void k_fill_of_node(const uint32_t* __restrict__ el, int64_t nel, int m,
                               const int64_t* __restrict__ start, uint32_t* __restrict__ cursor,
                               uint32_t* __restrict__ of_node) {
    int64_t total = nel * m;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        uint32_t v = el[t];
        uint32_t slot = atomicAdd(&cursor[v], 1u);
        of_node[start[v] + slot] = (uint32_t)(t / m);
    }
}

// Each node's elements in increasing order (the order of sparse.rs:35-40's counting sort).
__global__ void k_sort_segments(const int64_t* __restrict__ start, int64_t n,
                                uint32_t* __restrict__ of_node) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        int64_t b = start[v], e = start[v + 1];
        for (int64_t i = b + 1; i < e; ++i) {
            uint32_t key = of_node[i];
            int64_t j = i - 1;
            while (j >= b && of_node[j] > key) {
                of_node[j + 1] = of_node[j];
                --j;
            }
            of_node[j + 1] = key;
        }
    }
}

void build_incidence(const uint32_t* d_el, int64_t nel, int m, int64_t n, Incidence* inc,
                     cudaStream_t s) {
    DevBuf<uint32_t> count(n);
    count.zero(s);
    DevBuf<int> bad(1);
    bad.zero(s);
    k_count_nodes<<<blocks_for(nel * m, 256), 256, 0, s>>>(d_el, nel * m, (uint32_t)n, count.p,
                                                            bad.p);
    FG_CHECK_LAUNCH();
    if (fetch(bad.p, s)) throw Failure(FEMGPU_ERR_INVALID, "an element names a node past the last");
    inc->start.alloc(n + 1);
    exclusive_scan32(count.p, inc->start.p, n, s);
    count.zero(s);
    inc->of_node.alloc(nel * m);
    k_fill_of_node<<<blocks_for(nel * m, 256), 256, 0, s>>>(d_el, nel, m, inc->start.p, count.p,
                                                             inc->of_node.p);
    FG_CHECK_LAUNCH();
    k_sort_segments<<<blocks_for(n, 128), 128, 0, s>>>(inc->start.p, n, inc->of_node.p);
    FG_CHECK_LAUNCH();
    inc->n = n;
    inc->nel = nel;
    inc->m = m;
}

// ------------------------------------------------------------------ pattern (sparse.rs:22-65)
// One warp per row. The candidates of row i are i and the nodes of its elements. The warp
// emits them in increasing order without repeats by selection: each step takes the least
// candidate above the last one emitted (__reduce_min_sync). The first pass counts, the second
// writes; both visit the same candidates, so the rows match the reference's mark-and-sort.
constexpr int CACHE = 8;  // candidates per lane kept in registers (256 per row)

template <bool WRITE>
__global__ void k_pattern_rows(const uint32_t* __restrict__ el, int m,
                               const int64_t* __restrict__ start,
                               const uint32_t* __restrict__ of_node, int64_t n,
                               uint32_t* __restrict__ rowlen, const int64_t* __restrict__ ptr,
                               uint32_t* __restrict__ idx) {
    const int lane = threadIdx.x & 31;
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < n; i += warps) {
        int64_t b = start[i];
        int64_t c = 1 + (start[i + 1] - b) * m;
        auto cand = [&](int64_t t) -> uint32_t {
            if (t == 0) return (uint32_t)i;
            int64_t u = t - 1;
            return el[(int64_t)of_node[b + u / m] * m + u % m];
        };
        uint32_t mine[CACHE];
        bool cached = c <= 32 * CACHE;
        if (cached) {
#pragma unroll
            for (int k = 0; k < CACHE; ++k) {
                int64_t t = lane + 32 * k;
                mine[k] = t < c ? cand(t) : 0xffffffffu;
            }
        }
        uint64_t lo = 0;
        uint32_t count = 0, held = 0;
        int64_t base = WRITE ? ptr[i] : 0;
        for (;;) {
            uint32_t best = 0xffffffffu;
            if (cached) {
#pragma unroll
                for (int k = 0; k < CACHE; ++k)
                    if ((uint64_t)mine[k] >= lo && mine[k] < best) best = mine[k];
            } else {
                for (int64_t t = lane; t < c; t += 32) {
                    uint32_t v = cand(t);
                    if ((uint64_t)v >= lo && v < best) best = v;
                }
            }
            best = __reduce_min_sync(0xffffffffu, best);
            if (best == 0xffffffffu) break;
            if (WRITE) {
                if (lane == (int)(count & 31)) held = best;
                if ((count & 31) == 31) idx[base + (count & ~31u) + lane] = held;
            }
            ++count;
            lo = (uint64_t)best + 1;
        }
        if (WRITE) {
            uint32_t tail = count & 31;
            if ((uint32_t)lane < tail) idx[base + (count & ~31u) + lane] = held;
        } else if (lane == 0) {
            rowlen[i] = count;
        }
    }
}

void build_pattern(const uint32_t* d_el, const Incidence& inc, DevCsr* out, cudaStream_t s) {
    int64_t n = inc.n;
    DevBuf<uint32_t> len(n);
    int blocks = blocks_for(n * 32, 256, NUM_SMS * 64);
    k_pattern_rows<false><<<blocks, 256, 0, s>>>(d_el, inc.m, inc.start.p, inc.of_node.p, n,
                                                  len.p, nullptr, nullptr);
    FG_CHECK_LAUNCH();
    out->n = n;
    out->ptr.alloc(n + 1);
    exclusive_scan32(len.p, out->ptr.p, n, s);
    out->nnz = fetch(out->ptr.p + n, s);
    out->idx.alloc(out->nnz);
    k_pattern_rows<true><<<blocks, 256, 0, s>>>(d_el, inc.m, inc.start.p, inc.of_node.p, n,
                                                 nullptr, out->ptr.p, out->idx.p);
    FG_CHECK_LAUNCH();
    out->val.alloc(out->nnz);
    out->val.zero(s);
}

// The pattern of the unknowns 3 node + component from the pattern of the nodes: row 3v + c
// holds 3w, 3w + 1, 3w + 2 for each w of node row v (the reference builds it from the
// elements of 3 m unknowns, elastic_tet.rs:178-183, which gives the same rows). A node in no
// element keeps only its own unknown, as in the reference.
__global__ void k_dof_rowlen(const int64_t* __restrict__ nptr, const int64_t* __restrict__ start,
                             int64_t n, uint32_t* __restrict__ len) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        bool alone = start[v + 1] == start[v];
        uint32_t l = alone ? 1u : (uint32_t)(3 * (nptr[v + 1] - nptr[v]));
        len[3 * v] = len[3 * v + 1] = len[3 * v + 2] = l;
    }
}

__global__ void k_dof_fill(const int64_t* __restrict__ nptr, const uint32_t* __restrict__ nidx,
                           const int64_t* __restrict__ start, int64_t n,
                           const int64_t* __restrict__ ptr, uint32_t* __restrict__ idx) {
    const int lane = threadIdx.x & 31;
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = warp; v < n; v += warps) {
        if (start[v + 1] == start[v]) {
            if (lane < 3) idx[ptr[3 * v + lane]] = (uint32_t)(3 * v + lane);
            continue;
        }
        int64_t b = nptr[v], L = nptr[v + 1] - b;
        for (int c = 0; c < 3; ++c) {
            uint32_t* row = idx + ptr[3 * v + c];
            for (int64_t t = lane; t < 3 * L; t += 32) row[t] = 3 * nidx[b + t / 3] + (uint32_t)(t % 3);
        }
    }
}

void expand_dof_pattern(const DevCsr& node, const Incidence& inc, DevCsr* out, cudaStream_t s) {
    int64_t n = node.n;
    DevBuf<uint32_t> len(3 * n);
    k_dof_rowlen<<<blocks_for(n, 256), 256, 0, s>>>(node.ptr.p, inc.start.p, n, len.p);
    FG_CHECK_LAUNCH();
    out->n = 3 * n;
    out->ptr.alloc(3 * n + 1);
    exclusive_scan32(len.p, out->ptr.p, 3 * n, s);
    out->nnz = fetch(out->ptr.p + 3 * n, s);
    out->idx.alloc(out->nnz);
    k_dof_fill<<<blocks_for(n * 32, 256, NUM_SMS * 64), 256, 0, s>>>(
        node.ptr.p, node.idx.p, inc.start.p, n, out->ptr.p, out->idx.p);
    FG_CHECK_LAUNCH();
    out->val.alloc(out->nnz);
    out->val.zero(s);
}

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ int64_t lower_bound(const uint32_t* __restrict__ a, int64_t lo,
                                               int64_t hi, uint32_t key) {
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (a[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void load_corners(const double* __restrict__ xyz,
                                             const uint32_t* __restrict__ t, double p[4][3]) {
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) p[c][d] = xyz[3 * (int64_t)t[c] + d];
}

// ------------------------------------------------------------------ gather: P1 heat
// One thread per row: the row's elements in increasing order, each adding its row of the
// 4 x 4 conduction matrix. Every entry gets its terms in increasing element order, starting from
// 0.0, which is the sum that Csr::add_element forms (sparse.rs:75-86, heat.rs:925-927).
__global__ void k_gather_heat(const double* __restrict__ xyz, const uint32_t* __restrict__ el,
                              const double* __restrict__ coef, const int64_t* __restrict__ start,
                              const uint32_t* __restrict__ of_node, int64_t n,
                              const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                              double* __restrict__ val, int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r0 = ptr[i], r1 = ptr[i + 1];
        for (int64_t t = start[i]; t < start[i + 1]; ++t) {
            uint32_t e = of_node[t];
            const uint32_t* nodes = el + 4 * (int64_t)e;
            double p[4][3], g[4][3], v;
            load_corners(xyz, nodes, p);
            tet_gradients(p, g, &v);
            double k[3] = {coef[3 * (int64_t)e], coef[3 * (int64_t)e + 1],
                           coef[3 * (int64_t)e + 2]};
            int a = 0;
            while (a < 4 && nodes[a] != (uint32_t)i) ++a;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                int64_t at = lower_bound(idx, r0, r1, nodes[b]);
                if (at >= r1 || idx[at] != nodes[b]) {
                    atomicExch(bad, 1);
                    continue;
                }
                val[at] += conduction_entry(g, v, k, a, b);
            }
        }
    }
}

// ------------------------------------------------------------------ gather: hex8 heat
// heat.rs:1246-1273: entry (p, q) of the 8 x 8 conduction matrix of a box cell of sides s with
// conductivities k, the corners in VTK order (bit b of axis e of corner p in kHexBits): the sum
// over the axes d of k_d times, for each axis e in order, 1/h or -1/h (e = d) or h/3 or h/6.
__device__ __constant__ const int kHexBits[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                                    {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

__device__ __forceinline__ double hex_conduction_entry(const double s[3], const double k[3], int p,
                                                       int q) {
    double v = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double term = k[d];
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            const bool same = kHexBits[p][e] == kHexBits[q][e];
            term *= e == d ? (same ? 1.0 / s[e] : -1.0 / s[e]) : (same ? s[e] / 3.0 : s[e] / 6.0);
        }
        v += term;
    }
    return v;
}

// One thread per row, as k_gather_heat, for box cells (heat.rs:820-826): the cell's sides are
// its corner 6 minus its corner 0, the plane spacings of the grid.
__global__ void k_gather_hex_heat(const double* __restrict__ xyz, const uint32_t* __restrict__ el,
                                  const double* __restrict__ coef,
                                  const int64_t* __restrict__ start,
                                  const uint32_t* __restrict__ of_node, int64_t n,
                                  const int64_t* __restrict__ ptr,
                                  const uint32_t* __restrict__ idx, double* __restrict__ val,
                                  int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r0 = ptr[i], r1 = ptr[i + 1];
        for (int64_t t = start[i]; t < start[i + 1]; ++t) {
            uint32_t e = of_node[t];
            const uint32_t* nodes = el + 8 * (int64_t)e;
            double s[3], k[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                s[d] = xyz[3 * (int64_t)nodes[6] + d] - xyz[3 * (int64_t)nodes[0] + d];
                k[d] = coef[3 * (int64_t)e + d];
            }
            int a = 0;
            while (a < 8 && nodes[a] != (uint32_t)i) ++a;
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                int64_t at = lower_bound(idx, r0, r1, nodes[b]);
                if (at >= r1 || idx[at] != nodes[b]) {
                    atomicExch(bad, 1);
                    continue;
                }
                val[at] += hex_conduction_entry(s, k, a, b);
            }
        }
    }
}

// ------------------------------------------------------------------ gather: elasticity
// One warp per node v, for its 3 rows 3v + c. The element matrix rows 3 a + c of each element
// of v, in increasing element order; the lanes share the 3 x 3 m outputs of one element, each
// output the sum over the quadrature points in the reference's order (tet10.rs:93-118). The 3
// rows are accumulated in shared memory when they fit, else in place in global memory.
template <int NN>
struct ElasticShared {
    static constexpr int ROWCAP = 3 * 128;  // 3 x (node row length) doubles per component row
    double buf[3 * ROWCAP];
    double gr[NN == 10 ? 4 : 1][NN][3];
    int pos[NN];
};

// tet10.rs:181-205: the scalar of the consistent mass of points i and j, in units of V / 420.
__device__ __forceinline__ double tet10_mass_scalar(int i, int j) {
    if (i < 4 && j < 4) return i == j ? 6.0 : 1.0;
    if (i < 4 || j < 4) {
        const int c = i < 4 ? i : j, e = i < 4 ? j - 4 : i - 4;
        return (kEdges[e][0] == c || kEdges[e][1] == c) ? -4.0 : -6.0;
    }
    const int a0 = kEdges[i - 4][0], a1 = kEdges[i - 4][1];
    const int b0 = kEdges[j - 4][0], b1 = kEdges[j - 4][1];
    const int shared = (a0 == b0 || a0 == b1) + (a1 == b0 || a1 == b1);
    return shared == 2 ? 32.0 : (shared == 1 ? 16.0 : 8.0);
}

// MASS: the consistent mass of the 10-node tetrahedron (tet10.rs:173-212) with the density
// coef[e], in place of the stiffness: entry (3i + a, 3j + b) = density V / 420 scalar(i, j) for
// a = b, 0 else.
// ORTHO: coef holds the 9 constants of an orthotropic material per element
// (orthotropic_stiffness), else E and nu. Flags: 2 no stable material, 3 a modulus not above 0.
template <int NN, int WARPS, bool MASS = false, bool ORTHO = false>
__global__ void __launch_bounds__(32 * WARPS)
    k_gather_elastic(const double* __restrict__ xyz, const uint32_t* __restrict__ el,
                     const double* __restrict__ coef, const int64_t* __restrict__ start,
                     const uint32_t* __restrict__ of_node, int64_t nnodes,
                     const int64_t* __restrict__ nptr, const uint32_t* __restrict__ nidx,
                     const int64_t* __restrict__ ptr, double* __restrict__ val,
                     int* __restrict__ bad) {
    __shared__ ElasticShared<NN> sh[WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    ElasticShared<NN>& S = sh[w];
    constexpr int NQ = NN == 10 ? 4 : 1;
    constexpr int OUT = 9 * NN;
    for (int64_t v = blockIdx.x * (int64_t)WARPS + w; v < nnodes; v += (int64_t)gridDim.x * WARPS) {
        int64_t nb = nptr[v], L = nptr[v + 1] - nb;
        if (start[v + 1] == start[v]) continue;  // no element: the zero row stays
        int64_t rowlen = 3 * L;
        bool in_shared = rowlen <= ElasticShared<NN>::ROWCAP;
        double* buf = in_shared ? S.buf : val + ptr[3 * v];
        // Rows 3v, 3v+1 and 3v+2 are consecutive in the CSR, each 3 L long.
        for (int64_t t = lane; t < 3 * rowlen; t += 32) buf[t] = 0.0;
        __syncwarp();
        for (int64_t t = start[v]; t < start[v + 1]; ++t) {
            uint32_t e = of_node[t];
            const uint32_t* nodes = el + (int64_t)NN * e;
            if (lane < NN) {
                uint32_t j = nodes[lane];
                int64_t at = lower_bound(nidx, nb, nb + L, j);
                if (at >= nb + L || nidx[at] != j) {
                    atomicExch(bad, 1);
                    at = nb;
                }
                S.pos[lane] = (int)(at - nb);
            }
            double p[4][3], g[4][3], vol;
            load_corners(xyz, nodes, p);
            tet_gradients(p, g, &vol);
            Stiffness D;
            if (ORTHO) {
                const int st = orthotropic_stiffness(coef + 9 * (int64_t)e, &D);
                if (st && lane == 0) atomicExch(bad, st == 1 ? 3 : 2);
            } else if (!MASS &&
                       !isotropic_stiffness(coef[2 * (int64_t)e], coef[2 * (int64_t)e + 1], &D)) {
                if (lane == 0) atomicExch(bad, 2);
            }
            if (MASS) {
            } else if (NQ == 4) {
                if (lane < 4) {
                    double tab[10][3];
                    tet10_gradients(g, lane, tab);
#pragma unroll
                    for (int i = 0; i < 10; ++i)
#pragma unroll
                        for (int d = 0; d < 3; ++d) S.gr[lane][i][d] = tab[i][d];
                }
            } else if (lane < 4) {
#pragma unroll
                for (int d = 0; d < 3; ++d) S.gr[0][lane][d] = g[lane][d];
            }
            int an = 0;
            while (an < NN && nodes[an] != (uint32_t)v) ++an;
            __syncwarp();
            double wq = NQ == 4 ? vol / 4.0 : vol;
            const double wm = MASS ? coef[e] * vol / 420.0 : 0.0;
            for (int o = lane; o < OUT; o += 32) {
                int a = o / (3 * NN);
                int rem = o % (3 * NN);
                int j = rem / 3, b = rem % 3;
                double k = 0.0;
                if (MASS) {
                    k = a == b ? wm * tet10_mass_scalar(an, j) : 0.0;
                } else {
#pragma unroll
                    for (int q = 0; q < NQ; ++q)
                        k += wq * elastic_term(S.gr[q][an], S.gr[q][j], a, b, D);
                }
                buf[a * rowlen + 3 * S.pos[j] + b] += k;
            }
            __syncwarp();
        }
        if (in_shared) {
            double* out = val + ptr[3 * v];
            for (int64_t t = lane; t < 3 * rowlen; t += 32) out[t] = buf[t];
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------ box cells: elasticity
// The condensed element of a box cell (hex.rs:218-297) depends only on its 3 sides and its
// material, and a grid has few distinct cells (the plane spacings times the materials). So the
// cells are sorted into classes by the bits of those 12 numbers, each class's 24 x 24 matrix is
// made once on the device, and the rows are gathered from the class table.

// The words of each cell: the sides (corner 6 minus corner 0), the 9 orthotropic constants and,
// with `expansion` (width 15), the 3 expansion coefficients.
__global__ void k_hex_keys(const double* __restrict__ xyz, const uint32_t* __restrict__ el,
                           const double* __restrict__ coef, const double* __restrict__ expansion,
                           int width, int64_t nel, double* __restrict__ key) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t c0 = el[8 * e], c6 = el[8 * e + 6];
        double* k = key + width * e;
#pragma unroll
        for (int d = 0; d < 3; ++d) k[d] = xyz[3 * (int64_t)c6 + d] - xyz[3 * (int64_t)c0 + d];
#pragma unroll
        for (int d = 0; d < 9; ++d) k[3 + d] = coef[9 * e + d];
        if (width == 15)
#pragma unroll
            for (int d = 0; d < 3; ++d) k[12 + d] = expansion ? expansion[3 * e + d] : 0.0;
    }
}

// hex.rs:337-353: entry (3 a + c, 3 j + b) of the consistent mass of a box cell with the sides
// s and the density rho: rho times the product of the 1D masses s_d / 3 (a and j at the same end
// of axis d) or s_d / 6, for c = b; 0 else.
__device__ __forceinline__ double hex_mass_entry(const double* s, double rho, int a, int j, int c,
                                                 int b) {
    if (c != b) return 0.0;
    double v = 1.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) v *= hex_bit(a, d) == hex_bit(j, d) ? s[d] / 3.0 : s[d] / 6.0;
    return rho * v;
}

// One warp per node v, for its 3 rows 3v + c, as k_gather_elastic: the rows 3 a + c of the
// class matrix of each cell of v (a = v's corner), in increasing cell order. MASS: the box
// cell's consistent mass instead (coef = the density per cell, the sides from xyz).
template <int WARPS, bool MASS = false>
__global__ void __launch_bounds__(32 * WARPS)
    k_gather_hex_elastic(const uint32_t* __restrict__ el, const uint32_t* __restrict__ cls,
                         const double* __restrict__ table, const double* __restrict__ xyz,
                         const double* __restrict__ coef, const int64_t* __restrict__ start,
                         const uint32_t* __restrict__ of_node, int64_t nnodes,
                         const int64_t* __restrict__ nptr, const uint32_t* __restrict__ nidx,
                         const int64_t* __restrict__ ptr, double* __restrict__ val,
                         int* __restrict__ bad) {
    constexpr int ROWCAP = 3 * 64;
    __shared__ double sbuf[WARPS][3 * ROWCAP];
    __shared__ int spos[WARPS][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t v = blockIdx.x * (int64_t)WARPS + w; v < nnodes; v += (int64_t)gridDim.x * WARPS) {
        const int64_t nb = nptr[v], L = nptr[v + 1] - nb;
        if (start[v + 1] == start[v]) continue;
        const int64_t rowlen = 3 * L;
        const bool in_shared = rowlen <= ROWCAP;
        double* buf = in_shared ? sbuf[w] : val + ptr[3 * v];
        for (int64_t t = lane; t < 3 * rowlen; t += 32) buf[t] = 0.0;
        __syncwarp();
        for (int64_t t = start[v]; t < start[v + 1]; ++t) {
            const uint32_t e = of_node[t];
            const uint32_t* nodes = el + 8 * (int64_t)e;
            if (lane < 8) {
                const uint32_t j = nodes[lane];
                int64_t at = lower_bound(nidx, nb, nb + L, j);
                if (at >= nb + L || nidx[at] != j) {
                    atomicExch(bad, 1);
                    at = nb;
                }
                spos[w][lane] = (int)(at - nb);
            }
            int an = 0;
            while (an < 8 && nodes[an] != (uint32_t)v) ++an;
            __syncwarp();
            if (MASS) {
                double sd[3];
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    sd[d] = xyz[3 * (int64_t)nodes[6] + d] - xyz[3 * (int64_t)nodes[0] + d];
                const double rho = coef[e];
                for (int o = lane; o < 72; o += 32) {
                    const int c = o / 24, col = o % 24;
                    buf[c * rowlen + 3 * spos[w][col / 3] + col % 3] +=
                        hex_mass_entry(sd, rho, an, col / 3, c, col % 3);
                }
            } else {
                const double* m = table + 576 * (int64_t)cls[e] + 72 * an;  // rows 3 an .. +2
                for (int o = lane; o < 72; o += 32) {
                    const int c = o / 24, col = o % 24;
                    buf[c * rowlen + 3 * spos[w][col / 3] + col % 3] += m[o];
                }
            }
            __syncwarp();
        }
        if (in_shared) {
            double* out = val + ptr[3 * v];
            for (int64_t t = lane; t < 3 * rowlen; t += 32) out[t] = buf[t];
        }
        __syncwarp();
    }
}

void hex_elements(const double* d_keys, int64_t n, double* d_table, cudaStream_t s) {
    DevBuf<int> bad(1);
    bad.zero(s);
    k_hex_element<false><<<(unsigned)std::min<int64_t>(n, NUM_SMS * 16), HEX_THREADS, 0, s>>>(
        d_keys, 12, n, d_table, bad.p);
    FG_CHECK_LAUNCH();
    assembly_flag(fetch(bad.p, s));
}

void hex_modes(const double* d_keys, int64_t n, double* d_modes, cudaStream_t s) {
    DevBuf<int> bad(1);
    bad.zero(s);
    k_hex_element<true><<<(unsigned)std::min<int64_t>(n, NUM_SMS * 16), HEX_THREADS, 0, s>>>(
        d_keys, 15, n, d_modes, bad.p);
    FG_CHECK_LAUNCH();
    assembly_flag(fetch(bad.p, s));
}

// The classes of the cells, on the device: the cells sorted by a 64-bit hash of their words
// (FNV-1a), a class starting wherever the hash or any word differs from the previous sorted
// cell's (a collision that interleaves 2 keys makes extra classes of equal matrices, never a
// wrong one), numbered by a scan of the starts.
__global__ void k_key_hash(const double* __restrict__ key, int width, int64_t nel,
                           uint64_t* __restrict__ hash, uint32_t* __restrict__ pos) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x) {
        uint64_t h = 1469598103934665603ULL;
        for (int w = 0; w < width; ++w)
            h = (h ^ (uint64_t)__double_as_longlong(key[width * e + w])) * 1099511628211ULL;
        hash[e] = h;
        pos[e] = (uint32_t)e;
    }
}

__global__ void k_key_heads(const uint64_t* __restrict__ hash, const uint32_t* __restrict__ pos,
                            const double* __restrict__ key, int width, int64_t n,
                            uint32_t* __restrict__ head) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        bool starts = t == 0 || hash[t] != hash[t - 1];
        if (!starts) {
            const double* a = key + width * (int64_t)pos[t];
            const double* b = key + width * (int64_t)pos[t - 1];
            for (int w = 0; w < width && !starts; ++w)
                starts = __double_as_longlong(a[w]) != __double_as_longlong(b[w]);
        }
        head[t] = starts ? 1u : 0u;
    }
}

__global__ void k_key_classes(const uint32_t* __restrict__ head, const int64_t* __restrict__ run,
                              const uint32_t* __restrict__ pos, const double* __restrict__ key,
                              int width, int64_t n, uint32_t* __restrict__ cls,
                              double* __restrict__ keys) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = run[t + 1] - 1;  // the inclusive count of starts
        cls[pos[t]] = (uint32_t)c;
        if (head[t])
            for (int w = 0; w < width; ++w) keys[width * c + w] = key[width * (int64_t)pos[t] + w];
    }
}

int64_t hex_classes(const double* xyz, const uint32_t* el, const double* coef,
                    const double* expansion, int width, int64_t nel, DevBuf<uint32_t>* cls,
                    DevBuf<double>* keys, cudaStream_t s) {
    if (nel >= 0x7fffffffLL) throw Failure(FEMGPU_ERR_TOO_LARGE, "more than 2^31 box cells");
    DevBuf<double> d_key(width * nel);
    k_hex_keys<<<blocks_for(nel, 256), 256, 0, s>>>(xyz, el, coef, expansion, width, nel,
                                                    d_key.p);
    DevBuf<uint64_t> hash(nel), hash2(nel);
    DevBuf<uint32_t> pos(nel), pos2(nel), head(nel);
    k_key_hash<<<blocks_for(nel, 256), 256, 0, s>>>(d_key.p, width, nel, hash.p, pos.p);
    FG_CHECK_LAUNCH();
    size_t tmp = 0;
    FG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, hash.p, hash2.p, pos.p, pos2.p,
                                            (int)nel, 0, 64, s));
    DevBuf<uint8_t> t(tmp);
    FG_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, hash.p, hash2.p, pos.p, pos2.p, (int)nel,
                                            0, 64, s));
    k_key_heads<<<blocks_for(nel, 256), 256, 0, s>>>(hash2.p, pos2.p, d_key.p, width, nel,
                                                     head.p);
    FG_CHECK_LAUNCH();
    DevBuf<int64_t> run(nel + 1);
    exclusive_scan32(head.p, run.p, nel, s);
    const int64_t nclass = fetch(run.p + nel, s);
    cls->alloc(nel);
    keys->alloc(width * nclass);
    k_key_classes<<<blocks_for(nel, 256), 256, 0, s>>>(head.p, run.p, pos2.p, d_key.p, width, nel,
                                                       cls->p, keys->p);
    FG_CHECK_LAUNCH();
    FG_CUDA(cudaStreamSynchronize(s));
    return nclass;
}

// ------------------------------------------------------------------ colouring
// Jones-Plassmann: M. T. Jones and P. E. Plassmann, A parallel graph coloring heuristic, SIAM J.
// Sci. Comput. 14 (1993) 654-669. The priority of element e is the "lowbias32" hash of
// C. Wellons (2018); (priority, index) orders the elements. Each round has 2 launches: select
// (an uncoloured element above each uncoloured neighbour) then assign (the least colour that
// no coloured neighbour has). The selected elements of a round share no node, so the assignment
// reads only colours of earlier rounds.
__device__ __forceinline__ uint32_t lowbias32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

constexpr uint32_t UNSET = 0xffffffffu;

__global__ void k_colour_select(const uint32_t* __restrict__ el, int m, int64_t nel,
                                const int64_t* __restrict__ start,
                                const uint32_t* __restrict__ of_node,
                                const uint32_t* __restrict__ colour, uint8_t* __restrict__ sel) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x) {
        if (colour[e] != UNSET) {
            sel[e] = 0;
            continue;
        }
        uint64_t me = ((uint64_t)lowbias32((uint32_t)e) << 32) | (uint32_t)e;
        bool top = true;
        for (int a = 0; a < m && top; ++a) {
            uint32_t v = el[e * m + a];
            for (int64_t t = start[v]; t < start[v + 1]; ++t) {
                uint32_t f = of_node[t];
                if (f == (uint32_t)e || colour[f] != UNSET) continue;
                uint64_t other = ((uint64_t)lowbias32(f) << 32) | f;
                if (other > me) {
                    top = false;
                    break;
                }
            }
        }
        sel[e] = top;
    }
}

__global__ void k_colour_assign(const uint32_t* __restrict__ el, int m, int64_t nel,
                                const int64_t* __restrict__ start,
                                const uint32_t* __restrict__ of_node, uint32_t* __restrict__ colour,
                                const uint8_t* __restrict__ sel,
                                unsigned long long* __restrict__ left, int* __restrict__ most) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x) {
        if (!sel[e]) continue;
        uint64_t used[4] = {0, 0, 0, 0};
        for (int a = 0; a < m; ++a) {
            uint32_t v = el[e * m + a];
            for (int64_t t = start[v]; t < start[v + 1]; ++t) {
                uint32_t c = colour[of_node[t]];
                if (c != UNSET && c < 256) used[c >> 6] |= 1ull << (c & 63);
            }
        }
        uint32_t c = 0;
        while (c < 256 && ((used[c >> 6] >> (c & 63)) & 1)) ++c;
        colour[e] = c;  // c == 256 marks "more than 256 colours"
        atomicAdd(left, (unsigned long long)-1ll);
        atomicMax(most, (int)c + 1);
    }
}

int colour_elements(const uint32_t* d_el, const Incidence& inc, DevBuf<uint32_t>* colour,
                    cudaStream_t s) {
    int64_t nel = inc.nel;
    colour->alloc(nel);
    FG_CUDA(cudaMemsetAsync(colour->p, 0xff, nel * 4, s));
    DevBuf<uint8_t> sel(nel);
    DevBuf<unsigned long long> left(1);
    DevBuf<int> most(1);
    unsigned long long h_left = (unsigned long long)nel;
    FG_CUDA(cudaMemcpyAsync(left.p, &h_left, 8, cudaMemcpyHostToDevice, s));
    most.zero(s);
    int blocks = blocks_for(nel, 256, NUM_SMS * 32);
    for (int round = 0; h_left > 0; ++round) {
        if (round > 100000) throw Failure(FEMGPU_ERR_TIMEOUT, "the colouring did not finish");
        k_colour_select<<<blocks, 256, 0, s>>>(d_el, inc.m, nel, inc.start.p, inc.of_node.p,
                                               colour->p, sel.p);
        FG_CHECK_LAUNCH();
        k_colour_assign<<<blocks, 256, 0, s>>>(d_el, inc.m, nel, inc.start.p, inc.of_node.p,
                                               colour->p, sel.p, left.p, most.p);
        FG_CHECK_LAUNCH();
        h_left = fetch(left.p, s);
    }
    int nc = fetch(most.p, s);
    if (nc > 256) throw Failure(FEMGPU_ERR_TOO_LARGE, "the elements need more than 256 colours");
    return nc;
}

// ------------------------------------------------------------------ colour scatter
// Colour by colour, each element adds its whole matrix; elements of 1 colour share no row, so
// there are no write conflicts and no atomics. The terms of an entry are summed in colour order.
__global__ void k_scatter_heat(const double* __restrict__ xyz, const uint32_t* __restrict__ el,
                               const double* __restrict__ coef, const uint32_t* __restrict__ list,
                               int64_t count, const int64_t* __restrict__ ptr,
                               const uint32_t* __restrict__ idx, double* __restrict__ val,
                               int* __restrict__ bad) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count;
         t += (int64_t)gridDim.x * blockDim.x) {
        uint32_t e = list[t];
        const uint32_t* nodes = el + 4 * (int64_t)e;
        double p[4][3], g[4][3], v;
        load_corners(xyz, nodes, p);
        tet_gradients(p, g, &v);
        double k[3] = {coef[3 * (int64_t)e], coef[3 * (int64_t)e + 1], coef[3 * (int64_t)e + 2]};
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            int64_t r0 = ptr[nodes[a]], r1 = ptr[nodes[a] + 1];
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                int64_t at = lower_bound(idx, r0, r1, nodes[b]);
                if (at >= r1 || idx[at] != nodes[b]) {
                    atomicExch(bad, 1);
                    continue;
                }
                val[at] += conduction_entry(g, v, k, a, b);
            }
        }
    }
}

template <int NN, int WARPS>
__global__ void __launch_bounds__(32 * WARPS)
    k_scatter_elastic(const double* __restrict__ xyz, const uint32_t* __restrict__ el,
                      const double* __restrict__ coef, const uint32_t* __restrict__ list,
                      int64_t count, const int64_t* __restrict__ nptr,
                      const uint32_t* __restrict__ nidx, const int64_t* __restrict__ ptr,
                      double* __restrict__ val, int* __restrict__ bad) {
    constexpr int NQ = NN == 10 ? 4 : 1;
    struct Sh {
        double gr[NQ][NN][3];
        int pos[NN][NN];
    };
    __shared__ Sh sh[WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    Sh& S = sh[w];
    for (int64_t t = blockIdx.x * (int64_t)WARPS + w; t < count; t += (int64_t)gridDim.x * WARPS) {
        uint32_t e = list[t];
        const uint32_t* nodes = el + (int64_t)NN * e;
        for (int q = lane; q < NN * NN; q += 32) {
            int a = q / NN, b = q % NN;
            int64_t nb = nptr[nodes[a]], ne = nptr[nodes[a] + 1];
            int64_t at = lower_bound(nidx, nb, ne, nodes[b]);
            if (at >= ne || nidx[at] != nodes[b]) {
                atomicExch(bad, 1);
                at = nb;
            }
            S.pos[a][b] = (int)(at - nb);
        }
        double p[4][3], g[4][3], vol;
        load_corners(xyz, nodes, p);
        tet_gradients(p, g, &vol);
        Stiffness D;
        if (!isotropic_stiffness(coef[2 * (int64_t)e], coef[2 * (int64_t)e + 1], &D) && lane == 0)
            atomicExch(bad, 2);
        if (NQ == 4) {
            if (lane < 4) {
                double tab[10][3];
                tet10_gradients(g, lane, tab);
#pragma unroll
                for (int i = 0; i < 10; ++i)
#pragma unroll
                    for (int d = 0; d < 3; ++d) S.gr[lane][i][d] = tab[i][d];
            }
        } else if (lane < 4) {
#pragma unroll
            for (int d = 0; d < 3; ++d) S.gr[0][lane][d] = g[lane][d];
        }
        __syncwarp();
        double wq = NQ == 4 ? vol / 4.0 : vol;
        for (int o = lane; o < 9 * NN * NN; o += 32) {
            int row = o / (3 * NN), col = o % (3 * NN);
            int i = row / 3, a = row % 3, j = col / 3, b = col % 3;
            double k = 0.0;
#pragma unroll
            for (int q = 0; q < NQ; ++q) k += wq * elastic_term(S.gr[q][i], S.gr[q][j], a, b, D);
            uint32_t vi = nodes[i];
            val[ptr[3 * (int64_t)vi + a] + 3 * S.pos[i][j] + b] += k;
        }
        __syncwarp();
    }
}

__global__ void k_colour_histogram(const uint32_t* __restrict__ colour, int64_t nel,
                                   uint32_t* __restrict__ hist) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&hist[colour[e]], 1u);
}

__global__ void k_colour_fill(const uint32_t* __restrict__ colour, int64_t nel,
                              const int64_t* __restrict__ cstart, uint32_t* __restrict__ cursor,
                              uint32_t* __restrict__ list) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x) {
        uint32_t c = colour[e];
        list[cstart[c] + atomicAdd(&cursor[c], 1u)] = (uint32_t)e;
    }
}

// ------------------------------------------------------------------ assemble
void assemble(int kind, int mode, int64_t npoints, const double* d_xyz, int64_t nel,
              const uint32_t* d_el, const double* d_coef, Assembled* out, cudaStream_t s) {
    if (kind < 0 || kind > 7) throw Failure(FEMGPU_ERR_INVALID, "unknown element kind");
    if (mode < 0 || mode > 1) throw Failure(FEMGPU_ERR_INVALID, "unknown assembly mode");
    if (kind >= FEMGPU_P2_MASS && mode != FEMGPU_ASSEMBLE_GATHER)
        throw Failure(FEMGPU_ERR_INVALID,
                      "the mass, orthotropic materials and box cells assemble by rows "
                      "(FEMGPU_ASSEMBLE_GATHER)");
    const bool scalar = kind == FEMGPU_P1_HEAT || kind == FEMGPU_HEX8_HEAT;
    int nn = kind >= FEMGPU_HEX8_HEAT ? 8 : (kind >= FEMGPU_P2_ELASTIC ? 10 : 4);
    if (npoints >= 0xffffffffLL / 3)
        throw Failure(FEMGPU_ERR_TOO_LARGE, "more points than 32-bit unknown numbers hold");
    build_incidence(d_el, nel, nn, npoints, &out->inc, s);
    build_pattern(d_el, out->inc, &out->node, s);
    DevBuf<int> bad(1);
    bad.zero(s);
    DevCsr& K = out->matrix;
    if (scalar) {
        K.n = out->node.n;
        K.nnz = out->node.nnz;
        K.ptr = std::move(out->node.ptr);
        K.idx = std::move(out->node.idx);
        K.val = std::move(out->node.val);
        out->node.n = 0;
    } else {
        expand_dof_pattern(out->node, out->inc, &K, s);
    }
    K.val.zero(s);
    if (mode == FEMGPU_ASSEMBLE_GATHER) {
        if (kind == FEMGPU_P1_HEAT) {
            k_gather_heat<<<blocks_for(npoints, 128, NUM_SMS * 32), 128, 0, s>>>(
                d_xyz, d_el, d_coef, out->inc.start.p, out->inc.of_node.p, npoints, K.ptr.p,
                K.idx.p, K.val.p, bad.p);
        } else if (kind == FEMGPU_HEX8_HEAT) {
            k_gather_hex_heat<<<blocks_for(npoints, 128, NUM_SMS * 32), 128, 0, s>>>(
                d_xyz, d_el, d_coef, out->inc.start.p, out->inc.of_node.p, npoints, K.ptr.p,
                K.idx.p, K.val.p, bad.p);
        } else if (kind == FEMGPU_HEX8_ELASTIC) {
            DevBuf<double> keys, table;
            DevBuf<uint32_t> cls;
            const int64_t nclass =
                hex_classes(d_xyz, d_el, d_coef, nullptr, 12, nel, &cls, &keys, s);
            table.alloc(576 * nclass);
            k_hex_element<false><<<(unsigned)std::min<int64_t>(nclass, NUM_SMS * 16), HEX_THREADS,
                                   0, s>>>(keys.p, 12, nclass, table.p, bad.p);
            FG_CHECK_LAUNCH();
            k_gather_hex_elastic<4><<<blocks_for(npoints, 4, NUM_SMS * 64), 128, 0, s>>>(
                d_el, cls.p, table.p, nullptr, nullptr, out->inc.start.p, out->inc.of_node.p,
                npoints, out->node.ptr.p, out->node.idx.p, K.ptr.p, K.val.p, bad.p);
            FG_CHECK_LAUNCH();
            FG_CUDA(cudaStreamSynchronize(s));
        } else if (kind == FEMGPU_HEX8_MASS) {
            k_gather_hex_elastic<4, true><<<blocks_for(npoints, 4, NUM_SMS * 64), 128, 0, s>>>(
                d_el, nullptr, nullptr, d_xyz, d_coef, out->inc.start.p, out->inc.of_node.p,
                npoints, out->node.ptr.p, out->node.idx.p, K.ptr.p, K.val.p, bad.p);
            FG_CHECK_LAUNCH();
        } else if (kind == FEMGPU_P1_ELASTIC) {
            k_gather_elastic<4, 4><<<blocks_for(npoints, 4, NUM_SMS * 64), 128, 0, s>>>(
                d_xyz, d_el, d_coef, out->inc.start.p, out->inc.of_node.p, npoints,
                out->node.ptr.p, out->node.idx.p, K.ptr.p, K.val.p, bad.p);
        } else if (kind == FEMGPU_P2_ELASTIC_ORTHO) {
            k_gather_elastic<10, 4, false, true><<<blocks_for(npoints, 4, NUM_SMS * 64), 128, 0,
                                                   s>>>(
                d_xyz, d_el, d_coef, out->inc.start.p, out->inc.of_node.p, npoints,
                out->node.ptr.p, out->node.idx.p, K.ptr.p, K.val.p, bad.p);
        } else if (kind == FEMGPU_P2_MASS) {
            k_gather_elastic<10, 4, true><<<blocks_for(npoints, 4, NUM_SMS * 64), 128, 0, s>>>(
                d_xyz, d_el, d_coef, out->inc.start.p, out->inc.of_node.p, npoints,
                out->node.ptr.p, out->node.idx.p, K.ptr.p, K.val.p, bad.p);
        } else {
            k_gather_elastic<10, 4><<<blocks_for(npoints, 4, NUM_SMS * 64), 128, 0, s>>>(
                d_xyz, d_el, d_coef, out->inc.start.p, out->inc.of_node.p, npoints,
                out->node.ptr.p, out->node.idx.p, K.ptr.p, K.val.p, bad.p);
        }
        FG_CHECK_LAUNCH();
    } else {
        // The colouring needs only the corners: 2 tetrahedra share an edge point only if they
        // share both its corners.
        Incidence corners;
        const uint32_t* d_corners = d_el;
        DevBuf<uint32_t> c4;
        if (nn == 10) {
            c4.alloc(nel * 4);
            FG_CUDA(cudaMemcpy2DAsync(c4.p, 16, d_el, 40, 16, nel, cudaMemcpyDeviceToDevice, s));
            d_corners = c4.p;
            build_incidence(d_corners, nel, 4, npoints, &corners, s);
        }
        const Incidence& ci = nn == 10 ? corners : out->inc;
        DevBuf<uint32_t> colour;
        int nc = colour_elements(d_corners, ci, &colour, s);
        DevBuf<uint32_t> hist(nc), cursor(nc);
        hist.zero(s);
        cursor.zero(s);
        k_colour_histogram<<<blocks_for(nel, 256), 256, 0, s>>>(colour.p, nel, hist.p);
        DevBuf<int64_t> cstart(nc + 1);
        exclusive_scan32(hist.p, cstart.p, nc, s);
        DevBuf<uint32_t> list(nel);
        k_colour_fill<<<blocks_for(nel, 256), 256, 0, s>>>(colour.p, nel, cstart.p, cursor.p,
                                                           list.p);
        FG_CHECK_LAUNCH();
        std::vector<int64_t> hs(nc + 1);
        cstart.download(hs.data(), nc + 1, s);
        FG_CUDA(cudaStreamSynchronize(s));
        out->ncolours = nc;
        for (int c = 0; c < nc; ++c) {
            int64_t cnt = hs[c + 1] - hs[c];
            if (!cnt) continue;
            const uint32_t* l = list.p + hs[c];
            if (kind == FEMGPU_P1_HEAT)
                k_scatter_heat<<<blocks_for(cnt, 128), 128, 0, s>>>(
                    d_xyz, d_el, d_coef, l, cnt, K.ptr.p, K.idx.p, K.val.p, bad.p);
            else if (kind == FEMGPU_P1_ELASTIC)
                k_scatter_elastic<4, 4><<<blocks_for(cnt, 4, NUM_SMS * 64), 128, 0, s>>>(
                    d_xyz, d_el, d_coef, l, cnt, out->node.ptr.p, out->node.idx.p, K.ptr.p,
                    K.val.p, bad.p);
            else
                k_scatter_elastic<10, 4><<<blocks_for(cnt, 4, NUM_SMS * 64), 128, 0, s>>>(
                    d_xyz, d_el, d_coef, l, cnt, out->node.ptr.p, out->node.idx.p, K.ptr.p,
                    K.val.p, bad.p);
            FG_CHECK_LAUNCH();
        }
    }
    assembly_flag(fetch(bad.p, s));
}

void assembly_flag(int b) {
    if (b == 1) throw Failure(FEMGPU_ERR_PATTERN, "the pattern holds each element pair");
    if (b == 2)
        throw Failure(FEMGPU_ERR_MATERIAL,
                      "the Poisson ratios give no stable material (for an isotropic material, "
                      "nu must be between -1 and 0.5)");
    if (b == 3)
        throw Failure(FEMGPU_ERR_MATERIAL,
                      "the moduli must be above 0 and the Poisson ratios finite");
    if (b == 4)
        throw Failure(FEMGPU_ERR_INVALID,
                      "a box cell has a side not above 0: corner 6 must lie beyond corner 0 on "
                      "each axis");
    if (b == 5)
        throw Failure(FEMGPU_ERR_MATERIAL, "the incompatible modes of a box cell have no stiffness");
}

// ------------------------------------------------------------------ Quadratic (tet10.rs:244)
__global__ void k_edge_keys(const uint32_t* __restrict__ tets, int64_t ntet,
                            uint64_t* __restrict__ keys, uint32_t* __restrict__ pos) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 6 * ntet;
         t += (int64_t)gridDim.x * blockDim.x) {
        int64_t e = t / 6;
        int k = (int)(t % 6);
        uint32_t a = tets[4 * e + kEdges[k][0]], b = tets[4 * e + kEdges[k][1]];
        uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
        keys[t] = ((uint64_t)lo << 32) | hi;
        pos[t] = (uint32_t)t;
    }
}

__global__ void k_run_heads(const uint64_t* __restrict__ keys, int64_t m,
                            uint32_t* __restrict__ head) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m;
         t += (int64_t)gridDim.x * blockDim.x)
        head[t] = (t == 0 || keys[t] != keys[t - 1]) ? 1u : 0u;
}

__global__ void k_run_first(const uint32_t* __restrict__ head, const int64_t* __restrict__ run,
                            const uint32_t* __restrict__ pos, int64_t m,
                            uint32_t* __restrict__ first, uint32_t* __restrict__ rid) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m;
         t += (int64_t)gridDim.x * blockDim.x)
        if (head[t]) {
            int64_t r = run[t + 1] - 1;
            first[r] = pos[t];
            rid[r] = (uint32_t)r;
        }
}

__global__ void k_rank(const uint32_t* __restrict__ order, int64_t nrun,
                       uint32_t* __restrict__ rank) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nrun;
         q += (int64_t)gridDim.x * blockDim.x)
        rank[order[q]] = (uint32_t)q;
}

__global__ void k_edge_scatter(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ pos,
                               const int64_t* __restrict__ run, const uint32_t* __restrict__ rank,
                               int64_t m, uint32_t ncorner, uint32_t* __restrict__ tets10,
                               uint32_t* __restrict__ edges) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m;
         t += (int64_t)gridDim.x * blockDim.x) {
        uint32_t id = rank[run[t + 1] - 1];
        uint32_t p = pos[t];
        tets10[10 * (int64_t)(p / 6) + 4 + p % 6] = ncorner + id;
        if (t == 0 || keys[t] != keys[t - 1]) {
            edges[2 * (int64_t)id] = (uint32_t)(keys[t] >> 32);
            edges[2 * (int64_t)id + 1] = (uint32_t)keys[t];
        }
    }
}

__global__ void k_copy_corners(const uint32_t* __restrict__ tets, int64_t ntet,
                               uint32_t* __restrict__ tets10) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 4 * ntet;
         t += (int64_t)gridDim.x * blockDim.x)
        tets10[10 * (t / 4) + t % 4] = tets[t];
}

// The edges sorted by their corner pair (a stable radix sort keeps the places of 1 edge in
// increasing order, so the first is where it was first seen); the distinct edges ranked by the
// place of first sight, which is the numbering of the reference's HashMap walk.
int64_t quadratic(int64_t ncorner, int64_t ntet, const uint32_t* d_tets, uint32_t* d_tets10,
                  uint32_t* d_edges, cudaStream_t s) {
    int64_t m = 6 * ntet;
    if (m == 0) return 0;
    DevBuf<uint64_t> keys(m), keys2(m);
    DevBuf<uint32_t> pos(m), pos2(m);
    k_edge_keys<<<blocks_for(m, 256), 256, 0, s>>>(d_tets, ntet, keys.p, pos.p);
    FG_CHECK_LAUNCH();
    size_t tmp = 0;
    FG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys.p, keys2.p, pos.p, pos2.p, (int)m,
                                            0, 64, s));
    DevBuf<uint8_t> t(tmp);
    FG_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, keys.p, keys2.p, pos.p, pos2.p, (int)m, 0,
                                            64, s));
    DevBuf<uint32_t> head(m);
    k_run_heads<<<blocks_for(m, 256), 256, 0, s>>>(keys2.p, m, head.p);
    DevBuf<int64_t> run(m + 1);
    // run[t + 1] - 1 = the run of sorted place t (inclusive sum of heads).
    exclusive_scan32(head.p, run.p, m, s);
    int64_t nrun = fetch(run.p + m, s);
    DevBuf<uint32_t> first(nrun), rid(nrun), first2(nrun), rid2(nrun), rank(nrun);
    k_run_first<<<blocks_for(m, 256), 256, 0, s>>>(head.p, run.p, pos2.p, m, first.p, rid.p);
    tmp = 0;
    FG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, first.p, first2.p, rid.p, rid2.p,
                                            (int)nrun, 0, 32, s));
    DevBuf<uint8_t> t2(tmp);
    FG_CUDA(cub::DeviceRadixSort::SortPairs(t2.p, tmp, first.p, first2.p, rid.p, rid2.p,
                                            (int)nrun, 0, 32, s));
    k_rank<<<blocks_for(nrun, 256), 256, 0, s>>>(rid2.p, nrun, rank.p);
    k_copy_corners<<<blocks_for(4 * ntet, 256), 256, 0, s>>>(d_tets, ntet, d_tets10);
    k_edge_scatter<<<blocks_for(m, 256), 256, 0, s>>>(keys2.p, pos2.p, run.p, rank.p, m,
                                                      (uint32_t)ncorner, d_tets10, d_edges);
    FG_CHECK_LAUNCH();
    return nrun;
}

// ------------------------------------------------------------------ submatrix, reduced_rhs
__global__ void k_mark_keep(const int64_t* __restrict__ keep, int64_t nkeep, int64_t n,
                            uint32_t* __restrict__ fresh, int* __restrict__ bad) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nkeep;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = keep[k];
        if (i < 0 || i >= n) {
            atomicExch(bad, 1);
            continue;
        }
        if (atomicExch(&fresh[i], (uint32_t)k) != 0xffffffffu) atomicExch(bad, 2);
    }
}

__global__ void k_sub_count(const int64_t* __restrict__ keep, int64_t nkeep,
                            const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                            const uint32_t* __restrict__ fresh, uint32_t* __restrict__ len) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nkeep;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = keep[k];
        uint32_t c = 0;
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) c += fresh[idx[e]] != 0xffffffffu;
        len[k] = c;
    }
}

// sparse.rs:116-126 and the row sort of sparse.rs:137-148 (insertion sort, stable).
__global__ void k_sub_fill(const int64_t* __restrict__ keep, int64_t nkeep,
                           const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                           const double* __restrict__ val, const uint32_t* __restrict__ fresh,
                           const int64_t* __restrict__ optr, uint32_t* __restrict__ oidx,
                           double* __restrict__ oval) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nkeep;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = keep[k], o = optr[k], b = o;
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) {
            uint32_t j = fresh[idx[e]];
            if (j != 0xffffffffu) {
                oidx[o] = j;
                oval[o] = val[e];
                ++o;
            }
        }
        for (int64_t q = b + 1; q < o; ++q) {
            uint32_t key = oidx[q];
            double v = oval[q];
            int64_t r = q - 1;
            while (r >= b && oidx[r] > key) {
                oidx[r + 1] = oidx[r];
                oval[r + 1] = oval[r];
                --r;
            }
            oidx[r + 1] = key;
            oval[r + 1] = v;
        }
    }
}

void submatrix(const DevCsr& a, const int64_t* d_keep, int64_t nkeep, DevCsr* out,
               cudaStream_t s) {
    DevBuf<uint32_t> fresh(a.n);
    FG_CUDA(cudaMemsetAsync(fresh.p, 0xff, fresh.bytes(), s));
    DevBuf<int> bad(1);
    bad.zero(s);
    k_mark_keep<<<blocks_for(nkeep, 256), 256, 0, s>>>(d_keep, nkeep, a.n, fresh.p, bad.p);
    FG_CHECK_LAUNCH();
    int b = fetch(bad.p, s);
    if (b == 1) throw Failure(FEMGPU_ERR_INVALID, "a kept row is out of range");
    if (b == 2) throw Failure(FEMGPU_ERR_INVALID, "the kept rows hold an index twice");
    DevBuf<uint32_t> len(nkeep);
    k_sub_count<<<blocks_for(nkeep, 256), 256, 0, s>>>(d_keep, nkeep, a.ptr.p, a.idx.p, fresh.p,
                                                        len.p);
    out->n = nkeep;
    out->ptr.alloc(nkeep + 1);
    exclusive_scan32(len.p, out->ptr.p, nkeep, s);
    out->nnz = fetch(out->ptr.p + nkeep, s);
    out->idx.alloc(out->nnz);
    out->val.alloc(out->nnz);
    k_sub_fill<<<blocks_for(nkeep, 128), 128, 0, s>>>(d_keep, nkeep, a.ptr.p, a.idx.p, a.val.p,
                                                       fresh.p, out->ptr.p, out->idx.p,
                                                       out->val.p);
    FG_CHECK_LAUNCH();
}

// heat.rs:1219-1244 (steady): r = load_i - sum over the fixed columns j of a_ij t_j, in the
// order of the row.
__global__ void k_reduced_rhs(const int64_t* __restrict__ free, int64_t nfree,
                              const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                              const double* __restrict__ val, const uint32_t* __restrict__ fresh,
                              const double* __restrict__ load, const double* __restrict__ t,
                              double* __restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nfree;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = free[k];
        double r = load[i];
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) {
            uint32_t j = idx[e];
            if (fresh[j] == 0xffffffffu) r -= val[e] * t[j];
        }
        out[k] = r;
    }
}

void reduced_rhs(const DevCsr& a, const double* d_load, const double* d_t, const int64_t* d_free,
                 int64_t nfree, double* d_out, cudaStream_t s) {
    DevBuf<uint32_t> fresh(a.n);
    FG_CUDA(cudaMemsetAsync(fresh.p, 0xff, fresh.bytes(), s));
    DevBuf<int> bad(1);
    bad.zero(s);
    k_mark_keep<<<blocks_for(nfree, 256), 256, 0, s>>>(d_free, nfree, a.n, fresh.p, bad.p);
    FG_CHECK_LAUNCH();
    if (fetch(bad.p, s)) throw Failure(FEMGPU_ERR_INVALID, "the free list is not a set of rows");
    k_reduced_rhs<<<blocks_for(nfree, 256), 256, 0, s>>>(d_free, nfree, a.ptr.p, a.idx.p, a.val.p,
                                                         fresh.p, d_load, d_t, d_out);
    FG_CHECK_LAUNCH();
}

// sparse.rs:96-105 in FP64, 1 thread per row, the row's terms in order.
__global__ void k_csr_mul(int64_t n, const int64_t* __restrict__ ptr,
                          const uint32_t* __restrict__ idx, const double* __restrict__ val,
                          const double* __restrict__ x, double* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) s += val[e] * x[idx[e]];
        y[i] = s;
    }
}

void csr_mul(const DevCsr& a, const double* d_x, double* d_y, cudaStream_t s) {
    k_csr_mul<<<blocks_for(a.n, 256), 256, 0, s>>>(a.n, a.ptr.p, a.idx.p, a.val.p, d_x, d_y);
    FG_CHECK_LAUNCH();
}

}  // namespace femgpu
