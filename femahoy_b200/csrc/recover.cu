// Post-solve recovery of the 10-node tetrahedra on the device: the loop of
// elastic_tet.rs:367-427 (the strain and the stress at the 10 points of each cell, their mean at
// each point, the peak von Mises stress of each part) and the von Mises and principal stresses of
// the means (elastic_tet.rs:482-483).
//
// Layout in HBM, written once at setup: per cell a 128-byte record (the gradients of its 4
// volume coordinates, tet_gradients of heat.rs:983-1002, and its material number); per distinct
// material (E, nu, alpha) a 128-byte entry (D of hex.rs:58-114 and D alpha of
// elastic_tet.rs:164-170); the incidence of the assembly (the cells of each point in increasing
// order) and, beside it, the place (0-9) of the point in each of those cells. A recovery first
// copies u into 32 bytes per point, so that each point's displacement is 1 aligned 32-byte load.
//
// One thread per point walks its cells in increasing order, evaluates Tet10::strain_stress
// (tet10.rs:142-169) at its own volume coordinates in each, and sums. The reference adds the same
// terms to the same point in the same order, so the means are bit-identical with it. Each
// (cell, point) pair, a "visit", is evaluated exactly once, by the thread of its point. The unit
// is compiled with -fmad=false, so no multiply and add are fused.
//
// Peaks: the thread of each visit folds its von Mises stress into 3 running maxima of its part,
// each a 128-bit word updated by compare-and-swap: (value, ~key) for the peak and for the
// regular peak, where key = 10 cell + place orders the visits as the reference's loop, and
// (~key, value) for the first regular visit. The maximum of such words is the largest value and,
// among equal values, the smallest key: the reference's first strict maximum. Maxima are exact,
// so no order of the updates changes the result. With few parts the maxima live in shared memory
// per block and are folded into global memory at the end of the block.
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "assemble.cuh"
#include "common.cuh"
#include "elements.cuh"
#include "hex.cuh"
#include "rust_format.hpp"

namespace femgpu {

// One cell: the gradients of its 4 volume coordinates, its material, and its part with the
// `near` flag in the top bit (128 bytes, 4 aligned 32-byte loads).
struct alignas(32) CellRecord {
    double g[12];
    uint32_t mat;
    uint32_t tag;
    double pad[3];
};
static_assert(sizeof(CellRecord) == 128, "the cell record is 128 bytes");

// One material: D (normal 3 x 3 row-major, then G_yz, G_xz, G_xy) and D alpha (128 bytes).
struct alignas(32) MaterialEntry {
    double normal[9];
    double shear[3];
    double thermal[3];
    double pad;
};
static_assert(sizeof(MaterialEntry) == 128, "the material entry is 128 bytes");

constexpr int MAX_PARTS = 2048;
constexpr int SMEM_PARTS = 64;  // parts whose maxima a block keeps in shared memory
constexpr uint64_t NONE = ~0ull;
constexpr uint32_t NEAR_BIT = 0x80000000u;
typedef unsigned __int128 u128;

// tet10.rs:38, packed 4 bits per edge: the first and the second corner of edge k.
constexpr uint32_t EDGE_FIRST = 0x210010u;   // 0, 1, 0, 0, 1, 2
constexpr uint32_t EDGE_SECOND = 0x333221u;  // 1, 2, 2, 3, 3, 3

__device__ __forceinline__ int edge_corner(int k, int which) {
    return (int)(((which ? EDGE_SECOND : EDGE_FIRST) >> (4 * k)) & 0xfu);
}

// A 32-byte load through the read-only path; p is 32-byte aligned and not written by the kernel.
__device__ __forceinline__ void ld32(const double* p, double& a, double& b, double& c,
                                     double& d) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(a), "=d"(b), "=d"(c), "=d"(d)
        : "l"(p));
}

__device__ __forceinline__ bool is_nan_bits(uint64_t b) {
    return (b & 0x7fffffffffffffffull) > 0x7ff0000000000000ull;
}

// elastic.rs:977-983
__device__ __forceinline__ double mises6(const double s[6]) {
    double a = s[0] - s[1], b = s[1] - s[2], c = s[2] - s[0];
    return sqrt(0.5 * (a * a + b * b + c * c) + 3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

// elastic.rs:985-1002 (O. K. Smith, Comm. ACM 4 (1961) 168), largest first.
__device__ __forceinline__ void principal3(const double s[6], double out[3]) {
    double xx = s[0], yy = s[1], zz = s[2], xy = s[3], yz = s[4], xz = s[5];
    double q = (xx + yy + zz) / 3.0;
    double p1 = xy * xy + yz * yz + xz * xz;
    double p2 = (xx - q) * (xx - q) + (yy - q) * (yy - q) + (zz - q) * (zz - q) + 2.0 * p1;
    double p = sqrt(p2 / 6.0);
    if (p == 0.0) {
        out[0] = out[1] = out[2] = q;
        return;
    }
    double a = (xx - q) / p, b = (yy - q) / p, c = (zz - q) / p;
    double d = xy / p, e = yz / p, f = xz / p;
    double det = a * (b * c - e * e) - d * (d * c - e * f) + f * (d * e - b * f);
    double h = det / 2.0;
    if (h < -1.0) h = -1.0;  // f64::clamp, which keeps a NaN
    if (h > 1.0) h = 1.0;
    double phi = acos(h) / 3.0;
    const double pi = 3.141592653589793;
    double s1 = q + 2.0 * p * cos(phi);
    double s3 = q + 2.0 * p * cos(phi + 2.0 * pi / 3.0);
    out[0] = s1;
    out[1] = 3.0 * q - s1 - s3;
    out[2] = s3;
}

// Setup: D and D alpha of each distinct material (E, nu, alpha_x, alpha_y, alpha_z). Flag 2: no
// stable material (hex.rs:72-98).
__global__ void k_recover_materials(const double* __restrict__ in, int64_t nmat,
                                    MaterialEntry* __restrict__ out, int* __restrict__ bad) {
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < nmat;
         m += (int64_t)gridDim.x * blockDim.x) {
        const double* v = in + 5 * m;
        Stiffness D;
        if (!isotropic_stiffness(v[0], v[1], &D)) atomicExch(bad, 2);
        MaterialEntry r;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double s = -0.0;  // the Rust float sum starts from -0.0
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                r.normal[3 * i + j] = D.normal[i][j];
                s += D.normal[i][j] * v[2 + j];
            }
            r.thermal[i] = s;
            r.shear[i] = D.shear[i];
        }
        r.pad = 0.0;
        out[m] = r;
    }
}

// Setup: the record of each cell, with its part and `near` flag (a corner is singular:
// elastic_tet.rs:395). Flag 3: a part past the last.
__global__ void k_recover_cells(const double* __restrict__ xyz, const uint32_t* __restrict__ t10,
                                const uint32_t* __restrict__ mat,
                                const uint32_t* __restrict__ part, uint32_t nparts,
                                const uint8_t* __restrict__ singular, int64_t nel,
                                CellRecord* __restrict__ rec, int* __restrict__ bad) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t* t = t10 + 10 * e;
        double p[4][3];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int d = 0; d < 3; ++d) p[k][d] = xyz[3 * (int64_t)t[k] + d];
        double g[4][3], volume;
        tet_gradients(p, g, &volume);
        CellRecord r;
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int d = 0; d < 3; ++d) r.g[3 * k + d] = g[k][d];
        uint32_t pt = part ? part[e] : 0u;
        if (pt >= nparts) atomicExch(bad, 3);
        bool near = false;
        if (singular)
#pragma unroll
            for (int k = 0; k < 4; ++k) near = near || singular[t[k]] != 0;
        r.mat = mat[e];
        r.tag = (pt & ~NEAR_BIT) | (near ? NEAR_BIT : 0u);
        r.pad[0] = r.pad[1] = r.pad[2] = 0.0;
        rec[e] = r;
    }
}

// Setup: the place of point v in each of its cells (M points each). A cell that names the point
// twice is listed twice and takes its places in order, as the reference's loop over its points.
template <int M>
__global__ void k_visit_places(const uint32_t* __restrict__ t10, const int64_t* __restrict__ start,
                               const uint32_t* __restrict__ of_node, int64_t npoints,
                               uint8_t* __restrict__ place) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < npoints;
         v += (int64_t)gridDim.x * blockDim.x) {
        uint32_t last = 0xffffffffu;
        int lastc = -1;
        for (int64_t k = start[v]; k < start[v + 1]; ++k) {
            const uint32_t e = of_node[k];
            const uint32_t* t = t10 + M * (int64_t)e;
            int c = e == last ? lastc + 1 : 0;
            while (c < M && t[c] != (uint32_t)v) ++c;
            // c < M: the incidence was built from these cells.
            place[k] = (uint8_t)c;
            last = e;
            lastc = c;
        }
    }
}

// u (3 per point) into 4 per point, the 4th 0.
__global__ void k_pad_u(const double* __restrict__ u, int64_t npoints, double* __restrict__ u4) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < npoints;
         v += (int64_t)gridDim.x * blockDim.x) {
        const double a = u[3 * v], b = u[3 * v + 1], c = u[3 * v + 2];
        double2* o = reinterpret_cast<double2*>(u4 + 4 * v);
        o[0] = make_double2(a, b);
        o[1] = make_double2(c, 0.0);
    }
}

// Tet10::strain_stress (tet10.rs:142-169) of cell e (record rp, points t) at its point c,
// followed by reorder and tensor_strain (elastic.rs:967-975): sig and eps in the order xx, yy,
// zz, xy, yz, xz.
__device__ __forceinline__ void strain_stress_l(const CellRecord* __restrict__ rp,
                                                const MaterialEntry* __restrict__ mats,
                                                const uint32_t t[10], const double l[4],
                                                const double* __restrict__ u4,
                                                const double* __restrict__ dtemp,
                                                double sig[6], double eps[6], uint32_t* tag);

__device__ __forceinline__ void strain_stress_at(const CellRecord* __restrict__ rp,
                                                 const MaterialEntry* __restrict__ mats,
                                                 const uint32_t t[10], int c,
                                                 const double* __restrict__ u4,
                                                 const double* __restrict__ dtemp,
                                                 double sig[6], double eps[6], uint32_t* tag) {
    // node_coordinates (tet10.rs:216-228)
    double l[4];
    if (c < 4) {
#pragma unroll
        for (int k = 0; k < 4; ++k) l[k] = k == c ? 1.0 : 0.0;
    } else {
        const int i = edge_corner(c - 4, 0), j = edge_corner(c - 4, 1);
#pragma unroll
        for (int k = 0; k < 4; ++k) l[k] = (k == i || k == j) ? 0.5 : 0.0;
    }
    strain_stress_l(rp, mats, t, l, u4, dtemp, sig, eps, tag);
}

// Tet10::strain_stress (tet10.rs:142-169) of cell e at the volume coordinates l, with reorder
// and tensor_strain as above.
__device__ __forceinline__ void strain_stress_l(const CellRecord* __restrict__ rp,
                                                const MaterialEntry* __restrict__ mats,
                                                const uint32_t t[10], const double l[4],
                                                const double* __restrict__ u4,
                                                const double* __restrict__ dtemp,
                                                double sig[6], double eps[6], uint32_t* tag) {
    const double* rd = reinterpret_cast<const double*>(rp);
    double g[12];
#pragma unroll
    for (int k = 0; k < 3; ++k) ld32(rd + 4 * k, g[4 * k], g[4 * k + 1], g[4 * k + 2], g[4 * k + 3]);
    const uint2 mt = __ldg(reinterpret_cast<const uint2*>(rd + 12));
    const uint32_t mat = mt.x;
    *tag = mt.y;
    double e[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 10; ++i) {
        // The gradient of function i at l (tet10.rs:77-87).
        double gi[3];
        if (i < 4) {
            const double f = 4.0 * l[i] - 1.0;
#pragma unroll
            for (int d = 0; d < 3; ++d) gi[d] = f * g[3 * i + d];
        } else {
            const int a = edge_corner(i - 4, 0), b = edge_corner(i - 4, 1);
#pragma unroll
            for (int d = 0; d < 3; ++d) gi[d] = 4.0 * (l[a] * g[3 * b + d] + l[b] * g[3 * a + d]);
        }
        double ui[3], unused;
        ld32(u4 + 4 * (int64_t)t[i], ui[0], ui[1], ui[2], unused);
#pragma unroll
        for (int a = 0; a < 3; ++a) e[a] += gi[a] * ui[a];
        // SHEAR (tet10.rs:41): yz, xz, xy
        e[3] += gi[1] * ui[2] + gi[2] * ui[1];
        e[4] += gi[0] * ui[2] + gi[2] * ui[0];
        e[5] += gi[0] * ui[1] + gi[1] * ui[0];
    }
    double dt = -0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) dt += l[k] * (dtemp ? __ldg(dtemp + t[k]) : 0.0);
    const double* md = reinterpret_cast<const double*>(mats + mat);
    double w[16];
#pragma unroll
    for (int k = 0; k < 4; ++k) ld32(md + 4 * k, w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
    // w[0..9) normal, w[9..12) shear, w[12..15) thermal.
    double s[6];
#pragma unroll
    for (int a = 0; a < 3; ++a)  // hex.rs:128-139
        s[a] = w[3 * a] * e[0] + w[3 * a + 1] * e[1] + w[3 * a + 2] * e[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) s[3 + k] = w[9 + k] * e[3 + k];
#pragma unroll
    for (int a = 0; a < 3; ++a) s[a] -= w[12 + a] * dt;
    sig[0] = s[0];
    sig[1] = s[1];
    sig[2] = s[2];
    sig[3] = s[5];
    sig[4] = s[3];
    sig[5] = s[4];
    eps[0] = e[0];
    eps[1] = e[1];
    eps[2] = e[2];
    eps[3] = 0.5 * e[5];
    eps[4] = 0.5 * e[3];
    eps[5] = 0.5 * e[4];
}

// max(*a, v) by compare-and-swap. The high half of *a never decreases, so a v whose high half
// is below it is below *a and needs no atomic.
__device__ __forceinline__ void fold_max(u128* a, u128 v) {
    const unsigned long long vh = (unsigned long long)(v >> 64);
    const unsigned long long ch =
        *(reinterpret_cast<volatile unsigned long long*>(a) + 1);  // little-endian: high half
    if (vh < ch) return;
    u128 old = atomicCAS(a, (u128)0, (u128)0);  // an atomic read (0 stays 0)
    while (v > old) {
        const u128 prev = atomicCAS(a, old, v);
        if (prev == old) break;
        old = prev;  // another thread raised it: compare again
    }
}

// One thread per point: the sums of elastic_tet.rs:396-403 over the point's cells in
// increasing order, the means of elastic_tet.rs:419-425, and elastic_tet.rs:482-483. With
// PEAKS, the peaks of elastic_tet.rs:405-416 into `peak` (3 words per part: peak, regular peak,
// first regular visit), through shared memory when SMEM.
template <bool PEAKS, bool SMEM>
__global__ void __launch_bounds__(128, 4)
    k_recover_points(const CellRecord* __restrict__ rec, const MaterialEntry* __restrict__ mats,
                     const uint32_t* __restrict__ t10, const int64_t* __restrict__ start,
                     const uint32_t* __restrict__ of_node, const uint8_t* __restrict__ place,
                     const double* __restrict__ u4, const double* __restrict__ dtemp,
                     const uint8_t* __restrict__ singular, int64_t npoints, int nparts,
                     double* __restrict__ stress, double* __restrict__ strain,
                     double* __restrict__ mises_out, double* __restrict__ principal_out,
                     u128* __restrict__ peak) {
    extern __shared__ u128 peak_s[];
    u128* fold = SMEM ? peak_s : peak;
    if (PEAKS && SMEM) {
        for (int i = threadIdx.x; i < 3 * nparts; i += blockDim.x) peak_s[i] = 0;
        __syncthreads();
    }
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < npoints;
         v += (int64_t)gridDim.x * blockDim.x) {
        double ss[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        double se[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        const int64_t b = start[v], end = start[v + 1];
        const bool sing_v = PEAKS && singular && singular[v];
        for (int64_t k = b; k < end; ++k) {
            const uint32_t e = __ldg(of_node + k);
            const int c = __ldg(place + k);
            const uint2* row = reinterpret_cast<const uint2*>(t10 + 10 * (int64_t)e);
            uint32_t t[10];
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const uint2 w = __ldg(row + q);
                t[2 * q] = w.x;
                t[2 * q + 1] = w.y;
            }
            double sig[6], eps[6];
            uint32_t tg;
            strain_stress_at(rec + e, mats, t, c, u4, dtemp, sig, eps, &tg);
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                ss[i] += sig[i];
                se[i] += eps[i];
            }
            if (PEAKS) {
                const unsigned long long bits =
                    (unsigned long long)__double_as_longlong(mises6(sig));
                const unsigned long long key = 10ull * e + c;
                const int p = (int)(tg & ~NEAR_BIT);
                const bool reg = !(tg & NEAR_BIT) && !sing_v;
                const bool nan = is_nan_bits(bits);
                const u128 vk = ((u128)bits << 64) | (u128)(NONE - key);
                if (!nan) fold_max(fold + 3 * p, vk);
                if (reg) {
                    if (!nan) fold_max(fold + 3 * p + 1, vk);
                    fold_max(fold + 3 * p + 2, ((u128)(NONE - key) << 64) | (u128)bits);
                }
            }
        }
        int64_t count = end - b;
        const double cnt = (double)(count > 1 ? count : 1);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            ss[i] /= cnt;
            se[i] /= cnt;
            stress[6 * v + i] = ss[i];
            strain[6 * v + i] = se[i];
        }
        if (mises_out) mises_out[v] = mises6(ss);
        if (principal_out) {
            double pr[3];
            principal3(ss, pr);
#pragma unroll
            for (int i = 0; i < 3; ++i) principal_out[3 * v + i] = pr[i];
        }
    }
    if (PEAKS && SMEM) {
        __syncthreads();
        for (int i = threadIdx.x; i < 3 * nparts; i += blockDim.x)
            if (peak_s[i] != 0) fold_max(peak + i, peak_s[i]);
    }
}

// ------------------------------------------------------------------ box cells
// The box grid's loop (elastic.rs:615-660): Hex::strain_stress (hex.rs:311-335) at the 8 corners
// of each cell. Each distinct cell (sides, material, expansion) has a record of HEX_MODES values
// (hex.cuh: mode_u, mode_t, D, D alpha, the sides), made once at setup; each cell has its class
// and its part with the `near` flag (8 bytes). A run first forms the 9 mode amplitudes of each
// cell (a = mode_t T - mode_u u, hex.rs:316-326), once per cell, then 1 thread per point walks its
// cells in increasing order as for the tetrahedra.

// Setup: each cell's class and tag. Flag 3: a part past the last.
__global__ void k_recover_hex_cells(const uint32_t* __restrict__ hexes,
                                    const uint32_t* __restrict__ cls,
                                    const uint32_t* __restrict__ part, uint32_t nparts,
                                    const uint8_t* __restrict__ singular, int64_t nel,
                                    uint2* __restrict__ rec, int* __restrict__ bad) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t pt = part ? part[e] : 0u;
        if (pt >= nparts) atomicExch(bad, 3);
        bool near = false;
        if (singular)
#pragma unroll
            for (int k = 0; k < 8; ++k) near = near || singular[hexes[8 * e + k]] != 0;
        rec[e] = make_uint2(cls[e], (pt & ~NEAR_BIT) | (near ? NEAR_BIT : 0u));
    }
}

// The 9 mode amplitudes of each cell (hex.rs:316-326): a_i = sum_c mode_t[i][c] T_c, then minus
// sum_c mode_u[i][c] u_c, each from 0.0 in the reference's order; 12 values per cell.
__global__ void k_hex_amplitudes(const uint32_t* __restrict__ hexes, const uint2* __restrict__ rec,
                                 const double* __restrict__ modes, const double* __restrict__ u4,
                                 const double* __restrict__ dtemp, int64_t nel,
                                 double* __restrict__ amp) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x) {
        const double* m = modes + HEX_MODES * (int64_t)__ldg(&rec[e].x);
        double u[24], t[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const uint32_t v = __ldg(hexes + 8 * e + n);
            double unused;
            ld32(u4 + 4 * (int64_t)v, u[3 * n], u[3 * n + 1], u[3 * n + 2], unused);
            t[n] = dtemp ? __ldg(dtemp + v) : 0.0;
        }
        double* out = amp + 12 * e;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            double a = 0.0;
#pragma unroll
            for (int c = 0; c < 8; ++c) a += __ldg(m + HEX_MODE_T + 8 * i + c) * t[c];
#pragma unroll
            for (int c = 0; c < 24; ++c) a -= __ldg(m + HEX_MODE_U + 24 * i + c) * u[c];
            out[i] = a;
        }
        out[9] = out[10] = out[11] = 0.0;
    }
}

// Hex::strain_stress of cell e at its corner c (xi = -1 or 1 per axis), then reorder and
// tensor_strain (elastic.rs:967-975): sig and eps in the order xx, yy, zz, xy, yz, xz.
__device__ __forceinline__ void hex_strain_stress_at(const double* __restrict__ m,
                                                     const uint32_t t[8],
                                                     const double* __restrict__ a, int c,
                                                     const double* __restrict__ u4,
                                                     const double* __restrict__ dtemp,
                                                     double sig[6], double eps[6]) {
    double xi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) xi[d] = hex_bit(c, d) == 1 ? 1.0 : -1.0;
    const double* gc = m + HEX_GRAD + 33 * c;  // hex_gradients at this corner, made at setup
    double e[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 11; ++i) {
        const double g[3] = {__ldg(gc + 3 * i), __ldg(gc + 3 * i + 1), __ldg(gc + 3 * i + 2)};
        double ui[3];
        if (i < 8) {
            double unused;
            ld32(u4 + 4 * (int64_t)t[i], ui[0], ui[1], ui[2], unused);
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) ui[k] = __ldg(a + 3 * (i - 8) + k);
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) e[q] += g[q] * ui[q];
        // SHEAR (hex.rs:143): yz, xz, xy
        e[3] += g[1] * ui[2] + g[2] * ui[1];
        e[4] += g[0] * ui[2] + g[2] * ui[0];
        e[5] += g[0] * ui[1] + g[1] * ui[0];
    }
    double n[8];
    hex_shape(xi, n);
    double dt = -0.0;  // the Rust float sum starts from -0.0
#pragma unroll
    for (int k = 0; k < 8; ++k) dt += n[k] * (dtemp ? __ldg(dtemp + t[k]) : 0.0);
    double s[6];
#pragma unroll
    for (int q = 0; q < 3; ++q)  // hex.rs:128-139
        s[q] = __ldg(m + HEX_NORMAL + 3 * q) * e[0] + __ldg(m + HEX_NORMAL + 3 * q + 1) * e[1] +
               __ldg(m + HEX_NORMAL + 3 * q + 2) * e[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) s[3 + k] = __ldg(m + HEX_SHEAR + k) * e[3 + k];
#pragma unroll
    for (int q = 0; q < 3; ++q) s[q] -= __ldg(m + HEX_THERMAL + q) * dt;
    sig[0] = s[0];
    sig[1] = s[1];
    sig[2] = s[2];
    sig[3] = s[5];
    sig[4] = s[3];
    sig[5] = s[4];
    eps[0] = e[0];
    eps[1] = e[1];
    eps[2] = e[2];
    eps[3] = 0.5 * e[5];
    eps[4] = 0.5 * e[3];
    eps[5] = 0.5 * e[4];
}

// One thread per point, as k_recover_points, over the 8 corners of the box cells (the visit key
// of a peak is 8 cell + corner: the reference's loop order).
template <bool PEAKS, bool SMEM>
__global__ void __launch_bounds__(128, 4)
    k_recover_hex_points(const uint2* __restrict__ rec, const double* __restrict__ modes,
                         const double* __restrict__ amp, const uint32_t* __restrict__ hexes,
                         const int64_t* __restrict__ start, const uint32_t* __restrict__ of_node,
                         const uint8_t* __restrict__ place, const double* __restrict__ u4,
                         const double* __restrict__ dtemp, const uint8_t* __restrict__ singular,
                         int64_t npoints, int nparts, double* __restrict__ stress,
                         double* __restrict__ strain, double* __restrict__ mises_out,
                         double* __restrict__ principal_out, u128* __restrict__ peak) {
    extern __shared__ u128 peak_s[];
    u128* fold = SMEM ? peak_s : peak;
    if (PEAKS && SMEM) {
        for (int i = threadIdx.x; i < 3 * nparts; i += blockDim.x) peak_s[i] = 0;
        __syncthreads();
    }
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < npoints;
         v += (int64_t)gridDim.x * blockDim.x) {
        double ss[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        double se[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        const int64_t b = start[v], end = start[v + 1];
        const bool sing_v = PEAKS && singular && singular[v];
        for (int64_t k = b; k < end; ++k) {
            const uint32_t e = __ldg(of_node + k);
            const int c = __ldg(place + k);
            const uint4* row = reinterpret_cast<const uint4*>(hexes + 8 * (int64_t)e);
            const uint4 w0 = __ldg(row), w1 = __ldg(row + 1);
            const uint32_t t[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
            const uint2 r = __ldg(rec + e);
            double sig[6], eps[6];
            hex_strain_stress_at(modes + HEX_MODES * (int64_t)r.x, t, amp + 12 * (int64_t)e, c, u4,
                                 dtemp, sig, eps);
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                ss[i] += sig[i];
                se[i] += eps[i];
            }
            if (PEAKS) {
                const unsigned long long bits =
                    (unsigned long long)__double_as_longlong(mises6(sig));
                const unsigned long long key = 8ull * e + c;
                const int p = (int)(r.y & ~NEAR_BIT);
                const bool reg = !(r.y & NEAR_BIT) && !sing_v;
                const bool nan = is_nan_bits(bits);
                const u128 vk = ((u128)bits << 64) | (u128)(NONE - key);
                if (!nan) fold_max(fold + 3 * p, vk);
                if (reg) {
                    if (!nan) fold_max(fold + 3 * p + 1, vk);
                    fold_max(fold + 3 * p + 2, ((u128)(NONE - key) << 64) | (u128)bits);
                }
            }
        }
        const int64_t count = end - b;
        const double cnt = (double)(count > 1 ? count : 1);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            ss[i] /= cnt;
            se[i] /= cnt;
            stress[6 * v + i] = ss[i];
            strain[6 * v + i] = se[i];
        }
        if (mises_out) mises_out[v] = mises6(ss);
        if (principal_out) {
            double pr[3];
            principal3(ss, pr);
#pragma unroll
            for (int i = 0; i < 3; ++i) principal_out[3 * v + i] = pr[i];
        }
    }
    if (PEAKS && SMEM) {
        __syncthreads();
        for (int i = threadIdx.x; i < 3 * nparts; i += blockDim.x)
            if (peak_s[i] != 0) fold_max(peak + i, peak_s[i]);
    }
}

// The thermal and volume forces of the box cells (elastic.rs:386-405), 1 thread per point: over
// its cells in increasing order, f = sum_c load[3 a + d][c] T_c from 0.0 (a = the point's corner),
// plus accel_d times the volume / 8, added to force[3 v + d] from 0.0: the reference's order.
__global__ void k_hex_loads(const uint32_t* __restrict__ hexes, const uint32_t* __restrict__ cls,
                            const double* __restrict__ modes, const int64_t* __restrict__ start,
                            const uint32_t* __restrict__ of_node, const uint8_t* __restrict__ place,
                            const double* __restrict__ accel, const double* __restrict__ dtemp,
                            int64_t npoints, double* __restrict__ force) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < npoints;
         v += (int64_t)gridDim.x * blockDim.x) {
        double fv[3] = {0.0, 0.0, 0.0};
        for (int64_t k = start[v]; k < start[v + 1]; ++k) {
            const uint32_t e = __ldg(of_node + k);
            const int a = __ldg(place + k);
            const double* m = modes + HEX_MODES * (int64_t)__ldg(cls + e);
            double t[8];
#pragma unroll
            for (int c = 0; c < 8; ++c)
                t[c] = dtemp ? __ldg(dtemp + __ldg(hexes + 8 * (int64_t)e + c)) : 0.0;
            const double volume =
                __ldg(m + HEX_SIZE) * __ldg(m + HEX_SIZE + 1) * __ldg(m + HEX_SIZE + 2);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double f = 0.0;
#pragma unroll
                for (int c = 0; c < 8; ++c) f += __ldg(m + HEX_LOAD + 8 * (3 * a + d) + c) * t[c];
                f += (accel ? __ldg(accel + 3 * (int64_t)e + d) : 0.0) * volume / 8.0;
                fv[d] += f;
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) force[3 * v + d] = fv[d];
    }
}

// 1 thread per part: the reference's Peak (elastic_tet.rs:405-416, elastic.rs:636-650) from the
// 3 maxima; cells of `nn` points (`el`), the tag of cell e at tag[stride e]. The first regular
// visit stays the regular peak when its value is NaN, since no value is greater than NaN.
__global__ void k_peak_final(const u128* __restrict__ peak, int nparts,
                             const uint32_t* __restrict__ t10, int nn,
                             const uint32_t* __restrict__ tag, int stride,
                             const uint8_t* __restrict__ singular, femgpu_peak* __restrict__ out) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nparts) return;
    const u128 all = peak[3 * p], reg = peak[3 * p + 1], first = peak[3 * p + 2];
    femgpu_peak o;
    memset(&o, 0, sizeof(o));
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    if (all == 0) {
        o.mises = -inf;
        o.element = -1;
    } else {
        const uint64_t key = NONE - (uint64_t)all;
        o.mises = __longlong_as_double((long long)(uint64_t)(all >> 64));
        o.element = (int64_t)(key / nn);
        o.local = (int32_t)(key % nn);
        o.point = t10[key];
        o.singular =
            ((tag[stride * (key / nn)] & NEAR_BIT) || (singular && singular[o.point])) ? 1 : 0;
    }
    uint64_t rk = NONE;
    double rm = -inf;
    if (first != 0) {
        const uint64_t fbits = (uint64_t)first;
        if (is_nan_bits(fbits)) {
            rk = NONE - (uint64_t)(first >> 64);
            rm = __longlong_as_double((long long)fbits);
        } else {
            rk = NONE - (uint64_t)reg;
            rm = __longlong_as_double((long long)(uint64_t)(reg >> 64));
        }
    }
    if (rk == NONE) {
        o.regular_mises = -inf;
        o.regular_element = -1;
    } else {
        o.regular_mises = rm;
        o.regular_element = (int64_t)(rk / nn);
        o.regular_local = (int32_t)(rk % nn);
        o.regular_point = t10[rk];
    }
    out[p] = o;
}

}  // namespace femgpu

using namespace femgpu;

// ------------------------------------------------------------------ probes
// elastic_tet.rs:428-467 with cells_at (elastic_tet.rs:538-553): a probe takes the cells whose
// volume coordinates of its point are all >= -1e-9. k_probe_hits tests every (probe, cell) pair
// (a few probes against all cells, as the reference's search) and lists the hits; then 1 thread
// per probe sorts its hits and sums their shares in increasing cell order, the reference's
// order, so the values are bit-identical (the unit is built with -fmad=false).
constexpr int MAX_PROBE_HITS = 512;

// The volume coordinates of x in cell e: l[i] = sum_d g[i][d] (x[d] - p0[d]) for i >= 1 (a
// float sum from -0.0), l[0] = 1 - l[1] - l[2] - l[3].
__device__ __forceinline__ void probe_coordinates(const CellRecord& r, const double* p0,
                                                  const double x[3], double l[4]) {
#pragma unroll
    for (int i = 1; i < 4; ++i) {
        double sum = -0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) sum += r.g[3 * i + d] * (x[d] - p0[d]);
        l[i] = sum;
    }
    l[0] = 1.0 - l[1] - l[2] - l[3];
}

__global__ void k_probe_hits(const CellRecord* __restrict__ rec, const double* __restrict__ xyz,
                             const uint32_t* __restrict__ t10, int64_t nel,
                             const double* __restrict__ points, int64_t nprobes,
                             int* __restrict__ count, int64_t* __restrict__ hits) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nel * nprobes;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = k / nel, e = k % nel;
        const double x[3] = {points[3 * q], points[3 * q + 1], points[3 * q + 2]};
        const double* p0 = xyz + 3 * (int64_t)t10[10 * e];
        double l[4];
        probe_coordinates(rec[e], p0, x, l);
        if (l[0] >= -1e-9 && l[1] >= -1e-9 && l[2] >= -1e-9 && l[3] >= -1e-9) {
            const int slot = atomicAdd(count + q, 1);
            if (slot < MAX_PROBE_HITS) hits[q * MAX_PROBE_HITS + slot] = e;
        }
    }
}

__global__ void k_probe_values(const CellRecord* __restrict__ rec,
                               const MaterialEntry* __restrict__ mats,
                               const double* __restrict__ xyz, const uint32_t* __restrict__ t10,
                               const double* __restrict__ u4, const double* __restrict__ dtemp,
                               const double* __restrict__ temperature,
                               const double* __restrict__ points, int64_t nprobes,
                               const int* __restrict__ count, int64_t* __restrict__ hits,
                               double* __restrict__ disp, double* __restrict__ stress,
                               double* __restrict__ mises, double* __restrict__ temp) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nprobes;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int m = count[q];
        if (m < 1 || m > MAX_PROBE_HITS) continue;
        int64_t* h = hits + q * MAX_PROBE_HITS;
        for (int a = 1; a < m; ++a) {  // insertion sort: increasing cells
            const int64_t v = h[a];
            int b = a;
            while (b > 0 && h[b - 1] > v) {
                h[b] = h[b - 1];
                --b;
            }
            h[b] = v;
        }
        const double x[3] = {points[3 * q], points[3 * q + 1], points[3 * q + 2]};
        const double share = 1.0 / (double)m;
        double dsp[3] = {0.0, 0.0, 0.0}, sg[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, tv = 0.0;
        for (int k = 0; k < m; ++k) {
            const int64_t e = h[k];
            uint32_t t[10];
#pragma unroll
            for (int c = 0; c < 10; ++c) t[c] = t10[10 * e + c];
            double l[4];
            probe_coordinates(rec[e], xyz + 3 * (int64_t)t[0], x, l);
            // Tet10 shape functions (tet10.rs:51-60).
            double w[10];
#pragma unroll
            for (int i = 0; i < 4; ++i) w[i] = l[i] * (2.0 * l[i] - 1.0);
#pragma unroll
            for (int j = 0; j < 6; ++j) w[4 + j] = 4.0 * l[edge_corner(j, 0)] * l[edge_corner(j, 1)];
#pragma unroll
            for (int c = 0; c < 10; ++c) {
                double ui[3], unused;
                ld32(u4 + 4 * (int64_t)t[c], ui[0], ui[1], ui[2], unused);
#pragma unroll
                for (int a = 0; a < 3; ++a) dsp[a] += share * w[c] * ui[a];
            }
            double sig[6], eps[6];
            uint32_t tag;
            strain_stress_l(rec + e, mats, t, l, u4, dtemp, sig, eps, &tag);
#pragma unroll
            for (int i = 0; i < 6; ++i) sg[i] += share * sig[i];
            if (temperature) {
                double sum = -0.0;
#pragma unroll
                for (int c = 0; c < 4; ++c) sum += l[c] * temperature[t[c]];
                tv += share * sum;
            }
        }
        for (int a = 0; a < 3; ++a) disp[3 * q + a] = dsp[a];
        for (int i = 0; i < 6; ++i) stress[6 * q + i] = sg[i];
        mises[q] = mises6(sg);
        temp[q] = tv;
    }
}

struct femgpu_recovery {
    int64_t npoints = 0, nel = 0, nmat = 0;
    int nparts = 1;
    bool has_singular = false;
    // Box cells (femgpu_recovery_new_hex): t10 then holds 8 corners per cell.
    bool hex = false;
    DevBuf<uint2> hrec;
    DevBuf<double> hmodes, amp;
    Incidence inc;
    DevBuf<uint8_t> place;
    DevBuf<uint32_t> t10;
    DevBuf<double> xyz;  // the points (P2 cells), for the probes
    DevBuf<CellRecord> rec;
    DevBuf<MaterialEntry> mats;
    DevBuf<uint8_t> singular;
    DevBuf<double> u4;
    DevBuf<u128> peak;
    DevBuf<femgpu_peak> dpeaks;
    // Device copies for the host-pointer form.
    DevBuf<double> du, ddt, dstress, dstrain, dmises, dprincipal;
    cudaStream_t s = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0, last_bytes = 0.0;
    ~femgpu_recovery() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (s) cudaStreamDestroy(s);
    }

    void run(const double* u, const double* dtemp, double* stress, double* strain,
             double* mises, double* principal, femgpu_peak* peaks) {
        const bool want_peaks = peaks != nullptr;
        const uint8_t* sing = has_singular ? singular.p : nullptr;
        FG_CUDA(cudaEventRecord(ev0, s));
        k_pad_u<<<blocks_for(npoints, 256), 256, 0, s>>>(u, npoints, u4.p);
        FG_CHECK_LAUNCH();
        const int grid = blocks_for(npoints, 128, NUM_SMS * 64);
        if (hex) {
            run_hex(dtemp, stress, strain, mises, principal, peaks, grid);
            return;
        }
        if (!want_peaks) {
            k_recover_points<false, false><<<grid, 128, 0, s>>>(
                rec.p, mats.p, t10.p, inc.start.p, inc.of_node.p, place.p, u4.p, dtemp, sing,
                npoints, nparts, stress, strain, mises, principal, nullptr);
        } else {
            peak.zero(s);
            if (nparts <= SMEM_PARTS)
                k_recover_points<true, true><<<grid, 128, 3 * sizeof(u128) * nparts, s>>>(
                    rec.p, mats.p, t10.p, inc.start.p, inc.of_node.p, place.p, u4.p, dtemp, sing,
                    npoints, nparts, stress, strain, mises, principal, peak.p);
            else
                k_recover_points<true, false><<<grid, 128, 0, s>>>(
                    rec.p, mats.p, t10.p, inc.start.p, inc.of_node.p, place.p, u4.p, dtemp, sing,
                    npoints, nparts, stress, strain, mises, principal, peak.p);
        }
        FG_CHECK_LAUNCH();
        if (want_peaks) {
            k_peak_final<<<(nparts + 127) / 128, 128, 0, s>>>(
                peak.p, nparts, t10.p, 10, reinterpret_cast<const uint32_t*>(rec.p) + 25, 32, sing,
                dpeaks.p);
            FG_CHECK_LAUNCH();
        }
        FG_CUDA(cudaEventRecord(ev1, s));
        if (want_peaks) dpeaks.download(peaks, nparts, s);
        FG_CUDA(cudaStreamSynchronize(s));
        float ms = 0.f;
        FG_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        // Each array once: u read, written padded and read padded; the cell records and point
        // numbers; the incidence with its places; the outputs.
        last_bytes = npoints * (24.0 + 32.0 + 32.0) + nel * (sizeof(CellRecord) + 40.0) +
                     nmat * (double)sizeof(MaterialEntry) + (npoints + 1) * 8.0 +
                     10.0 * nel * 5.0 + (dtemp ? npoints * 8.0 : 0.0) + npoints * 96.0 +
                     (mises ? npoints * 8.0 : 0.0) + (principal ? npoints * 24.0 : 0.0) +
                     (want_peaks && has_singular ? npoints * 1.0 : 0.0);
    }

    void run_hex(const double* dtemp, double* stress, double* strain, double* mises,
                 double* principal, femgpu_peak* peaks, int grid) {
        const bool want_peaks = peaks != nullptr;
        const uint8_t* sing = has_singular ? singular.p : nullptr;
        k_hex_amplitudes<<<blocks_for(nel, 128, NUM_SMS * 32), 128, 0, s>>>(
            t10.p, hrec.p, hmodes.p, u4.p, dtemp, nel, amp.p);
        FG_CHECK_LAUNCH();
        if (!want_peaks) {
            k_recover_hex_points<false, false><<<grid, 128, 0, s>>>(
                hrec.p, hmodes.p, amp.p, t10.p, inc.start.p, inc.of_node.p, place.p, u4.p, dtemp,
                sing, npoints, nparts, stress, strain, mises, principal, nullptr);
        } else {
            peak.zero(s);
            if (nparts <= SMEM_PARTS)
                k_recover_hex_points<true, true><<<grid, 128, 3 * sizeof(u128) * nparts, s>>>(
                    hrec.p, hmodes.p, amp.p, t10.p, inc.start.p, inc.of_node.p, place.p, u4.p,
                    dtemp, sing, npoints, nparts, stress, strain, mises, principal, peak.p);
            else
                k_recover_hex_points<true, false><<<grid, 128, 0, s>>>(
                    hrec.p, hmodes.p, amp.p, t10.p, inc.start.p, inc.of_node.p, place.p, u4.p,
                    dtemp, sing, npoints, nparts, stress, strain, mises, principal, peak.p);
        }
        FG_CHECK_LAUNCH();
        if (want_peaks) {
            k_peak_final<<<(nparts + 127) / 128, 128, 0, s>>>(
                peak.p, nparts, t10.p, 8, reinterpret_cast<const uint32_t*>(hrec.p) + 1, 2, sing,
                dpeaks.p);
            FG_CHECK_LAUNCH();
        }
        FG_CUDA(cudaEventRecord(ev1, s));
        if (want_peaks) dpeaks.download(peaks, nparts, s);
        FG_CUDA(cudaStreamSynchronize(s));
        float ms = 0.f;
        FG_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        // Each array once: u read, written padded and read padded; the cells' corners, records
        // and amplitudes (written and read); the class records; the incidence with its places;
        // the outputs.
        last_bytes = npoints * (24.0 + 32.0 + 32.0) + nel * (32.0 + 8.0 + 2 * 96.0) +
                     nmat * HEX_MODES * 8.0 + (npoints + 1) * 8.0 + 8.0 * nel * 5.0 +
                     (dtemp ? npoints * 8.0 : 0.0) + npoints * 96.0 +
                     (mises ? npoints * 8.0 : 0.0) + (principal ? npoints * 24.0 : 0.0) +
                     (want_peaks && has_singular ? npoints * 1.0 : 0.0);
    }
};

namespace {
template <class F>
int recovery_guarded(F f) {
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
}  // namespace

extern "C" {

int femgpu_recovery_new(size_t npoints, const double* xyz, size_t nel, const uint32_t* tets10,
                        const double* coef, const double* expansion, const uint32_t* part,
                        size_t nparts, const uint8_t* singular, femgpu_recovery** out) {
    return recovery_guarded([&] {
        need(out != nullptr, "out is null");
        need(npoints > 0 && nel > 0, "an empty mesh");
        need(xyz && tets10 && coef, "a null mesh array");
        need(nparts >= 1, "no part");
        if (nparts > (size_t)MAX_PARTS)
            throw Failure(FEMGPU_ERR_TOO_LARGE, "more than 2048 parts");
        if (npoints >= 0xffffffffull || nel >= 0xffffffffull / 10)
            throw Failure(FEMGPU_ERR_TOO_LARGE, "more points or cells than 32-bit numbers hold");
        auto r = std::make_unique<femgpu_recovery>();
        FG_CUDA(cudaStreamCreateWithFlags(&r->s, cudaStreamNonBlocking));
        FG_CUDA(cudaEventCreate(&r->ev0));
        FG_CUDA(cudaEventCreate(&r->ev1));
        cudaStream_t s = r->s;
        r->npoints = (int64_t)npoints;
        r->nel = (int64_t)nel;
        r->nparts = (int)nparts;
        r->t10.upload(tets10, 10 * nel, s);
        build_incidence(r->t10.p, r->nel, 10, r->npoints, &r->inc, s);
        r->place.alloc(10 * nel);
        k_visit_places<10><<<blocks_for(r->npoints, 128, NUM_SMS * 32), 128, 0, s>>>(
            r->t10.p, r->inc.start.p, r->inc.of_node.p, r->npoints, r->place.p);
        FG_CHECK_LAUNCH();
        // The distinct materials (E, nu, alpha) by their bits, numbered in order of first sight.
        std::map<std::array<uint64_t, 5>, uint32_t> seen;
        std::vector<uint32_t> mat(nel);
        std::vector<double> table;
        for (size_t e = 0; e < nel; ++e) {
            double v[5] = {coef[2 * e], coef[2 * e + 1], 0.0, 0.0, 0.0};
            if (expansion)
                for (int k = 0; k < 3; ++k) v[2 + k] = expansion[3 * e + k];
            std::array<uint64_t, 5> key;
            std::memcpy(key.data(), v, sizeof(v));
            auto it = seen.emplace(key, (uint32_t)seen.size());
            if (it.second) table.insert(table.end(), v, v + 5);
            mat[e] = it.first->second;
        }
        r->nmat = (int64_t)seen.size();
        DevBuf<double> dxyz, dtable;
        DevBuf<uint32_t> dpart, dmat;
        dxyz.upload(xyz, 3 * npoints, s);
        dtable.upload(table.data(), table.size(), s);
        dmat.upload(mat.data(), nel, s);
        if (part) dpart.upload(part, nel, s);
        if (singular) {
            r->singular.upload(singular, npoints, s);
            r->has_singular = true;
        }
        r->mats.alloc(r->nmat);
        r->rec.alloc(nel);
        r->u4.alloc(4 * npoints);
        DevBuf<int> bad(1);
        bad.zero(s);
        k_recover_materials<<<blocks_for(r->nmat, 128), 128, 0, s>>>(dtable.p, r->nmat, r->mats.p,
                                                                     bad.p);
        FG_CHECK_LAUNCH();
        k_recover_cells<<<blocks_for(r->nel, 128, NUM_SMS * 32), 128, 0, s>>>(
            dxyz.p, r->t10.p, dmat.p, part ? dpart.p : nullptr, (uint32_t)nparts,
            singular ? r->singular.p : nullptr, r->nel, r->rec.p, bad.p);
        FG_CHECK_LAUNCH();
        int b = fetch(bad.p, s);
        if (b == 2)
            throw Failure(FEMGPU_ERR_MATERIAL,
                          "the Poisson ratios give no stable material (for an isotropic material, "
                          "nu must be between -1 and 0.5)");
        if (b == 3) throw Failure(FEMGPU_ERR_INVALID, "a cell names a part past the last");
        r->peak.alloc(3 * nparts);
        r->dpeaks.alloc(nparts);
        r->xyz = std::move(dxyz);
        FG_CUDA(cudaStreamSynchronize(s));
        *out = r.release();
    });
}

int femgpu_recovery_new_hex(size_t npoints, const double* xyz, size_t nel, const uint32_t* hexes,
                            const double* coef, const double* expansion, const uint32_t* part,
                            size_t nparts, const uint8_t* singular, femgpu_recovery** out) {
    return recovery_guarded([&] {
        need(out != nullptr, "out is null");
        need(npoints > 0 && nel > 0, "an empty mesh");
        need(xyz && hexes && coef, "a null mesh array");
        need(nparts >= 1, "no part");
        if (nparts > (size_t)MAX_PARTS)
            throw Failure(FEMGPU_ERR_TOO_LARGE, "more than 2048 parts");
        if (npoints >= 0xffffffffull || nel >= 0xffffffffull / 8)
            throw Failure(FEMGPU_ERR_TOO_LARGE, "more points or cells than 32-bit numbers hold");
        for (size_t k = 0; k < 8 * nel; ++k)
            need(hexes[k] < npoints, "a cell names a point past the last");
        auto r = std::make_unique<femgpu_recovery>();
        FG_CUDA(cudaStreamCreateWithFlags(&r->s, cudaStreamNonBlocking));
        FG_CUDA(cudaEventCreate(&r->ev0));
        FG_CUDA(cudaEventCreate(&r->ev1));
        cudaStream_t s = r->s;
        r->hex = true;
        r->npoints = (int64_t)npoints;
        r->nel = (int64_t)nel;
        r->nparts = (int)nparts;
        r->t10.upload(hexes, 8 * nel, s);
        build_incidence(r->t10.p, r->nel, 8, r->npoints, &r->inc, s);
        r->place.alloc(8 * nel);
        k_visit_places<8><<<blocks_for(r->npoints, 128, NUM_SMS * 32), 128, 0, s>>>(
            r->t10.p, r->inc.start.p, r->inc.of_node.p, r->npoints, r->place.p);
        FG_CHECK_LAUNCH();
        // The distinct cells (sides, material, expansion) and their recovery records.
        DevBuf<double> dxyz, dcoef, dexp, keys;
        DevBuf<uint32_t> cls, dpart;
        dxyz.upload(xyz, 3 * npoints, s);
        dcoef.upload(coef, 9 * nel, s);
        if (expansion) dexp.upload(expansion, 3 * nel, s);
        r->nmat = hex_classes(dxyz.p, r->t10.p, dcoef.p, expansion ? dexp.p : nullptr, 15,
                              r->nel, &cls, &keys, s);
        r->hmodes.alloc(HEX_MODES * r->nmat);
        hex_modes(keys.p, r->nmat, r->hmodes.p, s);
        if (part) dpart.upload(part, nel, s);
        if (singular) {
            r->singular.upload(singular, npoints, s);
            r->has_singular = true;
        }
        r->hrec.alloc(nel);
        r->amp.alloc(12 * nel);
        r->u4.alloc(4 * npoints);
        DevBuf<int> bad(1);
        bad.zero(s);
        k_recover_hex_cells<<<blocks_for(r->nel, 128, NUM_SMS * 32), 128, 0, s>>>(
            r->t10.p, cls.p, part ? dpart.p : nullptr, (uint32_t)nparts,
            singular ? r->singular.p : nullptr, r->nel, r->hrec.p, bad.p);
        FG_CHECK_LAUNCH();
        if (fetch(bad.p, s) == 3) throw Failure(FEMGPU_ERR_INVALID, "a cell names a part past the last");
        r->peak.alloc(3 * nparts);
        r->dpeaks.alloc(nparts);
        FG_CUDA(cudaStreamSynchronize(s));
        *out = r.release();
    });
}

int femgpu_hex_loads(size_t npoints, const double* xyz, size_t nel, const uint32_t* hexes,
                     const double* coef, const double* expansion, const double* accel,
                     const double* dtemp, double* force) {
    return recovery_guarded([&] {
        need(npoints > 0 && nel > 0, "an empty mesh");
        need(xyz && hexes && coef && force, "a null mesh array");
        if (npoints >= 0xffffffffull || nel >= 0xffffffffull / 8)
            throw Failure(FEMGPU_ERR_TOO_LARGE, "more points or cells than 32-bit numbers hold");
        for (size_t k = 0; k < 8 * nel; ++k)
            need(hexes[k] < npoints, "a cell names a point past the last");
        cudaStream_t s = cudaStreamPerThread;
        DevBuf<uint32_t> dh, cls;
        DevBuf<double> dxyz, dcoef, dexp, dacc, dt, keys, modes, df(3 * npoints);
        DevBuf<uint8_t> place;
        Incidence inc;
        dh.upload(hexes, 8 * nel, s);
        dxyz.upload(xyz, 3 * npoints, s);
        dcoef.upload(coef, 9 * nel, s);
        if (expansion) dexp.upload(expansion, 3 * nel, s);
        if (accel) dacc.upload(accel, 3 * nel, s);
        if (dtemp) dt.upload(dtemp, npoints, s);
        build_incidence(dh.p, (int64_t)nel, 8, (int64_t)npoints, &inc, s);
        place.alloc(8 * nel);
        k_visit_places<8><<<blocks_for((int64_t)npoints, 128, NUM_SMS * 32), 128, 0, s>>>(
            dh.p, inc.start.p, inc.of_node.p, (int64_t)npoints, place.p);
        FG_CHECK_LAUNCH();
        const int64_t nclass = hex_classes(dxyz.p, dh.p, dcoef.p, expansion ? dexp.p : nullptr,
                                           15, (int64_t)nel, &cls, &keys, s);
        modes.alloc(HEX_MODES * nclass);
        hex_modes(keys.p, nclass, modes.p, s);
        k_hex_loads<<<blocks_for((int64_t)npoints, 128, NUM_SMS * 32), 128, 0, s>>>(
            dh.p, cls.p, modes.p, inc.start.p, inc.of_node.p, place.p,
            accel ? dacc.p : nullptr, dtemp ? dt.p : nullptr, (int64_t)npoints, df.p);
        FG_CHECK_LAUNCH();
        df.download(force, 3 * npoints, s);
        FG_CUDA(cudaStreamSynchronize(s));
    });
}

int femgpu_recovery_run(femgpu_recovery* r, const double* u, const double* dtemp, double* stress,
                        double* strain, double* mises, double* principal, femgpu_peak* peaks) {
    return recovery_guarded([&] {
        need(r && u, "a null argument");
        cudaStream_t s = r->s;
        const size_t n = (size_t)r->npoints;
        r->du.upload(u, 3 * n, s);
        if (dtemp) r->ddt.upload(dtemp, n, s);
        if (r->dstress.count < 6 * n) r->dstress.alloc(6 * n);
        if (r->dstrain.count < 6 * n) r->dstrain.alloc(6 * n);
        if (mises && r->dmises.count < n) r->dmises.alloc(n);
        if (principal && r->dprincipal.count < 3 * n) r->dprincipal.alloc(3 * n);
        r->run(r->du.p, dtemp ? r->ddt.p : nullptr, r->dstress.p, r->dstrain.p,
               mises ? r->dmises.p : nullptr, principal ? r->dprincipal.p : nullptr, peaks);
        if (stress) r->dstress.download(stress, 6 * n, s);
        if (strain) r->dstrain.download(strain, 6 * n, s);
        if (mises) r->dmises.download(mises, n, s);
        if (principal) r->dprincipal.download(principal, 3 * n, s);
        FG_CUDA(cudaStreamSynchronize(s));
    });
}

int femgpu_recovery_run_device(femgpu_recovery* r, const double* u, const double* dtemp,
                               double* stress, double* strain, double* mises, double* principal,
                               femgpu_peak* peaks) {
    return recovery_guarded([&] {
        need(r && u && stress && strain, "a null argument");
        r->run(u, dtemp, stress, strain, mises, principal, peaks);
    });
}

int femgpu_recovery_probes(femgpu_recovery* r, const double* u, const double* dtemp,
                           const double* temperature, size_t nprobes, const double* points,
                           const char* const* names, double* displacement, double* stress,
                           double* mises, double* temp, int64_t* hits) {
    return recovery_guarded([&] {
        need(r && u && points && displacement && stress && mises && temp, "a null argument");
        need(!r->hex, "the probes take the cells of a P2 model");
        if (nprobes == 0) return;
        if (nprobes > (1u << 20)) throw Failure(FEMGPU_ERR_TOO_LARGE, "more than 2^20 probes");
        cudaStream_t s = r->s;
        const int64_t n = r->npoints, np = (int64_t)nprobes;
        r->du.upload(u, 3 * n, s);
        DevBuf<double> ddt, dtemp_abs, dpts(3 * np), ddisp(3 * np), dstress(6 * np),
            dmises(np), dtv(np);
        if (dtemp) ddt.upload(dtemp, n, s);
        if (temperature) dtemp_abs.upload(temperature, n, s);
        dpts.upload(points, 3 * np, s);
        DevBuf<int> count(np);
        DevBuf<int64_t> dhits(np * MAX_PROBE_HITS);
        count.zero(s);
        k_pad_u<<<blocks_for(n, 256), 256, 0, s>>>(r->du.p, n, r->u4.p);
        k_probe_hits<<<blocks_for(r->nel * np, 256, NUM_SMS * 64), 256, 0, s>>>(
            r->rec.p, r->xyz.p, r->t10.p, r->nel, dpts.p, np, count.p, dhits.p);
        k_probe_values<<<blocks_for(np, 64), 64, 0, s>>>(
            r->rec.p, r->mats.p, r->xyz.p, r->t10.p, r->u4.p, dtemp ? ddt.p : nullptr,
            temperature ? dtemp_abs.p : nullptr, dpts.p, np, count.p, dhits.p, ddisp.p,
            dstress.p, dmises.p, dtv.p);
        FG_CHECK_LAUNCH();
        std::vector<int> c(np);
        count.download(c.data(), np, s);
        ddisp.download(displacement, 3 * np, s);
        dstress.download(stress, 6 * np, s);
        dmises.download(mises, np, s);
        dtv.download(temp, np, s);
        FG_CUDA(cudaStreamSynchronize(s));
        for (int64_t q = 0; q < np; ++q) {
            if (hits) hits[q] = c[q];
            if (c[q] == 0) {
                // elastic_tet.rs:433-438
                const double* x = points + 3 * q;
                std::string name = names && names[q] ? names[q] : std::to_string(q);
                throw Failure(FEMGPU_ERR_INVALID, "probe " + name + " at (" + rust_display(x[0]) +
                                                      ", " + rust_display(x[1]) + ", " +
                                                      rust_display(x[2]) + ") is in no part");
            }
            if (c[q] > MAX_PROBE_HITS)
                throw Failure(FEMGPU_ERR_TOO_LARGE, "a probe point is in more than 512 cells");
        }
    });
}

int femgpu_recovery_last_time(const femgpu_recovery* r, double* ms, double* bytes) {
    return recovery_guarded([&] {
        need(r != nullptr, "a null handle");
        if (ms) *ms = r->last_ms;
        if (bytes) *bytes = r->last_bytes;
    });
}

size_t femgpu_recovery_bytes(const femgpu_recovery* r) {
    if (!r) return 0;
    return r->t10.bytes() + r->rec.bytes() + r->mats.bytes() + r->singular.bytes() +
           r->hrec.bytes() + r->hmodes.bytes() + r->amp.bytes() +
           r->place.bytes() + r->u4.bytes() + r->peak.bytes() + r->dpeaks.bytes() +
           r->xyz.bytes() +
           r->inc.start.bytes() +
           r->inc.of_node.bytes() + r->du.bytes() + r->ddt.bytes() + r->dstress.bytes() +
           r->dstrain.bytes() + r->dmises.bytes() + r->dprincipal.bytes();
}

void* femgpu_recovery_stream(const femgpu_recovery* r) { return r ? (void*)r->s : nullptr; }

void femgpu_recovery_free(femgpu_recovery* r) { delete r; }

}  // extern "C"
