// Element kernels of the path as device functions. Each follows the reference's expression
// order, and the files that include this one are compiled with -fmad=false, so every value is
// bit-identical with the Rust code (which never fuses a multiply and an add).
#pragma once
#include <cstdint>

namespace femgpu {

// tet10.rs:38: the 2 corners of each edge point, and tet10.rs:41: the axes of each shear.
__device__ __constant__ const int kEdges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
__device__ __constant__ const int kShear[3][2] = {{1, 2}, {0, 2}, {0, 1}};

// heat.rs:983-1002: the gradients of the 4 barycentric functions and the volume det / 6.
__device__ __forceinline__ void tet_gradients(const double p[4][3], double g[4][3],
                                              double* volume) {
    double e[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int d = 0; d < 3; ++d) e[k][d] = p[k + 1][d] - p[0][d];
    double det = e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1]) -
                 e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0]) +
                 e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0]);
    double r[3][3];
    // rows = [e1 x e2, e2 x e0, e0 x e1]
    const int A[3] = {1, 2, 0}, B[3] = {2, 0, 1};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double* a = e[A[k]];
        const double* b = e[B[k]];
        r[k][0] = a[1] * b[2] - a[2] * b[1];
        r[k][1] = a[2] * b[0] - a[0] * b[2];
        r[k][2] = a[0] * b[1] - a[1] * b[0];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[k + 1][d] = r[k][d] / det;
#pragma unroll
    for (int d = 0; d < 3; ++d) g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
    *volume = det / 6.0;
}

// heat.rs:972-981: entry (i, j) of V G^T K G; the Rust float sum equals ((t0 + t1) + t2).
__device__ __forceinline__ double conduction_entry(const double g[4][3], double v,
                                                   const double k[3], int i, int j) {
    double s = k[0] * g[i][0] * g[j][0];
    s = s + k[1] * g[i][1] * g[j][1];
    s = s + k[2] * g[i][2] * g[j][2];
    return v * s;
}

// hex.rs:120-124
struct Stiffness {
    double normal[3][3];
    double shear[3];
};

// hex.rs:58-64 and 69-114 for an isotropic material. Returns false when the constants give no
// stable material (hex.rs:72-98).
__device__ __forceinline__ bool isotropic_stiffness(double e, double nu, Stiffness* d) {
    double g = e / (2.0 * (1.0 + nu));
    if (!(isfinite(e) && e > 0.0 && isfinite(g) && g > 0.0) || !isfinite(nu)) return false;
    double s[3][3] = {{1.0 / e, -nu / e, -nu / e}, {-nu / e, 1.0 / e, -nu / e},
                      {-nu / e, -nu / e, 1.0 / e}};
    double det = s[0][0] * (s[1][1] * s[2][2] - s[1][2] * s[2][1]) -
                 s[0][1] * (s[1][0] * s[2][2] - s[1][2] * s[2][0]) +
                 s[0][2] * (s[1][0] * s[2][1] - s[1][1] * s[2][0]);
    double minor = s[0][0] * s[1][1] - s[0][1] * s[1][0];
    if (!(minor > 0.0 && det > 1e-12 * s[0][0] * s[1][1] * s[2][2])) return false;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            d->normal[i][j] = (s[j1][i1] * s[j2][i2] - s[j1][i2] * s[j2][i1]) / det;
        }
    d->shear[0] = g;
    d->shear[1] = g;
    d->shear[2] = g;
    return true;
}

// hex.rs:69-114 for an orthotropic material, c = E_x, E_y, E_z, nu_xy, nu_xz, nu_yz, G_xy,
// G_xz, G_yz (the fields of Orthotropic, hex.rs:47-55). Returns 0, or 1 when a modulus is not
// above 0 or a ratio not finite (hex.rs:72-79), 2 when the constants give no stable material
// (hex.rs:88-98).
__device__ __forceinline__ int orthotropic_stiffness(const double* c, Stiffness* d) {
    const double ex = c[0], ey = c[1], ez = c[2];
    const double nxy = c[3], nxz = c[4], nyz = c[5];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        ok = ok && isfinite(c[k]) && c[k] > 0.0 && isfinite(c[6 + k]) && c[6 + k] > 0.0 &&
             isfinite(c[3 + k]);
    if (!ok) return 1;
    double s[3][3] = {{1.0 / ex, -nxy / ex, -nxz / ex},
                      {-nxy / ex, 1.0 / ey, -nyz / ey},
                      {-nxz / ex, -nyz / ey, 1.0 / ez}};
    double det = s[0][0] * (s[1][1] * s[2][2] - s[1][2] * s[2][1]) -
                 s[0][1] * (s[1][0] * s[2][2] - s[1][2] * s[2][0]) +
                 s[0][2] * (s[1][0] * s[2][1] - s[1][1] * s[2][0]);
    double minor = s[0][0] * s[1][1] - s[0][1] * s[1][0];
    if (!(minor > 0.0 && det > 1e-12 * s[0][0] * s[1][1] * s[2][2])) return 2;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            d->normal[i][j] = (s[j1][i1] * s[j2][i2] - s[j1][i2] * s[j2][i1]) / det;
        }
    d->shear[0] = c[8];  // G_yz
    d->shear[1] = c[7];  // G_xz
    d->shear[2] = c[6];  // G_xy
    return 0;
}

// tet10.rs:101-112: the (a, b) term of B^T D B between 2 function gradients.
__device__ __forceinline__ double elastic_term(const double* gi, const double* gj, int a, int b,
                                               const Stiffness& d) {
    double v = gi[a] * gj[b] * d.normal[a][b];
    if (a == b) {
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            int p = kShear[s][0], q = kShear[s][1];
            if (p == a)
                v += gi[q] * gj[q] * d.shear[s];
            else if (q == a)
                v += gi[p] * gj[p] * d.shear[s];
        }
    } else {
        v += gi[b] * gj[a] * d.shear[3 - a - b];
    }
    return v;
}

// tet10.rs:44-48 and 77-87: the gradients of the 10 functions at quadrature point q.
__device__ __forceinline__ void tet10_gradients(const double g[4][3], int q, double out[10][3]) {
    const double A = 0.5854101966249685, B = 0.1381966011250105;
    double l[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) l[c] = (c == q) ? A : B;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) out[i][d] = (4.0 * l[i] - 1.0) * g[i][d];
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        int i = kEdges[e][0], j = kEdges[e][1];
#pragma unroll
        for (int d = 0; d < 3; ++d) out[4 + e][d] = 4.0 * (l[i] * g[j][d] + l[j] * g[i][d]);
    }
}

}  // namespace femgpu
