// The box cell of the grid with 9 incompatible modes (crates/fem/src/hex.rs:146-309) on the
// device: 1 block per distinct cell (a class: its sides and material). Included by the assembly
// and the recovery units, both compiled with -fmad=false: every sum and solve runs in the
// reference's order with separate roundings, so the results equal the reference's bit for bit.
#pragma once
#include "common.cuh"
#include "elements.cuh"

namespace femgpu {

// The local bits of corner n in VTK order (hex.rs:34-43): 000 100 110 010 001 101 111 011. The
// Gauss points of the 2 x 2 x 2 rule take the same order (hex.rs:212-216).
__device__ __forceinline__ int hex_bit(int n, int d) {
    return d == 0 ? ((n + 1) >> 1) & 1 : (d == 1 ? (n >> 1) & 1 : n >> 2);
}

// hex.rs:146-160: the gradients of the 8 corner functions and the 3 mode functions (1 - xi^2
// along each axis) at the local point xi of a box with the sides `size`.
__device__ __forceinline__ void hex_gradients(const double* size, const double* xi,
                                              double g[11][3]) {
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        double s[3], f[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            s[d] = hex_bit(n, d) == 1 ? 1.0 : -1.0;
            f[d] = 0.5 * (1.0 + s[d] * xi[d]);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) g[n][d] = s[d] / size[d] * f[(d + 1) % 3] * f[(d + 2) % 3];
    }
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[8 + m][d] = m == d ? -4.0 * xi[d] / size[d] : 0.0;
}

// hex.rs:164-178: the 8 corner functions at xi, each a product from 1.0.
__device__ __forceinline__ void hex_shape(const double* xi, double n[8]) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        double v = 1.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) v *= hex_bit(c, d) == 1 ? 0.5 * (1.0 + xi[d]) : 0.5 * (1.0 - xi[d]);
        n[c] = v;
    }
}

constexpr int HEX_THREADS = 128;

// The recovery record of a class (HEX_MODES doubles, 32-byte aligned): mode_u (9 x 24), mode_t
// (9 x 8), D (normal 3 x 3, then G_yz, G_xz, G_xy), D alpha, the sides, the gradients of the 11
// functions at each of the 8 corners (hex.rs:146-160 at xi = -1 or 1: 33 per corner), and the
// condensed load of a unit temperature change at each corner (hex.rs:283-289, 24 x 8).
constexpr int HEX_MODE_U = 0, HEX_MODE_T = 216, HEX_NORMAL = 288, HEX_SHEAR = 297,
              HEX_THERMAL = 300, HEX_SIZE = 303, HEX_GRAD = 320, HEX_LOAD = 584,
              HEX_MODES = 776;

// One block per class of `key` (`width` words each: 3 sides, 9 orthotropic constants, with
// MODES 3 expansion coefficients). hex.rs:218-297: the 33 x 33 stiffness of the 11 functions x 3
// components summed over the Gauss points in their order (jac = the volume / 8), the Cholesky
// factor of the 9 x 9 block of the modes (hex.rs:355-372) and its solves (hex.rs:374-389).
// !MODES: out gets the condensed 24 x 24 stiffness (576 per class). MODES: also the 33 x 8
// thermal load, and out gets the recovery record (mode_u, mode_t of hex.rs:262-273 and D, D
// alpha, the sides). Flags: 2 no stable material, 3 a modulus not above 0, 4 a side not above 0,
// 5 the modes' block not positive.
template <bool MODES>
__global__ void __launch_bounds__(HEX_THREADS)
    k_hex_element(const double* __restrict__ key, int width, int64_t nclass,
                  double* __restrict__ out_all, int* __restrict__ bad) {
    __shared__ double g[8][11][3];
    __shared__ double nsh[8][8];
    __shared__ double k[33][33];
    __shared__ double lt[MODES ? 33 : 1][8];
    __shared__ double l[9][9];
    __shared__ double x[9][32];
    __shared__ double thermal[3];
    __shared__ int ok;
    const int t = threadIdx.x;
    for (int64_t cl = blockIdx.x; cl < nclass; cl += gridDim.x) {
        const double* size = key + width * cl;
        Stiffness D;
        const int st = orthotropic_stiffness(size + 3, &D);
        bool sides = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) sides = sides && isfinite(size[d]) && size[d] > 0.0;
        if (t == 0) {
            ok = st == 0 && sides;
            if (st) atomicExch(bad, st == 1 ? 3 : 2);
            else if (!sides) atomicExch(bad, 4);
        }
        if (MODES && t < 3) {  // D alpha, the Rust float sum from -0.0
            double s = -0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) s += D.normal[t][j] * size[12 + j];
            thermal[t] = s;
        }
        if (t < 8) {
            const double p = 1.0 / sqrt(3.0);
            double xi[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) xi[d] = hex_bit(t, d) == 1 ? p : -p;
            double gt[11][3], nt[8];
            hex_gradients(size, xi, gt);
            hex_shape(xi, nt);
            for (int i = 0; i < 11; ++i)
#pragma unroll
                for (int d = 0; d < 3; ++d) g[t][i][d] = gt[i][d];
#pragma unroll
            for (int c = 0; c < 8; ++c) nsh[t][c] = nt[c];
        }
        __syncthreads();
        if (ok) {
            const double jac = size[0] * size[1] * size[2] / 8.0;
            for (int o = t; o < 33 * 33; o += HEX_THREADS) {
                const int r = o / 33, c = o % 33;
                const int i = r / 3, a = r % 3, j = c / 3, b = c % 3;
                double v = 0.0;
#pragma unroll
                for (int q = 0; q < 8; ++q) v += jac * elastic_term(g[q][i], g[q][j], a, b, D);
                k[r][c] = v;
            }
            if (MODES)  // hex.rs:256-260: l[3 i + a][c] += jac g_i[a] thermal[a] N_c
                for (int o = t; o < 33 * 8; o += HEX_THREADS) {
                    const int r = o / 8, c = o % 8, i = r / 3, a = r % 3;
                    double v = 0.0;
#pragma unroll
                    for (int q = 0; q < 8; ++q) v += jac * g[q][i][a] * thermal[a] * nsh[q][c];
                    lt[r][c] = v;
                }
        }
        __syncthreads();
        if (ok && t == 0) {  // cholesky9
            for (int j = 0; j < 9; ++j) {
                double d = k[24 + j][24 + j];
                for (int c = 0; c < j; ++c) d -= l[j][c] * l[j][c];
                if (!(d > 0.0)) {
                    ok = 0;
                    atomicExch(bad, 5);
                    break;
                }
                d = sqrt(d);
                l[j][j] = d;
                for (int i = j + 1; i < 9; ++i) {
                    double v = k[24 + i][24 + j];
                    for (int c = 0; c < j; ++c) v -= l[i][c] * l[j][c];
                    l[i][j] = v / d;
                }
            }
        }
        __syncthreads();
        // solve9 on column t of K_mu (t < 24) or of the modes' thermal load (24 <= t < 32).
        if (ok && (t < 24 || (MODES && t < 32))) {
            double b[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) b[i] = t < 24 ? k[24 + i][t] : lt[MODES ? 24 + i : 0][t - 24];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
#pragma unroll
                for (int q = 0; q < i; ++q) b[i] -= l[i][q] * b[q];
                b[i] /= l[i][i];
            }
#pragma unroll
            for (int i = 8; i >= 0; --i) {
#pragma unroll
                for (int q = i + 1; q < 9; ++q) b[i] -= l[q][i] * b[q];
                b[i] /= l[i][i];
            }
#pragma unroll
            for (int i = 0; i < 9; ++i) x[i][t] = b[i];
        }
        __syncthreads();
        if (!MODES) {
            double* out = out_all + 576 * cl;
            for (int o = t; o < 576; o += HEX_THREADS) {
                const int r = o / 24, c = o % 24;
                double v = 0.0;
                if (ok) {
                    v = k[r][c];
#pragma unroll
                    for (int i = 0; i < 9; ++i) v -= k[r][24 + i] * x[i][c];
                }
                out[o] = v;
            }
        } else {
            double* out = out_all + HEX_MODES * cl;
            for (int o = t; o < 192; o += HEX_THREADS) {  // lc = l - K_um mode_t
                const int r = o / 8, c = o % 8;
                double v = 0.0;
                if (ok) {
                    v = lt[MODES ? r : 0][c];
#pragma unroll
                    for (int i = 0; i < 9; ++i) v -= k[r][24 + i] * x[i][24 + c];
                }
                out[HEX_LOAD + o] = v;
            }
            if (t < 8) {  // the gradients at corner t
                double xi[3], gc[11][3];
#pragma unroll
                for (int d = 0; d < 3; ++d) xi[d] = hex_bit(t, d) == 1 ? 1.0 : -1.0;
                hex_gradients(size, xi, gc);
                for (int i = 0; i < 11; ++i)
#pragma unroll
                    for (int d = 0; d < 3; ++d) out[HEX_GRAD + 33 * t + 3 * i + d] = gc[i][d];
            }
            for (int o = t; o < HEX_GRAD; o += HEX_THREADS) {
                double v = 0.0;
                if (o < HEX_MODE_T)
                    v = ok ? x[o / 24][o % 24] : 0.0;
                else if (o < HEX_NORMAL)
                    v = ok ? x[(o - HEX_MODE_T) / 8][24 + (o - HEX_MODE_T) % 8] : 0.0;
                else if (o < HEX_SHEAR)
                    v = D.normal[(o - HEX_NORMAL) / 3][(o - HEX_NORMAL) % 3];
                else if (o < HEX_THERMAL)
                    v = D.shear[o - HEX_SHEAR];
                else if (o < HEX_SIZE)
                    v = thermal[o - HEX_THERMAL];
                else if (o < HEX_SIZE + 3)
                    v = size[o - HEX_SIZE];
                out[o] = v;
            }
        }
        __syncthreads();
    }
}

}  // namespace femgpu
