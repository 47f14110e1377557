// The dense generalized eigenproblem of the modes' Rayleigh-Ritz step on the device: K q =
// lambda M q for the p x p projections of the subspace iteration (p = max(2 q, q + 8) <= 128 for
// q <= 64 modes), the step the reference takes with eigen.rs:183-331.
//
// Method (1 block of 1024 threads; the matrices in a global scratch that stays in L2):
//   1. D = diag(M)^-1/2 and the Cholesky factor L of D M D (a unit diagonal keeps the factor
//      accurate when the subspace vectors differ in scale, as in the reference); a pivot at or
//      below 1e-14 means dependent vectors, the reference's test and text;
//   2. C = L^-1 (D K D) L^-T by triangular solves, 1 thread per column, then symmetrized;
//   3. the eigenpairs of C by the parallel Jacobi method: each round rotates n / 2 disjoint
//      pairs at once (the round-robin order of Brent and Luk, SIAM J. Sci. Stat. Comput. 6 (1985)
//      69-84: element 0 fixed, the others shifted by 1 each round), the columns then the rows,
//      n - 1 rounds a sweep, until the off-diagonal norm is at most 1e-15 of the norm or 100
//      sweeps (the reference's test, its sequential cyclic order replaced by the parallel one);
//   4. the eigenvalues ascending (a stable rank: equal values keep their order) and Q = D L^-T V,
//      so that Q^T M Q = I.
// The results equal the reference's to rounding; an eigenvector of a repeated eigenvalue may be
// any orthonormal basis of its space, as with any method.
#include <cmath>

#include "common.cuh"

namespace femgpu {
namespace {

constexpr int EIG_TH = 1024;
constexpr int EIG_MAX = 1024;  // the largest n (1 thread per column)

__device__ double block_sum(double v, double* red) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) red[32] = t;
    }
    __syncthreads();
    return red[32];
}

// work: L, C, V (n x n each, row-major), d (n). status: 1 M not positive definite, 2 dependent
// vectors.
__global__ void __launch_bounds__(EIG_TH)
    k_dense_generalized(int n, const double* __restrict__ K, const double* __restrict__ M,
                        double* __restrict__ work, double* __restrict__ values,
                        double* __restrict__ Q, int* __restrict__ status) {
    __shared__ double red[33];
    __shared__ int stop;
    __shared__ double cs[EIG_MAX / 2], sn[EIG_MAX / 2];
    __shared__ int pp[EIG_MAX / 2], pq[EIG_MAX / 2], pos[EIG_MAX];
    const int tid = threadIdx.x;
    const size_t nn = (size_t)n * n;
    double* L = work;
    double* C = work + nn;
    double* V = work + 2 * nn;
    double* d = work + 3 * nn;
    if (tid == 0) stop = 0;
    __syncthreads();
    // 1. The scale and the factor of D M D.
    for (int i = tid; i < n; i += blockDim.x) {
        const double mi = M[(size_t)i * n + i];
        if (!(mi > 0.0)) atomicExch(&stop, 1);
        d[i] = 1.0 / sqrt(mi);
    }
    __syncthreads();
    if (stop) {
        if (tid == 0) *status = 1;
        return;
    }
    for (size_t t = tid; t < nn; t += blockDim.x) {
        const int i = (int)(t / n), j = (int)(t % n);
        L[t] = j <= i ? M[t] * d[i] * d[j] : 0.0;
    }
    __syncthreads();
    for (int j = 0; j < n; ++j) {
        if (tid == 0) {
            const double s = L[(size_t)j * n + j];
            if (!(s > 1e-14))
                stop = 2;
            else
                L[(size_t)j * n + j] = sqrt(s);
        }
        __syncthreads();
        if (stop) {
            if (tid == 0) *status = 2;
            return;
        }
        const double ljj = L[(size_t)j * n + j];
        for (int i = j + 1 + tid; i < n; i += blockDim.x) L[(size_t)i * n + j] /= ljj;
        __syncthreads();
        const int w = n - j - 1;
        for (int t = tid; t < w * w; t += blockDim.x) {
            const int i = j + 1 + t / w, c = j + 1 + t % w;
            if (c <= i) L[(size_t)i * n + c] -= L[(size_t)i * n + j] * L[(size_t)c * n + j];
        }
        __syncthreads();
    }
    // 2. W = L^-1 (D K D) into V, then C = L^-1 W^T; column j by thread j.
    for (int j = tid; j < n; j += blockDim.x)
        for (int i = 0; i < n; ++i) {
            double v = K[(size_t)i * n + j] * d[i] * d[j];
            for (int c = 0; c < i; ++c) v -= L[(size_t)i * n + c] * V[(size_t)c * n + j];
            V[(size_t)i * n + j] = v / L[(size_t)i * n + i];
        }
    __syncthreads();
    for (int j = tid; j < n; j += blockDim.x)
        for (int i = 0; i < n; ++i) {
            double v = V[(size_t)j * n + i];
            for (int c = 0; c < i; ++c) v -= L[(size_t)i * n + c] * C[(size_t)c * n + j];
            C[(size_t)i * n + j] = v / L[(size_t)i * n + i];
        }
    __syncthreads();
    for (size_t t = tid; t < nn; t += blockDim.x) {
        const int i = (int)(t / n), j = (int)(t % n);
        if (j < i) {
            const double v = 0.5 * (C[t] + C[(size_t)j * n + i]);
            C[t] = v;
            C[(size_t)j * n + i] = v;
        }
    }
    for (size_t t = tid; t < nn; t += blockDim.x) V[t] = (t / n == t % n) ? 1.0 : 0.0;
    __syncthreads();
    // 3. Parallel Jacobi.
    double ss = 0.0;
    for (size_t t = tid; t < nn; t += blockDim.x) ss += C[t] * C[t];
    const double norm = sqrt(block_sum(ss, red));
    const int N = n + (n & 1);  // an odd n gets a dummy index n, never rotated
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (size_t t = tid; t < nn; t += blockDim.x)
            if (t / n != t % n) off += C[t] * C[t];
        off = block_sum(off, red);
        if (!(sqrt(off) > 1e-15 * norm)) break;
        for (int k = tid; k < N; k += blockDim.x) pos[k] = k;
        __syncthreads();
        for (int round = 0; round < N - 1; ++round) {
            for (int k = tid; k < N / 2; k += blockDim.x) {
                int p = pos[k], q = pos[N - 1 - k];
                if (p > q) {
                    const int t = p;
                    p = q;
                    q = t;
                }
                double c = 1.0, s = 0.0;
                if (q < n) {
                    const double apq = C[(size_t)p * n + q];
                    if (apq != 0.0) {
                        const double tau = (C[(size_t)q * n + q] - C[(size_t)p * n + p]) / (2.0 * apq);
                        const double t = tau >= 0.0 ? 1.0 / (tau + hypot(tau, 1.0))
                                                    : -1.0 / (-tau + hypot(tau, 1.0));
                        c = 1.0 / hypot(t, 1.0);
                        s = t * c;
                    }
                }
                pp[k] = p;
                pq[k] = q;
                cs[k] = c;
                sn[k] = s;
            }
            __syncthreads();
            // The columns p, q of C and of V.
            for (int t = tid; t < (N / 2) * n; t += blockDim.x) {
                const int k = t / n, r = t % n;
                const int p = pp[k], q = pq[k];
                if (q >= n || sn[k] == 0.0) continue;
                const double c = cs[k], s = sn[k];
                double x = C[(size_t)r * n + p], y = C[(size_t)r * n + q];
                C[(size_t)r * n + p] = c * x - s * y;
                C[(size_t)r * n + q] = s * x + c * y;
                x = V[(size_t)r * n + p];
                y = V[(size_t)r * n + q];
                V[(size_t)r * n + p] = c * x - s * y;
                V[(size_t)r * n + q] = s * x + c * y;
            }
            __syncthreads();
            // The rows p, q of C.
            for (int t = tid; t < (N / 2) * n; t += blockDim.x) {
                const int k = t / n, r = t % n;
                const int p = pp[k], q = pq[k];
                if (q >= n || sn[k] == 0.0) continue;
                const double c = cs[k], s = sn[k];
                const double x = C[(size_t)p * n + r], y = C[(size_t)q * n + r];
                C[(size_t)p * n + r] = c * x - s * y;
                C[(size_t)q * n + r] = s * x + c * y;
            }
            __syncthreads();
            // The next round's pairs: element 0 fixed, the others shifted by 1.
            int moved = 0;
            if (tid < N) moved = tid == 0 ? pos[0] : (tid == 1 ? pos[N - 1] : pos[tid - 1]);
            __syncthreads();
            if (tid < N) pos[tid] = moved;
            __syncthreads();
        }
    }
    // 4. Ascending (stable) and Q = D L^-T V, column by column.
    for (int i = tid; i < n; i += blockDim.x) {
        const double a = C[(size_t)i * n + i];
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const double b = C[(size_t)j * n + j];
            rank += (b < a) || (b == a && j < i);
        }
        values[rank] = a;
        pos[i] = rank;
    }
    __syncthreads();
    for (int j = tid; j < n; j += blockDim.x) {
        const int col = pos[j];
        for (int i = n - 1; i >= 0; --i) {
            double v = V[(size_t)i * n + j];
            for (int r = i + 1; r < n; ++r) v -= L[(size_t)r * n + i] * Q[(size_t)r * n + col];
            Q[(size_t)i * n + col] = v / L[(size_t)i * n + i];
        }
    }
    __syncthreads();
    for (size_t t = tid; t < nn; t += blockDim.x) Q[t] *= d[t / n];
}

}  // namespace

// K q = lambda M q for symmetric row-major n x n device matrices (n <= 1024): values (n) and Q
// (n x n, the vectors as columns) on the device, on `s`. Throws the reference's texts.
void dense_generalized_device(const double* k, const double* m, int n, double* values,
                              double* q, cudaStream_t s) {
    if (n < 1 || n > EIG_MAX)
        throw Failure(FEMGPU_ERR_TOO_LARGE, "the dense eigenproblem takes 1 to 1024 unknowns");
    DevBuf<double> work(3 * (size_t)n * n + n);
    DevBuf<int> status(1);
    status.zero(s);
    k_dense_generalized<<<1, EIG_TH, 0, s>>>(n, k, m, work.p, values, q, status.p);
    FG_CHECK_LAUNCH();
    const int st = fetch(status.p, s);
    if (st == 1) throw Failure(FEMGPU_ERR_NOT_SPD, "the projected mass matrix is not positive definite");
    if (st == 2)
        throw Failure(FEMGPU_ERR_NOT_SPD,
                      "the projected mass matrix is singular: the subspace vectors are dependent");
}

}  // namespace femgpu
