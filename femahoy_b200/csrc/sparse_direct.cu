// The multifrontal sparse Cholesky factor on the device (sparse_direct.cuh).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>

#include "rust_format.hpp"
#include "dense_factor.cuh"
#include "sparse_direct.cuh"

namespace femgpu {
namespace {

constexpr double PIVOT = 1e-10;     // cholesky.rs:22
constexpr int SMALL_ROWS = 128;     // fronts factored in shared memory by 1 block
constexpr int CHUNK = 4096;         // entries of an update matrix per extend-add block
constexpr int TH = 256;

// The front of supernode s: m x m, column-major.
struct Fronts {
    const int64_t* first;
    const int64_t* rows_ptr;
    const uint32_t* rows;
    const int64_t* foff;
    double* f;
};

__device__ __forceinline__ int64_t lower_bound(const uint32_t* r, int64_t m, uint32_t v) {
    int64_t lo = 0, hi = m;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (r[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// The entries of A in the lower part of each front (cholesky.rs:60-72), 1 thread per column,
// and each column's diagonal of A.
__global__ void k_assemble_fronts(int64_t n, const int64_t* __restrict__ perm,
                                  const int64_t* __restrict__ iperm,
                                  const int64_t* __restrict__ aptr,
                                  const uint32_t* __restrict__ aidx,
                                  const double* __restrict__ aval,
                                  const int32_t* __restrict__ col2sn, Fronts fr,
                                  double* __restrict__ diag0) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int s = col2sn[j];
        const int64_t r0 = fr.rows_ptr[s], m = fr.rows_ptr[s + 1] - r0;
        const uint32_t* R = fr.rows + r0;
        double* F = fr.f + fr.foff[s] + (j - fr.first[s]) * m;
        const int64_t old = perm[j];
        double d = 0.0;
        for (int64_t e = aptr[old]; e < aptr[old + 1]; ++e) {
            const int64_t i = iperm[aidx[e]];
            if (i == j) d = aval[e];
            if (i >= j) F[lower_bound(R, m, (uint32_t)i)] += aval[e];
        }
        diag0[j] = d;
    }
}

// Extend-add (cholesky.rs:74-86): chunk (child c, part q) adds the lower triangle of a part of
// c's update matrix into its parent's front at the parent's rows.
__global__ void k_extend_add(const int2* __restrict__ chunk, Fronts fr,
                             const int64_t* __restrict__ parent,
                             const uint32_t* __restrict__ relind,
                             const int64_t* __restrict__ relind_off) {
    const int c = chunk[blockIdx.x].x;
    const int64_t q = chunk[blockIdx.x].y;
    const int64_t mc = fr.rows_ptr[c + 1] - fr.rows_ptr[c];
    const int64_t kc = fr.first[c + 1] - fr.first[c];
    const int64_t mu = mc - kc;
    const int64_t p = parent[c];
    const int64_t mp = fr.rows_ptr[p + 1] - fr.rows_ptr[p];
    const double* U = fr.f + fr.foff[c] + kc * mc + kc;
    double* F = fr.f + fr.foff[p];
    const uint32_t* rel = relind + relind_off[c];
    const int64_t end = min(mu * mu, (q + 1) * (int64_t)CHUNK);
    for (int64_t t = q * CHUNK + threadIdx.x; t < end; t += blockDim.x) {
        const int64_t col = t / mu, row = t % mu;
        if (row < col) continue;
        F[rel[row] + (int64_t)rel[col] * mp] += U[row + col * mc];
    }
}

// Partial Cholesky of the first k columns of a front in shared memory (cholesky.rs:173-225):
// each pivot checked against PIVOT times its column's diagonal of A, its column scaled, and the
// rest of the lower triangle updated (right-looking); 1 block per front of at most SMALL_ROWS.
__global__ void __launch_bounds__(TH)
    k_front_small(const int64_t* __restrict__ list, Fronts fr,
                  const double* __restrict__ diag0, unsigned long long* __restrict__ status) {
    extern __shared__ double S[];
    __shared__ int stop;
    const int64_t s = list[blockIdx.x];
    const int64_t j0 = fr.first[s];
    const int m = (int)(fr.rows_ptr[s + 1] - fr.rows_ptr[s]);
    const int k = (int)(fr.first[s + 1] - j0);
    double* F = fr.f + fr.foff[s];
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) S[t] = F[t];
    if (threadIdx.x == 0) stop = 0;
    __syncthreads();
    for (int j = 0; j < k; ++j) {
        if (threadIdx.x == 0) {
            const double d = S[j + j * m];
            if (!(d > PIVOT * fabs(diag0[j0 + j]))) {
                atomicMin(status, (unsigned long long)(j0 + j));
                stop = 1;
            } else {
                S[j + j * m] = sqrt(d);
            }
        }
        __syncthreads();
        if (stop) break;
        const double inv = 1.0 / S[j + j * m];
        for (int r = j + 1 + threadIdx.x; r < m; r += blockDim.x) S[r + j * m] *= inv;
        __syncthreads();
        // The lower triangle of the trailing block, column by column.
        const int w = m - j - 1;
        for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
            const int c = j + 1 + t / w, r = j + 1 + t % w;
            if (r >= c) S[r + c * m] -= S[r + j * m] * S[c + j * m];
        }
        __syncthreads();
    }
    __syncthreads();
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) F[t] = S[t];
}

__global__ void k_permute_in(int64_t n, const int64_t* __restrict__ perm,
                             const double* __restrict__ b, double* __restrict__ y) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        y[j] = b[perm[j]];
}

__global__ void k_permute_out(int64_t n, const int64_t* __restrict__ perm,
                              const double* __restrict__ y, double* __restrict__ x) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        x[perm[j]] = y[j];
}

// The product forms of a supernode's triangular solves, when the inverse W = L11^-1 of its
// diagonal block is kept (k x k, column-major): z1 = W z1 and z2 -= L21 z1 in the forward
// direction, x1 = W^T t in the backward one. The vector is staged in shared memory 1024 values
// at a time; tmp is the supernode's own range of a scratch vector (its columns j0 .. j0 + k).
constexpr int ZS = 1024;

__device__ void forward_by_inverse(const double* __restrict__ W, const double* __restrict__ F,
                                   int64_t m, int64_t k, double* __restrict__ z,
                                   double* __restrict__ tmp) {
    __shared__ double zs[ZS];
    for (int64_t i = threadIdx.x; i < k; i += blockDim.x) tmp[i] = 0.0;
    for (int64_t c0 = 0; c0 < k; c0 += ZS) {
        const int cnt = (int)min((int64_t)ZS, k - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) zs[t] = z[c0 + t];
        __syncthreads();
        for (int64_t i = c0 + threadIdx.x; i < k; i += blockDim.x) {
            const int hi = (int)min((int64_t)cnt, i - c0 + 1);  // W lower: j <= i
            double acc = 0.0;
            for (int j = 0; j < hi; ++j) acc += W[i + (c0 + j) * k] * zs[j];
            tmp[i] += acc;
        }
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < k; i += blockDim.x) z[i] = tmp[i];
    // z2 -= L21 z1, z1 staged again.
    for (int64_t c0 = 0; c0 < k; c0 += ZS) {
        const int cnt = (int)min((int64_t)ZS, k - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) zs[t] = z[c0 + t];
        __syncthreads();
        for (int64_t r = k + threadIdx.x; r < m; r += blockDim.x) {
            double acc = 0.0;
            for (int j = 0; j < cnt; ++j) acc += F[r + (c0 + j) * m] * zs[j];
            z[r] -= acc;
        }
    }
    __syncthreads();
}

__device__ void backward_by_inverse(const double* __restrict__ W, int64_t k,
                                    double* __restrict__ z, double* __restrict__ tmp) {
    __shared__ double ts[ZS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int64_t j = threadIdx.x; j < k; j += blockDim.x) tmp[j] = 0.0;
    for (int64_t c0 = 0; c0 < k; c0 += ZS) {
        const int cnt = (int)min((int64_t)ZS, k - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) ts[t] = z[c0 + t];
        __syncthreads();
        // x1[j] += sum over rows i of the chunk with i >= j of W[i][j] t[i] (column j of W is
        // contiguous): a warp per column.
        for (int64_t j = warp; j < k && j < c0 + cnt; j += nw) {
            const int lo = (int)max((int64_t)0, j - c0);
            const double* col = W + c0 + j * k;
            double acc = 0.0;
            for (int t = lo + lane; t < cnt; t += 32) acc += col[t] * ts[t];
            for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) tmp[j] += acc;
        }
    }
    __syncthreads();
    for (int64_t j = threadIdx.x; j < k; j += blockDim.x) z[j] = tmp[j];
    __syncthreads();
}

// Forward solve of supernode s (1 block): z = its part of y and its children's updates (added
// child by child in increasing order), then L11 z1 = z1 and z2 -= L21 z1 by blocks of 32 columns;
// z1 goes to y, z2 is the update for the parent.
__global__ void __launch_bounds__(TH)
    k_forward(const int64_t* __restrict__ list, Fronts fr, const int64_t* __restrict__ zoff,
              const int64_t* __restrict__ child_ptr, const int64_t* __restrict__ child,
              const uint32_t* __restrict__ relind, const int64_t* __restrict__ relind_off,
              double* __restrict__ work, double* __restrict__ y,
              const int64_t* __restrict__ winv_off, const double* __restrict__ winv,
              double* __restrict__ tmp) {
    const int64_t s = list[blockIdx.x];
    const int64_t j0 = fr.first[s];
    const int64_t m = fr.rows_ptr[s + 1] - fr.rows_ptr[s], k = fr.first[s + 1] - j0;
    const double* F = fr.f + fr.foff[s];
    double* z = work + zoff[s];
    for (int64_t t = threadIdx.x; t < m; t += blockDim.x) z[t] = t < k ? y[j0 + t] : 0.0;
    __syncthreads();
    for (int64_t ci = child_ptr[s]; ci < child_ptr[s + 1]; ++ci) {
        const int64_t c = child[ci];
        const int64_t kc = fr.first[c + 1] - fr.first[c];
        const int64_t mu = fr.rows_ptr[c + 1] - fr.rows_ptr[c] - kc;
        const double* zc = work + zoff[c] + kc;
        const uint32_t* rel = relind + relind_off[c];
        for (int64_t t = threadIdx.x; t < mu; t += blockDim.x) z[rel[t]] += zc[t];
        __syncthreads();
    }
    if (winv_off && winv_off[s] >= 0) {
        forward_by_inverse(winv + winv_off[s], F, m, k, z, tmp + j0);
        for (int64_t t = threadIdx.x; t < k; t += blockDim.x) y[j0 + t] = z[t];
        return;
    }
    // The columns in blocks of 32: warp 0 solves the block's triangle with shuffles (lane i
    // holds row jb + i), then every thread takes rows below the block and subtracts the block's
    // 32 columns times the solved values: 2 barriers per 32 columns instead of 2 per column.
    __shared__ double zb[32];
    for (int64_t jb = 0; jb < k; jb += 32) {
        const int kb = (int)min((int64_t)32, k - jb);
        if (threadIdx.x < 32) {
            // Lane l holds row jb + l of the block's triangle in registers (all loads issued
            // before the serial steps, which then only shuffle).
            const int l = threadIdx.x;
            double row[32];
#pragma unroll
            for (int j = 0; j < 32; ++j)
                row[j] = (j < kb && l < kb && j <= l) ? F[(jb + l) + (jb + j) * m] : 0.0;
            double x = l < kb ? z[jb + l] : 0.0;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                if (j < kb) {
                    if (l == j) x = x / row[j];
                    const double xj = __shfl_sync(0xffffffffu, x, j);
                    if (l > j) x -= row[j] * xj;
                }
            }
            if (l < kb) {
                z[jb + l] = x;
                zb[l] = x;
            }
        }
        __syncthreads();
        for (int64_t r = jb + kb + threadIdx.x; r < m; r += blockDim.x) {
            double acc = 0.0;
            for (int j = 0; j < kb; ++j) acc += F[r + (jb + j) * m] * zb[j];
            z[r] -= acc;
        }
        __syncthreads();
    }
    for (int64_t t = threadIdx.x; t < k; t += blockDim.x) y[j0 + t] = z[t];
}

// Backward solve of supernode s (1 block), its ancestors done: t_j = y_j - sum over the rows
// below of L[r][j] x_r (a warp per column), then L11^T x1 = t.
__global__ void __launch_bounds__(TH)
    k_backward(const int64_t* __restrict__ list, Fronts fr, const int64_t* __restrict__ zoff,
               double* __restrict__ work, double* __restrict__ y,
               const int64_t* __restrict__ winv_off, const double* __restrict__ winv,
               double* __restrict__ tmp) {
    const int64_t s = list[blockIdx.x];
    const int64_t j0 = fr.first[s];
    const int64_t r0 = fr.rows_ptr[s];
    const int64_t m = fr.rows_ptr[s + 1] - r0, k = fr.first[s + 1] - j0;
    const uint32_t* R = fr.rows + r0;
    const double* F = fr.f + fr.foff[s];
    double* z = work + zoff[s];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    // The solved values of the rows below (y at R[r], r >= k) gathered into shared memory a
    // chunk at a time, so that each warp's column sums read the front coalesced and x from
    // shared memory, with no dependent global loads.
    constexpr int XG = 1024;
    __shared__ double xg[XG];
    for (int64_t t = threadIdx.x; t < k; t += blockDim.x) z[t] = y[j0 + t];
    for (int64_t r0 = k; r0 < m; r0 += XG) {
        const int cnt = (int)min((int64_t)XG, m - r0);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) xg[t] = y[R[r0 + t]];
        __syncthreads();
        for (int64_t j = warp; j < k; j += nw) {
            const double* col = F + r0 + j * m;
            double acc = 0.0;
            for (int t = lane; t < cnt; t += 32) acc += col[t] * xg[t];
            for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) z[j] -= acc;
        }
    }
    __syncthreads();
    if (winv_off && winv_off[s] >= 0) {
        backward_by_inverse(winv + winv_off[s], k, z, tmp + j0);
        for (int64_t t = threadIdx.x; t < k; t += blockDim.x) y[j0 + t] = z[t];
        return;
    }
    // L11^T x1 = t in blocks of 32 from the last: warp 0 solves the block's triangle with
    // shuffles, then every row above the block subtracts the block's solved values times its
    // row of L (the 32 entries contiguous in the column-major front).
    __shared__ double zb[32];
    for (int64_t je = k; je > 0; je -= 32) {
        const int64_t jb = je >= 32 ? je - 32 : 0;
        const int kb = (int)(je - jb);
        if (threadIdx.x < 32) {
            // Lane l holds column jb + l of the block's triangle (contiguous in the front).
            const int l = threadIdx.x;
            double col[32];
#pragma unroll
            for (int j = 0; j < 32; ++j)
                col[j] = (j < kb && l < kb && j >= l) ? F[(jb + j) + (jb + l) * m] : 0.0;
            double x = l < kb ? z[jb + l] : 0.0;
#pragma unroll
            for (int j = 31; j >= 0; --j) {
                if (j < kb) {
                    if (l == j) x = x / col[j];
                    const double xj = __shfl_sync(0xffffffffu, x, j);
                    if (l < j) x -= col[j] * xj;
                }
            }
            if (l < kb) {
                z[jb + l] = x;
                zb[l] = x;
            }
        }
        __syncthreads();
        for (int64_t i = threadIdx.x; i < jb; i += blockDim.x) {
            double acc = 0.0;
            for (int j = 0; j < kb; ++j) acc += F[(jb + j) + i * m] * zb[j];
            z[i] -= acc;
        }
        __syncthreads();
    }
    for (int64_t t = threadIdx.x; t < k; t += blockDim.x) y[j0 + t] = z[t];
}

}  // namespace

void SparseFactor::factor(const HostCsr& a, const double* xyz, cudaStream_t s) {
    n_ = a.n;
    // The reference's fill-reducing order (order.rs) and the analysis in it.
    Supernodal S = analyse_factor(a, nested_dissection(a, xyz));
    ns_ = S.ns;
    entries_ = S.entries;
    flops_ = S.flops;
    host_first_ = S.first;
    m_.resize(ns_);
    k_.resize(ns_);
    std::vector<int64_t> foff(ns_), zoff(ns_);
    size_t fv = 0, zv = 0;
    for (int64_t t = 0; t < ns_; ++t) {
        m_[t] = S.rows_ptr[t + 1] - S.rows_ptr[t];
        k_[t] = S.first[t + 1] - S.first[t];
        foff[t] = (int64_t)fv;
        zoff[t] = (int64_t)zv;
        fv += (size_t)(m_[t] * m_[t]);
        zv += (size_t)m_[t];
    }
    front_values_ = fv;
    if (fv > ((size_t)96 << 30) / 8)
        throw Failure(FEMGPU_ERR_TOO_LARGE,
                      "the frontal matrices of the sparse factor need more than 96 GiB");
    // Children (increasing), relative indices of each child's update rows in its parent.
    std::vector<int64_t> cptr(ns_ + 1, 0), clist;
    for (int64_t t = 0; t < ns_; ++t)
        if (S.parent[t] >= 0) cptr[S.parent[t] + 1] += 1;
    for (int64_t t = 0; t < ns_; ++t) cptr[t + 1] += cptr[t];
    clist.resize(cptr[ns_]);
    std::vector<int64_t> fill(cptr.begin(), cptr.end() - 1);
    std::vector<int> rank(ns_, 0);
    for (int64_t t = 0; t < ns_; ++t)
        if (S.parent[t] >= 0) {
            rank[t] = (int)(fill[S.parent[t]] - cptr[S.parent[t]]);
            clist[fill[S.parent[t]]++] = t;
        }
    std::vector<int64_t> roff(ns_, 0);
    std::vector<uint32_t> rel;
    for (int64_t c = 0; c < ns_; ++c) {
        roff[c] = (int64_t)rel.size();
        const int64_t p = S.parent[c];
        if (p < 0) continue;
        const uint32_t* Rp = S.rows.data() + S.rows_ptr[p];
        for (int64_t t = S.rows_ptr[c] + k_[c]; t < S.rows_ptr[c + 1]; ++t)
            rel.push_back((uint32_t)(std::lower_bound(Rp, Rp + m_[p], S.rows[t]) - Rp));
    }
    // The level schedule.
    height_ = 0;
    for (int h : S.height) height_ = std::max<int64_t>(height_, h);
    small_.assign(height_ + 1, {});
    large_.assign(height_ + 1, {});
    std::vector<std::vector<int64_t>> all(height_ + 1);
    for (int64_t t = 0; t < ns_; ++t) {
        (m_[t] <= SMALL_ROWS ? small_ : large_)[S.height[t]].push_back(t);
        all[S.height[t]].push_back(t);
    }
    std::vector<int64_t> sl, ll;
    small_at_.assign(1, 0);
    level_at_.assign(1, 0);
    for (int64_t h = 0; h <= height_; ++h) {
        sl.insert(sl.end(), small_[h].begin(), small_[h].end());
        small_at_.push_back((int64_t)sl.size());
        ll.insert(ll.end(), all[h].begin(), all[h].end());
        level_at_.push_back((int64_t)ll.size());
    }
    // Extend-add chunks per (height of the parent, rank of the child).
    std::vector<int2> ch;
    chunks_.clear();
    for (int64_t h = 1; h <= height_; ++h) {
        int maxrank = -1;
        for (int64_t p : all[h]) maxrank = std::max<int>(maxrank, (int)(cptr[p + 1] - cptr[p]) - 1);
        for (int r = 0; r <= maxrank; ++r) {
            Chunks c{(int)h, r, (int64_t)ch.size(), 0};
            for (int64_t p : all[h]) {
                if (cptr[p + 1] - cptr[p] <= r) continue;
                const int64_t cc = clist[cptr[p] + r];
                const int64_t mu = m_[cc] - k_[cc];
                const int64_t parts = (mu * mu + CHUNK - 1) / CHUNK;
                for (int64_t q = 0; q < parts; ++q) ch.push_back(int2{(int)cc, (int)q});
            }
            c.count = (int64_t)ch.size() - c.at;
            if (c.count) chunks_.push_back(c);
        }
    }
    if (ns_ >= INT_MAX) throw Failure(FEMGPU_ERR_TOO_LARGE, "too many supernodes");
    // Device arrays.
    std::vector<int32_t> col2sn(n_);
    for (int64_t t = 0; t < ns_; ++t)
        for (int64_t j = S.first[t]; j < S.first[t + 1]; ++j) col2sn[j] = (int32_t)t;
    perm_.upload(S.perm.data(), n_, s);
    DevBuf<int64_t> iperm;
    iperm.upload(S.iperm.data(), n_, s);
    first_.upload(S.first.data(), ns_ + 1, s);
    rows_ptr_.upload(S.rows_ptr.data(), ns_ + 1, s);
    rows_.upload(S.rows.data(), S.rows.size(), s);
    foff_.upload(foff.data(), ns_, s);
    host_foff_ = foff;
    zoff_.upload(zoff.data(), ns_, s);
    child_ptr_.upload(cptr.data(), ns_ + 1, s);
    child_.upload(clist.data(), std::max<size_t>(1, clist.size()), s);
    relind_.upload(rel.data(), std::max<size_t>(1, rel.size()), s);
    relind_off_.upload(roff.data(), ns_, s);
    small_list_.upload(sl.data(), std::max<size_t>(1, sl.size()), s);
    level_list_.upload(ll.data(), std::max<size_t>(1, ll.size()), s);
    chunk_.upload(ch.data(), std::max<size_t>(1, ch.size()), s);
    DevBuf<int64_t> parent;
    parent.upload(S.parent.data(), ns_, s);
    DevBuf<int32_t> dcol2sn;
    dcol2sn.upload(col2sn.data(), n_, s);
    fronts_.alloc(fv);
    FG_CUDA(cudaMemsetAsync(fronts_.p, 0, fv * sizeof(double), s));
    work_.alloc(std::max<size_t>(1, zv));
    y_.alloc(n_);
    DevBuf<int64_t> aptr;
    DevBuf<uint32_t> aidx;
    DevBuf<double> aval, diag0(n_);
    aptr.upload(a.ptr.data(), n_ + 1, s);
    aidx.upload(a.idx.data(), a.nnz(), s);
    aval.upload(a.val.data(), a.nnz(), s);
    DevBuf<unsigned long long> status(1);
    FG_CUDA(cudaMemsetAsync(status.p, 0xff, sizeof(unsigned long long), s));
    const Fronts fr{first_.p, rows_ptr_.p, rows_.p, foff_.p, fronts_.p};
    k_assemble_fronts<<<blocks_for(n_, TH), TH, 0, s>>>(n_, perm_.p, iperm.p, aptr.p, aidx.p,
                                                       aval.p, dcol2sn.p, fr, diag0.p);
    FG_CHECK_LAUNCH();
    const size_t smem = (size_t)SMALL_ROWS * SMALL_ROWS * sizeof(double);
    FG_CUDA(cudaFuncSetAttribute(k_front_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    size_t ci = 0;
    for (int64_t h = 0; h <= height_; ++h) {
        for (; ci < chunks_.size() && chunks_[ci].height == h; ++ci)
            k_extend_add<<<(unsigned)chunks_[ci].count, TH, 0, s>>>(
                chunk_.p + chunks_[ci].at, fr, parent.p, relind_.p, relind_off_.p);
        const int64_t ns_small = small_at_[h + 1] - small_at_[h];
        if (ns_small > 0) {
            int mmax = 0;
            for (int64_t t : small_[h]) mmax = std::max<int>(mmax, (int)m_[t]);
            k_front_small<<<(unsigned)ns_small, TH, (size_t)mmax * mmax * sizeof(double), s>>>(
                small_list_.p + small_at_[h], fr, diag0.p, status.p);
        }
        for (int64_t t : large_[h])
            dense_partial_cholesky(fronts_.p + foff[t], m_[t], k_[t], diag0.p + S.first[t],
                                   S.first[t], status.p, s);
        FG_CHECK_LAUNCH();
    }
    unsigned long long bad = fetch(status.p, s);
    if (bad != ~0ull) {
        const int64_t j = (int64_t)bad;
        const double d = fetch(diag0.p + j, s);
        char buf[320];
        std::snprintf(buf, sizeof buf,
                      "the matrix is not positive definite: the pivot of column %lld is 0 or less "
                      "to the precision of the arithmetic (its diagonal is %s)",
                      (long long)S.perm[j], rust_exp_shortest(d).c_str());
        throw Failure(FEMGPU_ERR_NOT_SPD, buf);
    }
    FG_CUDA(cudaStreamSynchronize(s));
}

namespace {

// The lower triangle of the k x k diagonal block of front F (leading dimension m) into L (leading
// dimension k), zeros above: 1 member of the copy per blockIdx.y.
struct BlockCopy {
    const double* F;
    double* L;
    int64_t m, k;
};

__global__ void k_copy_blocks(const BlockCopy* __restrict__ c) {
    const BlockCopy b = c[blockIdx.y];
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < b.k * b.k;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t % b.k, j = t / b.k;
        b.L[t] = i >= j ? b.F[i + j * b.m] : 0.0;
    }
}

}  // namespace

void SparseFactor::invert_blocks(int64_t min_cols, cudaStream_t s) {
    std::vector<int64_t> off(ns_, -1);
    std::vector<int64_t> members;
    int64_t total = 0, kmax = 0;
    for (int64_t t = 0; t < ns_; ++t)
        if (k_[t] >= min_cols) {
            off[t] = total;
            total += k_[t] * k_[t];
            members.push_back(t);
            kmax = std::max(kmax, k_[t]);
        }
    if (members.empty()) return;
    if (members.size() > 65535) throw Failure(FEMGPU_ERR_TOO_LARGE, "too many large supernodes");
    winv_.alloc(total);
    tmp_.alloc(std::max<int64_t>(n_, 1));
    DevBuf<double> lc(total);
    std::vector<BlockCopy> bc;
    std::vector<int64_t> ns;
    std::vector<double*> ls, ws;
    for (int64_t t : members) {
        bc.push_back({fronts_.p + host_foff_[t], lc.p + off[t], m_[t], k_[t]});
        ns.push_back(k_[t]);
        ls.push_back(lc.p + off[t]);
        ws.push_back(winv_.p + off[t]);
    }
    DevBuf<BlockCopy> dbc;
    dbc.upload(bc.data(), bc.size(), s);
    k_copy_blocks<<<dim3((unsigned)blocks_for(kmax * kmax, TH, 256), (unsigned)bc.size()), TH, 0,
                    s>>>(dbc.p);
    FG_CHECK_LAUNCH();
    DenseBatchWork w;
    triangular_inverse_batch(ns, ls, ws, &w, s);
    winv_off_.upload(off.data(), ns_, s);
    FG_CUDA(cudaStreamSynchronize(s));
}

void SparseFactor::solve(const double* b, double* x, cudaStream_t s) {
    const Fronts fr{first_.p, rows_ptr_.p, rows_.p, foff_.p, fronts_.p};
    k_permute_in<<<blocks_for(n_, TH), TH, 0, s>>>(n_, perm_.p, b, y_.p);
    for (int64_t h = 0; h <= height_; ++h) {
        const int64_t cnt = level_at_[h + 1] - level_at_[h];
        if (cnt)
            k_forward<<<(unsigned)cnt, TH, 0, s>>>(level_list_.p + level_at_[h], fr, zoff_.p,
                                                   child_ptr_.p, child_.p, relind_.p,
                                                   relind_off_.p, work_.p, y_.p, winv_off_.p,
                                                   winv_.p, tmp_.p);
    }
    for (int64_t h = height_; h >= 0; --h) {
        const int64_t cnt = level_at_[h + 1] - level_at_[h];
        if (cnt)
            k_backward<<<(unsigned)cnt, TH, 0, s>>>(level_list_.p + level_at_[h], fr, zoff_.p,
                                                    work_.p, y_.p, winv_off_.p, winv_.p,
                                                    tmp_.p);
    }
    k_permute_out<<<blocks_for(n_, TH), TH, 0, s>>>(n_, perm_.p, y_.p, x);
    FG_CHECK_LAUNCH();
}

size_t SparseFactor::solve_launches() const {
    size_t c = 2;
    for (int64_t h = 0; h <= height_; ++h)
        if (level_at_[h + 1] > level_at_[h]) c += 2;
    return c;
}

size_t SparseFactor::bytes() const {
    return fronts_.bytes() + work_.bytes() + y_.bytes() + perm_.bytes() + first_.bytes() +
           rows_ptr_.bytes() + rows_.bytes() + foff_.bytes() + zoff_.bytes() +
           child_ptr_.bytes() + child_.bytes() + relind_.bytes() + relind_off_.bytes() +
           small_list_.bytes() + level_list_.bytes() + chunk_.bytes() + winv_.bytes() +
           tmp_.bytes() + winv_off_.bytes();
}

std::string SparseFactor::describe() const {
    char buf[256];
    int64_t nl = 0, mmax = 0;
    for (const auto& l : large_) nl += (int64_t)l.size();
    for (int64_t m : m_) mmax = std::max(mmax, m);
    std::snprintf(buf, sizeof buf,
                  "sparse multifrontal factor: %lld supernodes, %lld levels, %lld fronts above %d "
                  "rows (largest %lld), L entries %llu, flops %.3g, front values %zu\n",
                  (long long)ns_, (long long)height_ + 1, (long long)nl, SMALL_ROWS,
                  (long long)mmax, (unsigned long long)entries_, flops_, front_values_);
    return buf;
}

}  // namespace femgpu
