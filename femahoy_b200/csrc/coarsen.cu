// The multigrid hierarchy on the device (coarsen.cuh): plane coarsening with its prolongation,
// transposes and the sparse products of the Galerkin operator P^T A P.
#include <cub/cub.cuh>

#include <algorithm>

#include "coarsen.cuh"

namespace femgpu {
namespace {

constexpr int TH = 256;

// The interpolation of each fine plane of one axis: the 2 coarse planes it takes its value from
// (equal for a plane that is kept) and their linear weights from the plane coordinates.
struct AxisMaps {
    const uint32_t* c[3];  // 2 per fine plane
    const double* w[3];    // 2 per fine plane
    uint64_t dims[3];      // coarse planes per axis
    int comps;
};

// The at most 8 (coarse key, weight) pairs of fine row i, keys increasing. The key of a coarse
// unknown is comp + comps (x + dims_x (y + dims_y z)), so increasing keys are grid order.
__device__ int interp_row(int64_t i, const uint32_t* __restrict__ pts,
                          const uint8_t* __restrict__ comp, const int64_t* __restrict__ aptr,
                          const uint32_t* __restrict__ aidx, const double* __restrict__ aval,
                          const AxisMaps& m, uint64_t key[8], double wt[8]) {
    uint32_t f[3], c0[3], c1[3];
    double w0[3], w1[3];
    bool between[3];
    bool any = false;
    for (int d = 0; d < 3; ++d) {
        f[d] = pts[3 * i + d];
        c0[d] = m.c[d][2 * f[d]];
        c1[d] = m.c[d][2 * f[d] + 1];
        w0[d] = m.w[d][2 * f[d]];
        w1[d] = m.w[d][2 * f[d] + 1];
        between[d] = c0[d] != c1[d];
        any |= between[d];
    }
    if (m.comps == 1 && any) {
        // The operator weights of a scalar between 2 coarse planes: minus its row's couplings to
        // the fine plane below and to the one above, each summed in the row's order.
        double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {0.0, 0.0, 0.0};
        for (int64_t k = aptr[i]; k < aptr[i + 1]; ++k) {
            const uint32_t j = aidx[k];
            const double v = aval[k];
            for (int d = 0; d < 3; ++d) {
                if (!between[d]) continue;
                const uint32_t g = pts[3 * (int64_t)j + d];
                if (g + 1 == f[d])
                    lo[d] -= v;
                else if (g == f[d] + 1)
                    hi[d] -= v;
            }
        }
        for (int d = 0; d < 3; ++d)
            if (between[d] && lo[d] > 0.0 && hi[d] > 0.0) {
                w0[d] = lo[d] / (lo[d] + hi[d]);
                w1[d] = hi[d] / (lo[d] + hi[d]);
            }
    }
    const uint64_t cc = comp[i];
    int cnt = 0;
    for (int a = 0; a < 2; ++a) {
        const uint64_t cx = a ? c1[0] : c0[0];
        const double wx = a ? w1[0] : w0[0];
        for (int b = 0; b < 2; ++b) {
            const uint64_t cy = b ? c1[1] : c0[1];
            const double wy = b ? w1[1] : w0[1];
            for (int e = 0; e < 2; ++e) {
                const uint64_t cz = e ? c1[2] : c0[2];
                const double wz = e ? w1[2] : w0[2];
                const double w = wx * wy * wz;
                if (w == 0.0) continue;
                const uint64_t kk = cc + m.comps * (cx + m.dims[0] * (cy + m.dims[1] * cz));
                // Insert in key order.
                int at = cnt;
                while (at > 0 && key[at - 1] > kk) {
                    key[at] = key[at - 1];
                    wt[at] = wt[at - 1];
                    --at;
                }
                key[at] = kk;
                wt[at] = w;
                ++cnt;
            }
        }
    }
    return cnt;
}

template <bool FILL>
__global__ void k_interp(int64_t n, const uint32_t* __restrict__ pts,
                         const uint8_t* __restrict__ comp, const int64_t* __restrict__ aptr,
                         const uint32_t* __restrict__ aidx, const double* __restrict__ aval,
                         AxisMaps m, uint32_t* __restrict__ count, const int64_t* __restrict__ ptr,
                         uint64_t* __restrict__ keys, double* __restrict__ vals) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t key[8];
        double wt[8];
        const int c = interp_row(i, pts, comp, aptr, aidx, aval, m, key, wt);
        if (!FILL) {
            count[i] = (uint32_t)c;
        } else {
            const int64_t at = ptr[i];
            for (int k = 0; k < c; ++k) {
                keys[at + k] = key[k];
                vals[at + k] = wt[k];
            }
        }
    }
}

// The coarse column of each entry: the rank of its key among the distinct keys.
__global__ void k_key_rank(int64_t nnz, const uint64_t* __restrict__ keys,
                           const uint64_t* __restrict__ uniq, int64_t nu,
                           uint32_t* __restrict__ idx) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[e];
        int64_t lo = 0, hi = nu;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (uniq[mid] < k)
                lo = mid + 1;
            else
                hi = mid;
        }
        idx[e] = (uint32_t)lo;
    }
}

// The grid point and component of each coarse unknown from its key.
__global__ void k_key_points(int64_t nu, const uint64_t* __restrict__ uniq, int comps,
                             uint64_t dx, uint64_t dy, uint32_t* __restrict__ pts,
                             uint8_t* __restrict__ comp) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nu;
         q += (int64_t)gridDim.x * blockDim.x) {
        uint64_t k = uniq[q];
        comp[q] = (uint8_t)(k % comps);
        k /= comps;
        pts[3 * q] = (uint32_t)(k % dx);
        k /= dx;
        pts[3 * q + 1] = (uint32_t)(k % dy);
        pts[3 * q + 2] = (uint32_t)(k / dy);
    }
}

// The first entry of each row from the sorted (row << 32 | column) keys.
__global__ void k_rows_from_keys(int64_t rows, const uint64_t* __restrict__ keys, int64_t nnz,
                                 int64_t* __restrict__ ptr) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= rows;
         r += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t want = (uint64_t)r << 32;
        int64_t lo = 0, hi = nnz;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (keys[mid] < want)
                lo = mid + 1;
            else
                hi = mid;
        }
        ptr[r] = lo;
    }
}

__global__ void k_transpose_keys(int64_t rows, const int64_t* __restrict__ ptr,
                                 const uint32_t* __restrict__ idx, uint64_t* __restrict__ keys) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows;
         i += (int64_t)gridDim.x * blockDim.x)
        for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
            keys[k] = ((uint64_t)idx[k] << 32) | (uint64_t)i;
}

__global__ void k_low_words(int64_t n, const uint64_t* __restrict__ keys,
                            uint32_t* __restrict__ idx) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x)
        idx[k] = (uint32_t)(keys[k] & 0xffffffffu);
}

// Row i of C = A B by 1 warp with the row's columns in a hash table in shared memory (SPG_TAB
// slots, linear probing, a slot claimed by compare-and-swap): for each entry a_ij of A's row in
// order, the lanes take B's row j, 32 entries at a time, and add a_ij b_jk into column k's
// slot. B's row has distinct columns, so no 2 lanes meet in a slot within a step, and each
// entry of C is summed in A's row order, whatever the lanes' timing (a slot's first product is
// stored, not added to 0): the coarse operators are the same bits every time. The counting
// pass counts the claimed slots;
// the filling pass writes the row's columns increasing (each entry's rank among the row's
// columns) with their sums at ptr[i]. A row of more than SPG_CAP columns sets *overflow.
constexpr int SPG_TAB = 1024, SPG_CAP = 512, SPG_WARPS = 4;
constexpr uint32_t SPG_EMPTY = 0xffffffffu;

// Shared memory per warp: the table's keys, and for the filling pass its sums and the row's
// columns compacted.
template <bool FILL>
constexpr size_t spg_smem() {
    return (size_t)SPG_WARPS *
           (SPG_TAB * sizeof(uint32_t) + (FILL ? SPG_TAB * sizeof(double) + SPG_CAP * 4 : 0));
}

template <bool FILL>
__global__ void __launch_bounds__(32 * SPG_WARPS)
    k_spgemm_warp(int64_t rows, const int64_t* __restrict__ aptr,
                  const uint32_t* __restrict__ aidx, const double* __restrict__ aval,
                  const int64_t* __restrict__ bptr, const uint32_t* __restrict__ bidx,
                  const double* __restrict__ bval, uint32_t* __restrict__ count,
                  const int64_t* __restrict__ cptr, uint32_t* __restrict__ cidx,
                  double* __restrict__ cval, int* __restrict__ overflow) {
    extern __shared__ __align__(16) unsigned char spg_raw[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* vals = reinterpret_cast<double*>(spg_raw) + (size_t)w * SPG_TAB;  // FILL only
    uint32_t* keys = reinterpret_cast<uint32_t*>(
                         spg_raw + (FILL ? (size_t)SPG_WARPS * SPG_TAB * sizeof(double) : 0)) +
                     (size_t)w * SPG_TAB;
    uint32_t* ck = reinterpret_cast<uint32_t*>(
                       spg_raw + (size_t)SPG_WARPS * SPG_TAB * (sizeof(double) + 4)) +
                   (size_t)w * SPG_CAP;  // FILL only
    const int64_t nwarps = (int64_t)gridDim.x * SPG_WARPS;
    for (int64_t i = blockIdx.x * (int64_t)SPG_WARPS + w; i < rows; i += nwarps) {
        for (int t = lane; t < SPG_TAB; t += 32) keys[t] = SPG_EMPTY;
        __syncwarp();
        int claimed = 0;  // slots this lane claimed
        bool full = false;
        for (int64_t ka = aptr[i]; ka < aptr[i + 1]; ++ka) {
            const uint32_t j = aidx[ka];
            const double a = aval[ka];
            const int64_t b0 = bptr[j], b1 = bptr[j + 1];
            for (int64_t kb = b0 + lane; kb < b1 && !full; kb += 32) {
                const uint32_t c = bidx[kb];
                uint32_t h = (c * 2654435761u) >> (32 - 10);
                for (int probes = 0;; ++probes) {
                    if (probes == SPG_TAB) {
                        full = true;
                        break;
                    }
                    const uint32_t k = *(volatile uint32_t*)&keys[h];
                    if (k == c) {
                        if (FILL) vals[h] += a * bval[kb];
                        break;
                    }
                    if (k == SPG_EMPTY) {
                        const uint32_t old = atomicCAS(&keys[h], SPG_EMPTY, c);
                        if (old == SPG_EMPTY) {
                            if (FILL) vals[h] = a * bval[kb];
                            ++claimed;
                            break;
                        }
                        if (old == c) {
                            if (FILL) vals[h] += a * bval[kb];
                            break;
                        }
                    }
                    h = (h + 1) & (SPG_TAB - 1);
                }
            }
            __syncwarp();
        }
        int m = claimed;
        for (int o = 16; o; o >>= 1) m += __shfl_xor_sync(0xffffffffu, m, o);
        full = __any_sync(0xffffffffu, full) || m > SPG_CAP;
        if (full) {
            if (lane == 0) {
                atomicExch(overflow, 1);
                if (!FILL) count[i] = 0;
            }
            __syncwarp();
            continue;
        }
        if (!FILL) {
            if (lane == 0) count[i] = (uint32_t)m;
        } else {
            // The row's columns compacted, then each claimed slot's rank among them is its place
            // in the output (the columns increasing).
            int base = 0;
            for (int t0 = 0; t0 < SPG_TAB; t0 += 32) {
                const uint32_t c = keys[t0 + lane];
                const bool p = c != SPG_EMPTY;
                const unsigned bal = __ballot_sync(0xffffffffu, p);
                if (p) ck[base + __popc(bal & ((1u << lane) - 1u))] = c;
                base += __popc(bal);
            }
            __syncwarp();
            const int64_t at = cptr[i];
            for (int t = lane; t < SPG_TAB; t += 32) {
                const uint32_t c = keys[t];
                if (c == SPG_EMPTY) continue;
                int rank = 0;
                for (int u = 0; u < m; ++u) rank += ck[u] < c;
                cidx[at + rank] = c;
                cval[at + rank] = vals[t];
            }
        }
        __syncwarp();
    }
}

int key_bits(uint64_t maxkey) {
    int b = 1;
    while (b < 64 && (maxkey >> b) != 0) ++b;
    return b;
}

// C = A B with A's rows (aptr, aidx, aval; `rows` of them) and B (bptr, bidx, bval, `cols`
// columns).
void spgemm(int64_t rows, const int64_t* aptr, const uint32_t* aidx, const double* aval,
            const int64_t* bptr, const uint32_t* bidx, const double* bval, int64_t cols,
            DevBuf<int64_t>* cptr, DevBuf<uint32_t>* cidx, DevBuf<double>* cval, int64_t* cnnz,
            cudaStream_t s) {
    DevBuf<uint32_t> count(rows > 0 ? rows : 1);
    DevBuf<int> overflow(1);
    overflow.zero(s);
    // 1 warp per row, the row's columns hashed in shared memory.
    const int blocks = blocks_for(rows, SPG_WARPS, NUM_SMS * 16);
    FG_CUDA(cudaFuncSetAttribute(k_spgemm_warp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)spg_smem<true>()));
    k_spgemm_warp<false><<<blocks, 32 * SPG_WARPS, spg_smem<false>(), s>>>(
        rows, aptr, aidx, aval, bptr, bidx, bval, count.p, nullptr, nullptr, nullptr, overflow.p);
    FG_CHECK_LAUNCH();
    if (fetch(overflow.p, s))
        throw Failure(FEMGPU_ERR_TOO_LARGE, "a row of a coarse operator has more than 512 entries");
    cptr->alloc(rows + 1);
    exclusive_scan32(count.p, cptr->p, rows, s);
    int64_t nnz = fetch(cptr->p + rows, s);
    cidx->alloc(nnz > 0 ? nnz : 1);
    cval->alloc(nnz > 0 ? nnz : 1);
    k_spgemm_warp<true><<<blocks, 32 * SPG_WARPS, spg_smem<true>(), s>>>(
        rows, aptr, aidx, aval, bptr, bidx, bval, nullptr, cptr->p, cidx->p, cval->p,
        overflow.p);
    FG_CHECK_LAUNCH();
    (void)cols;
    *cnnz = nnz;
}

}  // namespace

void grid_upload(const HostLevel& h, DevGrid* d, cudaStream_t s) {
    d->planes = h.planes;
    d->n = (int64_t)h.points.size();
    int comps = 1;
    for (uint8_t c : h.comp) comps = std::max(comps, (int)c + 1);
    d->comps = comps;
    std::vector<uint32_t> flat(3 * h.points.size());
    for (size_t k = 0; k < h.points.size(); ++k)
        for (int a = 0; a < 3; ++a) flat[3 * k + a] = h.points[k][a];
    d->pts.upload(flat.data(), flat.size(), s);
    d->comp.upload(h.comp.data(), h.comp.size(), s);
    FG_CUDA(cudaStreamSynchronize(s));
}

HostLevel grid_download(const DevGrid& d, cudaStream_t s) {
    HostLevel h;
    h.planes = d.planes;
    std::vector<uint32_t> flat(3 * d.n);
    d.pts.download(flat.data(), flat.size(), s);
    h.comp.resize(d.n);
    d.comp.download(h.comp.data(), d.n, s);
    FG_CUDA(cudaStreamSynchronize(s));
    h.points.resize(d.n);
    for (int64_t k = 0; k < d.n; ++k)
        for (int a = 0; a < 3; ++a) h.points[k][a] = flat[3 * k + a];
    return h;
}

bool coarsen_grid(const DevGrid& fine, const DevCsr& a, int axes, DevRect* p, DevGrid* coarse,
                  cudaStream_t s) {
    if (axes == 0) axes = 7;
    // The planes kept along each axis and the map of each fine plane (host: a few hundred
    // planes at most per axis).
    std::array<std::vector<uint32_t>, 3> mc;
    std::array<std::vector<double>, 3> mw;
    std::array<std::vector<double>, 3> cplanes;
    bool any = false;
    for (int d = 0; d < 3; ++d) {
        const std::vector<double>& pl = fine.planes[d];
        const size_t n = pl.size();
        std::vector<size_t> keep;
        const bool halve = n > 2 && ((axes >> d) & 1);
        any |= halve;
        for (size_t i = 0; i < n; i += halve ? 2 : 1) keep.push_back(i);
        if (halve && keep.back() != n - 1) keep.push_back(n - 1);
        mc[d].resize(2 * n);
        mw[d].resize(2 * n);
        size_t c = 0;
        for (size_t i = 0; i < n; ++i) {
            while (keep[c] < i) ++c;
            if (keep[c] == i) {
                mc[d][2 * i] = mc[d][2 * i + 1] = (uint32_t)c;
                mw[d][2 * i] = 1.0;
                mw[d][2 * i + 1] = 0.0;
            } else {
                const size_t lo = keep[c - 1], hi = keep[c];
                const double w = (pl[i] - pl[lo]) / (pl[hi] - pl[lo]);
                mc[d][2 * i] = (uint32_t)(c - 1);
                mc[d][2 * i + 1] = (uint32_t)c;
                mw[d][2 * i] = 1.0 - w;
                mw[d][2 * i + 1] = w;
            }
        }
        for (size_t i : keep) cplanes[d].push_back(pl[i]);
    }
    if (!any) return false;
    std::array<DevBuf<uint32_t>, 3> dc;
    std::array<DevBuf<double>, 3> dw;
    AxisMaps m{};
    for (int d = 0; d < 3; ++d) {
        dc[d].upload(mc[d].data(), mc[d].size(), s);
        dw[d].upload(mw[d].data(), mw[d].size(), s);
        m.c[d] = dc[d].p;
        m.w[d] = dw[d].p;
        m.dims[d] = cplanes[d].size();
    }
    m.comps = fine.comps;
    const int64_t n = fine.n;
    const int blocks = blocks_for(n, TH);
    DevBuf<uint32_t> count(n);
    k_interp<false><<<blocks, TH, 0, s>>>(n, fine.pts.p, fine.comp.p, a.ptr.p, a.idx.p, a.val.p, m,
                                         count.p, nullptr, nullptr, nullptr);
    FG_CHECK_LAUNCH();
    p->rows = n;
    p->ptr.alloc(n + 1);
    exclusive_scan32(count.p, p->ptr.p, n, s);
    const int64_t nnz = fetch(p->ptr.p + n, s);
    p->nnz = nnz;
    DevBuf<uint64_t> keys(nnz), sorted(nnz);
    p->val.alloc(nnz);
    k_interp<true><<<blocks, TH, 0, s>>>(n, fine.pts.p, fine.comp.p, a.ptr.p, a.idx.p, a.val.p, m,
                                        nullptr, p->ptr.p, keys.p, p->val.p);
    FG_CHECK_LAUNCH();
    // The coarse unknowns: the distinct keys, in increasing (grid) order.
    const uint64_t maxkey =
        (uint64_t)fine.comps * m.dims[0] * m.dims[1] * m.dims[2];
    const int bits = key_bits(maxkey);
    size_t tmp = 0;
    FG_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, keys.p, sorted.p, (int)nnz, 0, bits, s));
    DevBuf<uint8_t> t1(tmp);
    FG_CUDA(cub::DeviceRadixSort::SortKeys(t1.p, tmp, keys.p, sorted.p, (int)nnz, 0, bits, s));
    DevBuf<uint64_t> uniq(nnz);
    DevBuf<int64_t> nu_d(1);
    size_t tmp2 = 0;
    FG_CUDA(cub::DeviceSelect::Unique(nullptr, tmp2, sorted.p, uniq.p, nu_d.p, (int)nnz, s));
    DevBuf<uint8_t> t2(tmp2);
    FG_CUDA(cub::DeviceSelect::Unique(t2.p, tmp2, sorted.p, uniq.p, nu_d.p, (int)nnz, s));
    const int64_t nu = fetch(nu_d.p, s);
    p->cols = nu;
    p->idx.alloc(nnz);
    k_key_rank<<<blocks_for(nnz, TH), TH, 0, s>>>(nnz, keys.p, uniq.p, nu, p->idx.p);
    coarse->planes = cplanes;
    coarse->n = nu;
    coarse->comps = fine.comps;
    coarse->pts.alloc(3 * nu);
    coarse->comp.alloc(nu);
    k_key_points<<<blocks_for(nu, TH), TH, 0, s>>>(nu, uniq.p, fine.comps, m.dims[0], m.dims[1],
                                                  coarse->pts.p, coarse->comp.p);
    FG_CHECK_LAUNCH();
    FG_CUDA(cudaStreamSynchronize(s));
    return true;
}

void transpose_rect(const DevRect& p, DevRect* t, cudaStream_t s) {
    const int64_t nnz = p.nnz;
    DevBuf<uint64_t> keys(nnz > 0 ? nnz : 1), sorted(nnz > 0 ? nnz : 1);
    DevBuf<double> vals(nnz > 0 ? nnz : 1);
    k_transpose_keys<<<blocks_for(p.rows, TH), TH, 0, s>>>(p.rows, p.ptr.p, p.idx.p, keys.p);
    FG_CHECK_LAUNCH();
    const int bits = 32 + key_bits((uint64_t)std::max<int64_t>(p.cols, 1));
    size_t tmp = 0;
    FG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys.p, sorted.p, p.val.p, vals.p,
                                            (int)nnz, 0, bits, s));
    DevBuf<uint8_t> t1(tmp);
    FG_CUDA(cub::DeviceRadixSort::SortPairs(t1.p, tmp, keys.p, sorted.p, p.val.p, vals.p,
                                            (int)nnz, 0, bits, s));
    t->rows = p.cols;
    t->cols = p.rows;
    t->nnz = nnz;
    t->ptr.alloc(p.cols + 1);
    k_rows_from_keys<<<blocks_for(p.cols + 1, TH), TH, 0, s>>>(p.cols, sorted.p, nnz, t->ptr.p);
    t->idx.alloc(nnz > 0 ? nnz : 1);
    k_low_words<<<blocks_for(nnz, TH), TH, 0, s>>>(nnz, sorted.p, t->idx.p);
    FG_CHECK_LAUNCH();
    t->val = std::move(vals);
    FG_CUDA(cudaStreamSynchronize(s));
}

void galerkin_product(const DevRect& p, const DevCsr& a, DevCsr* out, cudaStream_t s) {
    if (p.nnz >= 0x7fffffff)
        throw Failure(FEMGPU_ERR_TOO_LARGE, "a prolongation with 2^31 entries or more");
    // A P (fine rows, coarse columns), then P^T (A P).
    DevBuf<int64_t> apptr;
    DevBuf<uint32_t> apidx;
    DevBuf<double> apval;
    int64_t apnnz = 0;
    spgemm(a.n, a.ptr.p, a.idx.p, a.val.p, p.ptr.p, p.idx.p, p.val.p, p.cols, &apptr, &apidx,
           &apval, &apnnz, s);
    DevRect r;
    transpose_rect(p, &r, s);
    out->n = p.cols;
    spgemm(r.rows, r.ptr.p, r.idx.p, r.val.p, apptr.p, apidx.p, apval.p, p.cols, &out->ptr,
           &out->idx, &out->val, &out->nnz, s);
    FG_CUDA(cudaStreamSynchronize(s));
}

HostRect rect_download(const DevRect& d, cudaStream_t s) {
    HostRect h;
    h.rows = d.rows;
    h.cols = d.cols;
    h.ptr.resize(d.rows + 1);
    h.idx.resize(d.nnz);
    h.val.resize(d.nnz);
    d.ptr.download(h.ptr.data(), d.rows + 1, s);
    d.idx.download(h.idx.data(), d.nnz, s);
    d.val.download(h.val.data(), d.nnz, s);
    FG_CUDA(cudaStreamSynchronize(s));
    return h;
}

void rect_upload(const HostRect& h, DevRect* d, cudaStream_t s) {
    d->rows = h.rows;
    d->cols = h.cols;
    d->nnz = (int64_t)h.idx.size();
    d->ptr.upload(h.ptr.data(), h.ptr.size(), s);
    d->idx.upload(h.idx.data(), h.idx.size(), s);
    d->val.upload(h.val.data(), h.val.size(), s);
    FG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace femgpu
