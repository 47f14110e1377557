// Offset forms and the 3x3-block SELL form built on the device (offsets.cuh).
#include <algorithm>

#include "block3.cuh"
#include "offsets.cuh"
#include "ops.cuh"

namespace femgpu {
namespace {

constexpr int TH = 256;
constexpr unsigned long long EMPTY_SLOT = ~0ull;
static_assert(B3C == 32, "k_b3_check maps the block rows of a slice to the lanes of a warp");
static_assert(TH % 32 == 0, "whole warps");

// Inserts o into the table of `slots` values (EMPTY_SLOT marks a free one). Slots are taken in
// order, each by 1 compare-and-swap, so a value is in 1 slot only and a reader that meets a free
// slot has seen every value inserted before it. False when o is new and the table is full.
__device__ __forceinline__ bool slot_insert(unsigned long long* tab, int slots,
                                            unsigned long long o) {
    for (int k = 0; k < slots; ++k) {
        const unsigned long long v = *(volatile unsigned long long*)(tab + k);
        if (v == o) return true;
        if (v == EMPTY_SLOT) {
            const unsigned long long old = atomicCAS(tab + k, EMPTY_SLOT, o);
            if (old == EMPTY_SLOT || old == o) return true;
        }
    }
    return false;
}

// g[0, MAXK): the global table; g[MAXK], g[MAXK + 1]: upper and diagonal entries; g[MAXK + 2]:
// set when some table ran full.
template <bool STENCIL>
__global__ void k_scan_offsets(const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                               int64_t rows, int limit, int* __restrict__ base,
                               unsigned long long* g) {
    __shared__ unsigned long long tab[MAXK];
    __shared__ unsigned long long su, sd;
    __shared__ int full;
    for (int k = threadIdx.x; k < MAXK; k += blockDim.x) tab[k] = EMPTY_SLOT;
    if (threadIdx.x == 0) {
        su = 0;
        sd = 0;
        full = 0;
    }
    __syncthreads();
    unsigned long long up = 0, dg = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (*(volatile int*)&full) break;
        const int64_t b = ptr[i], e = ptr[i + 1];
        int64_t origin = i;
        if (!STENCIL) {
            uint32_t m = 0xffffffffu;
            for (int64_t k = b; k < e; ++k) m = min(m, idx[k]);
            origin = e > b ? (int64_t)m : 0;
            base[i] = (int)origin;
        }
        for (int64_t k = b; k < e; ++k) {
            const int64_t o = (int64_t)idx[k] - origin;
            if (STENCIL) {
                if (o < 0) continue;
                ++up;
                dg += o == 0;
            }
            if (!slot_insert(tab, limit, (unsigned long long)o)) {
                full = 1;
                break;
            }
        }
    }
    atomicAdd(&su, up);
    atomicAdd(&sd, dg);
    __syncthreads();
    if (threadIdx.x < MAXK && tab[threadIdx.x] != EMPTY_SLOT)
        if (!slot_insert(g, limit, tab[threadIdx.x])) atomicExch(g + MAXK + 2, 1ull);
    if (threadIdx.x == 0) {
        if (full) atomicExch(g + MAXK + 2, 1ull);
        atomicAdd(g + MAXK, su);
        atomicAdd(g + MAXK + 1, sd);
    }
}

struct OffsetList {
    int K;
    int64_t v[MAXK];
};

template <class T, bool STENCIL>
__global__ void k_fill_offsets(const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                               const double* __restrict__ val, int64_t rows,
                               const int* __restrict__ base, OffsetList offs, int64_t ld,
                               T* __restrict__ coef) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t origin = STENCIL ? i : (int64_t)base[i];
        for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            const int64_t o = (int64_t)idx[k] - origin;
            if (STENCIL && o < 0) continue;
            int lo = 0, hi = offs.K - 1;  // offs.v sorted, o among them
            while (lo < hi) {
                const int mid = (lo + hi) / 2;
                if (offs.v[mid] < o)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            coef[(int64_t)lo * ld + i] = (T)val[k];
        }
    }
}

// Block row I = thread g (the threads of a warp are the 32 block rows of 1 slice, and every warp
// runs the loop the same number of times): flags a block row whose 3 rows differ in columns or
// whose columns are not aligned triples, and writes each slice's entries (its widest block row,
// in blocks, times B3C).
__global__ void k_b3_check(const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                           int64_t nb, int64_t nslices, int64_t* __restrict__ ent,
                           int* __restrict__ bad) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nslices * B3C;
         g += (int64_t)gridDim.x * blockDim.x) {
        unsigned w = 0;
        if (g < nb) {
            const int64_t r0 = 3 * g, p0 = ptr[r0];
            const int64_t len = ptr[r0 + 1] - p0;
            bool good = len % 3 == 0;
            for (int q = 1; q < 3 && good; ++q) {
                const int64_t pq = ptr[r0 + q];
                if (ptr[r0 + q + 1] - pq != len) good = false;
                for (int64_t k = 0; k < len && good; ++k)
                    if (idx[pq + k] != idx[p0 + k]) good = false;
            }
            for (int64_t k = 0; k < len && good; k += 3) {
                const uint32_t c = idx[p0 + k];
                if (c % 3 != 0 || idx[p0 + k + 1] != c + 1 || idx[p0 + k + 2] != c + 2)
                    good = false;
            }
            if (!good) atomicOr(bad, 1);
            w = (unsigned)(len / 3);
        }
        const unsigned wmax = __reduce_max_sync(0xffffffffu, w);
        if ((threadIdx.x & 31) == 0) ent[g / B3C] = (int64_t)wmax * B3C;
    }
}

template <class T>
__global__ void k_b3_fill(const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                          const double* __restrict__ val, int64_t nb,
                          const int64_t* __restrict__ sptr, uint32_t* __restrict__ col,
                          T* __restrict__ vals) {
    for (int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; I < nb;
         I += (int64_t)gridDim.x * blockDim.x) {
        const int64_t sl = I / B3C, r = I % B3C, base = sptr[sl];
        const int w = (int)((sptr[sl + 1] - base) / B3C);
        const int wi = (int)((ptr[3 * I + 1] - ptr[3 * I]) / 3);
        for (int k = 0; k < w; ++k) {
            const int64_t blk = base + (int64_t)k * B3C + r;
            if (k < wi) {
                col[blk] = idx[ptr[3 * I] + 3 * k] / 3;
                for (int q = 0; q < 3; ++q)
                    for (int c = 0; c < 3; ++c)
                        vals[blk * 9 + 3 * q + c] = (T)val[ptr[3 * I + q] + 3 * k + c];
            } else {
                col[blk] = (uint32_t)I;  // padding: value 0, the block row's own x
            }
        }
    }
}

template <class T>
__global__ void k_reciprocal(int64_t n, const double* __restrict__ d, T* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (T)(1.0 / d[i]);
}

template <class T>
__global__ void k_to(int64_t n, const double* __restrict__ a, T* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (T)a[i];
}

}  // namespace

bool scan_offsets(const int64_t* ptr, const uint32_t* idx, int64_t rows, bool stencil, int limit,
                  int* base, OffsetScan* out, cudaStream_t s) {
    limit = std::min(limit, MAXK);
    DevBuf<unsigned long long> g(MAXK + 3);
    FG_CUDA(cudaMemsetAsync(g.p, 0xff, MAXK * sizeof(unsigned long long), s));
    FG_CUDA(cudaMemsetAsync(g.p + MAXK, 0, 3 * sizeof(unsigned long long), s));
    if (rows > 0) {
        if (stencil)
            k_scan_offsets<true><<<blocks_for(rows, TH), TH, 0, s>>>(ptr, idx, rows, limit, base,
                                                                      g.p);
        else
            k_scan_offsets<false><<<blocks_for(rows, TH), TH, 0, s>>>(ptr, idx, rows, limit,
                                                                       base, g.p);
        FG_CHECK_LAUNCH();
    }
    std::vector<unsigned long long> h = g.to_host(s);
    if (h[MAXK + 2]) return false;
    out->offs.clear();
    for (int k = 0; k < MAXK; ++k)
        if (h[k] != EMPTY_SLOT) out->offs.push_back((int64_t)h[k]);
    std::sort(out->offs.begin(), out->offs.end());
    out->upper = (int64_t)h[MAXK];
    out->diag = (int64_t)h[MAXK + 1];
    return true;
}

template <class T>
void fill_offsets(const int64_t* ptr, const uint32_t* idx, const double* val, int64_t rows,
                  bool stencil, const int* base, const std::vector<int64_t>& offs, int64_t ld,
                  T* coef, cudaStream_t s) {
    if (offs.empty() || offs.size() > (size_t)MAXK)
        throw Failure(FEMGPU_ERR_TOO_LARGE, "an offset form of more than 32 offsets");
    FG_CUDA(cudaMemsetAsync(coef, 0, offs.size() * (size_t)ld * sizeof(T), s));
    if (rows == 0) return;
    OffsetList l{};
    l.K = (int)offs.size();
    for (size_t k = 0; k < offs.size(); ++k) l.v[k] = offs[k];
    if (stencil)
        k_fill_offsets<T, true><<<blocks_for(rows, TH), TH, 0, s>>>(ptr, idx, val, rows, base, l,
                                                                     ld, coef);
    else
        k_fill_offsets<T, false><<<blocks_for(rows, TH), TH, 0, s>>>(ptr, idx, val, rows, base,
                                                                      l, ld, coef);
    FG_CHECK_LAUNCH();
}

template <class T>
bool make_bsell3_device(const DevCsr& a, DevBuf<int64_t>* sptr, DevBuf<uint32_t>* col,
                        DevBuf<T>* val, cudaStream_t s) {
    if (a.n % 3 != 0 || a.n / 3 >= 0x7fffffff || a.n == 0) return false;
    const int64_t nb = a.n / 3, nslices = (nb + B3C - 1) / B3C;
    DevBuf<int64_t> ent(nslices);
    DevBuf<int> bad(1);
    bad.zero(s);
    k_b3_check<<<blocks_for(nslices * B3C, TH), TH, 0, s>>>(a.ptr.p, a.idx.p, nb, nslices, ent.p,
                                                             bad.p);
    FG_CHECK_LAUNCH();
    if (fetch(bad.p, s)) return false;
    sptr->alloc(nslices + 1);
    exclusive_scan(ent.p, sptr->p, nslices, s);
    const int64_t blocks = fetch(sptr->p + nslices, s);
    col->alloc(blocks);
    val->alloc((size_t)blocks * 9);
    col->zero(s);
    val->zero(s);
    k_b3_fill<T><<<blocks_for(nb, TH), TH, 0, s>>>(a.ptr.p, a.idx.p, a.val.p, nb, sptr->p, col->p,
                                                   val->p);
    FG_CHECK_LAUNCH();
    return true;
}

template <class T>
void reciprocal(int64_t n, const double* d, T* dinv, cudaStream_t s) {
    if (n == 0) return;
    k_reciprocal<T><<<blocks_for(n, TH), TH, 0, s>>>(n, d, dinv);
    FG_CHECK_LAUNCH();
}

template <class T>
void convert_values(int64_t n, const double* a, T* b, cudaStream_t s) {
    if (n == 0) return;
    k_to<T><<<blocks_for(n, TH), TH, 0, s>>>(n, a, b);
    FG_CHECK_LAUNCH();
}

template void fill_offsets<float>(const int64_t*, const uint32_t*, const double*, int64_t, bool,
                                  const int*, const std::vector<int64_t>&, int64_t, float*,
                                  cudaStream_t);
template void fill_offsets<double>(const int64_t*, const uint32_t*, const double*, int64_t, bool,
                                   const int*, const std::vector<int64_t>&, int64_t, double*,
                                   cudaStream_t);
template bool make_bsell3_device<float>(const DevCsr&, DevBuf<int64_t>*, DevBuf<uint32_t>*,
                                        DevBuf<float>*, cudaStream_t);
template bool make_bsell3_device<double>(const DevCsr&, DevBuf<int64_t>*, DevBuf<uint32_t>*,
                                         DevBuf<double>*, cudaStream_t);
template void reciprocal<float>(int64_t, const double*, float*, cudaStream_t);
template void reciprocal<double>(int64_t, const double*, double*, cudaStream_t);
template void convert_values<float>(int64_t, const double*, float*, cudaStream_t);
template void convert_values<double>(int64_t, const double*, double*, cudaStream_t);

}  // namespace femgpu
