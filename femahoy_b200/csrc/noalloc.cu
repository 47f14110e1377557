// femgpu_reduced_rhs_noalloc: the right side of the free unknowns (heat.rs:1219-1244, steady
// form), for callers that must not allocate device memory.
//
// Who needs it: a caller that shares the GPU with other work in flight, such as a loop serving
// many solves on several streams, cannot afford cudaMalloc/cudaFree, because cudaFree waits for
// the whole device and would stall every other stream; and a caller whose device memory is
// already held by its own pool allocator cannot count on a fresh cudaMalloc succeeding. This
// entry point takes every input and output from the caller, and keeps the one piece of scratch
// it needs (the map from a row to its place in the free list) in a fixed array inside the
// library, so it never allocates.
//
// Limits and sharing: the scratch holds FEMGPU_NOALLOC_MAX_ROWS entries (16 MiB, reserved on
// every GPU that loads the library until the process exits), so the matrix may have at most
// that many rows. All calls share the array and it keeps the last call's contents; each call
// clears what it uses first. Calls whose work overlaps on the GPU (from several host threads,
// or on several streams without ordering between them) race on the array and must not be made.
// Each call waits for its own stream before it returns (to read its argument checks), so it
// cannot be made while that stream is being captured into a CUDA graph.
//
// Compiled with -fmad=false, like the assembly, so its sums equal the reference's bit for bit.
#include <mutex>

#include "common.cuh"

namespace femgpu {
namespace {

// The scratch: for each row, its place in the free list, or 0xffffffff for a fixed row. The
// last entry past the rows is not used; a separate word holds the argument-check flag.
static __device__ __align__(256) uint32_t g_noalloc_place[FEMGPU_NOALLOC_MAX_ROWS];
static __device__ __align__(256) int g_noalloc_bad;

// The device addresses of the 2 arrays for each device, found once per device with that device
// current. In host code the names above are host-side stand-ins, not device addresses.
struct Symbols {
    uint32_t* place = nullptr;
    int* bad = nullptr;
};
constexpr int MAX_DEVICES = 64;
Symbols g_symbols[MAX_DEVICES];
std::once_flag g_once[MAX_DEVICES];
cudaError_t g_symbol_error[MAX_DEVICES];

// The argument checks, 1 bit each in the flag word (several may be set at once).
constexpr int BAD_ROW = 1;         // a free row outside 0..n
constexpr int BAD_TWICE = 2;       // a free row listed twice
constexpr int BAD_ORDER = 4;       // the free rows not increasing
constexpr int BAD_COLUMN = 8;      // a column index of a free row outside 0..n

__global__ void k_noalloc_mark(const int64_t* __restrict__ free, int64_t nfree, int64_t n,
                               uint32_t* __restrict__ place, int* __restrict__ bad) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nfree;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = free[k];
        if (k > 0 && free[k - 1] >= i) atomicOr(bad, BAD_ORDER);
        if (i < 0 || i >= n) {
            atomicOr(bad, BAD_ROW);
            continue;
        }
        if (atomicExch(&place[i], (uint32_t)k) != 0xffffffffu) atomicOr(bad, BAD_TWICE);
    }
}

// r_k = load_i - sum over the fixed columns j of row i (in the row's order) of a_ij t_j, for the
// free row i = free[k]: the same expression and order as the allocating entry point. A row or a
// column outside 0..n is flagged and not read.
__global__ void k_noalloc_rhs(const int64_t* __restrict__ free, int64_t nfree, int64_t n,
                              const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                              const double* __restrict__ val, const uint32_t* __restrict__ place,
                              const double* __restrict__ load, const double* __restrict__ t,
                              double* __restrict__ out, int* __restrict__ bad) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nfree;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = free[k];
        if (i < 0 || i >= n) continue;
        double r = load[i];
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) {
            uint32_t j = idx[e];
            if (j >= n) {
                atomicOr(bad, BAD_COLUMN);
                continue;
            }
            if (place[j] == 0xffffffffu) r -= val[e] * t[j];
        }
        out[k] = r;
    }
}

// The device addresses of the scratch for the current device (set up on its first use).
Symbols symbols_for_current_device() {
    int dev = 0;
    FG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES)
        throw Failure(FEMGPU_ERR_INVALID, "device ordinal past the library's table");
    std::call_once(g_once[dev], [dev] {
        Symbols s;
        cudaError_t e = cudaGetSymbolAddress((void**)&s.place, g_noalloc_place);
        if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&s.bad, g_noalloc_bad);
        g_symbol_error[dev] = e;
        if (e == cudaSuccess) g_symbols[dev] = s;
    });
    if (g_symbol_error[dev] != cudaSuccess)
        throw Failure(FEMGPU_ERR_CUDA, std::string("cudaGetSymbolAddress failed: ") +
                                           cudaGetErrorString(g_symbol_error[dev]));
    return g_symbols[dev];
}

}  // namespace

void reduced_rhs_noalloc(int64_t n, const int64_t* ptr, const uint32_t* idx, const double* val,
                         const double* load, const double* t, const int64_t* free, int64_t nfree,
                         double* out, cudaStream_t s) {
    if (n < 0 || n > (int64_t)FEMGPU_NOALLOC_MAX_ROWS)
        throw Failure(FEMGPU_ERR_TOO_LARGE,
                      "femgpu_reduced_rhs_noalloc takes at most FEMGPU_NOALLOC_MAX_ROWS "
                      "(4194304) rows: its scratch is a fixed array");
    if (nfree < 0 || nfree > n) throw Failure(FEMGPU_ERR_INVALID, "more free rows than rows");
    if (n == 0 || nfree == 0) return;
    Symbols sym = symbols_for_current_device();
    FG_CUDA(cudaMemsetAsync(sym.place, 0xff, (size_t)n * sizeof(uint32_t), s));
    FG_CUDA(cudaMemsetAsync(sym.bad, 0, sizeof(int), s));
    int blocks = blocks_for(nfree, 256);
    k_noalloc_mark<<<blocks, 256, 0, s>>>(free, nfree, n, sym.place, sym.bad);
    k_noalloc_rhs<<<blocks, 256, 0, s>>>(free, nfree, n, ptr, idx, val, sym.place, load, t, out,
                                         sym.bad);
    FG_CHECK_LAUNCH();
    // 1 wait per call, for the argument checks of both kernels.
    int bad = 0;
    FG_CUDA(cudaMemcpyAsync(&bad, sym.bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    if (bad & BAD_ROW) throw Failure(FEMGPU_ERR_INVALID, "a free row is out of range");
    if (bad & BAD_TWICE) throw Failure(FEMGPU_ERR_INVALID, "the free rows hold a row twice");
    if (bad & BAD_ORDER) throw Failure(FEMGPU_ERR_INVALID, "the free rows are not increasing");
    if (bad & BAD_COLUMN)
        throw Failure(FEMGPU_ERR_INVALID, "a column index of a free row is out of range");
}

}  // namespace femgpu

extern "C" int femgpu_reduced_rhs_noalloc(size_t n, const int64_t* ptr, const uint32_t* idx,
                                          const double* val, const double* load, const double* t,
                                          const int64_t* free, size_t nfree, double* out,
                                          void* stream) {
    try {
        if (!ptr || !idx || !val || !load || !t || !free || !out)
            throw femgpu::Failure(FEMGPU_ERR_INVALID, "a null device array");
        femgpu::reduced_rhs_noalloc((int64_t)n, ptr, idx, val, load, t, free, (int64_t)nfree, out,
                                    (cudaStream_t)stream);
        return FEMGPU_OK;
    } catch (const femgpu::Failure& e) {
        femgpu::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        femgpu::set_last_error(e.what());
        return FEMGPU_ERR_INVALID;
    }
}
