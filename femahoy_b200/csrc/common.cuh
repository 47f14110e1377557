// Shared definitions of the femgpu CUDA library: status codes, error state, device buffers and
// the launch geometry of the B200 (148 SMs).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "femgpu.h"

namespace femgpu {

// A failure carrying a status code of femgpu.h and the reference's error text.
struct Failure : std::runtime_error {
    int code;
    Failure(int c, const std::string& s) : std::runtime_error(s), code(c) {}
};

void set_last_error(const std::string& s);

#define FG_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            throw ::femgpu::Failure(FEMGPU_ERR_CUDA, std::string("CUDA error: ") +    \
                                                         cudaGetErrorString(e_) +     \
                                                         " at " __FILE__ ":" +        \
                                                         std::to_string(__LINE__));   \
    } while (0)

#define FG_CHECK_LAUNCH() FG_CUDA(cudaGetLastError())

constexpr int NUM_SMS = 148;

inline int blocks_for(int64_t n, int threads, int cap = NUM_SMS * 16) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

// An owned device allocation of `count` elements of T.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t count = 0;
    DevBuf() = default;
    explicit DevBuf(size_t n) { alloc(n); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), count(o.count) {
        o.p = nullptr;
        o.count = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            count = o.count;
            o.p = nullptr;
            o.count = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t n) {
        release();
        count = n;
        if (n) FG_CUDA(cudaMalloc(&p, n * sizeof(T)));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        count = 0;
    }
    size_t bytes() const { return count * sizeof(T); }
    void upload(const T* h, size_t n, cudaStream_t s) {
        if (n > count) alloc(n);
        if (n) FG_CUDA(cudaMemcpyAsync(p, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void download(T* h, size_t n, cudaStream_t s) const {
        if (n) FG_CUDA(cudaMemcpyAsync(h, p, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    std::vector<T> to_host(cudaStream_t s) const {
        std::vector<T> v(count);
        download(v.data(), count, s);
        FG_CUDA(cudaStreamSynchronize(s));
        return v;
    }
    void zero(cudaStream_t s) {
        if (count) FG_CUDA(cudaMemsetAsync(p, 0, bytes(), s));
    }
};

// A device CSR matrix with both triangles, sorted columns (sparse.rs:12-17).
struct DevCsr {
    int64_t n = 0;
    int64_t nnz = 0;
    DevBuf<int64_t> ptr;
    DevBuf<uint32_t> idx;
    DevBuf<double> val;
};

// Exclusive prefix sum of `n` counts into `out` (n + 1 values; out[n] = total), on `s`.
void exclusive_scan(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s);
void exclusive_scan32(const uint32_t* in, int64_t* out, int64_t n, cudaStream_t s);

// Programmatic dependent launch. The kernels of a PCG iteration are launched so that each may
// start while the one before it drains; every such kernel first waits (griddepcontrol.wait) for
// the completion and the memory of the kernel before it, so it reads what it would have read
// without the attribute. On the short kernels of the coarse levels the launch latency this
// hides is most of their time.
// (An explicit early trigger, griddepcontrol.launch_dependents after the wait, measured no
// better on the 128^3 heat solve; the blocks trigger when they exit.)
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
static void launch(bool pdl, void (*kernel)(KArgs...), int grid, int block, cudaStream_t s,
                   Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr{};
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? &attr : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    FG_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

// The same with `smem` bytes of dynamic shared memory.
template <typename... KArgs, typename... Args>
static void launch_smem(bool pdl, void (*kernel)(KArgs...), int grid, int block, size_t smem,
                        cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr{};
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? &attr : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    FG_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

// A scalar from device memory.
template <class T>
T fetch(const T* d, cudaStream_t s) {
    T h;
    FG_CUDA(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    return h;
}

}  // namespace femgpu
