// The reactions of a solved elastic model: K u - f at the fixed unknowns, summed per fixed face
// set and per point support, with the force imbalance (elastic::reactions, elastic.rs:772-839,
// called by elastic.rs:585 and elastic_tet.rs:352).
//
// Layout. Only the fixed unknowns matter, a thin boundary layer of the model (config 3 fixes
// 5,043 of 2,022,243 unknowns), so the work is:
//   1. k_fixed_flags + exclusive scan + k_fixed_list: the fixed unknowns in increasing order;
//   2. k_fixed_residual: a thread per fixed unknown forms (K u)_i - f_i, the row's products
//      summed in column order (Csr::mul, sparse.rs:96-105), so r_i has the reference's bits;
//   3. k_reaction_sums: 1 block; each thread owns 1 sum (the gross magnitude, the 3 totals, the 3
//      components of each load) and adds its terms in increasing unknown order, the order of
//      the reference's loop, so every sum has the reference's bits.
// Compiled with -fmad=false: no product is fused into a sum, as in the Rust code.
#include <cmath>

#include "common.cuh"
#include "solver.cuh"

namespace femgpu {
namespace {

constexpr int TH = 256;

__global__ void k_fixed_flags(const uint8_t* __restrict__ fixed, int64_t n,
                              uint32_t* __restrict__ flag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        flag[i] = fixed[i] != 0;
}

__global__ void k_fixed_list(const uint8_t* __restrict__ fixed, const int64_t* __restrict__ at,
                             int64_t n, int64_t* __restrict__ list) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        if (fixed[i]) list[at[i]] = i;
}

// r_k = (K u)_i - f_i for the k-th fixed unknown i.
__global__ void k_fixed_residual(const int64_t* __restrict__ list, int64_t nfixed,
                                 const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                                 const double* __restrict__ val, const double* __restrict__ u,
                                 const double* __restrict__ f, double* __restrict__ r) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nfixed;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = list[k];
        double s = 0.0;
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) s += val[e] * u[idx[e]];
        r[k] = s - f[i];
    }
}

// Sum q < 1 is the gross magnitude, q in 1..3 the total of component q - 1, q >= 4 the
// component (q - 4) % 3 of load (q - 4) / 3. Each walks the fixed unknowns in increasing order.
__global__ void k_reaction_sums(const int64_t* __restrict__ list, const double* __restrict__ r,
                                int64_t nfixed, const uint32_t* __restrict__ owner,
                                int64_t nloads, double gross0, double ax, double ay, double az,
                                double* __restrict__ sums) {
    const int64_t nsums = 4 + 3 * nloads;
    for (int64_t q = threadIdx.x; q < nsums; q += blockDim.x) {
        double acc;
        if (q == 0) {
            acc = gross0;
            for (int64_t k = 0; k < nfixed; ++k) acc += fabs(r[k]);
        } else if (q < 4) {
            const int c = (int)(q - 1);
            acc = c == 0 ? ax : (c == 1 ? ay : az);
            for (int64_t k = 0; k < nfixed; ++k)
                if (list[k] % 3 == c) acc += r[k];
        } else {
            const int64_t load = (q - 4) / 3;
            const int c = (int)((q - 4) % 3);
            acc = 0.0;
            for (int64_t k = 0; k < nfixed; ++k) {
                const int64_t i = list[k];
                if (i % 3 == c && (int64_t)owner[i] == load) acc += r[k];
            }
        }
        sums[q] = acc;
    }
}

}  // namespace

void reactions(const DevCsr& k, const double* u, const double* f, const uint8_t* fixed,
               const uint32_t* owner, int64_t nloads, const double applied[3], double gross0,
               double* load_force, double* total, double* gross, double* imbalance,
               cudaStream_t s) {
    const int64_t n = k.n;
    DevBuf<double> du(n), df(n);
    DevBuf<uint8_t> dfix(n);
    DevBuf<uint32_t> downer(n), flag(n);
    DevBuf<int64_t> at(n + 1);
    FG_CUDA(cudaMemcpyAsync(du.p, u, n * 8, cudaMemcpyHostToDevice, s));
    FG_CUDA(cudaMemcpyAsync(df.p, f, n * 8, cudaMemcpyHostToDevice, s));
    FG_CUDA(cudaMemcpyAsync(dfix.p, fixed, n, cudaMemcpyHostToDevice, s));
    FG_CUDA(cudaMemcpyAsync(downer.p, owner, n * 4, cudaMemcpyHostToDevice, s));
    k_fixed_flags<<<blocks_for(n, TH), TH, 0, s>>>(dfix.p, n, flag.p);
    FG_CHECK_LAUNCH();
    exclusive_scan32(flag.p, at.p, n, s);
    int64_t nfixed = 0;
    FG_CUDA(cudaMemcpyAsync(&nfixed, at.p + n, 8, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    const int64_t nsums = 4 + 3 * nloads;
    DevBuf<double> sums(nsums);
    if (nfixed > 0) {
        DevBuf<int64_t> list(nfixed);
        DevBuf<double> r(nfixed);
        k_fixed_list<<<blocks_for(n, TH), TH, 0, s>>>(dfix.p, at.p, n, list.p);
        k_fixed_residual<<<blocks_for(nfixed, TH), TH, 0, s>>>(list.p, nfixed, k.ptr.p, k.idx.p,
                                                              k.val.p, du.p, df.p, r.p);
        k_reaction_sums<<<1, 1024, 0, s>>>(list.p, r.p, nfixed, downer.p, nloads, gross0,
                                           applied[0], applied[1], applied[2], sums.p);
        FG_CHECK_LAUNCH();
        std::vector<double> h(nsums);
        FG_CUDA(cudaMemcpyAsync(h.data(), sums.p, nsums * 8, cudaMemcpyDeviceToHost, s));
        FG_CUDA(cudaStreamSynchronize(s));
        *gross = h[0];
        for (int c = 0; c < 3; ++c) total[c] = h[1 + c];
        for (int64_t q = 0; q < 3 * nloads; ++q) load_force[q] = h[4 + q];
    } else {
        *gross = gross0;
        for (int c = 0; c < 3; ++c) total[c] = applied[c];
        for (int64_t q = 0; q < 3 * nloads; ++q) load_force[q] = 0.0;
    }
    // elastic.rs:827-831: the largest |total| over the gross forces (f64::max skips a NaN, as
    // fmax does).
    double m = 0.0;
    for (int c = 0; c < 3; ++c) m = std::fmax(m, std::fabs(total[c]));
    *imbalance = *gross > 0.0 ? m / *gross : 0.0;
}

}  // namespace femgpu

extern "C" int femgpu_reactions(const femgpu_csr* k, const double* u, const double* force,
                                const uint8_t* fixed, const uint32_t* owner, size_t nloads,
                                const double* applied, double gross, double* load_force,
                                double* total, double* gross_out, double* imbalance) {
    try {
        if (!k || !u || !force || !fixed || !owner || !applied || !total || !gross_out ||
            !imbalance || (nloads > 0 && !load_force))
            throw femgpu::Failure(FEMGPU_ERR_INVALID, "a null array");
        if (k->m.n % 3 != 0)
            throw femgpu::Failure(FEMGPU_ERR_INVALID, "the matrix is not 3 unknowns per point");
        if (nloads > (size_t)1 << 20)
            throw femgpu::Failure(FEMGPU_ERR_TOO_LARGE, "more than 1048576 loads");
        cudaStream_t s = nullptr;
        FG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            femgpu::reactions(k->m, u, force, fixed, owner, (int64_t)nloads, applied, gross,
                              load_force, total, gross_out, imbalance, s);
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
        return FEMGPU_OK;
    } catch (const femgpu::Failure& e) {
        femgpu::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        femgpu::set_last_error(e.what());
        return FEMGPU_ERR_INVALID;
    }
}
