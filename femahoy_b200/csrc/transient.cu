// The transient heat loop on the device: backward Euler with the lumped capacity, the loop of
// heat.rs:686-733. Per step: the right side of the free points (heat::reduced_rhs with the
// capacity term, heat.rs:1219-1244), 1 solve of (K + C/dt) on the free unknowns warm-started
// from the last temperatures, the temperatures of the free points, K T, the rates
// C (T - T_prev) / dt and the energy sums of heat.rs:535-547. The matrix, its solver (the
// multigrid hierarchy or the dense factor) and all vectors stay on the device for the whole run;
// only the temperatures of the output steps and their 3 energy sums come back.
//
// Built with -fmad=false: the right side, K + C/dt and the rates keep the reference's separate
// roundings, bit for bit.
#include <cmath>
#include <memory>
#include <vector>

#include "assemble.cuh"
#include "common.cuh"
#include "solver.cuh"

namespace femgpu {

constexpr int TT = 256;

// heat.rs:691-696: a_full.val[diagonal] += capacity[i] / dt. Flag 1: a row without a diagonal.
__global__ void k_add_capacity(int64_t n, const int64_t* __restrict__ ptr,
                               const uint32_t* __restrict__ idx, double* __restrict__ val,
                               const double* __restrict__ cap, double dt, int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = ptr[i], hi = ptr[i + 1];
        while (lo < hi) {  // the columns of a row are sorted
            int64_t mid = (lo + hi) / 2;
            if (idx[mid] < (uint32_t)i)
                lo = mid + 1;
            else
                hi = mid;
        }
        if (lo < ptr[i + 1] && idx[lo] == (uint32_t)i)
            val[lo] += cap[i] / dt;
        else
            atomicExch(bad, 1);
    }
}

// heat.rs:1219-1244 with Some((capacity, dt)): load + C/dt T minus the fixed columns of A T, in
// the row's column order.
__global__ void k_transient_rhs(int64_t nfree, const int64_t* __restrict__ free,
                                const int64_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                                const double* __restrict__ val, const uint8_t* __restrict__ isfree,
                                const double* __restrict__ load, const double* __restrict__ t,
                                const double* __restrict__ cap, double dt,
                                double* __restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nfree;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = free[k];
        double r = load[i];
        r += cap[i] / dt * t[i];
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) {
            const uint32_t j = idx[e];
            if (!isfree[j]) r -= val[e] * t[j];
        }
        out[k] = r;
    }
}

__global__ void k_take_free(int64_t nfree, const int64_t* __restrict__ free,
                            const double* __restrict__ t, double* __restrict__ x) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nfree;
         k += (int64_t)gridDim.x * blockDim.x)
        x[k] = t[free[k]];
}

__global__ void k_put_free(int64_t nfree, const int64_t* __restrict__ free,
                           const double* __restrict__ x, double* __restrict__ t) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nfree;
         k += (int64_t)gridDim.x * blockDim.x)
        t[free[k]] = x[k];
}

// The rates C (T - T_prev) / dt (heat.rs:726-728) and, per block, the partial sums of
// heat.rs:535-547 with no radiation: stored = sum rate, fixed = sum over the fixed points of
// q = K T + rate - load, and the sum of |rate| and |q|. 1 point per thread, 1 grid pass.
__global__ void __launch_bounds__(TT)
    k_rate_energy(int64_t n, const double* __restrict__ cap, const double* __restrict__ t,
                  const double* __restrict__ prev, double dt, const double* __restrict__ kt,
                  const double* __restrict__ load, const uint8_t* __restrict__ isfree,
                  double* __restrict__ rate, double* __restrict__ partial) {
    double s = 0.0, f = 0.0, g = 0.0;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) {
        const double r = cap[i] * (t[i] - prev[i]) / dt;
        rate[i] = r;
        s = r;
        g = fabs(r);
        if (!isfree[i]) {
            const double q = kt[i] + r - load[i] - 0.0;
            f = q;
            g += fabs(q);
        }
    }
    __shared__ double sh[3][TT / 32];
    for (int o = 16; o; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        f += __shfl_xor_sync(0xffffffffu, f, o);
        g += __shfl_xor_sync(0xffffffffu, g, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][w] = s;
        sh[1][w] = f;
        sh[2][w] = g;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0, c = 0.0;
        for (int k = 0; k < TT / 32; ++k) {
            a += sh[0][k];
            b += sh[1][k];
            c += sh[2][k];
        }
        partial[3 * blockIdx.x] = a;
        partial[3 * blockIdx.x + 1] = b;
        partial[3 * blockIdx.x + 2] = c;
    }
}

// The block partials summed in block order by 1 thread (a deterministic result).
__global__ void k_energy_total(const double* __restrict__ partial, int64_t nblocks,
                               double* __restrict__ out) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int64_t k = 0; k < nblocks; ++k) {
        a += partial[3 * k];
        b += partial[3 * k + 1];
        c += partial[3 * k + 2];
    }
    out[0] = a;
    out[1] = b;
    out[2] = c;
}

}  // namespace femgpu

using namespace femgpu;

struct femgpu_transient {
    femgpu_solver* solver = nullptr;
    int64_t n = 0, nfree = 0;
    double dt = 0.0;
    DevCsr k;      // the conductivity matrix: K T for the energy
    DevCsr afull;  // K + C/dt: the fixed columns of the right side
    DevBuf<double> cap, load, t, prev, rhs, x, kt, rate, partial, energy;
    DevBuf<int64_t> free;
    DevBuf<uint8_t> isfree;
    ~femgpu_transient() {
        if (solver) femgpu_solver_free(solver);
    }
};

namespace {
template <class F>
int transient_guarded(F f) {
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

void copy_csr(const DevCsr& a, DevCsr* out, cudaStream_t s) {
    out->n = a.n;
    out->nnz = a.nnz;
    out->ptr.alloc(a.n + 1);
    out->idx.alloc(a.nnz);
    out->val.alloc(a.nnz);
    FG_CUDA(cudaMemcpyAsync(out->ptr.p, a.ptr.p, out->ptr.bytes(), cudaMemcpyDeviceToDevice, s));
    FG_CUDA(cudaMemcpyAsync(out->idx.p, a.idx.p, out->idx.bytes(), cudaMemcpyDeviceToDevice, s));
    FG_CUDA(cudaMemcpyAsync(out->val.p, a.val.p, out->val.bytes(), cudaMemcpyDeviceToDevice, s));
}
}  // namespace

extern "C" {

int femgpu_transient_new(const femgpu_csr* k, const double* capacity, double dt,
                         const int64_t* free, size_t nfree, const femgpu_unknowns* unknowns,
                         int method, const femgpu_crossover* crossover,
                         const femgpu_options* options, femgpu_transient** out) {
    return transient_guarded([&] {
        need(k && capacity && free && unknowns && out, "null argument");
        need(std::isfinite(dt) && dt > 0.0, "the time step must be above 0");
        const int64_t n = k->m.n;
        need(nfree > 0 && (int64_t)nfree <= n, "the free points must be 1 to n");
        for (size_t q = 0; q < nfree; ++q) {
            need(free[q] >= 0 && free[q] < n, "a free point past the last");
            need(q == 0 || free[q] > free[q - 1], "the free points must increase");
        }
        auto tr = std::make_unique<femgpu_transient>();
        tr->n = n;
        tr->nfree = (int64_t)nfree;
        tr->dt = dt;
        cudaStream_t s = nullptr;  // setup on the legacy stream, synchronized before the solver
        copy_csr(k->m, &tr->k, s);
        copy_csr(k->m, &tr->afull, s);
        tr->cap.upload(capacity, n, s);
        tr->free.upload(free, nfree, s);
        std::vector<uint8_t> mark(n, 0);
        for (size_t q = 0; q < nfree; ++q) mark[free[q]] = 1;
        tr->isfree.upload(mark.data(), n, s);
        DevBuf<int> bad(1);
        bad.zero(s);
        k_add_capacity<<<blocks_for(n, TT), TT, 0, s>>>(n, tr->afull.ptr.p, tr->afull.idx.p,
                                                        tr->afull.val.p, tr->cap.p, dt, bad.p);
        FG_CHECK_LAUNCH();
        if (fetch(bad.p, s)) throw Failure(FEMGPU_ERR_INVALID, "a diagonal");
        femgpu_csr sub;
        submatrix(tr->afull, tr->free.p, tr->nfree, &sub.m, s);
        FG_CUDA(cudaStreamSynchronize(s));
        // heat.rs:697-703: Crossover::Unknowns(TRANSIENT_DIRECT_LIMIT), 40,000 in the reference;
        // the direct solver of this library holds at most 16,384 unknowns.
        femgpu_crossover c{0, 40000, 0.0, 0, 0};  // TRANSIENT_DIRECT_LIMIT, solve.rs:24
        if (crossover) c = *crossover;
        int rc = femgpu_solver_new(&sub, unknowns, method, &c, options, &tr->solver);
        if (rc != FEMGPU_OK) {
            char buf[1024];
            femgpu_last_error(buf, sizeof buf);
            throw Failure(rc, buf);
        }
        const int64_t nb = (n + TT - 1) / TT;
        tr->load.alloc(n);
        tr->t.alloc(n);
        tr->prev.alloc(n);
        tr->kt.alloc(n);
        tr->rate.alloc(n);
        tr->rhs.alloc(nfree);
        tr->x.alloc(nfree);
        tr->partial.alloc(3 * nb);
        tr->energy.alloc(3);
        *out = tr.release();
    });
}

femgpu_solver* femgpu_transient_solver(femgpu_transient* tr) { return tr ? tr->solver : nullptr; }

int femgpu_transient_run(femgpu_transient* tr, size_t steps, const double* load,
                         double* temperature, size_t output_every, double* frames,
                         femgpu_energy* energies, const volatile int* cancel,
                         femgpu_stats* stats) {
    return transient_guarded([&] {
        need(tr && load && temperature, "null argument");
        SolverImpl& sv = tr->solver->impl;
        cudaStream_t s = sv.stream();
        const int64_t n = tr->n, nf = tr->nfree;
        const int64_t nb = (n + TT - 1) / TT;
        const int gf = blocks_for(nf, TT), gn = blocks_for(n, TT);
        const size_t every = output_every ? output_every : 1;
        femgpu_stats total{};
        tr->load.upload(load, n, s);
        tr->t.upload(temperature, n, s);
        k_take_free<<<gf, TT, 0, s>>>(nf, tr->free.p, tr->t.p, tr->x.p);
        FG_CHECK_LAUNCH();
        size_t frame = 0;
        for (size_t step = 1; step <= steps; ++step) {
            if (cancel && *cancel) throw Failure(FEMGPU_ERR_CANCELLED, "cancelled");
            FG_CUDA(cudaMemcpyAsync(tr->prev.p, tr->t.p, n * 8, cudaMemcpyDeviceToDevice, s));
            k_transient_rhs<<<gf, TT, 0, s>>>(nf, tr->free.p, tr->afull.ptr.p, tr->afull.idx.p,
                                               tr->afull.val.p, tr->isfree.p, tr->load.p,
                                               tr->t.p, tr->cap.p, tr->dt, tr->rhs.p);
            FG_CHECK_LAUNCH();
            femgpu_stats st{};
            sv.solve(tr->rhs.p, tr->x.p, cancel, &st);
            total.iterations += st.iterations;
            total.residual = st.residual;
            total.true_residual = std::max(total.true_residual, st.true_residual);
            total.seconds += st.seconds;
            total.launches += st.launches + 4;
            k_put_free<<<gf, TT, 0, s>>>(nf, tr->free.p, tr->x.p, tr->t.p);
            FG_CHECK_LAUNCH();
            if (step % every != 0 && step != steps) continue;
            // K T (Csr::mul, heat.rs:725), the rates and the energy sums of this output step.
            csr_mul(tr->k, tr->t.p, tr->kt.p, s);
            k_rate_energy<<<(int)nb, TT, 0, s>>>(n, tr->cap.p, tr->t.p, tr->prev.p, tr->dt,
                                                 tr->kt.p, tr->load.p, tr->isfree.p, tr->rate.p,
                                                 tr->partial.p);
            k_energy_total<<<1, 1, 0, s>>>(tr->partial.p, nb, tr->energy.p);
            FG_CHECK_LAUNCH();
            total.launches += 3;
            if (frames) tr->t.download(frames + frame * (size_t)n, n, s);
            if (energies) {
                double e[3];
                tr->energy.download(e, 3, s);
                FG_CUDA(cudaStreamSynchronize(s));
                energies[frame] = femgpu_energy{e[0], e[1], e[2]};
            }
            ++frame;
        }
        tr->t.download(temperature, n, s);
        FG_CUDA(cudaStreamSynchronize(s));
        if (stats) *stats = total;
    });
}

void femgpu_transient_free(femgpu_transient* tr) { delete tr; }

}  // extern "C"
