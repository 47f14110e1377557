// Post-solve recovery of the 10-node tetrahedra on the device: the loop of
// elastic_tet.rs:367-427 (the strain and the stress at the 10 points of each cell, their mean at
// each point, the peak von Mises stress of each part) and the von Mises and principal stresses of
// the means (elastic_tet.rs:482-483).
//
// Layout in HBM. Setup writes one 224-byte record per cell: the gradients of its 4 volume
// coordinates (tet_gradients, heat.rs:983-1002), its stiffness D (hex.rs:58-114) and D alpha
// (elastic_tet.rs:164-170). The incidence of the assembly lists the cells of each point in
// increasing order. A recovery is one thread per point: it walks its cells in that order,
// evaluates Tet10::strain_stress (tet10.rs:142-169) at its own volume coordinates in each, and
// sums. The reference adds the same terms to the same point in the same order, so the means
// are bit-identical with it. Each (cell, point) pair is evaluated exactly once, by the thread of
// its point. The unit is compiled with -fmad=false, so no multiply and add are fused.
//
// Peaks: the thread that evaluates pair (cell e, point c) writes its von Mises stress to
// vm[10 e + c]. Each block reduces a contiguous range of pairs per part in shared memory, then
// 1 thread per part combines the blocks: the largest value, and among equal values the smallest
// index, which is the first in the reference's (cell, point) order. Maximum and minimum are
// exact, so no order of the reduction changes the result.
#include <cmath>
#include <cstring>
#include <memory>

#include "assemble.cuh"
#include "common.cuh"
#include "elements.cuh"

namespace femgpu {

// One cell's constants: 27 values and a pad, 224 bytes (7 sectors of 32 bytes).
struct CellRecord {
    double g[4][3];
    double normal[3][3];
    double shear[3];
    double thermal[3];
    double pad;
};
static_assert(sizeof(CellRecord) == 224, "the cell record is 224 bytes");

constexpr int MAX_PARTS = 2048;
constexpr int PEAK_THREADS = 256;
constexpr int PEAK_BLOCKS = 2 * NUM_SMS;
constexpr uint64_t NONE = ~0ull;
constexpr uint32_t NEAR_BIT = 0x80000000u;

struct PeakPartial {
    uint64_t max_all, key_all, max_reg, key_reg, first_reg;
};

// tet10.rs:38, packed 4 bits per edge: the first and the second corner of edge k.
constexpr uint32_t EDGE_FIRST = 0x210010u;   // 0, 1, 0, 0, 1, 2
constexpr uint32_t EDGE_SECOND = 0x333221u;  // 1, 2, 2, 3, 3, 3

__device__ __forceinline__ bool is_nan_bits(uint64_t b) {
    return (b & 0x7fffffffffffffffull) > 0x7ff0000000000000ull;
}

// elastic.rs:977-983
__device__ __forceinline__ double mises6(const double s[6]) {
    double a = s[0] - s[1], b = s[1] - s[2], c = s[2] - s[0];
    return sqrt(0.5 * (a * a + b * b + c * c) + 3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

// elastic.rs:985-1002 (O. K. Smith, Comm. ACM 4 (1961) 168), largest first.
__device__ __forceinline__ void principal3(const double s[6], double out[3]) {
    double xx = s[0], yy = s[1], zz = s[2], xy = s[3], yz = s[4], xz = s[5];
    double q = (xx + yy + zz) / 3.0;
    double p1 = xy * xy + yz * yz + xz * xz;
    double p2 = (xx - q) * (xx - q) + (yy - q) * (yy - q) + (zz - q) * (zz - q) + 2.0 * p1;
    double p = sqrt(p2 / 6.0);
    if (p == 0.0) {
        out[0] = out[1] = out[2] = q;
        return;
    }
    double a = (xx - q) / p, b = (yy - q) / p, c = (zz - q) / p;
    double d = xy / p, e = yz / p, f = xz / p;
    double det = a * (b * c - e * e) - d * (d * c - e * f) + f * (d * e - b * f);
    double h = det / 2.0;
    if (h < -1.0) h = -1.0;  // f64::clamp, which keeps a NaN
    if (h > 1.0) h = 1.0;
    double phi = acos(h) / 3.0;
    const double pi = 3.141592653589793;
    double s1 = q + 2.0 * p * cos(phi);
    double s3 = q + 2.0 * p * cos(phi + 2.0 * pi / 3.0);
    out[0] = s1;
    out[1] = 3.0 * q - s1 - s3;
    out[2] = s3;
}

// Setup: the record, and the part and the `near` flag of each cell (a corner is singular:
// elastic_tet.rs:395). Flags: 2 no stable material, 3 a part past the last.
__global__ void k_recover_cells(const double* __restrict__ xyz, const uint32_t* __restrict__ t10,
                                const double* __restrict__ coef,
                                const double* __restrict__ expansion,
                                const uint32_t* __restrict__ part, uint32_t nparts,
                                const uint8_t* __restrict__ singular, int64_t nel,
                                CellRecord* __restrict__ rec, uint32_t* __restrict__ tag,
                                int* __restrict__ bad) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t* t = t10 + 10 * e;
        double p[4][3];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int d = 0; d < 3; ++d) p[k][d] = xyz[3 * (int64_t)t[k] + d];
        CellRecord r;
        double volume;
        tet_gradients(p, r.g, &volume);
        Stiffness D;
        if (!isotropic_stiffness(coef[2 * e], coef[2 * e + 1], &D)) atomicExch(bad, 2);
        double alpha[3] = {0.0, 0.0, 0.0};
        if (expansion)
#pragma unroll
            for (int k = 0; k < 3; ++k) alpha[k] = expansion[3 * e + k];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double s = -0.0;  // the Rust float sum starts from -0.0
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                r.normal[i][j] = D.normal[i][j];
                s += D.normal[i][j] * alpha[j];
            }
            r.thermal[i] = s;
            r.shear[i] = D.shear[i];
        }
        r.pad = 0.0;
        rec[e] = r;
        uint32_t pt = part ? part[e] : 0u;
        if (pt >= nparts) atomicExch(bad, 3);
        bool near = false;
        if (singular)
#pragma unroll
            for (int k = 0; k < 4; ++k) near = near || singular[t[k]] != 0;
        tag[e] = (pt & ~NEAR_BIT) | (near ? NEAR_BIT : 0u);
    }
}

// Tet10::strain_stress (tet10.rs:142-169) of cell `r` at its point c, followed by reorder and
// tensor_strain (elastic.rs:967-975): sig and eps in the order xx, yy, zz, xy, yz, xz.
__device__ __forceinline__ void strain_stress_at(const CellRecord* __restrict__ rp,
                                                 const uint32_t* __restrict__ t, int c,
                                                 const double* __restrict__ u,
                                                 const double* __restrict__ dtemp,
                                                 double sig[6], double eps[6]) {
    const double2* r2 = reinterpret_cast<const double2*>(rp);
    double w[28];
#pragma unroll
    for (int k = 0; k < 14; ++k) {
        double2 v = __ldg(r2 + k);
        w[2 * k] = v.x;
        w[2 * k + 1] = v.y;
    }
    // w[0..12) g, w[12..21) normal, w[21..24) shear, w[24..27) thermal.
    double l[4] = {0.0, 0.0, 0.0, 0.0};  // node_coordinates (tet10.rs:216-228)
    if (c < 4) {
        l[0] = c == 0 ? 1.0 : 0.0;
        l[1] = c == 1 ? 1.0 : 0.0;
        l[2] = c == 2 ? 1.0 : 0.0;
        l[3] = c == 3 ? 1.0 : 0.0;
    } else {
        int i = (EDGE_FIRST >> (4 * (c - 4))) & 0xf, j = (EDGE_SECOND >> (4 * (c - 4))) & 0xf;
#pragma unroll
        for (int k = 0; k < 4; ++k) l[k] = (k == i || k == j) ? 0.5 : 0.0;
    }
    double e[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 10; ++i) {
        // The gradient of function i at l (tet10.rs:77-87).
        double gi[3];
        if (i < 4) {
#pragma unroll
            for (int d = 0; d < 3; ++d) gi[d] = (4.0 * l[i] - 1.0) * w[3 * i + d];
        } else {
            const int a = kEdges[i - 4][0], b = kEdges[i - 4][1];
#pragma unroll
            for (int d = 0; d < 3; ++d) gi[d] = 4.0 * (l[a] * w[3 * b + d] + l[b] * w[3 * a + d]);
        }
        const int64_t base = 3 * (int64_t)t[i];
        double ui[3] = {u[base], u[base + 1], u[base + 2]};
#pragma unroll
        for (int a = 0; a < 3; ++a) e[a] += gi[a] * ui[a];
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const int a = kShear[s][0], b = kShear[s][1];
            e[3 + s] += gi[a] * ui[b] + gi[b] * ui[a];
        }
    }
    double dt = -0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) dt += l[k] * (dtemp ? dtemp[t[k]] : 0.0);
    double s[6];
#pragma unroll
    for (int a = 0; a < 3; ++a)  // hex.rs:128-139
        s[a] = w[12 + 3 * a] * e[0] + w[12 + 3 * a + 1] * e[1] + w[12 + 3 * a + 2] * e[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) s[3 + k] = w[21 + k] * e[3 + k];
#pragma unroll
    for (int a = 0; a < 3; ++a) s[a] -= w[24 + a] * dt;
    sig[0] = s[0];
    sig[1] = s[1];
    sig[2] = s[2];
    sig[3] = s[5];
    sig[4] = s[3];
    sig[5] = s[4];
    eps[0] = e[0];
    eps[1] = e[1];
    eps[2] = e[2];
    eps[3] = 0.5 * e[5];
    eps[4] = 0.5 * e[3];
    eps[5] = 0.5 * e[4];
}

// One thread per point: the sums of elastic_tet.rs:396-403 over the point's cells in
// increasing order, the means of elastic_tet.rs:419-425, and elastic_tet.rs:482-483.
template <bool PEAKS>
__global__ void __launch_bounds__(128)
    k_recover_points(const CellRecord* __restrict__ rec, const uint32_t* __restrict__ t10,
                     const int64_t* __restrict__ start, const uint32_t* __restrict__ of_node,
                     const double* __restrict__ u, const double* __restrict__ dtemp,
                     int64_t npoints, double* __restrict__ stress, double* __restrict__ strain,
                     double* __restrict__ mises_out, double* __restrict__ principal_out,
                     double* __restrict__ vm) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < npoints;
         v += (int64_t)gridDim.x * blockDim.x) {
        double ss[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        double se[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        const int64_t b = start[v], end = start[v + 1];
        uint32_t last = 0xffffffffu;
        int lastc = -1;
        for (int64_t k = b; k < end; ++k) {
            const uint32_t e = of_node[k];
            const uint32_t* t = t10 + 10 * (int64_t)e;
            // The point's place in the cell; a cell that names the point twice is listed twice
            // and takes its places in order, as the reference's loop over c.
            int c = e == last ? lastc + 1 : 0;
            while (c < 10 && t[c] != (uint32_t)v) ++c;
            if (c >= 10) continue;  // not reached: the incidence lists exactly these places
            last = e;
            lastc = c;
            double sig[6], eps[6];
            strain_stress_at(rec + e, t, c, u, dtemp, sig, eps);
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                ss[i] += sig[i];
                se[i] += eps[i];
            }
            if (PEAKS) vm[10 * (int64_t)e + c] = mises6(sig);
        }
        int64_t count = end - b;
        const double cnt = (double)(count > 1 ? count : 1);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            ss[i] /= cnt;
            se[i] /= cnt;
            stress[6 * v + i] = ss[i];
            strain[6 * v + i] = se[i];
        }
        if (mises_out) mises_out[v] = mises6(ss);
        if (principal_out) {
            double pr[3];
            principal3(ss, pr);
#pragma unroll
            for (int i = 0; i < 3; ++i) principal_out[3 * v + i] = pr[i];
        }
    }
}

// Each block: the pairs [10 e0, 10 e1) of its range of cells, per part in shared memory
// (5 x nparts words). Pass A takes the maxima and the first regular pair; pass B the smallest
// pair index at each maximum.
__global__ void __launch_bounds__(PEAK_THREADS)
    k_peak_blocks(const double* __restrict__ vm, const uint32_t* __restrict__ tag,
                  const uint32_t* __restrict__ t10, const uint8_t* __restrict__ singular,
                  int64_t nel, int nparts, int64_t chunk, PeakPartial* __restrict__ partial) {
    extern __shared__ unsigned long long sm[];
    unsigned long long* mall = sm;
    unsigned long long* kall = sm + nparts;
    unsigned long long* mreg = sm + 2 * nparts;
    unsigned long long* kreg = sm + 3 * nparts;
    unsigned long long* freg = sm + 4 * nparts;
    for (int p = threadIdx.x; p < nparts; p += blockDim.x) {
        mall[p] = 0;
        mreg[p] = 0;
        kall[p] = NONE;
        kreg[p] = NONE;
        freg[p] = NONE;
    }
    __syncthreads();
    const int64_t e0 = blockIdx.x * chunk;
    const int64_t e1 = e0 + chunk < nel ? e0 + chunk : nel;
    for (int pass = 0; pass < 2; ++pass) {
        for (int64_t i = 10 * e0 + threadIdx.x; i < 10 * e1; i += blockDim.x) {
            const uint32_t tg = tag[i / 10];
            const int p = (int)(tg & ~NEAR_BIT);
            const bool reg = !(tg & NEAR_BIT) && !(singular && singular[t10[i]]);
            const unsigned long long bits = (unsigned long long)__double_as_longlong(vm[i]);
            const bool nan = is_nan_bits(bits);
            if (pass == 0) {
                if (!nan) atomicMax(&mall[p], bits);
                if (reg) {
                    if (!nan) atomicMax(&mreg[p], bits);
                    atomicMin(&freg[p], (unsigned long long)i);
                }
            } else if (!nan) {
                if (bits == mall[p]) atomicMin(&kall[p], (unsigned long long)i);
                if (reg && bits == mreg[p]) atomicMin(&kreg[p], (unsigned long long)i);
            }
        }
        __syncthreads();
    }
    for (int p = threadIdx.x; p < nparts; p += blockDim.x)
        partial[(int64_t)blockIdx.x * nparts + p] =
            PeakPartial{mall[p], kall[p], mreg[p], kreg[p], freg[p]};
}

__device__ __forceinline__ void combine(uint64_t m, uint64_t k, uint64_t* bm, uint64_t* bk) {
    if (k == NONE) return;
    if (*bk == NONE || m > *bm || (m == *bm && k < *bk)) {
        *bm = m;
        *bk = k;
    }
}

// 1 thread per part: the blocks combined, and the reference's Peak (elastic_tet.rs:405-416):
// the first regular pair stays the regular peak when its value is NaN, since no value is
// greater than NaN.
__global__ void k_peak_final(const PeakPartial* __restrict__ partial, int nblocks, int nparts,
                             const double* __restrict__ vm, const uint32_t* __restrict__ t10,
                             const uint32_t* __restrict__ tag,
                             const uint8_t* __restrict__ singular, femgpu_peak* __restrict__ out) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nparts) return;
    uint64_t mall = 0, kall = NONE, mreg = 0, kreg = NONE, freg = NONE;
    for (int b = 0; b < nblocks; ++b) {
        const PeakPartial q = partial[(int64_t)b * nparts + p];
        combine(q.max_all, q.key_all, &mall, &kall);
        combine(q.max_reg, q.key_reg, &mreg, &kreg);
        if (q.first_reg < freg) freg = q.first_reg;
    }
    femgpu_peak o;
    memset(&o, 0, sizeof(o));
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    if (kall == NONE) {
        o.mises = -inf;
        o.element = -1;
    } else {
        o.mises = __longlong_as_double((long long)mall);
        o.element = (int64_t)(kall / 10);
        o.local = (int32_t)(kall % 10);
        o.point = t10[kall];
        o.singular = ((tag[kall / 10] & NEAR_BIT) || (singular && singular[o.point])) ? 1 : 0;
    }
    uint64_t rk = NONE;
    double rm = -inf;
    if (freg != NONE) {
        const uint64_t fb = (uint64_t)__double_as_longlong(vm[freg]);
        if (is_nan_bits(fb)) {
            rk = freg;
            rm = vm[freg];
        } else {
            rk = kreg;
            rm = __longlong_as_double((long long)mreg);
        }
    }
    if (rk == NONE) {
        o.regular_mises = -inf;
        o.regular_element = -1;
    } else {
        o.regular_mises = rm;
        o.regular_element = (int64_t)(rk / 10);
        o.regular_local = (int32_t)(rk % 10);
        o.regular_point = t10[rk];
    }
    out[p] = o;
}

}  // namespace femgpu

using namespace femgpu;

struct femgpu_recovery {
    int64_t npoints = 0, nel = 0;
    int nparts = 1;
    bool has_singular = false;
    Incidence inc;
    DevBuf<uint32_t> t10;
    DevBuf<CellRecord> rec;
    DevBuf<uint32_t> tag;
    DevBuf<uint8_t> singular;
    DevBuf<double> vm;
    DevBuf<PeakPartial> partial;
    DevBuf<femgpu_peak> dpeaks;
    int peak_blocks = 1;
    int64_t chunk = 1;
    // Device copies for the host-pointer form.
    DevBuf<double> du, ddt, dstress, dstrain, dmises, dprincipal;
    cudaStream_t s = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0, last_bytes = 0.0;
    ~femgpu_recovery() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (s) cudaStreamDestroy(s);
    }

    void run(const double* u, const double* dtemp, double* stress, double* strain,
             double* mises, double* principal, femgpu_peak* peaks) {
        const bool want_peaks = peaks != nullptr;
        if (want_peaks && vm.count < (size_t)(10 * nel)) vm.alloc(10 * nel);
        FG_CUDA(cudaEventRecord(ev0, s));
        const int grid = blocks_for(npoints, 128, NUM_SMS * 64);
        if (want_peaks)
            k_recover_points<true><<<grid, 128, 0, s>>>(rec.p, t10.p, inc.start.p, inc.of_node.p,
                                                        u, dtemp, npoints, stress, strain, mises,
                                                        principal, vm.p);
        else
            k_recover_points<false><<<grid, 128, 0, s>>>(rec.p, t10.p, inc.start.p,
                                                         inc.of_node.p, u, dtemp, npoints,
                                                         stress, strain, mises, principal,
                                                         nullptr);
        FG_CHECK_LAUNCH();
        if (want_peaks) {
            const size_t smem = 5 * sizeof(unsigned long long) * (size_t)nparts;
            k_peak_blocks<<<peak_blocks, PEAK_THREADS, smem, s>>>(
                vm.p, tag.p, t10.p, has_singular ? singular.p : nullptr, nel, nparts, chunk,
                partial.p);
            FG_CHECK_LAUNCH();
            k_peak_final<<<(nparts + 127) / 128, 128, 0, s>>>(
                partial.p, peak_blocks, nparts, vm.p, t10.p, tag.p,
                has_singular ? singular.p : nullptr, dpeaks.p);
            FG_CHECK_LAUNCH();
        }
        FG_CUDA(cudaEventRecord(ev1, s));
        if (want_peaks) dpeaks.download(peaks, nparts, s);
        FG_CUDA(cudaStreamSynchronize(s));
        float ms = 0.f;
        FG_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        // The cell records, the cells' point numbers, the incidence and u once; the outputs once;
        // for the peaks the pair values written and read once and the cell tags.
        double bytes = nel * (sizeof(CellRecord) + 10.0 * 4) + (npoints + 1) * 8.0 +
                       10.0 * nel * 4 + npoints * 24.0 + (dtemp ? npoints * 8.0 : 0.0) +
                       npoints * 96.0 + (mises ? npoints * 8.0 : 0.0) +
                       (principal ? npoints * 24.0 : 0.0);
        if (want_peaks) bytes += nel * (80.0 + 80.0 + 4.0) + (has_singular ? nel * 10.0 : 0.0);
        last_bytes = bytes;
    }
};

namespace {
template <class F>
int recovery_guarded(F f) {
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
}  // namespace

extern "C" {

int femgpu_recovery_new(size_t npoints, const double* xyz, size_t nel, const uint32_t* tets10,
                        const double* coef, const double* expansion, const uint32_t* part,
                        size_t nparts, const uint8_t* singular, femgpu_recovery** out) {
    return recovery_guarded([&] {
        need(out != nullptr, "out is null");
        need(npoints > 0 && nel > 0, "an empty mesh");
        need(xyz && tets10 && coef, "a null mesh array");
        need(nparts >= 1, "no part");
        if (nparts > (size_t)MAX_PARTS)
            throw Failure(FEMGPU_ERR_TOO_LARGE, "more than 2048 parts");
        if (npoints >= 0xffffffffull || nel >= 0xffffffffull / 10)
            throw Failure(FEMGPU_ERR_TOO_LARGE, "more points or cells than 32-bit numbers hold");
        auto r = std::make_unique<femgpu_recovery>();
        FG_CUDA(cudaStreamCreateWithFlags(&r->s, cudaStreamNonBlocking));
        FG_CUDA(cudaEventCreate(&r->ev0));
        FG_CUDA(cudaEventCreate(&r->ev1));
        cudaStream_t s = r->s;
        r->npoints = (int64_t)npoints;
        r->nel = (int64_t)nel;
        r->nparts = (int)nparts;
        r->t10.upload(tets10, 10 * nel, s);
        build_incidence(r->t10.p, r->nel, 10, r->npoints, &r->inc, s);
        DevBuf<double> dxyz, dcoef, dexp;
        DevBuf<uint32_t> dpart;
        dxyz.upload(xyz, 3 * npoints, s);
        dcoef.upload(coef, 2 * nel, s);
        if (expansion) dexp.upload(expansion, 3 * nel, s);
        if (part) dpart.upload(part, nel, s);
        if (singular) {
            r->singular.upload(singular, npoints, s);
            r->has_singular = true;
        }
        r->rec.alloc(nel);
        r->tag.alloc(nel);
        DevBuf<int> bad(1);
        bad.zero(s);
        k_recover_cells<<<blocks_for(r->nel, 128, NUM_SMS * 32), 128, 0, s>>>(
            dxyz.p, r->t10.p, dcoef.p, expansion ? dexp.p : nullptr, part ? dpart.p : nullptr,
            (uint32_t)nparts, singular ? r->singular.p : nullptr, r->nel, r->rec.p, r->tag.p,
            bad.p);
        FG_CHECK_LAUNCH();
        int b = fetch(bad.p, s);
        if (b == 2)
            throw Failure(FEMGPU_ERR_MATERIAL,
                          "the Poisson ratios give no stable material (for an isotropic material, "
                          "nu must be between -1 and 0.5)");
        if (b == 3) throw Failure(FEMGPU_ERR_INVALID, "a cell names a part past the last");
        r->chunk = (r->nel + PEAK_BLOCKS - 1) / PEAK_BLOCKS;
        r->peak_blocks = (int)((r->nel + r->chunk - 1) / r->chunk);
        r->partial.alloc((size_t)r->peak_blocks * nparts);
        r->dpeaks.alloc(nparts);
        const size_t smem = 5 * sizeof(unsigned long long) * nparts;
        if (smem > 48 * 1024)
            FG_CUDA(cudaFuncSetAttribute(k_peak_blocks,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        FG_CUDA(cudaStreamSynchronize(s));
        *out = r.release();
    });
}

int femgpu_recovery_run(femgpu_recovery* r, const double* u, const double* dtemp, double* stress,
                        double* strain, double* mises, double* principal, femgpu_peak* peaks) {
    return recovery_guarded([&] {
        need(r && u, "a null argument");
        cudaStream_t s = r->s;
        const size_t n = (size_t)r->npoints;
        r->du.upload(u, 3 * n, s);
        if (dtemp) r->ddt.upload(dtemp, n, s);
        if (r->dstress.count < 6 * n) r->dstress.alloc(6 * n);
        if (r->dstrain.count < 6 * n) r->dstrain.alloc(6 * n);
        if (mises && r->dmises.count < n) r->dmises.alloc(n);
        if (principal && r->dprincipal.count < 3 * n) r->dprincipal.alloc(3 * n);
        r->run(r->du.p, dtemp ? r->ddt.p : nullptr, r->dstress.p, r->dstrain.p,
               mises ? r->dmises.p : nullptr, principal ? r->dprincipal.p : nullptr, peaks);
        if (stress) r->dstress.download(stress, 6 * n, s);
        if (strain) r->dstrain.download(strain, 6 * n, s);
        if (mises) r->dmises.download(mises, n, s);
        if (principal) r->dprincipal.download(principal, 3 * n, s);
        FG_CUDA(cudaStreamSynchronize(s));
    });
}

int femgpu_recovery_run_device(femgpu_recovery* r, const double* u, const double* dtemp,
                               double* stress, double* strain, double* mises, double* principal,
                               femgpu_peak* peaks) {
    return recovery_guarded([&] {
        need(r && u && stress && strain, "a null argument");
        r->run(u, dtemp, stress, strain, mises, principal, peaks);
    });
}

int femgpu_recovery_last_time(const femgpu_recovery* r, double* ms, double* bytes) {
    return recovery_guarded([&] {
        need(r != nullptr, "a null handle");
        if (ms) *ms = r->last_ms;
        if (bytes) *bytes = r->last_bytes;
    });
}

size_t femgpu_recovery_bytes(const femgpu_recovery* r) {
    if (!r) return 0;
    return r->t10.bytes() + r->rec.bytes() + r->tag.bytes() + r->singular.bytes() +
           r->vm.bytes() + r->partial.bytes() + r->dpeaks.bytes() + r->inc.start.bytes() +
           r->inc.of_node.bytes() + r->du.bytes() + r->ddt.bytes() + r->dstress.bytes() +
           r->dstrain.bytes() + r->dmises.bytes() + r->dprincipal.bytes();
}

void* femgpu_recovery_stream(const femgpu_recovery* r) { return r ? (void*)r->s : nullptr; }

void femgpu_recovery_free(femgpu_recovery* r) { delete r; }

}  // extern "C"
