// The C ABI of femgpu.h: argument checks, host <-> device copies and the translation of
// failures into status codes with the reference's messages.
#include <cstring>
#include <string>

#include "assemble.cuh"
#include "common.cuh"
#include "hierarchy.hpp"
#include "solver.cuh"
#include "coarsen.cuh"
#include "symbolic.hpp"

namespace femgpu {

static thread_local std::string g_last_error;

void set_last_error(const std::string& s) { g_last_error = s; }

template <class F>
static int guarded(F f) {
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

// A stream for calls that have no handle (assembly, utilities).
static cudaStream_t util_stream() {
    static thread_local cudaStream_t s = nullptr;
    if (!s) FG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
}

static void require(bool ok, const char* what) {
    if (!ok) throw Failure(FEMGPU_ERR_INVALID, what);
}

}  // namespace femgpu

using namespace femgpu;

extern "C" {

size_t femgpu_last_error(char* buf, size_t len) {
    const std::string& e = g_last_error;
    if (buf && len) {
        size_t k = std::min(len - 1, e.size());
        std::memcpy(buf, e.data(), k);
        buf[k] = 0;
    }
    return e.size();
}

const char* femgpu_version(void) { return "femgpu 0.1 (sm_100a)"; }

static int assemble_impl(int kind, int mode, size_t npoints, const double* xyz, size_t nel,
                         const uint32_t* nodes, const double* coef, femgpu_csr** out,
                         bool device) {
    return guarded([&] {
        require(out != nullptr, "out is null");
        require(npoints > 0 && nel > 0, "an empty mesh");
        require(xyz && nodes && coef, "a null mesh array");
        cudaStream_t s = util_stream();
        int nn = kind >= FEMGPU_HEX8_HEAT ? 8 : (kind >= FEMGPU_P2_ELASTIC ? 10 : 4);
        int nc = (kind == FEMGPU_P1_HEAT || kind == FEMGPU_HEX8_HEAT)
                     ? 3
                     : (kind == FEMGPU_P2_MASS || kind == FEMGPU_HEX8_MASS
                            ? 1
                            : (kind == FEMGPU_P2_ELASTIC_ORTHO || kind == FEMGPU_HEX8_ELASTIC ? 9
                                                                                             : 2));
        DevBuf<double> dx, dc;
        DevBuf<uint32_t> de;
        const double* px = xyz;
        const double* pc = coef;
        const uint32_t* pe = nodes;
        if (!device) {
            dx.upload(xyz, 3 * npoints, s);
            de.upload(nodes, nn * nel, s);
            dc.upload(coef, nc * nel, s);
            px = dx.p;
            pc = dc.p;
            pe = de.p;
        }
        Assembled a;
        assemble(kind, mode, (int64_t)npoints, px, (int64_t)nel, pe, pc, &a, s);
        FG_CUDA(cudaStreamSynchronize(s));
        auto* h = new femgpu_csr;
        h->m = std::move(a.matrix);
        *out = h;
    });
}

int femgpu_assemble(int kind, int mode, size_t npoints, const double* xyz, size_t nel,
                    const uint32_t* nodes, const double* coef, femgpu_csr** out) {
    return assemble_impl(kind, mode, npoints, xyz, nel, nodes, coef, out, false);
}

int femgpu_assemble_device(int kind, int mode, size_t npoints, const double* xyz, size_t nel,
                           const uint32_t* nodes, const double* coef, femgpu_csr** out) {
    return assemble_impl(kind, mode, npoints, xyz, nel, nodes, coef, out, true);
}

int femgpu_pattern(size_t n, size_t nel, int m, const uint32_t* elements, femgpu_csr** out) {
    return guarded([&] {
        require(out && elements && m > 0 && n > 0, "invalid pattern arguments");
        cudaStream_t s = util_stream();
        DevBuf<uint32_t> de;
        de.upload(elements, (size_t)m * nel, s);
        Incidence inc;
        build_incidence(de.p, (int64_t)nel, m, (int64_t)n, &inc, s);
        auto* h = new femgpu_csr;
        build_pattern(de.p, inc, &h->m, s);
        FG_CUDA(cudaStreamSynchronize(s));
        *out = h;
    });
}

int femgpu_colour(size_t n, size_t nel, int m, const uint32_t* elements, uint32_t* colour,
                  int* ncolours) {
    return guarded([&] {
        require(elements && colour && ncolours && m > 0, "invalid colouring arguments");
        cudaStream_t s = util_stream();
        DevBuf<uint32_t> de;
        de.upload(elements, (size_t)m * nel, s);
        Incidence inc;
        build_incidence(de.p, (int64_t)nel, m, (int64_t)n, &inc, s);
        DevBuf<uint32_t> c;
        *ncolours = colour_elements(de.p, inc, &c, s);
        c.download(colour, nel, s);
        FG_CUDA(cudaStreamSynchronize(s));
    });
}

int femgpu_quadratic(size_t ncorner, size_t ntet, const uint32_t* tets, uint32_t* tets10,
                     uint32_t* edges, size_t* nedges) {
    return guarded([&] {
        require(tets && tets10 && edges && nedges, "a null array");
        cudaStream_t s = util_stream();
        DevBuf<uint32_t> dt, d10(10 * ntet), de(12 * ntet);
        dt.upload(tets, 4 * ntet, s);
        int64_t ne = quadratic((int64_t)ncorner, (int64_t)ntet, dt.p, d10.p, de.p, s);
        d10.download(tets10, 10 * ntet, s);
        de.download(edges, 2 * ne, s);
        FG_CUDA(cudaStreamSynchronize(s));
        *nedges = (size_t)ne;
    });
}

int femgpu_csr_info(const femgpu_csr* a, size_t* n, size_t* nnz) {
    return guarded([&] {
        require(a != nullptr, "null matrix");
        if (n) *n = (size_t)a->m.n;
        if (nnz) *nnz = (size_t)a->m.nnz;
    });
}

int femgpu_csr_download(const femgpu_csr* a, int64_t* ptr, uint32_t* idx, double* val) {
    return guarded([&] {
        require(a != nullptr, "null matrix");
        cudaStream_t s = util_stream();
        if (ptr) a->m.ptr.download(ptr, a->m.n + 1, s);
        if (idx) a->m.idx.download(idx, a->m.nnz, s);
        if (val) a->m.val.download(val, a->m.nnz, s);
        FG_CUDA(cudaStreamSynchronize(s));
    });
}

int femgpu_csr_upload(size_t n, const int64_t* ptr, const uint32_t* idx, const double* val,
                      femgpu_csr** out) {
    return guarded([&] {
        require(out && ptr && (ptr[n] == 0 || (idx && val)), "null CSR arrays");
        require(ptr[0] == 0, "ptr[0] must be 0");
        for (size_t i = 0; i < n; ++i) require(ptr[i + 1] >= ptr[i], "ptr must not decrease");
        cudaStream_t s = util_stream();
        auto* h = new femgpu_csr;
        h->m.n = (int64_t)n;
        h->m.nnz = ptr[n];
        h->m.ptr.upload(ptr, n + 1, s);
        h->m.idx.upload(idx, (size_t)ptr[n], s);
        h->m.val.upload(val, (size_t)ptr[n], s);
        FG_CUDA(cudaStreamSynchronize(s));
        *out = h;
    });
}

int femgpu_csr_submatrix(const femgpu_csr* a, const int64_t* keep, size_t nkeep,
                         femgpu_csr** out) {
    return guarded([&] {
        require(a && keep && out, "null argument");
        cudaStream_t s = util_stream();
        DevBuf<int64_t> dk;
        dk.upload(keep, nkeep, s);
        auto* h = new femgpu_csr;
        try {
            submatrix(a->m, dk.p, (int64_t)nkeep, &h->m, s);
            FG_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int femgpu_csr_mul(const femgpu_csr* a, const double* x, double* y) {
    return guarded([&] {
        require(a && x && y, "null argument");
        cudaStream_t s = util_stream();
        DevBuf<double> dx, dy(a->m.n);
        dx.upload(x, a->m.n, s);
        csr_mul(a->m, dx.p, dy.p, s);
        dy.download(y, a->m.n, s);
        FG_CUDA(cudaStreamSynchronize(s));
    });
}

int femgpu_reduced_rhs(const femgpu_csr* a, const double* load, const double* t,
                       const int64_t* free, size_t nfree, double* out) {
    return guarded([&] {
        require(a && load && t && free && out, "null argument");
        cudaStream_t s = util_stream();
        DevBuf<double> dl, dt, dout(nfree);
        DevBuf<int64_t> df;
        dl.upload(load, a->m.n, s);
        dt.upload(t, a->m.n, s);
        df.upload(free, nfree, s);
        reduced_rhs(a->m, dl.p, dt.p, df.p, (int64_t)nfree, dout.p, s);
        dout.download(out, nfree, s);
        FG_CUDA(cudaStreamSynchronize(s));
    });
}

void femgpu_csr_free(femgpu_csr* a) { delete a; }

int femgpu_prolongation(size_t npoints, const double* points, size_t corners, size_t nedges,
                        const uint32_t* edges, size_t nfree, const int64_t* free, size_t* nnz,
                        size_t* ncoarse, int64_t* p_ptr, uint32_t* p_idx, double* p_val,
                        double* coarse_xyz) {
    return guarded([&] {
        require(points && edges && free, "null argument");
        for (size_t k = 0; k < nfree; ++k) {
            require(free[k] >= 0 && (size_t)free[k] < 3 * npoints, "a free unknown out of range");
            require(k == 0 || free[k] > free[k - 1], "the free unknowns must increase");
            if ((size_t)(free[k] / 3) >= corners)
                require((size_t)(free[k] / 3) - corners < nedges, "an edge point out of range");
        }
        HostRect p;
        std::vector<double> xyz;
        prolongation(points, (int64_t)npoints, (int64_t)corners, edges, (int64_t)nedges, free,
                     (int64_t)nfree, &p, &xyz);
        if (nnz) *nnz = p.idx.size();
        if (ncoarse) *ncoarse = (size_t)p.cols;
        if (p_ptr) std::memcpy(p_ptr, p.ptr.data(), p.ptr.size() * 8);
        if (p_idx) std::memcpy(p_idx, p.idx.data(), p.idx.size() * 4);
        if (p_val) std::memcpy(p_val, p.val.data(), p.val.size() * 8);
        if (coarse_xyz) std::memcpy(coarse_xyz, xyz.data(), xyz.size() * 8);
    });
}

static HostCells host_cells(const femgpu_cells* c, const femgpu_unknowns* u) {
    HostCells h;
    if (!c || !c->count) return h;
    require(u->kind == FEMGPU_UNKNOWNS_GRID, "cells need grid unknowns");
    require(c->origin && c->cls && c->matrices && c->nclass > 0, "a null cell array");
    h.origin.resize(c->count);
    for (size_t i = 0; i < c->count; ++i) {
        for (int d = 0; d < 3; ++d) {
            require(c->origin[3 * i + d] + 1 < u->nplanes[d], "a cell past the planes");
            h.origin[i][d] = c->origin[3 * i + d];
        }
        require(c->cls[i] < c->nclass, "a cell class past the matrices");
    }
    h.cls.assign(c->cls, c->cls + c->count);
    h.table.assign(c->matrices, c->matrices + 576 * c->nclass);
    return h;
}

static HostLevel host_level(const femgpu_unknowns* u, int64_t n) {
    require(u->points && u->comp, "a grid level needs its points and components");
    HostLevel lv;
    for (int d = 0; d < 3; ++d) {
        require(u->planes[d] && u->nplanes[d] > 0, "empty planes");
        lv.planes[d].assign(u->planes[d], u->planes[d] + u->nplanes[d]);
    }
    lv.points.resize(n);
    for (int64_t k = 0; k < n; ++k)
        for (int d = 0; d < 3; ++d) {
            require(u->points[3 * k + d] < u->nplanes[d], "a grid point past its planes");
            lv.points[k][d] = u->points[3 * k + d];
        }
    lv.comp.assign(u->comp, u->comp + n);
    return lv;
}

static int solver_new_impl(const femgpu_csr* a, const femgpu_unknowns* u, int method,
                           const femgpu_crossover* crossover, const femgpu_options* options,
                           const femgpu_cells* cells, femgpu_solver** out);

int femgpu_solver_new(const femgpu_csr* a, const femgpu_unknowns* u, int method,
                      const femgpu_crossover* crossover, const femgpu_options* options,
                      femgpu_solver** out) {
    return solver_new_impl(a, u, method, crossover, options, nullptr, out);
}

int femgpu_solver_new_cells(const femgpu_csr* a, const femgpu_unknowns* u, int method,
                            const femgpu_crossover* crossover, const femgpu_options* options,
                            const femgpu_cells* cells, femgpu_solver** out) {
    return solver_new_impl(a, u, method, crossover, options, cells, out);
}

int femgpu_hex_mass(size_t count, const double* sizes, const double* density, double* out) {
    return guarded([&] {
        require(count > 0 && sizes && density && out, "null or empty cells");
        for (size_t e = 0; e < count; ++e) {
            const double* s = sizes + 3 * e;
            double* m = out + 576 * e;
            std::fill(m, m + 576, 0.0);
            for (int i = 0; i < 8; ++i)
                for (int j = 0; j < 8; ++j) {
                    double v = 1.0;  // the product of the 1D masses, from 1.0
                    for (int d = 0; d < 3; ++d) {
                        const int bi = d == 0 ? ((i + 1) >> 1) & 1 : (d == 1 ? (i >> 1) & 1 : i >> 2);
                        const int bj = d == 0 ? ((j + 1) >> 1) & 1 : (d == 1 ? (j >> 1) & 1 : j >> 2);
                        v *= bi == bj ? s[d] / 3.0 : s[d] / 6.0;
                    }
                    for (int a = 0; a < 3; ++a) m[(3 * i + a) * 24 + 3 * j + a] = density[e] * v;
                }
        }
    });
}

int femgpu_hex_elements(size_t count, const double* keys, double* matrices) {
    return guarded([&] {
        require(count > 0 && keys && matrices, "null or empty cell keys");
        cudaStream_t s = util_stream();
        DevBuf<double> dk, dt(576 * count);
        dk.upload(keys, 12 * count, s);
        hex_elements(dk.p, (int64_t)count, dt.p, s);
        dt.download(matrices, 576 * count, s);
        FG_CUDA(cudaStreamSynchronize(s));
    });
}

int femgpu_symbolic_counts(const femgpu_csr* a, const femgpu_unknowns* u, uint64_t* entries,
                           double* flops) {
    return guarded([&] {
        require(a && u && entries && flops, "null argument");
        require(u->kind != FEMGPU_UNKNOWNS_QUADRATIC || u->xyz, "quadratic needs coordinates");
        HostCsr m = download_csr(a->m, util_stream());
        std::vector<double> xyz((size_t)3 * m.n);
        if (u->kind == FEMGPU_UNKNOWNS_GRID) {
            HostLevel lv = host_level(u, m.n);
            for (int64_t k = 0; k < m.n; ++k)
                for (int d = 0; d < 3; ++d) xyz[3 * k + d] = lv.planes[d][lv.points[k][d]];
        } else {
            require(u->xyz != nullptr, "points need coordinates");
            std::copy(u->xyz, u->xyz + 3 * m.n, xyz.begin());
        }
        factor_figures(m, nested_dissection(m, xyz.data()), entries, flops);
    });
}

int femgpu_coarse_matrix(const femgpu_csr* a, const femgpu_unknowns* u,
                         const femgpu_cells* cells, int level, size_t* n, size_t* nnz,
                         int64_t* ptr, uint32_t* idx, double* val, uint32_t* points,
                         uint8_t* comp) {
    return guarded([&] {
        require(a && u && n && nnz, "null argument");
        require(u->kind == FEMGPU_UNKNOWNS_GRID, "coarse matrices need grid unknowns");
        require(level >= 1, "level 1 is the first coarse level");
        cudaStream_t s = util_stream();
        HostLevel lv = host_level(u, a->m.n);
        HostCells stored, first = host_cells(cells, u);
        const int threads = host_threads();
        DevGrid grid;
        grid_upload(lv, &grid, s);
        DevCsr held;
        const DevCsr* cur = &a->m;
        for (int l = 1; l <= level; ++l) {
            DevRect p;
            DevGrid coarse;
            require(coarsen_grid(grid, *cur, 7, &p, &coarse, s),
                    "the grid does not coarsen that far");
            DevCsr next;
            if (!first.empty()) {
                HostCells nxt;
                HostCsr m = by_cells(grid_download(grid, s), stored.empty() ? first : stored,
                                     grid_download(coarse, s), &nxt, threads);
                stored = std::move(nxt);
                upload_csr(m, &next, s);
            } else {
                galerkin_product(p, *cur, &next, s);
            }
            held = std::move(next);
            cur = &held;
            grid = std::move(coarse);
        }
        *n = (size_t)held.n;
        *nnz = (size_t)held.nnz;
        if (points || comp) {
            HostLevel h = grid_download(grid, s);
            for (int64_t k = 0; k < grid.n; ++k) {
                if (points)
                    for (int d = 0; d < 3; ++d) points[3 * k + d] = h.points[k][d];
                if (comp) comp[k] = h.comp[k];
            }
        }
        if (!ptr) return;
        require(idx && val, "null output arrays");
        HostCsr m = download_csr(held, s);
        std::copy(m.ptr.begin(), m.ptr.end(), ptr);
        std::copy(m.idx.begin(), m.idx.end(), idx);
        std::copy(m.val.begin(), m.val.end(), val);
    });
}

static int solver_new_impl(const femgpu_csr* a, const femgpu_unknowns* u, int method,
                           const femgpu_crossover* crossover, const femgpu_options* options,
                           const femgpu_cells* cells, femgpu_solver** out) {
    return guarded([&] {
        require(a && u && out, "null argument");
        require(method >= -1 && method <= 1, "unknown method");
        femgpu_crossover c{0, 3000, 0.0, 0, 0};  // Crossover::Unknowns(STEADY_DIRECT_LIMIT)
        if (crossover) c = *crossover;
        Options o;
        if (options) {
            o.precision = options->precision;
            o.degree = options->degree;
            o.lower = options->lower;
            o.sell_c = options->sell_c;
            o.coarsest = options->coarsest > 0 ? options->coarsest : DEVICE_COARSEST;
            o.max_levels = options->max_levels > 0 ? options->max_levels : 30;
            o.graph = options->graph != 2;
            o.format = options->format;
            o.tail = options->tail;
            o.pdl = options->launch == 0 ? 1 : 0;
            o.values = options->values;
            o.tiles = options->tiles;
            o.axes = options->axes ? options->axes : 7;
            o.stencil = options->stencil;
            o.l2 = options->l2;
            o.smoother = options->smoother ? options->smoother : 4;
            o.cluster = options->cluster;
            o.upper = options->upper;
        }
        require(o.cluster == 0 || o.cluster == 1, "cluster is 0 (off) or 1 (on)");
        require(o.upper == 0.0 || (o.upper >= 0.5 && o.upper <= 4.0),
                "upper is 0 (1.1) or a multiple of lambda_max in [0.5, 4]");
        require(o.smoother == 1 || o.smoother == 4,
                "smoother is 1 (the first-kind Chebyshev polynomial) or 0 or 4 (the fourth kind)");
        require(o.l2 == 0 || o.l2 == 1, "l2 is 0 (plain loads) or 1 (the coarsest inverse "
                                        "persisting in L2)");
        require(o.stencil >= 0 && o.stencil <= 4,
                "stencil is 0 (autotuned), 1 (runtime K), 2 (compile-time K), 3 (2 rows per "
                "thread) or 4 (marching planes)");
        require(o.tiles >= 0 && o.tiles <= 2, "tiles is 0 (autotuned), 1 (off) or 2 (on)");
        require(o.axes >= 1 && o.axes <= 7, "axes is a mask of the axes x (1), y (2), z (4)");
        require(o.values >= 0 && o.values <= 3,
                "values is 0 (default), 1 (FP32), 2 (FP16 stencil coefficients) or 3 (an FP16 "
                "coarsest inverse)");
        require(o.precision == FEMGPU_FP64 || o.precision == FEMGPU_MIXED, "unknown precision");
        require(o.sell_c == 0 || o.sell_c == 8 || o.sell_c == 16 || o.sell_c == 32 ||
                    o.sell_c == 64,
                "the SELL chunk height must be 8, 16, 32 or 64");
        require(o.degree >= 0 && o.degree <= 16, "the Chebyshev degree must be 1 to 16");
        require(o.format == 0 || o.format == 1, "the format is 0 (stencil where possible) or 1");
        int64_t n = a->m.n;
        if (u->kind == FEMGPU_UNKNOWNS_GRID) {
            require(u->points && u->comp, "a grid level needs its points and components");
            for (int d = 0; d < 3; ++d) require(u->planes[d] && u->nplanes[d] > 0, "empty planes");
            for (int64_t k = 0; k < n; ++k)
                for (int d = 0; d < 3; ++d)
                    require(u->points[3 * k + d] < u->nplanes[d], "a grid point past its planes");
        } else if (u->kind == FEMGPU_UNKNOWNS_POINTS) {
            require(u->xyz != nullptr, "points need coordinates");
        } else if (u->kind == FEMGPU_UNKNOWNS_QUADRATIC) {
            require(u->p_ptr && u->p_idx && u->p_val && u->coarse_xyz, "quadratic needs P");
            require(u->p_ptr[0] == 0, "P ptr[0] must be 0");
            for (int64_t k = 0; k < u->p_ptr[n]; ++k)
                require(u->p_idx[k] < u->p_cols, "a column of P past its columns");
        } else {
            throw Failure(FEMGPU_ERR_INVALID, "unknown unknowns kind");
        }
        HostCells hc = host_cells(cells, u);
        require(hc.empty() || o.axes == 7,
                "the coarse matrices from the cells need every axis coarsened (axes 0 or 7)");
        auto* s = new femgpu_solver;
        try {
            s->impl.create(a->m, *u, method, c, o, hc.empty() ? nullptr : &hc);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

int femgpu_solver_set_wait_limit(femgpu_solver* s, uint32_t polls) {
    return guarded([&] {
        require(s != nullptr, "null solver");
        s->impl.set_wait_limit(polls);
    });
}

int femgpu_solver_set_max_iter(femgpu_solver* s, size_t max_iter) {
    return guarded([&] {
        require(s != nullptr, "null solver");
        s->impl.max_iter = max_iter;
    });
}

int femgpu_solver_set_tol(femgpu_solver* s, double tol) {
    return guarded([&] {
        require(s != nullptr && tol >= 0.0, "a tolerance must be 0 or more");
        s->impl.tol = tol;
    });
}

int femgpu_solver_method(const femgpu_solver* s) { return s ? s->impl.method() : -1; }

int femgpu_solver_levels(const femgpu_solver* s, size_t* sizes, int cap) {
    if (!s) return 0;
    auto v = s->impl.level_sizes();
    for (int i = 0; i < (int)v.size() && i < cap; ++i)
        if (sizes) sizes[i] = (size_t)v[i];
    return (int)v.size();
}

size_t femgpu_solver_bytes(const femgpu_solver* s) { return s ? s->impl.bytes() : 0; }

size_t femgpu_solver_describe(const femgpu_solver* s, char* buf, size_t len) {
    if (!s) return 0;
    std::string d = s->impl.describe();
    if (buf && len) {
        size_t k = std::min(len - 1, d.size());
        std::memcpy(buf, d.data(), k);
        buf[k] = 0;
    }
    return d.size();
}

int femgpu_solver_solve(femgpu_solver* s, const double* b, double* x, const volatile int* cancel,
                        femgpu_stats* stats) {
    return guarded([&] {
        require(s && b && x, "null argument");
        s->impl.solve_host(b, x, cancel, stats);
    });
}

int femgpu_solver_solve_zero(femgpu_solver* s, const double* b, double* x,
                             const volatile int* cancel, femgpu_stats* stats) {
    return guarded([&] {
        require(s && b && x, "null argument");
        s->impl.solve_host_zero(b, x, cancel, stats);
    });
}

int femgpu_solver_solve_device(femgpu_solver* s, const double* b, double* x,
                               const volatile int* cancel, femgpu_stats* stats) {
    return guarded([&] {
        require(s && b && x, "null argument");
        s->impl.solve(b, x, cancel, stats);
    });
}

int femgpu_solver_precondition_device(femgpu_solver* s, const double* r, double* z) {
    return guarded([&] {
        require(s && r && z, "null argument");
        s->impl.precondition(r, z);
    });
}

void femgpu_solver_free(femgpu_solver* s) { delete s; }

size_t femgpu_solver_breakdown(femgpu_solver* s, char* buf, size_t len) {
    std::string d;
    int rc = guarded([&] { d = s->impl.breakdown(); });
    if (rc != FEMGPU_OK) return 0;
    if (buf && len) {
        size_t k = std::min(len - 1, d.size());
        std::memcpy(buf, d.data(), k);
        buf[k] = 0;
    }
    return d.size();
}

void* femgpu_solver_stream(const femgpu_solver* s) {
    return s ? (void*)s->impl.stream() : nullptr;
}

int femgpu_solver_kernel_time(femgpu_solver* s, int which, int reps, double* ms, double* bytes) {
    return guarded([&] {
        require(s && ms && bytes, "null argument");
        require(which == 0 || which == 1, "which is 0 (smoother step) or 1 (FP64 operator)");
        s->impl.kernel_time(which, reps, ms, bytes);
    });
}

}  // extern "C"
