// Oracle (test infrastructure): a C interface over the restatement, loaded with ctypes by the
// tests, the smoke check and the CPU-baseline leg of the benchmark. Handles own C++ objects;
// a function that fails returns a negative status and writes the reference's error text to
// the caller's buffer.
#include <atomic>
#include <cstring>
#include <memory>
#include <thread>

#include "oracle.hpp"

using namespace orc;

namespace {
void put_error(char* buf, size_t len, const char* what) {
    if (buf && len) {
        std::strncpy(buf, what, len - 1);
        buf[len - 1] = 0;
    }
}
Csr* C(void* h) { return static_cast<Csr*>(h); }
Rect* R(void* h) { return static_cast<Rect*>(h); }

Level make_level(const double* px, size_t nx, const double* py, size_t ny, const double* pz,
                 size_t nz, const uint32_t* points, const uint8_t* comp, size_t n) {
    Level l;
    l.planes[0].assign(px, px + nx);
    l.planes[1].assign(py, py + ny);
    l.planes[2].assign(pz, pz + nz);
    l.points.resize(n);
    for (size_t k = 0; k < n; ++k)
        for (int d = 0; d < 3; ++d) l.points[k][d] = points[3 * k + d];
    l.comp.assign(comp, comp + n);
    return l;
}
vector<Vec3> make_points(const double* xyz, size_t n) {
    vector<Vec3> v(n);
    for (size_t k = 0; k < n; ++k) v[k] = {xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]};
    return v;
}

// Element loops share the work among threads by element range only when the caller asks for
// it (the values are independent per element; the assembly itself is sequential).
void tet_points(const double* xyz, const uint32_t* t, Vec3 p[4]) {
    for (int c = 0; c < 4; ++c)
        for (int d = 0; d < 3; ++d) p[c][d] = xyz[3 * (size_t)t[c] + d];
}
}  // namespace

extern "C" {

void orc_set_threads(int n) { set_threads(n); }

// ---------------------------------------------------------------- Csr
void* orc_pattern(size_t n, const uint32_t* elements, size_t nel, int m) {
    return new Csr(pattern(n, elements, nel, m));
}
void* orc_csr_import(size_t n, const int64_t* ptr, const uint32_t* idx, const double* val) {
    Csr* a = new Csr;
    a->n = n;
    a->ptr.assign(ptr, ptr + n + 1);
    size_t nnz = (size_t)ptr[n];
    a->idx.assign(idx, idx + nnz);
    a->val.assign(val, val + nnz);
    return a;
}
void orc_csr_info(void* h, size_t* n, size_t* nnz) {
    *n = C(h)->n;
    *nnz = C(h)->idx.size();
}
void orc_csr_export(void* h, int64_t* ptr, uint32_t* idx, double* val) {
    Csr* a = C(h);
    for (size_t i = 0; i <= a->n; ++i) ptr[i] = (int64_t)a->ptr[i];
    if (idx) std::memcpy(idx, a->idx.data(), a->idx.size() * 4);
    if (val) std::memcpy(val, a->val.data(), a->val.size() * 8);
}
void orc_csr_free(void* h) { delete C(h); }
int orc_add_element(void* h, const uint32_t* nodes, int m, const double* ke, char* err,
                    size_t len) {
    try {
        C(h)->add_element(nodes, m, ke);
        return 0;
    } catch (const std::exception& e) {
        put_error(err, len, e.what());
        return -1;
    }
}
void orc_mul(void* h, const double* x, double* y) { C(h)->mul(x, y); }
void* orc_submatrix(void* h, const int64_t* keep, size_t nkeep) {
    vector<size_t> k(keep, keep + nkeep);
    return new Csr(C(h)->submatrix(k));
}
void orc_reduced_rhs(void* h, const double* load, const double* t, const int64_t* free,
                     size_t nfree, double* out) {
    vector<size_t> f(free, free + nfree);
    vector<double> r = reduced_rhs(*C(h), load, t, f);
    std::memcpy(out, r.data(), nfree * 8);
}

void orc_reactions(void* h, const double* u, const double* force, const uint8_t* fixed,
                   const uint32_t* owner, size_t nloads, const double* applied, double gross,
                   double* load_force, double* total, double* gross_out, double* imbalance) {
    reactions(*C(h), u, force, fixed, owner, nloads, applied, gross, load_force, total,
              gross_out, imbalance);
}

// ---------------------------------------------------------------- elements
void orc_tet_gradients(const double* p12, double* g12, double* volume) {
    Vec3 p[4], g[4];
    for (int c = 0; c < 4; ++c)
        for (int d = 0; d < 3; ++d) p[c][d] = p12[3 * c + d];
    tet_gradients(p, g, volume);
    for (int c = 0; c < 4; ++c)
        for (int d = 0; d < 3; ++d) g12[3 * c + d] = g[c][d];
}
int orc_isotropic(double e, double nu, double* normal9, double* shear3, char* err, size_t len) {
    try {
        Stiffness d = isotropic_stiffness(e, nu);
        std::memcpy(normal9, d.normal, 72);
        std::memcpy(shear3, d.shear, 24);
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}
// The element matrix of 1 tetrahedron: kind 0 = P1 heat (4 x 4, `coef` = 3 conductivities),
// 1 = P1 elasticity (12 x 12, `coef` = E, nu), 2 = P2 elasticity (30 x 30, `coef` = E, nu).
int orc_element_matrix(int kind, const double* p12, const double* coef, double* ke) {
    Vec3 p[4], g[4];
    double v;
    for (int c = 0; c < 4; ++c)
        for (int d = 0; d < 3; ++d) p[c][d] = p12[3 * c + d];
    tet_gradients(p, g, &v);
    if (kind == 0) {
        tet_conduction(g, v, Vec3{coef[0], coef[1], coef[2]}, ke);
        return 0;
    }
    if (kind == 3) {
        tet10_mass(v, coef[0], ke);
        return 0;
    }
    if (kind == 4) {
        tet10_stiffness(g, v, orthotropic_stiffness(coef, coef + 3, coef + 6), ke);
        return 0;
    }
    Stiffness d = isotropic_stiffness(coef[0], coef[1]);
    if (kind == 1)
        tet4_stiffness(g, v, d, ke);
    else
        tet10_stiffness(g, v, d, ke);
    return 0;
}

// hex.rs:218-297: the condensed 24 x 24 stiffness of a box cell with the sides `size` and the
// orthotropic constants `c` (Ex, Ey, Ez, nu_xy, nu_xz, nu_yz, G_xy, G_xz, G_yz).
int orc_hex8_stiffness(const double* size, const double* c, double* kc, char* err, size_t len) {
    try {
        hex8_stiffness(size, orthotropic_stiffness(c, c + 3, c + 6), kc);
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}

// eigen.rs:183-269 (row-major n x n); -1 and the reference's text on failure.
int orc_dense_generalized(const double* k, const double* m, int n, double* values, double* q,
                          char* err, size_t len) {
    std::string e;
    if (!dense_generalized(k, m, n, values, q, &e)) {
        put_error(err, len, e.c_str());
        return -1;
    }
    return 0;
}
// eigen.rs:274-331; `a` is overwritten.
void orc_dense_jacobi(double* a, int n, double* values, double* v) {
    dense_jacobi(a, n, values, v);
}

// Assemble all the elements of a mesh into the pattern `h`, in increasing element order
// (heat.rs:920-927, elastic_tet.rs:183-193, modes.rs:470-476). kind as orc_element_matrix;
// `nodes` are 4 corners (kind 0, 1), 10 points (kind 2, 3, 4) or 8 box corners (kind 5, 6) per
// element; `coef` has 3 (kinds 0, 5), 2 (kinds 1, 2), 1 (kind 3: the density) or 9 (kinds 4, 6:
// an orthotropic material) values per element.
// The scalar nodes of kinds 1 and 2 become the unknowns 3 node + component.
int orc_assemble(void* h, int kind, const double* xyz, const uint32_t* nodes, size_t nel,
                 const double* coef, char* err, size_t len) {
    try {
        Csr* a = C(h);
        if (kind == 5) {  // heat.rs:820-826: box cells, the sides from corners 0 and 6
            double ke[64];
            for (size_t e = 0; e < nel; ++e) {
                const uint32_t* t = nodes + 8 * e;
                double s[3], k[3];
                for (int d = 0; d < 3; ++d) {
                    s[d] = xyz[3 * (size_t)t[6] + d] - xyz[3 * (size_t)t[0] + d];
                    k[d] = coef[3 * e + d];
                }
                hex_conduction(s, k, ke);
                a->add_element(t, 8, ke);
            }
            return 0;
        }
        if (kind == 7) {  // modes.rs:363-370: box cells, hex::mass per cell
            vector<double> me(576);
            uint32_t dofs[24];
            for (size_t e = 0; e < nel; ++e) {
                const uint32_t* t = nodes + 8 * e;
                double s[3];
                for (int d = 0; d < 3; ++d)
                    s[d] = xyz[3 * (size_t)t[6] + d] - xyz[3 * (size_t)t[0] + d];
                hex8_mass(s, coef[e], me.data());
                for (int k = 0; k < 24; ++k) dofs[k] = 3 * t[k / 3] + (uint32_t)(k % 3);
                a->add_element(dofs, 24, me.data());
            }
            return 0;
        }
        if (kind == 6) {  // elastic.rs:386-391: box cells, Hex::new per cell
            vector<double> kc(576);
            uint32_t dofs[24];
            for (size_t e = 0; e < nel; ++e) {
                const uint32_t* t = nodes + 8 * e;
                const double* c = coef + 9 * e;  // Orthotropic {e, nu, g} (hex.rs:47-55)
                double s[3];
                for (int d = 0; d < 3; ++d)
                    s[d] = xyz[3 * (size_t)t[6] + d] - xyz[3 * (size_t)t[0] + d];
                hex8_stiffness(s, orthotropic_stiffness(c, c + 3, c + 6), kc.data());
                for (int k = 0; k < 24; ++k) dofs[k] = 3 * t[k / 3] + (uint32_t)(k % 3);
                a->add_element(dofs, 24, kc.data());
            }
            return 0;
        }
        int mn = kind >= 2 ? 10 : 4;
        int m = kind == 0 ? 4 : 3 * mn;
        vector<double> ke(m * m);
        vector<uint32_t> dofs(m);
        for (size_t e = 0; e < nel; ++e) {
            const uint32_t* t = nodes + e * mn;
            Vec3 p[4], g[4];
            double v;
            tet_points(xyz, t, p);
            tet_gradients(p, g, &v);
            if (kind == 0) {
                const double* k = coef + 3 * e;
                tet_conduction(g, v, Vec3{k[0], k[1], k[2]}, ke.data());
                a->add_element(t, 4, ke.data());
                continue;
            }
            if (kind == 3) {
                tet10_mass(v, coef[e], ke.data());  // modes.rs:475: the density per element
            } else if (kind == 4) {
                const double* c = coef + 9 * e;  // Orthotropic {e, nu, g} (hex.rs:47-55)
                tet10_stiffness(g, v, orthotropic_stiffness(c, c + 3, c + 6), ke.data());
            } else {
                Stiffness d = isotropic_stiffness(coef[2 * e], coef[2 * e + 1]);
                if (kind == 1)
                    tet4_stiffness(g, v, d, ke.data());
                else
                    tet10_stiffness(g, v, d, ke.data());
            }
            for (int k = 0; k < m; ++k) dofs[k] = 3 * t[k / 3] + (uint32_t)(k % 3);
            a->add_element(dofs.data(), m, ke.data());
        }
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}

// tet10.rs:244-272. Writes the edges (2 per edge) and the 10-point tetrahedra; returns the
// number of edges. `edges` must hold 2 * 6 * ntet values.
size_t orc_quadratic(const double* xyz, size_t ncorner, const uint32_t* tets, size_t ntet,
                     uint32_t* edges, uint32_t* tets10) {
    vector<Vec3> pts = make_points(xyz, ncorner);
    vector<array<uint32_t, 4>> t(ntet);
    for (size_t e = 0; e < ntet; ++e)
        for (int c = 0; c < 4; ++c) t[e][c] = tets[4 * e + c];
    Quadratic q = quadratic(pts, t);
    for (size_t k = 0; k < q.edges.size(); ++k) {
        edges[2 * k] = q.edges[k][0];
        edges[2 * k + 1] = q.edges[k][1];
    }
    for (size_t e = 0; e < ntet; ++e)
        for (int c = 0; c < 10; ++c) tets10[10 * e + c] = q.tets[e][c];
    return q.edges.size();
}

int orc_colour(size_t n, const uint32_t* elements, size_t nel, int m, uint32_t* colour) {
    int nc = 0;
    vector<uint32_t> c = colour_elements(n, elements, nel, m, &nc);
    std::memcpy(colour, c.data(), nel * 4);
    return nc;
}
uint32_t orc_colour_priority(uint32_t e) { return colour_priority(e); }

// ---------------------------------------------------------------- Rect
void* orc_rect_import(size_t rows, size_t cols, const int64_t* ptr, const uint32_t* idx,
                      const double* val) {
    Rect* p = new Rect;
    p->rows = rows;
    p->cols = cols;
    p->ptr.assign(ptr, ptr + rows + 1);
    size_t nnz = (size_t)ptr[rows];
    p->idx.assign(idx, idx + nnz);
    p->val.assign(val, val + nnz);
    return p;
}
void orc_rect_info(void* h, size_t* rows, size_t* cols, size_t* nnz) {
    *rows = R(h)->rows;
    *cols = R(h)->cols;
    *nnz = R(h)->idx.size();
}
void orc_rect_export(void* h, int64_t* ptr, uint32_t* idx, double* val) {
    Rect* p = R(h);
    for (size_t i = 0; i <= p->rows; ++i) ptr[i] = (int64_t)p->ptr[i];
    std::memcpy(idx, p->idx.data(), p->idx.size() * 4);
    std::memcpy(val, p->val.data(), p->val.size() * 8);
}
void orc_rect_free(void* h) { delete R(h); }
void orc_rect_mul(void* h, const double* x, double* y) { R(h)->mul(x, y); }
void orc_rect_mul_transpose(void* h, const double* x, double* y) { R(h)->mul_transpose(x, y); }
void* orc_galerkin(void* p, void* a) { return new Csr(R(p)->galerkin(*C(a))); }

// multigrid.rs:329-452. Returns P (a Rect handle) or null; the coarse level's points and
// components go to `cpoints` (3 per unknown) and `ccomp`, sized like the fine level.
void* orc_coarsen(void* a, const double* px, size_t nx, const double* py, size_t ny,
                  const double* pz, size_t nz, const uint32_t* points, const uint8_t* comp,
                  size_t n, uint32_t* cpoints, uint8_t* ccomp, size_t* cn) {
    Level fine = make_level(px, nx, py, ny, pz, nz, points, comp, n);
    Rect* p = new Rect;
    Level coarse;
    if (!coarsen(fine, *C(a), p, &coarse)) {
        delete p;
        return nullptr;
    }
    *cn = coarse.points.size();
    for (size_t k = 0; k < coarse.points.size(); ++k)
        for (int d = 0; d < 3; ++d) cpoints[3 * k + d] = coarse.points[k][d];
    std::memcpy(ccomp, coarse.comp.data(), coarse.comp.size());
    return p;
}

// multigrid.rs:458-608 after coarsen (multigrid.rs:329-452): the coarse matrix from the cells
// (origin 3 per cell, its class, 576 values per class), or null; the coarse level as
// orc_coarsen writes it.
void* orc_by_cells(void* a, const double* px, size_t nx, const double* py, size_t ny,
                   const double* pz, size_t nz, const uint32_t* points, const uint8_t* comp,
                   size_t n, size_t ncells, const uint32_t* origin, const uint32_t* cls,
                   const double* table, size_t nclass, uint32_t* cpoints, uint8_t* ccomp,
                   size_t* cn) {
    Level fine = make_level(px, nx, py, ny, pz, nz, points, comp, n);
    Cells cells;
    cells.origin.resize(ncells);
    for (size_t i = 0; i < ncells; ++i)
        for (int d = 0; d < 3; ++d) cells.origin[i][d] = origin[3 * i + d];
    cells.cls.assign(cls, cls + ncells);
    cells.table.assign(table, table + 576 * nclass);
    Rect p;
    Level coarse;
    if (!coarsen(fine, *C(a), &p, &coarse)) return nullptr;
    Cells next;
    Csr* out = new Csr(by_cells(fine, cells, coarse, &next));
    *cn = coarse.points.size();
    for (size_t k = 0; k < coarse.points.size(); ++k)
        for (int d = 0; d < 3; ++d) cpoints[3 * k + d] = coarse.points[k][d];
    std::memcpy(ccomp, coarse.comp.data(), coarse.comp.size());
    return out;
}

// pmultigrid.rs:104-151. Returns P; the coarse points go to `cxyz` (3 per coarse unknown;
// room for 3 * nfree values).
void* orc_prolongation(const double* points, size_t npoints, size_t corners,
                       const uint32_t* edges, size_t nedges, const int64_t* free, size_t nfree,
                       double* cxyz, size_t* ncoarse) {
    vector<Vec3> pts = make_points(points, npoints);
    vector<array<uint32_t, 2>> e(nedges);
    for (size_t k = 0; k < nedges; ++k) e[k] = {edges[2 * k], edges[2 * k + 1]};
    vector<size_t> f(free, free + nfree);
    Rect* p = new Rect;
    vector<Vec3> xyz;
    prolongation(pts, corners, e, f, p, &xyz);
    *ncoarse = xyz.size();
    for (size_t k = 0; k < xyz.size(); ++k)
        for (int d = 0; d < 3; ++d) cxyz[3 * k + d] = xyz[k][d];
    return p;
}

// ---------------------------------------------------------------- direct
void orc_nested_dissection(void* a, const double* xyz, int64_t* order) {
    vector<size_t> o = nested_dissection(*C(a), make_points(xyz, C(a)->n));
    for (size_t k = 0; k < o.size(); ++k) order[k] = (int64_t)o[k];
}
// Factor and solve in place; returns 0 or -1 with the error text. `entries` gets the factor's
// entries (symbolic.rs:162).
int orc_direct_solve(void* a, const double* xyz, double* b, uint64_t* entries, char* err,
                     size_t len) {
    try {
        Symbolic sym = analyse(*C(a), nested_dissection(*C(a), make_points(xyz, C(a)->n)));
        if (entries) *entries = sym.entries();
        Cholesky ch = factor(sym, *C(a));
        ch.solve(b);
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}

// ---------------------------------------------------------------- Solver
struct OSolver {
    Solver s;
};

// unknowns kind 0 = Grid (planes, points, comp), 1 = Points (xyz), 2 = Quadratic (xyz of each
// unknown, P as a Rect handle, coarse xyz). method -1 none, 0 direct, 1 multigrid.
// crossover: flops_rule 0 -> Unknowns(unknowns); 1 -> Flops{flops, entries, flat}.
void* orc_solver_new(void* a, int kind, const double* px, size_t nx, const double* py,
                     size_t ny, const double* pz, size_t nz, const uint32_t* points,
                     const uint8_t* comp, const double* xyz, void* p, const double* cxyz,
                     size_t ncoarse, int method, int flops_rule, size_t unknowns, double flops,
                     uint64_t entries, int flat, size_t ncells, const uint32_t* origin,
                     const uint32_t* cls, const double* table, size_t nclass, char* err,
                     size_t len) {
    try {
        Unknowns u;
        size_t n = C(a)->n;
        u.kind = (Unknowns::Kind)kind;
        if (kind == 0) u.level = make_level(px, nx, py, ny, pz, nz, points, comp, n);
        if (kind == 0 && ncells) {  // multigrid.rs:62-68: the cells of a displacement model
            u.cells.origin.resize(ncells);
            for (size_t i = 0; i < ncells; ++i)
                for (int d = 0; d < 3; ++d) u.cells.origin[i][d] = origin[3 * i + d];
            u.cells.cls.assign(cls, cls + ncells);
            for (size_t i = 0; i < ncells; ++i)
                if (cls[i] >= nclass) throw Error("a cell class is out of range");
            u.cells.table.assign(table, table + 576 * nclass);
        }
        if (kind >= 1) u.points = make_points(xyz, n);
        if (kind == 2) {
            u.p = *R(p);
            u.coarse = make_points(cxyz, ncoarse);
        }
        Crossover c;
        c.flops_rule = flops_rule != 0;
        c.unknowns = unknowns;
        c.flops = flops;
        c.entries = entries;
        c.flat = flat != 0;
        auto* s = new OSolver;
        s->s = Solver::make(*C(a), std::move(u), method, c);
        return s;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return nullptr;
    }
}
void orc_solver_free(void* s) { delete static_cast<OSolver*>(s); }
// A copy of the matrix of multigrid level `l` (null when the solver has no such level).
void* orc_solver_level_matrix(void* s, size_t l) {
    auto* o = static_cast<OSolver*>(s);
    if (o->s.inner != Solver::MG || l >= o->s.mg.a.size()) return nullptr;
    return new Csr(o->s.mg.a[l]);
}
int orc_solver_method(void* s) { return (int)static_cast<OSolver*>(s)->s.method(); }
size_t orc_solver_levels(void* s) {
    auto* o = static_cast<OSolver*>(s);
    return o->s.inner == Solver::MG ? o->s.mg.levels() : (o->s.inner == Solver::PMG ? 2 : 1);
}
size_t orc_solver_level_size(void* s, size_t l) {
    auto* o = static_cast<OSolver*>(s);
    if (o->s.inner == Solver::MG) return o->s.mg.a[l].n;
    if (o->s.inner == Solver::PMG) return l == 0 ? o->s.a.n : o->s.pmg.coarse_unknowns;
    return o->s.a.n;
}
// `cancel` (may be null) is read before each PCG iteration, as the reference's `cancelled`.
int orc_solver_solve(void* s, const double* b, double* x, double tol, size_t max_iter,
                     const volatile int* cancel, size_t* iterations, double* residual,
                     char* err, size_t len) {
    auto* o = static_cast<OSolver*>(s);
    try {
        if (tol > 0) o->s.tol = tol;
        if (max_iter > 0) o->s.max_iter = max_iter;
        Stats st = o->s.solve(b, x, [cancel] { return cancel && *cancel != 0; });
        *iterations = st.iterations;
        *residual = st.residual;
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}
// multigrid.rs:692-753 with a caller's preconditioner (a C function; NULL: z = r).
int orc_pcg(void* a, const double* b, double* x, void (*pre)(const double*, double*, size_t, void*),
            void* ctx, double tol, size_t max_iter, const volatile int* cancel,
            size_t* iterations, double* residual, char* err, size_t len) {
    try {
        const size_t n = C(a)->n;
        Convergence c = pcg(
            *C(a), b, x,
            [&](const double* r, double* z) {
                if (pre)
                    pre(r, z, n, ctx);
                else
                    std::copy(r, r + n, z);
            },
            tol, max_iter, [cancel] { return cancel && *cancel != 0; });
        *iterations = c.iterations;
        *residual = c.residual;
        return 0;
    } catch (const std::exception& e) {
        put_error(err, len, e.what());
        return -1;
    }
}

// z = M^-1 r of the solver's preconditioner (1 V-cycle).
void orc_solver_precondition(void* s, const double* r, double* z) {
    auto* o = static_cast<OSolver*>(s);
    if (o->s.inner == Solver::MG)
        o->s.mg.apply(r, z);
    else if (o->s.inner == Solver::PMG)
        o->s.pmg.apply(o->s.a, r, z);
}

// heat.rs:691-696 on the matrix `h`; -1 and the reference's text when a row has no diagonal.
int orc_add_capacity(void* h, const double* capacity, double dt, char* err, size_t len) {
    try {
        add_capacity(C(h), capacity, dt);
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}
// heat.rs:1219-1244 with the capacity term of a transient step.
void orc_reduced_rhs_transient(void* h, const double* load, const double* t, const int64_t* free,
                               size_t nfree, const double* capacity, double dt, double* out) {
    vector<size_t> f(free, free + nfree);
    vector<double> r = reduced_rhs(*C(h), load, t, f, capacity, dt);
    std::copy(r.begin(), r.end(), out);
}
void orc_transient_energy(size_t n, const double* kt, const double* rate, const double* load,
                          const uint8_t* fixed, double* out) {
    transient_energy(n, kt, rate, load, fixed, out);
}

// elastic_tet.rs:367-427 and 482-483 (see recover_tet10). Optional arrays may be null;
// `peaks` holds nparts entries.
int orc_recover(size_t npoints, const double* xyz, size_t nel, const uint32_t* tets10,
                const double* coef, const double* expansion, const double* dtemp,
                const double* u, const uint32_t* part, size_t nparts, const uint8_t* singular,
                double* stress, double* strain, double* mises_out, double* principal_out,
                void* peaks, char* err, size_t len) {
    try {
        recover_tet10(npoints, xyz, nel, tets10, coef, expansion, dtemp, u, part, nparts,
                      singular, stress, strain, mises_out, principal_out,
                      static_cast<RecoveryPeak*>(peaks));
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}
// elastic_tet.rs:428-467 (see probes_tet10).
long orc_probes(const double* xyz, size_t nel, const uint32_t* tets10, const double* coef,
                const double* expansion, const double* dtemp, const double* temperature,
                const double* u, size_t nprobes, const double* points, double* displacement,
                double* stress, double* mises_out, double* temp_out, int64_t* hits) {
    return probes_tet10(xyz, nel, tets10, coef, expansion, dtemp, temperature, u, nprobes,
                        points, displacement, stress, mises_out, temp_out, hits);
}
// elastic.rs:615-660 and 709-710 (see recover_hex8), as orc_recover.
int orc_recover_hex(size_t npoints, const double* xyz, size_t nel, const uint32_t* hexes,
                    const double* coef, const double* expansion, const double* dtemp,
                    const double* u, const uint32_t* part, size_t nparts, const uint8_t* singular,
                    double* stress, double* strain, double* mises_out, double* principal_out,
                    void* peaks, char* err, size_t len) {
    try {
        recover_hex8(npoints, xyz, nel, hexes, coef, expansion, dtemp, u, part, nparts, singular,
                     stress, strain, mises_out, principal_out, static_cast<RecoveryPeak*>(peaks));
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}
// symbolic.rs:162-182 of the analysis of `a` in the nested dissection order of `xyz` (order.rs).
void orc_symbolic_counts(void* a, const double* xyz, uint64_t* entries, double* flops) {
    Symbolic sym = analyse(*C(a), nested_dissection(*C(a), make_points(xyz, C(a)->n)));
    *entries = sym.entries();
    *flops = sym.flops();
}
// hex.rs:337-353
void orc_hex8_mass(const double* size, double density, double* m) { hex8_mass(size, density, m); }
// elastic.rs:386-405 (see hex_loads).
int orc_hex_loads(size_t npoints, const double* xyz, size_t nel, const uint32_t* hexes,
                  const double* coef, const double* expansion, const double* accel,
                  const double* dtemp, double* force, char* err, size_t len) {
    try {
        hex_loads(npoints, xyz, nel, hexes, coef, expansion, accel, dtemp, force);
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}
// hex.rs:218-335 for 1 box cell: its load (24 x 8) and mode matrices (9 x 24, 9 x 8), and the
// strain and stress at xi for the corner values u and t.
int orc_hex8_element(const double* size, const double* c, const double* alpha, double* k,
                     double* load, double* mode_u, double* mode_t, char* err, size_t len) {
    try {
        HexElement h;
        hex8_element(size, orthotropic_stiffness(c, c + 3, c + 6), alpha, &h);
        std::memcpy(k, h.k, sizeof(h.k));
        std::memcpy(load, h.load, sizeof(h.load));
        std::memcpy(mode_u, h.mode_u, sizeof(h.mode_u));
        std::memcpy(mode_t, h.mode_t, sizeof(h.mode_t));
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}
int orc_hex8_strain_stress(const double* size, const double* c, const double* alpha,
                           const double* xi, const double* u, const double* t, double* e,
                           double* s, char* err, size_t len) {
    try {
        HexElement h;
        hex8_element(size, orthotropic_stiffness(c, c + 3, c + 6), alpha, &h);
        hex8_strain_stress(h, xi, u, t, e, s);
        return 0;
    } catch (const std::exception& x) {
        put_error(err, len, x.what());
        return -1;
    }
}

}  // extern "C"
