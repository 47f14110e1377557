// Oracle (test infrastructure): the iterative solver. Restates
// crates/fem/src/multigrid.rs:43-452 and 683-753 (grid hierarchy with the Galerkin coarse
// matrices, line Gauss-Seidel, V-cycle, PCG), crates/fem/src/pmultigrid.rs:1-151 and
// crates/fem/src/solve.rs:87-250 (the solver dispatch).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <tuple>

#include "oracle.hpp"

namespace orc {

std::string rust_lower_exp(double v, int digits) {
    if (v != v) return "NaN";
    if (v == HUGE_VAL) return "inf";
    if (v == -HUGE_VAL) return "-inf";
    char text[48];
    int p = digits >= 0 ? digits : 0;
    for (;; ++p) {
        std::snprintf(text, sizeof text, "%.*e", p, v);
        if (digits >= 0 || p >= 16 || std::strtod(text, nullptr) == v) break;
    }
    // Split "d.ddde+XX" into the mantissa and the exponent's value.
    char* e = std::strchr(text, 'e');
    long ex = std::strtol(e + 1, nullptr, 10);
    *e = '\0';
    return std::string(text) + "e" + std::to_string(ex);
}

static const size_t COARSEST = 3000;  // multigrid.rs:50

// multigrid.rs:201-277
Lines Lines::make(const Level& level, int axis, const Csr& a) {
    int u = axis == 0 ? 1 : 0;
    int v = axis == 2 ? 1 : 2;
    size_t n = level.points.size();
    Lines L;
    L.order.resize(n);
    for (size_t k = 0; k < n; ++k) L.order[k] = (uint32_t)k;
    auto key = [&](uint32_t k) {
        const auto& p = level.points[k];
        return std::make_tuple(p[v], p[u], p[axis], level.comp[k]);
    };
    std::sort(L.order.begin(), L.order.end(),
              [&](uint32_t x, uint32_t y) { return key(x) < key(y); });
    bool have_last = false;
    array<uint32_t, 3> last{};
    for (size_t r = 0; r < n; ++r) {
        const auto& p = level.points[L.order[r]];
        bool next = have_last && last[u] == p[u] && last[v] == p[v] &&
                    (last[axis] == p[axis] || last[axis] + 1 == p[axis]);
        if (!next) L.start.push_back(r);
        last = p;
        have_last = true;
    }
    L.start.push_back(n);
    L.line.assign(n, 0);
    L.place.assign(n, 0);
    for (size_t l = 0; l + 1 < L.start.size(); ++l)
        for (size_t r = L.start[l]; r < L.start[l + 1]; ++r) {
            L.line[L.order[r]] = (uint32_t)l;
            L.place[L.order[r]] = (uint32_t)r;
        }
    size_t comps = 1;
    for (uint8_t c : level.comp) comps = std::max(comps, (size_t)c + 1);
    size_t band = 2 * comps - 1, w = band + 1;
    L.band = band;
    L.factor.assign(n * w, 0.0);
    for (size_t l = 0; l + 1 < L.start.size(); ++l)
        for (size_t r = L.start[l]; r < L.start[l + 1]; ++r) {
            size_t i = L.order[r];
            size_t first = std::max(r >= band ? r - band : 0, L.start[l]);
            for (size_t c = first; c <= r; ++c) {
                size_t e;
                double s = a.find(i, L.order[c], &e) ? a.val[e] : 0.0;
                size_t lo = std::max(first, c >= band ? c - band : 0);
                for (size_t k = lo; k < c; ++k)
                    s -= L.factor[r * w + band + k - r] * L.factor[c * w + band + k - c];
                if (c == r) {
                    if (!(s > 0.0))
                        throw Error(
                            "the matrix is not positive definite: a part can move with no "
                            "strain");
                    L.factor[r * w + band] = std::sqrt(s);
                } else {
                    L.factor[r * w + band + c - r] = s / L.factor[c * w + band];
                }
            }
        }
    return L;
}

// multigrid.rs:280-323
void Lines::sweep(const Csr& a, const double* b, double* x, bool forward) const {
    size_t w = band + 1;
    vector<double> y;
    auto solve = [&](size_t l) {
        size_t first = start[l], end = start[l + 1];
        y.clear();
        for (size_t r = first; r < end; ++r) {
            size_t i = order[r];
            double s = b[i];
            for (size_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
                size_t j = a.idx[k];
                size_t pj = place[j];
                size_t dist = pj > r ? pj - r : r - pj;
                bool near = line[j] == l && dist <= band;
                if (!near) s -= a.val[k] * x[j];
            }
            y.push_back(s);
        }
        for (size_t r = first; r < end; ++r) {
            double s = y[r - first];
            size_t lo = std::max(r >= band ? r - band : 0, first);
            for (size_t k = lo; k < r; ++k) s -= factor[r * w + band + k - r] * y[k - first];
            y[r - first] = s / factor[r * w + band];
        }
        for (size_t r = end; r-- > first;) {
            double s = y[r - first];
            for (size_t k = r + 1; k < std::min(r + w, end); ++k)
                s -= factor[k * w + band + r - k] * y[k - first];
            y[r - first] = s / factor[r * w + band];
        }
        for (size_t r = first; r < end; ++r) x[order[r]] = y[r - first];
    };
    size_t lines = start.size() - 1;
    if (forward)
        for (size_t l = 0; l < lines; ++l) solve(l);
    else
        for (size_t l = lines; l-- > 0;) solve(l);
}

// multigrid.rs:329-452
bool coarsen(const Level& fine, const Csr& a, Rect* pout, Level* cout) {
    struct W {
        uint32_t c;
        double w;
    };
    array<vector<array<W, 2>>, 3> map;
    array<vector<double>, 3> planes;
    bool any = false;
    for (int d = 0; d < 3; ++d) {
        const auto& p = fine.planes[d];
        size_t n = p.size();
        vector<size_t> keep;
        if (n <= 2) {
            for (size_t i = 0; i < n; ++i) keep.push_back(i);
        } else {
            any = true;
            for (size_t i = 0; i < n; i += 2) keep.push_back(i);
            if (keep.back() != n - 1) keep.push_back(n - 1);
        }
        for (size_t i : keep) planes[d].push_back(p[i]);
        size_t c = 0;
        map[d].resize(n);
        for (size_t i = 0; i < n; ++i) {
            while (keep[c] < i) ++c;
            if (keep[c] == i) {
                map[d][i] = {W{(uint32_t)c, 1.0}, W{(uint32_t)c, 0.0}};
            } else {
                size_t lo = keep[c - 1], hi = keep[c];
                double w = (p[i] - p[lo]) / (p[hi] - p[lo]);
                map[d][i] = {W{(uint32_t)(c - 1), 1.0 - w}, W{(uint32_t)c, w}};
            }
        }
    }
    if (!any) return false;
    size_t dims[3] = {planes[0].size(), planes[1].size(), planes[2].size()};
    size_t comps = 1;
    for (uint8_t c : fine.comp) comps = std::max(comps, (size_t)c + 1);
    auto flat = [&](const array<uint32_t, 3>& q, uint8_t c) {
        return c + comps * (q[0] + dims[0] * (q[1] + dims[1] * (size_t)q[2]));
    };
    vector<uint32_t> number(comps * dims[0] * dims[1] * dims[2], UINT32_MAX);
    Level coarse;
    coarse.planes = planes;
    Rect p;
    p.rows = fine.points.size();
    p.ptr.push_back(0);
    vector<std::pair<uint32_t, double>> pairs;
    for (size_t row = 0; row < fine.points.size(); ++row) {
        size_t start = p.idx.size();
        const auto& f = fine.points[row];
        uint8_t c = fine.comp[row];
        array<array<W, 2>, 3> weights;
        for (int d = 0; d < 3; ++d) {
            auto w = map[d][f[d]];
            if (w[0].c != w[1].c && comps == 1) {
                double lo = 0.0, hi = 0.0;
                for (size_t k = a.ptr[row]; k < a.ptr[row + 1]; ++k) {
                    const auto& g = fine.points[a.idx[k]];
                    if (g[d] + 1 == f[d])
                        lo -= a.val[k];
                    else if (g[d] == f[d] + 1)
                        hi -= a.val[k];
                }
                if (lo > 0.0 && hi > 0.0) {
                    w[0].w = lo / (lo + hi);
                    w[1].w = hi / (lo + hi);
                }
            }
            weights[d] = w;
        }
        for (const W& x : weights[0])
            for (const W& y : weights[1])
                for (const W& z : weights[2]) {
                    double w = x.w * y.w * z.w;
                    if (w == 0.0) continue;
                    array<uint32_t, 3> q = {x.c, y.c, z.c};
                    uint32_t& slot = number[flat(q, c)];
                    if (slot == UINT32_MAX) {
                        slot = (uint32_t)coarse.points.size();
                        coarse.points.push_back(q);
                        coarse.comp.push_back(c);
                    }
                    p.idx.push_back(slot);
                    p.val.push_back(w);
                }
        pairs.clear();
        for (size_t k = start; k < p.idx.size(); ++k) pairs.push_back({p.idx[k], p.val[k]});
        std::sort(pairs.begin(), pairs.end(),
                  [](const auto& s, const auto& t) { return s.first < t.first; });
        for (size_t k = 0; k < pairs.size(); ++k) {
            p.idx[start + k] = pairs[k].first;
            p.val[start + k] = pairs[k].second;
        }
        p.ptr.push_back(p.idx.size());
    }
    p.cols = coarse.points.size();
    *pout = std::move(p);
    *cout = std::move(coarse);
    return true;
}

static vector<Vec3> level_xyz(const Level& level) {
    vector<Vec3> xyz(level.points.size());
    for (size_t k = 0; k < level.points.size(); ++k)
        for (int d = 0; d < 3; ++d) xyz[k][d] = level.planes[d][level.points[k][d]];
    return xyz;
}

// The local bits of the 8 corners of a cell in VTK order (hex.rs:34-43).
static const int CORNER[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                 {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

// multigrid.rs:616-652: the modes of a coarse cell to keep (3 d + c for the mode along axis d of
// component c): a Cholesky factor of the Gram matrix of each component's 11 functions, corners
// first, skipping a pivot below 1e-6 of its diagonal.
static array<bool, 9> kept_modes(const double gram[3][11][11]) {
    array<bool, 9> keep{};
    for (int c = 0; c < 3; ++c) {
        const auto& g = gram[c];
        double l[11][11] = {};
        bool used[11] = {};
        for (int j = 0; j < 11; ++j) {
            double d = g[j][j];
            for (int k = 0; k < j; ++k)
                if (used[k]) d -= l[j][k] * l[j][k];
            if (!(d > 1e-6 * g[j][j])) continue;
            used[j] = true;
            d = std::sqrt(d);
            l[j][j] = d;
            for (int i = j + 1; i < 11; ++i) {
                double v = g[i][j];
                for (int k = 0; k < j; ++k)
                    if (used[k]) v -= l[i][k] * l[j][k];
                l[i][j] = v / d;
            }
            if (j >= 8) keep[3 * (j - 8) + c] = true;
        }
    }
    return keep;
}

// multigrid.rs:654-681: symmetric Gauss elimination of the kept modes with energy from the
// 33 x 33 matrix `k`; the 24 x 24 block of the corners.
static void condense_modes(double* k, const array<bool, 9>& keep, double* out) {
    for (int m = 24; m < 33; ++m) {
        if (!keep[m - 24]) continue;
        const double pivot = k[m * 33 + m];
        double scale = 0.0;
        for (int i = 0; i < 33; ++i) scale = std::fmax(scale, std::fabs(k[i * 33 + i]));
        if (!(pivot > 1e-12 * scale)) continue;
        for (int i = 0; i < 33; ++i) {
            const double f = k[i * 33 + m] / pivot;
            if (i == m || f == 0.0) continue;
            for (int j = 0; j < 33; ++j) k[i * 33 + j] -= f * k[m * 33 + j];
        }
    }
    for (int r = 0; r < 24; ++r)
        for (int c = 0; c < 24; ++c) out[r * 24 + c] = k[r * 33 + c];
}

// multigrid.rs:458-608. The fine cells of each coarse cell are summed in increasing fine-cell
// order (the reference groups them by an unstable sort, which leaves that order open).
Csr by_cells(const Level& fine, const Cells& cells, const Level& coarse, Cells* next) {
    size_t fd[3], cd[3];
    for (int d = 0; d < 3; ++d) {
        fd[d] = fine.planes[d].size();
        cd[d] = coarse.planes[d].size();
    }
    auto index = [](const array<uint32_t, 3>& q, size_t c, const size_t* dims) {
        return c + 3 * (q[0] + dims[0] * (q[1] + dims[1] * (size_t)q[2]));
    };
    vector<bool> free(3 * fd[0] * fd[1] * fd[2], false);
    for (size_t k = 0; k < fine.points.size(); ++k) free[index(fine.points[k], fine.comp[k], fd)] = true;
    vector<uint32_t> number(3 * cd[0] * cd[1] * cd[2], UINT32_MAX);
    for (size_t k = 0; k < coarse.points.size(); ++k)
        number[index(coarse.points[k], coarse.comp[k], cd)] = (uint32_t)k;
    // The kept planes of each axis (multigrid.rs:341-346) and the coarse cell of each fine one.
    array<vector<uint32_t>, 3> interval;
    for (int d = 0; d < 3; ++d) {
        vector<size_t> keep;
        if (fd[d] <= 2) {
            for (size_t i = 0; i < fd[d]; ++i) keep.push_back(i);
        } else {
            for (size_t i = 0; i < fd[d]; i += 2) keep.push_back(i);
            if (keep.back() != fd[d] - 1) keep.push_back(fd[d] - 1);
        }
        size_t c = 0;
        for (size_t i = 0; i < fd[d]; ++i) {
            while (c + 2 < keep.size() && keep[c + 1] <= i) ++c;
            interval[d].push_back((uint32_t)c);
        }
    }
    const size_t nf = cells.origin.size();
    vector<std::pair<uint32_t, array<uint32_t, 3>>> order(nf);
    for (size_t f = 0; f < nf; ++f) {
        const auto& o = cells.origin[f];
        order[f] = {(uint32_t)f, {interval[0][o[0]], interval[1][o[1]], interval[2][o[2]]}};
    }
    std::stable_sort(order.begin(), order.end(), [](const auto& a, const auto& b) {
        return std::tie(a.second[2], a.second[1], a.second[0]) <
               std::tie(b.second[2], b.second[1], b.second[0]);
    });
    next->origin.clear();
    next->cls.clear();
    next->table.clear();
    vector<double> k(33 * 33);
    size_t start = 0;
    while (start < order.size()) {
        const auto cc = order[start].second;
        size_t end = start;
        while (end < order.size() && order[end].second == cc) ++end;
        double lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
            lo[d] = coarse.planes[d][cc[d]];
            hi[d] = coarse.planes[d][cc[d] + 1];
        }
        std::fill(k.begin(), k.end(), 0.0);
        double gram[3][11][11] = {};
        for (size_t t = start; t < end; ++t) {
            const uint32_t f = order[t].first;
            const double* kf = cells.element(f);
            const auto& o = cells.origin[f];
            double phi[8][3][11] = {};
            for (int n = 0; n < 8; ++n) {
                array<uint32_t, 3> q;
                double xi[3];
                for (int d = 0; d < 3; ++d) {
                    q[d] = o[d] + (uint32_t)CORNER[n][d];
                    xi[d] = 2.0 * (fine.planes[d][q[d]] - lo[d]) / (hi[d] - lo[d]) - 1.0;
                }
                double corner[8];
                for (int m = 0; m < 8; ++m) {  // hex.rs:164-178
                    double v = 1.0;
                    for (int d = 0; d < 3; ++d)
                        v *= CORNER[m][d] == 1 ? 0.5 * (1.0 + xi[d]) : 0.5 * (1.0 - xi[d]);
                    corner[m] = v;
                }
                for (int c = 0; c < 3; ++c) {
                    if (!free[index(q, c, fd)]) continue;
                    double* fn = phi[n][c];
                    for (int m = 0; m < 8; ++m) fn[m] = corner[m];
                    for (int d = 0; d < 3; ++d) fn[8 + d] = 1.0 - xi[d] * xi[d];
                    for (int a = 0; a < 11; ++a)
                        for (int b = 0; b < 11; ++b) gram[c][a][b] += fn[a] * fn[b];
                }
            }
            double kt[24][33] = {};  // Kf T
            for (int r = 0; r < 24; ++r)
                for (int m = 0; m < 8; ++m)
                    for (int c = 0; c < 3; ++c) {
                        const double v = kf[r * 24 + 3 * m + c];
                        if (v != 0.0)
                            for (int a = 0; a < 11; ++a) kt[r][3 * a + c] += v * phi[m][c][a];
                    }
            for (int n = 0; n < 8; ++n)  // K += T^T kt
                for (int c = 0; c < 3; ++c)
                    for (int a = 0; a < 11; ++a) {
                        const double w = phi[n][c][a];
                        if (w == 0.0) continue;
                        double* out = k.data() + (3 * a + c) * 33;
                        for (int j = 0; j < 33; ++j) out[j] += w * kt[3 * n + c][j];
                    }
        }
        const size_t at = next->table.size();
        next->table.resize(at + 576);
        condense_modes(k.data(), kept_modes(gram), next->table.data() + at);
        next->cls.push_back((uint32_t)next->origin.size());
        next->origin.push_back(cc);
        start = end;
    }
    // Assemble on the coarse unknowns (the kept corners of each coarse cell).
    const size_t ncells = next->origin.size();
    vector<vector<std::pair<int, uint32_t>>> ids(ncells);
    vector<uint32_t> globals;
    vector<size_t> gstart{0};
    for (size_t e = 0; e < ncells; ++e) {
        for (int n = 0; n < 8; ++n) {
            array<uint32_t, 3> q;
            for (int d = 0; d < 3; ++d) q[d] = next->origin[e][d] + (uint32_t)CORNER[n][d];
            for (int c = 0; c < 3; ++c) {
                const uint32_t g = number[index(q, c, cd)];
                if (g != UINT32_MAX) ids[e].push_back({3 * n + c, g});
            }
        }
        for (const auto& rg : ids[e]) globals.push_back(rg.second);
        gstart.push_back(globals.size());
    }
    Csr a = pattern_lists(coarse.points.size(), globals, gstart);
    vector<double> ke;
    for (size_t e = 0; e < ncells; ++e) {
        ke.clear();
        const double* m = next->table.data() + 576 * e;
        for (const auto& r : ids[e])
            for (const auto& c : ids[e]) ke.push_back(m[r.first * 24 + c.first]);
        a.add_element(globals.data() + gstart[e], (int)ids[e].size(), ke.data());
    }
    return a;
}

// multigrid.rs:84-139.
Multigrid Multigrid::make(const Csr& a0, Level level, const Cells* cells) {
    Multigrid mg;
    mg.a.push_back(a0);
    Cells stored;
    bool have = false;
    for (;;) {
        const Csr& a = mg.a.back();
        if (a.n <= COARSEST || mg.p.size() >= 30) break;
        Rect p;
        Level coarse;
        if (!coarsen(level, a, &p, &coarse)) break;
        if (coarse.points.size() * 10 > a.n * 9) break;
        mg.lines.push_back({Lines::make(level, 0, a), Lines::make(level, 1, a),
                            Lines::make(level, 2, a)});
        Csr ac;
        if (cells && !cells->empty()) {
            Cells nxt;
            ac = by_cells(level, have ? stored : *cells, coarse, &nxt);
            stored = std::move(nxt);
            have = true;
        } else {
            ac = p.galerkin(a);
        }
        mg.a.push_back(std::move(ac));
        mg.p.push_back(std::move(p));
        level = std::move(coarse);
    }
    const Csr& a = mg.a.back();
    Symbolic sym = analyse(a, nested_dissection(a, level_xyz(level)));
    mg.coarse = factor(sym, a);
    return mg;
}

// multigrid.rs:147-149
void Multigrid::apply(const double* r, double* z) const { cycle(0, r, z); }

// multigrid.rs:151-179
void Multigrid::cycle(size_t l, const double* b, double* x) const {
    if (l + 1 == a.size()) {
        std::copy(b, b + a[l].n, x);
        coarse.solve(x);
        return;
    }
    const Csr& A = a[l];
    const Rect& P = p[l];
    std::fill(x, x + A.n, 0.0);
    for (int d = 0; d < 3; ++d) lines[l][d].sweep(A, b, x, true);
    vector<double> r(A.n);
    A.mul(x, r.data());
    for (size_t i = 0; i < A.n; ++i) r[i] = b[i] - r[i];
    vector<double> rc(P.cols), ec(P.cols);
    P.mul_transpose(r.data(), rc.data());
    cycle(l + 1, rc.data(), ec.data());
    P.mul(ec.data(), r.data());
    for (size_t i = 0; i < A.n; ++i) x[i] += r[i];
    for (int d = 3; d-- > 0;) lines[l][d].sweep(A, b, x, false);
}

static double dot(const double* u, const double* v, size_t n) {
    if (n == 0) return -0.0;
    const size_t t = (size_t)threads();
    if (t > 1 && n >= 65536) {
        // The all-cores baseline: fixed chunks, their sums added in chunk order.
        std::vector<double> part(t, 0.0);
        std::vector<std::thread> pool;
        for (size_t k = 0; k < t; ++k)
            pool.emplace_back([&, k] {
                double s = 0.0;
                for (size_t i = n * k / t; i < n * (k + 1) / t; ++i) s += u[i] * v[i];
                part[k] = s;
            });
        for (auto& th : pool) th.join();
        double s = 0.0;
        for (double p : part) s += p;
        return s;
    }
    double s = u[0] * v[0];
    for (size_t i = 1; i < n; ++i) s += u[i] * v[i];
    return s;
}

// multigrid.rs:692-753
Convergence pcg(const Csr& a, const double* b, double* x,
                const std::function<void(const double*, double*)>& precondition, double tol,
                size_t max_iter, const std::function<bool()>& cancelled) {
    size_t n = a.n;
    double norm_b = std::sqrt(dot(b, b, n));
    if (norm_b == 0.0) {
        std::fill(x, x + n, 0.0);
        return {0, 0.0};
    }
    vector<double> r(n), z(n, 0.0), q(n, 0.0);
    a.mul(x, r.data());
    for (size_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
    precondition(r.data(), z.data());
    vector<double> p(z);
    double rz = dot(r.data(), z.data(), n);
    for (size_t it = 0; it <= max_iter; ++it) {
        double residual = std::sqrt(dot(r.data(), r.data(), n)) / norm_b;
        if (residual <= tol) return {it, residual};
        if (it == max_iter) {
            char buf[200];
            std::snprintf(buf, sizeof buf,
                          "conjugate gradients did not converge: the residual is %s after %zu "
                          "iterations",
                          rust_lower_exp(residual, 2).c_str(), max_iter);
            throw Error(buf);
        }
        if (cancelled()) throw Error("cancelled");
        a.mul(p.data(), q.data());
        double alpha = rz / dot(p.data(), q.data(), n);
        for (size_t i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
        }
        precondition(r.data(), z.data());
        double rz_new = dot(r.data(), z.data(), n);
        double beta = rz_new / rz;
        rz = rz_new;
        for (size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    throw Error("the loop returns");
}

// pmultigrid.rs:33
static const int SWEEPS = 2;

// pmultigrid.rs:46-60
PMultigrid PMultigrid::make(const Csr& a, Rect p, const vector<Vec3>& coarse) {
    PMultigrid mg;
    Csr ac = p.galerkin(a);
    Symbolic sym = analyse(ac, nested_dissection(ac, coarse));
    mg.coarse = factor(sym, ac);
    mg.diag = a.diagonal();
    for (double d : mg.diag)
        if (!(d > 0.0)) throw Error("the matrix has a diagonal entry that is not above 0");
    mg.coarse_unknowns = p.cols;
    mg.p = std::move(p);
    return mg;
}

// pmultigrid.rs:63-98
void PMultigrid::apply(const Csr& a, const double* r, double* z) const {
    size_t n = a.n;
    std::fill(z, z + n, 0.0);
    auto row = [&](size_t i) {
        double s = r[i];
        for (size_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
            size_t j = a.idx[k];
            if (j != i) s -= a.val[k] * z[j];
        }
        return s / diag[i];
    };
    for (int s = 0; s < SWEEPS; ++s)
        for (size_t i = 0; i < n; ++i) z[i] = row(i);
    vector<double> az(n);
    a.mul(z, az.data());
    vector<double> res(n);
    for (size_t i = 0; i < n; ++i) res[i] = r[i] - az[i];
    vector<double> rc(p.cols);
    p.mul_transpose(res.data(), rc.data());
    coarse.solve(rc.data());
    p.mul(rc.data(), az.data());
    for (size_t i = 0; i < n; ++i) z[i] += az[i];
    for (int s = 0; s < SWEEPS; ++s)
        for (size_t i = n; i-- > 0;) z[i] = row(i);
}

// pmultigrid.rs:104-151
void prolongation(const vector<Vec3>& points, size_t corners,
                  const vector<array<uint32_t, 2>>& edges, const vector<size_t>& free, Rect* pout,
                  vector<Vec3>* xyz) {
    vector<uint32_t> coarse(3 * corners, UINT32_MAX);
    xyz->clear();
    for (size_t i : free)
        if (i < 3 * corners) {
            coarse[i] = (uint32_t)xyz->size();
            xyz->push_back(points[i / 3]);
        }
    Rect p;
    p.rows = free.size();
    p.ptr.push_back(0);
    for (size_t i : free) {
        size_t v = i / 3, c = i % 3;
        if (v < corners) {
            p.idx.push_back(coarse[i]);
            p.val.push_back(1.0);
        } else {
            vector<uint32_t> ends;
            for (uint32_t a : edges[v - corners]) {
                uint32_t k = coarse[3 * (size_t)a + c];
                if (k != UINT32_MAX) ends.push_back(k);
            }
            std::sort(ends.begin(), ends.end());
            for (uint32_t k : ends) {
                p.idx.push_back(k);
                p.val.push_back(0.5);
            }
        }
        p.ptr.push_back(p.idx.size());
    }
    p.cols = xyz->size();
    *pout = std::move(p);
}

// solve.rs:92-183
Solver Solver::make(Csr a, Unknowns unknowns, int method, Crossover crossover) {
    Solver s;
    auto choose_direct = [&](const std::function<Symbolic()>& symbolic, Symbolic* out) {
        if (method == (int)Method::Direct) {
            *out = symbolic();
            return true;
        }
        if (method == (int)Method::Multigrid) return false;
        if (!crossover.flops_rule) {
            if (a.n <= crossover.unknowns) {
                *out = symbolic();
                return true;
            }
            return false;
        }
        Symbolic sym = symbolic();
        if (sym.entries() <= crossover.entries &&
            (crossover.flat || sym.flops() <= crossover.flops * (double)a.n)) {
            *out = std::move(sym);
            return true;
        }
        return false;
    };
    if (unknowns.kind == Unknowns::Quadratic) {
        Symbolic sym;
        bool direct = choose_direct(
            [&] { return analyse(a, nested_dissection(a, unknowns.points)); }, &sym);
        if (direct) {
            s.chol = factor(sym, a);
            s.inner = Direct;
        } else {
            s.pmg = PMultigrid::make(a, std::move(unknowns.p), unknowns.coarse);
            s.inner = PMG;
        }
        s.a = std::move(a);
        return s;
    }
    if (unknowns.kind == Unknowns::Points) {
        if (method == (int)Method::Multigrid)
            throw Error("multigrid needs the box grid: a mesh of tetrahedra has the direct solver");
        Symbolic sym = analyse(a, nested_dissection(a, unknowns.points));
        s.chol = factor(sym, a);
        s.inner = Direct;
        s.a = std::move(a);
        return s;
    }
    Symbolic sym;
    bool direct = choose_direct(
        [&] { return analyse(a, nested_dissection(a, level_xyz(unknowns.level))); }, &sym);
    if (direct) {
        s.chol = factor(sym, a);
        s.inner = Direct;
    } else {
        s.mg = Multigrid::make(a, std::move(unknowns.level), &unknowns.cells);
        s.inner = MG;
    }
    s.a = std::move(a);
    return s;
}

// solve.rs:199-250
Stats Solver::solve(const double* b, double* x, const std::function<bool()>& cancelled) const {
    size_t n = a.n;
    if (inner == Direct) {
        std::copy(b, b + n, x);
        chol.solve(x);
        vector<double> ax(n);
        a.mul(x, ax.data());
        double bn = 0, rn = 0;
        if (n) {
            bn = b[0] * b[0];
            double d = b[0] - ax[0];
            rn = d * d;
        } else {
            bn = rn = -0.0;
        }
        for (size_t i = 1; i < n; ++i) {
            bn += b[i] * b[i];
            double d = b[i] - ax[i];
            rn += d * d;
        }
        bn = std::sqrt(bn);
        rn = std::sqrt(rn);
        return {0, bn > 0.0 ? rn / bn : rn};
    }
    Convergence c;
    if (inner == MG)
        c = pcg(a, b, x, [&](const double* r, double* z) { mg.apply(r, z); }, tol, max_iter,
                cancelled);
    else
        c = pcg(a, b, x, [&](const double* r, double* z) { pmg.apply(a, r, z); }, tol, max_iter,
                cancelled);
    return {c.iterations, c.residual};
}

}  // namespace orc
