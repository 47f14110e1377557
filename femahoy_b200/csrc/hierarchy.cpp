// Host setup steps of the multigrid hierarchy (see hierarchy.hpp): the coarse matrices from the
// cells, the crossover's counts, the P2 -> P1 prolongation and the grid level of points.
// Compiled with -ffp-contract=off so that the cells' coarse matrices are formed with the
// reference's roundings.
#include "hierarchy.hpp"

#include <algorithm>
#include <cmath>
#include <map>
#include <thread>
#include <tuple>

namespace femgpu {

int host_threads() {
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)std::min(h, 64u) : 1;
}

// ------------------------------------------------------------------ cells (multigrid.rs:458)
namespace {

const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                           {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};  // hex.rs:34-43

size_t grid_index(const std::array<uint32_t, 3>& q, size_t c, const size_t* dims) {
    return c + 3 * (q[0] + dims[0] * (q[1] + dims[1] * (size_t)q[2]));
}

// multigrid.rs:616-652: per component, a Cholesky factor of the Gram matrix of the 11 fields
// that skips the pivots below 1e-6 of their diagonal; a mode whose pivot stays is kept.
std::array<bool, 9> keep_modes(const double (*gram)[11][11]) {
    std::array<bool, 9> keep{};
    for (int c = 0; c < 3; ++c) {
        double l[11][11] = {};
        bool used[11] = {};
        for (int j = 0; j < 11; ++j) {
            double d = gram[c][j][j];
            for (int k = 0; k < j; ++k)
                if (used[k]) d -= l[j][k] * l[j][k];
            if (!(d > 1e-6 * gram[c][j][j])) continue;
            used[j] = true;
            d = std::sqrt(d);
            l[j][j] = d;
            for (int i = j + 1; i < 11; ++i) {
                double v = gram[c][i][j];
                for (int k = 0; k < j; ++k)
                    if (used[k]) v -= l[i][k] * l[j][k];
                l[i][j] = v / d;
            }
            if (j >= 8) keep[3 * (j - 8) + c] = true;
        }
    }
    return keep;
}

// multigrid.rs:654-681: symmetric elimination of the kept modes with energy; the corner block.
void condense33(double* k, const std::array<bool, 9>& keep, double* out) {
    for (int m = 24; m < 33; ++m) {
        if (!keep[m - 24]) continue;
        const double pivot = k[m * 33 + m];
        double scale = 0.0;
        for (int i = 0; i < 33; ++i) scale = std::fmax(scale, std::fabs(k[i * 33 + i]));
        if (!(pivot > 1e-12 * scale)) continue;
        for (int i = 0; i < 33; ++i) {
            const double f = k[i * 33 + m] / pivot;
            if (i == m || f == 0.0) continue;
            const double* km = k + m * 33;
            double* ki = k + i * 33;
            for (int j = 0; j < 33; ++j) ki[j] -= f * km[j];
        }
    }
    for (int r = 0; r < 24; ++r)
        for (int c = 0; c < 24; ++c) out[r * 24 + c] = k[r * 33 + c];
}

}  // namespace

HostCsr by_cells(const HostLevel& fine, const HostCells& cells, const HostLevel& coarse,
                 HostCells* next, int threads) {
    size_t fd[3], cd[3];
    for (int d = 0; d < 3; ++d) {
        fd[d] = fine.planes[d].size();
        cd[d] = coarse.planes[d].size();
    }
    std::vector<uint8_t> free(3 * fd[0] * fd[1] * fd[2], 0);
    for (size_t k = 0; k < fine.points.size(); ++k)
        free[grid_index(fine.points[k], fine.comp[k], fd)] = 1;
    std::vector<uint32_t> number(3 * cd[0] * cd[1] * cd[2], UINT32_MAX);
    for (size_t k = 0; k < coarse.points.size(); ++k)
        number[grid_index(coarse.points[k], coarse.comp[k], cd)] = (uint32_t)k;
    // The coarse cell of each fine plane interval along each axis: the planes kept by the
    // coarsening are every other one and the last (multigrid.rs:341-346, 491-502).
    std::array<std::vector<uint32_t>, 3> interval;
    for (int d = 0; d < 3; ++d) {
        std::vector<size_t> keep;
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
    // The fine cells grouped by coarse cell in (z, y, x) order, each group in increasing fine
    // order: a counting sort on the coarse cell's index.
    const size_t nf = cells.origin.size();
    const size_t ncc = (cd[0] - 1) * (cd[1] - 1) * (cd[2] - 1);
    std::vector<uint32_t> of(nf);
    std::vector<size_t> count(ncc + 1, 0);
    for (size_t f = 0; f < nf; ++f) {
        const auto& o = cells.origin[f];
        of[f] = interval[0][o[0]] +
                (uint32_t)((cd[0] - 1) * (interval[1][o[1]] + (cd[1] - 1) * interval[2][o[2]]));
        count[of[f] + 1] += 1;
    }
    for (size_t c = 0; c < ncc; ++c) count[c + 1] += count[c];
    std::vector<uint32_t> member(nf);
    {
        std::vector<size_t> at(count.begin(), count.end() - 1);
        for (size_t f = 0; f < nf; ++f) member[at[of[f]]++] = (uint32_t)f;
    }
    std::vector<uint32_t> groups;  // the coarse cells that hold fine cells, in order
    for (size_t c = 0; c < ncc; ++c)
        if (count[c + 1] > count[c]) groups.push_back((uint32_t)c);
    const size_t ng = groups.size();
    next->origin.resize(ng);
    next->cls.resize(ng);
    next->table.assign(576 * ng, 0.0);
    for (size_t g = 0; g < ng; ++g) {
        const uint32_t c = groups[g];
        next->origin[g] = {(uint32_t)(c % (cd[0] - 1)),
                           (uint32_t)(c / (cd[0] - 1) % (cd[1] - 1)),
                           (uint32_t)(c / ((cd[0] - 1) * (cd[1] - 1)))};
        next->cls[g] = (uint32_t)g;
    }
    // Each coarse cell's matrix: kt = Kf T for each fine cell, K += T^T kt (multigrid.rs:
    // 533-569), then the mode selection and the condensation.
    auto work = [&](size_t g0, size_t g1) {
        std::vector<double> k(33 * 33);
        for (size_t g = g0; g < g1; ++g) {
            const auto& cc = next->origin[g];
            double lo[3], hi[3];
            for (int d = 0; d < 3; ++d) {
                lo[d] = coarse.planes[d][cc[d]];
                hi[d] = coarse.planes[d][cc[d] + 1];
            }
            std::fill(k.begin(), k.end(), 0.0);
            double gram[3][11][11] = {};
            const uint32_t c = groups[g];
            for (size_t t = count[c]; t < count[c + 1]; ++t) {
                const uint32_t f = member[t];
                const double* kf = cells.table.data() + 576 * (size_t)cells.cls[f];
                const auto& o = cells.origin[f];
                double phi[8][3][11] = {};
                for (int n = 0; n < 8; ++n) {
                    std::array<uint32_t, 3> q;
                    double xi[3];
                    for (int d = 0; d < 3; ++d) {
                        q[d] = o[d] + (uint32_t)kCorner[n][d];
                        xi[d] = 2.0 * (fine.planes[d][q[d]] - lo[d]) / (hi[d] - lo[d]) - 1.0;
                    }
                    double corner[8];
                    for (int m = 0; m < 8; ++m) {  // hex.rs:164-178
                        double v = 1.0;
                        for (int d = 0; d < 3; ++d)
                            v *= kCorner[m][d] == 1 ? 0.5 * (1.0 + xi[d]) : 0.5 * (1.0 - xi[d]);
                        corner[m] = v;
                    }
                    for (int cmp = 0; cmp < 3; ++cmp) {
                        if (!free[grid_index(q, cmp, fd)]) continue;
                        double* fn = phi[n][cmp];
                        for (int m = 0; m < 8; ++m) fn[m] = corner[m];
                        for (int d = 0; d < 3; ++d) fn[8 + d] = 1.0 - xi[d] * xi[d];
                        for (int a = 0; a < 11; ++a)
                            for (int b = 0; b < 11; ++b) gram[cmp][a][b] += fn[a] * fn[b];
                    }
                }
                double kt[24][33] = {};
                for (int r = 0; r < 24; ++r)
                    for (int m = 0; m < 8; ++m)
                        for (int cmp = 0; cmp < 3; ++cmp) {
                            const double v = kf[r * 24 + 3 * m + cmp];
                            if (v != 0.0)
                                for (int a = 0; a < 11; ++a)
                                    kt[r][3 * a + cmp] += v * phi[m][cmp][a];
                        }
                for (int n = 0; n < 8; ++n)
                    for (int cmp = 0; cmp < 3; ++cmp)
                        for (int a = 0; a < 11; ++a) {
                            const double w = phi[n][cmp][a];
                            if (w == 0.0) continue;
                            double* out = k.data() + (3 * a + cmp) * 33;
                            const double* row = kt[3 * n + cmp];
                            for (int j = 0; j < 33; ++j) out[j] += w * row[j];
                        }
            }
            condense33(k.data(), keep_modes(gram), next->table.data() + 576 * g);
        }
    };
    threads = std::max(1, std::min<int>(threads, (int)std::max<size_t>(1, ng / 64)));
    {
        std::vector<std::thread> pool;
        for (int t = 1; t < threads; ++t)
            pool.emplace_back(work, ng * t / threads, ng * (t + 1) / threads);
        work(0, ng / threads);
        for (auto& th : pool) th.join();
    }
    // The unknowns of each coarse cell (its corners' free components) and the cells of each
    // coarse unknown, in cell order.
    const size_t nc = coarse.points.size();
    std::vector<uint8_t> nloc(ng, 0);
    std::vector<uint8_t> loc(24 * ng);
    std::vector<uint32_t> glob(24 * ng);
    std::vector<int64_t> rcount(nc + 1, 0);
    for (size_t g = 0; g < ng; ++g) {
        for (int n = 0; n < 8; ++n) {
            std::array<uint32_t, 3> q;
            for (int d = 0; d < 3; ++d) q[d] = next->origin[g][d] + (uint32_t)kCorner[n][d];
            for (int cmp = 0; cmp < 3; ++cmp) {
                const uint32_t id = number[grid_index(q, cmp, cd)];
                if (id == UINT32_MAX) continue;
                loc[24 * g + nloc[g]] = (uint8_t)(3 * n + cmp);
                glob[24 * g + nloc[g]] = id;
                nloc[g] += 1;
                rcount[id + 1] += 1;
            }
        }
    }
    for (size_t i = 0; i < nc; ++i) rcount[i + 1] += rcount[i];
    std::vector<uint32_t> rcell(rcount[nc]);
    std::vector<uint8_t> rslot(rcount[nc]);
    {
        std::vector<int64_t> at(rcount.begin(), rcount.end() - 1);
        for (size_t g = 0; g < ng; ++g)
            for (int s = 0; s < nloc[g]; ++s) {
                const uint32_t id = glob[24 * g + s];
                rcell[at[id]] = (uint32_t)g;
                rslot[at[id]] = (uint8_t)s;
                at[id] += 1;
            }
    }
    // Csr::pattern (each row: itself and the unknowns of its cells, sorted) and add_element in
    // cell order, row by row (sparse.rs:22-86): each entry sums its cells in increasing order.
    HostCsr a;
    a.n = (int64_t)nc;
    std::vector<int64_t> len(nc);
    auto rows = [&](size_t i0, size_t i1, bool fill) {
        std::vector<uint32_t> row;
        std::vector<int64_t> mark(nc, -1);
        for (size_t i = i0; i < i1; ++i) {
            row.clear();
            row.push_back((uint32_t)i);
            mark[i] = (int64_t)i;
            for (int64_t t = rcount[i]; t < rcount[i + 1]; ++t) {
                const size_t g = rcell[t];
                for (int s = 0; s < nloc[g]; ++s) {
                    const uint32_t j = glob[24 * g + s];
                    if (mark[j] != (int64_t)i) {
                        mark[j] = (int64_t)i;
                        row.push_back(j);
                    }
                }
            }
            std::sort(row.begin(), row.end());
            if (!fill) {
                len[i] = (int64_t)row.size();
                continue;
            }
            const int64_t base = a.ptr[i];
            for (size_t k = 0; k < row.size(); ++k) {
                a.idx[base + k] = row[k];
                a.val[base + k] = 0.0;
            }
            for (int64_t t = rcount[i]; t < rcount[i + 1]; ++t) {
                const size_t g = rcell[t];
                const double* m = next->table.data() + 576 * g;
                const int r = loc[24 * g + rslot[t]];
                for (int s = 0; s < nloc[g]; ++s) {
                    const uint32_t j = glob[24 * g + s];
                    const int64_t at =
                        std::lower_bound(row.begin(), row.end(), j) - row.begin() + base;
                    a.val[at] += m[r * 24 + loc[24 * g + s]];
                }
            }
        }
    };
    auto split = [&](bool fill) {
        int tr = std::max(1, std::min<int>(threads, (int)std::max<size_t>(1, nc / 256)));
        std::vector<std::thread> pool;
        for (int t = 1; t < tr; ++t)
            pool.emplace_back(rows, nc * t / tr, nc * (t + 1) / tr, fill);
        rows(0, nc / tr, fill);
        for (auto& th : pool) th.join();
    };
    split(false);
    a.ptr.assign(nc + 1, 0);
    for (size_t i = 0; i < nc; ++i) a.ptr[i + 1] = a.ptr[i] + len[i];
    a.idx.assign(a.ptr[nc], 0);
    a.val.assign(a.ptr[nc], 0.0);
    split(true);
    return a;
}

void prolongation(const double* points, int64_t npoints, int64_t corners, const uint32_t* edges,
                  int64_t nedges, const int64_t* free, int64_t nfree, HostRect* pout,
                  std::vector<double>* xyz) {
    (void)npoints;
    (void)nedges;
    // The coarse unknown of each free corner unknown (pmultigrid.rs:110-118).
    std::vector<uint32_t> coarse(3 * (size_t)corners, UINT32_MAX);
    xyz->clear();
    uint32_t nc = 0;
    for (int64_t k = 0; k < nfree; ++k) {
        int64_t i = free[k];
        if (i < 3 * corners) {
            coarse[i] = nc++;
            for (int d = 0; d < 3; ++d) xyz->push_back(points[3 * (i / 3) + d]);
        }
    }
    HostRect p;
    p.rows = nfree;
    p.ptr.reserve(nfree + 1);
    p.ptr.push_back(0);
    for (int64_t k = 0; k < nfree; ++k) {
        int64_t i = free[k];
        int64_t v = i / 3, c = i % 3;
        if (v < corners) {
            p.idx.push_back(coarse[i]);
            p.val.push_back(1.0);
        } else {
            // Half of each free corner of the edge (pmultigrid.rs:127-137).
            uint32_t ends[2];
            int ne = 0;
            for (int e = 0; e < 2; ++e) {
                uint32_t a = edges[2 * (v - corners) + e];
                uint32_t q = coarse[3 * (size_t)a + c];
                if (q != UINT32_MAX) ends[ne++] = q;
            }
            if (ne == 2 && ends[1] < ends[0]) std::swap(ends[0], ends[1]);
            for (int e = 0; e < ne; ++e) {
                p.idx.push_back(ends[e]);
                p.val.push_back(0.5);
            }
        }
        p.ptr.push_back((int64_t)p.idx.size());
    }
    p.cols = nc;
    *pout = std::move(p);
}

HostLevel level_of_points(const double* xyz, int64_t n, const uint8_t* comp) {
    HostLevel lv;
    for (int d = 0; d < 3; ++d) {
        std::vector<double> v(n);
        for (int64_t k = 0; k < n; ++k) v[k] = xyz[3 * k + d];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        lv.planes[d] = std::move(v);
    }
    lv.points.resize(n);
    lv.comp.resize(n);
    std::map<std::array<uint32_t, 3>, uint8_t> seen;
    for (int64_t k = 0; k < n; ++k) {
        std::array<uint32_t, 3> q;
        for (int d = 0; d < 3; ++d) {
            const auto& pl = lv.planes[d];
            q[d] = (uint32_t)(std::lower_bound(pl.begin(), pl.end(), xyz[3 * k + d]) - pl.begin());
        }
        lv.points[k] = q;
        if (comp) {
            lv.comp[k] = comp[k];
        } else {
            uint8_t& r = seen[q];
            lv.comp[k] = r++;
        }
    }
    return lv;
}

}  // namespace femgpu
