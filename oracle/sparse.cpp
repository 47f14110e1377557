// Oracle (test infrastructure): restatement of crates/fem/src/sparse.rs.
#include <algorithm>
#include <numeric>
#include <thread>

#include "oracle.hpp"

namespace orc {

// sparse.rs:22-65. Counting sort of the elements of each node, then for each row a mark
// de-duplication of the nodes of its elements, plus the row itself, and a sort. Element k is
// nodes[start[k] .. start[k + 1]].
Csr pattern_lists(size_t n, const vector<uint32_t>& nodes, const vector<size_t>& start) {
    const size_t nel = start.size() - 1;
    vector<size_t> count(n + 1, 0);
    for (uint32_t v : nodes) count[v + 1] += 1;
    for (size_t i = 0; i < n; ++i) count[i + 1] += count[i];
    vector<uint32_t> of_node(count[n]);
    vector<size_t> next(count);
    for (size_t k = 0; k < nel; ++k)
        for (size_t t = start[k]; t < start[k + 1]; ++t) {
            uint32_t v = nodes[t];
            of_node[next[v]] = (uint32_t)k;
            next[v] += 1;
        }
    Csr out;
    out.n = n;
    out.ptr.reserve(n + 1);
    out.ptr.push_back(0);
    vector<size_t> mark(n, SIZE_MAX);
    vector<uint32_t> row;
    for (size_t i = 0; i < n; ++i) {
        row.clear();
        mark[i] = i;
        row.push_back((uint32_t)i);
        for (size_t t = count[i]; t < count[i + 1]; ++t) {
            const size_t k = of_node[t];
            for (size_t b = start[k]; b < start[k + 1]; ++b) {
                uint32_t v = nodes[b];
                if (mark[v] != i) {
                    mark[v] = i;
                    row.push_back(v);
                }
            }
        }
        std::sort(row.begin(), row.end());
        out.idx.insert(out.idx.end(), row.begin(), row.end());
        out.ptr.push_back(out.idx.size());
    }
    out.val.assign(out.idx.size(), 0.0);
    return out;
}

Csr pattern(size_t n, const uint32_t* elements, size_t nel, int m) {
    vector<size_t> count(n + 1, 0);
    for (size_t e = 0; e < nel; ++e)
        for (int a = 0; a < m; ++a) count[elements[e * m + a] + 1] += 1;
    for (size_t i = 0; i < n; ++i) count[i + 1] += count[i];
    vector<uint32_t> of_node(count[n]);
    vector<size_t> next(count);
    for (size_t k = 0; k < nel; ++k)
        for (int a = 0; a < m; ++a) {
            uint32_t v = elements[k * m + a];
            of_node[next[v]] = (uint32_t)k;
            next[v] += 1;
        }
    Csr out;
    out.n = n;
    out.ptr.reserve(n + 1);
    out.ptr.push_back(0);
    vector<size_t> mark(n, SIZE_MAX);
    vector<uint32_t> row;
    for (size_t i = 0; i < n; ++i) {
        row.clear();
        mark[i] = i;
        row.push_back((uint32_t)i);
        for (size_t t = count[i]; t < count[i + 1]; ++t) {
            const uint32_t* el = elements + (size_t)of_node[t] * m;
            for (int b = 0; b < m; ++b) {
                uint32_t v = el[b];
                if (mark[v] != i) {
                    mark[v] = i;
                    row.push_back(v);
                }
            }
        }
        std::sort(row.begin(), row.end());
        out.idx.insert(out.idx.end(), row.begin(), row.end());
        out.ptr.push_back(out.idx.size());
    }
    out.val.assign(out.idx.size(), 0.0);
    return out;
}

// sparse.rs:68-71
bool Csr::find(size_t i, size_t j, size_t* at) const {
    auto b = idx.begin() + ptr[i], e = idx.begin() + ptr[i + 1];
    auto it = std::lower_bound(b, e, (uint32_t)j);
    if (it == e || *it != (uint32_t)j) return false;
    *at = (size_t)(it - idx.begin());
    return true;
}

// sparse.rs:75-86. Element order and `+=` as in the reference, so each value is the sum of
// its element contributions in increasing element order.
void Csr::add_element(const uint32_t* nodes, int m, const double* ke) {
    for (int a = 0; a < m; ++a) {
        size_t i = nodes[a];
        for (int b = 0; b < m; ++b) {
            size_t k;
            if (!find(i, nodes[b], &k)) throw Error("the pattern holds each element pair");
            val[k] += ke[a * m + b];
        }
    }
}

// sparse.rs:89-93
vector<double> Csr::diagonal() const {
    vector<double> d(n, 0.0);
    for (size_t i = 0; i < n; ++i) {
        size_t k;
        if (find(i, i, &k)) d[i] = val[k];
    }
    return d;
}

// sparse.rs:96-105
static int g_threads = 1;
void set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int threads() { return g_threads; }

// Each row is summed by 1 thread in column order, so the product is the same on any number of
// threads.
void Csr::mul(const double* x, double* y) const {
    auto rows = [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) {
            double s = 0.0;
            for (size_t k = ptr[i]; k < ptr[i + 1]; ++k) s += val[k] * x[idx[k]];
            y[i] = s;
        }
    };
    const size_t t = (size_t)g_threads;
    if (t <= 1 || n < 65536) {
        rows(0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t k = 0; k < t; ++k) pool.emplace_back(rows, n * k / t, n * (k + 1) / t);
    for (auto& th : pool) th.join();
}

// sparse.rs:137-148
static void sort_row(uint32_t* idx, double* val, size_t len) {
    bool sorted = true;
    for (size_t k = 1; k < len; ++k)
        if (!(idx[k - 1] < idx[k])) sorted = false;
    if (sorted) return;
    vector<std::pair<uint32_t, double>> pairs(len);
    for (size_t k = 0; k < len; ++k) pairs[k] = {idx[k], val[k]};
    std::sort(pairs.begin(), pairs.end(),
              [](const auto& p, const auto& q) { return p.first < q.first; });
    for (size_t k = 0; k < len; ++k) {
        idx[k] = pairs[k].first;
        val[k] = pairs[k].second;
    }
}

// sparse.rs:108-135
Csr Csr::submatrix(const vector<size_t>& keep) const {
    vector<uint32_t> fresh(n, UINT32_MAX);
    for (size_t k = 0; k < keep.size(); ++k) fresh[keep[k]] = (uint32_t)k;
    Csr out;
    out.n = keep.size();
    out.ptr.reserve(keep.size() + 1);
    out.ptr.push_back(0);
    for (size_t i : keep) {
        size_t start = out.idx.size();
        for (size_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            uint32_t j = fresh[idx[k]];
            if (j != UINT32_MAX) {
                out.idx.push_back(j);
                out.val.push_back(val[k]);
            }
        }
        sort_row(out.idx.data() + start, out.val.data() + start, out.idx.size() - start);
        out.ptr.push_back(out.idx.size());
    }
    return out;
}

// sparse.rs:212-220
void Rect::mul(const double* x, double* y) const {
    for (size_t i = 0; i < rows; ++i) {
        double s = 0.0;
        for (size_t k = ptr[i]; k < ptr[i + 1]; ++k) s += val[k] * x[idx[k]];
        y[i] = s;
    }
}

// sparse.rs:223-230
void Rect::mul_transpose(const double* x, double* y) const {
    std::fill(y, y + cols, 0.0);
    for (size_t i = 0; i < rows; ++i)
        for (size_t k = ptr[i]; k < ptr[i + 1]; ++k) y[idx[k]] += val[k] * x[i];
}

// sparse.rs:233-292: the transpose of P by counting sort, then Gustavson's method with a dense
// accumulator for each coarse row.
Csr Rect::galerkin(const Csr& a) const {
    size_t nc = cols;
    vector<size_t> tptr(nc + 1, 0);
    for (uint32_t j : idx) tptr[j + 1] += 1;
    for (size_t j = 0; j < nc; ++j) tptr[j + 1] += tptr[j];
    vector<uint32_t> tidx(idx.size());
    vector<double> tval(idx.size());
    vector<size_t> next(tptr);
    for (size_t i = 0; i < rows; ++i)
        for (size_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            size_t j = idx[k];
            tidx[next[j]] = (uint32_t)i;
            tval[next[j]] = val[k];
            next[j] += 1;
        }
    vector<double> acc(nc, 0.0);
    vector<size_t> mark(nc, SIZE_MAX);
    Csr out;
    out.n = nc;
    out.ptr.reserve(nc + 1);
    out.ptr.push_back(0);
    vector<uint32_t> row;
    for (size_t c = 0; c < nc; ++c) {
        row.clear();
        for (size_t t = tptr[c]; t < tptr[c + 1]; ++t) {
            size_t i = tidx[t];
            double pic = tval[t];
            for (size_t ka = a.ptr[i]; ka < a.ptr[i + 1]; ++ka) {
                size_t l = a.idx[ka];
                double aval = a.val[ka] * pic;
                for (size_t kp = ptr[l]; kp < ptr[l + 1]; ++kp) {
                    size_t d = idx[kp];
                    if (mark[d] != c) {
                        mark[d] = c;
                        acc[d] = 0.0;
                        row.push_back((uint32_t)d);
                    }
                    acc[d] += aval * val[kp];
                }
            }
        }
        std::sort(row.begin(), row.end());
        for (uint32_t d : row) {
            out.idx.push_back(d);
            out.val.push_back(acc[d]);
        }
        out.ptr.push_back(out.idx.size());
    }
    return out;
}

}  // namespace orc
