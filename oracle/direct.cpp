// Oracle (test infrastructure): the sparse direct solver, the FP64 direct oracle of each parity
// test. Restates crates/fem/src/order.rs:1-179 (nested dissection),
// crates/fem/src/symbolic.rs:1-266 (elimination tree, postorder, column counts, supernodes)
// and crates/fem/src/cholesky.rs:15-225 (multifrontal supernodal Cholesky).
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "oracle.hpp"

namespace orc {

// ------------------------------------------------------------------ order.rs
static const size_t LEAF = 64;                                  // order.rs:15
static const double CUTS[5] = {0.3, 0.4, 0.5, 0.6, 0.7};        // order.rs:56

// order.rs:143-179
static void separator_size(const Csr& a, const vector<size_t>& set, const vector<Vec3>& xyz,
                           vector<uint8_t>& side, int axis, double cut, size_t* sep,
                           size_t* small) {
    size_t nleft = 0;
    for (size_t v : set) {
        if (xyz[v][axis] < cut) {
            nleft += 1;
            side[v] = 1;
        } else {
            side[v] = 2;
        }
    }
    size_t sl = 0, sr = 0;
    for (size_t v : set) {
        uint8_t mine = side[v], other = 3 - mine;
        bool touches = false;
        for (size_t k = a.ptr[v]; k < a.ptr[v + 1]; ++k)
            if (side[a.idx[k]] == other) {
                touches = true;
                break;
            }
        if (touches) (mine == 1 ? sl : sr) += 1;
    }
    for (size_t v : set) side[v] = 0;
    *sep = std::min(sl, sr);
    *small = std::min(nleft, set.size() - nleft);
}

// order.rs:66-139
static bool split(const Csr& a, const vector<size_t>& set, const vector<Vec3>& xyz,
                  vector<uint8_t>& side, vector<size_t>* left_out, vector<size_t>* right_out,
                  vector<size_t>* sep_out) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t v : set)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::fmin(lo[d], xyz[v][d]);
            hi[d] = std::fmax(hi[d], xyz[v][d]);
        }
    bool have = false;
    double best_cost = 0, best_cut = 0;
    int best_axis = 0;
    vector<double> values;
    for (int axis = 0; axis < 3; ++axis) {
        if (hi[axis] <= lo[axis]) continue;
        values.clear();
        for (size_t v : set) values.push_back(xyz[v][axis]);
        std::sort(values.begin(), values.end());
        for (double q : CUTS) {
            size_t at = std::min((size_t)((double)values.size() * q), values.size() - 1);
            double cut = values[at];
            if (cut <= lo[axis]) {
                bool found = false;
                for (double x : values)
                    if (x > lo[axis]) {
                        cut = x;
                        found = true;
                        break;
                    }
                if (!found) continue;
            }
            size_t sep, small;
            separator_size(a, set, xyz, side, axis, cut, &sep, &small);
            double cost = (double)sep / std::sqrt(2.0 * (double)small / (double)set.size());
            if (!have || cost < best_cost) {
                have = true;
                best_cost = cost;
                best_cut = cut;
                best_axis = axis;
            }
        }
    }
    if (!have) return false;
    vector<size_t> left, right;
    for (size_t v : set) (xyz[v][best_axis] < best_cut ? left : right).push_back(v);
    for (size_t v : left) side[v] = 1;
    for (size_t v : right) side[v] = 2;
    auto touches = [&](size_t v, uint8_t other) {
        for (size_t k = a.ptr[v]; k < a.ptr[v + 1]; ++k)
            if (side[a.idx[k]] == other) return true;
        return false;
    };
    vector<size_t> sep_left, sep_right;
    for (size_t v : left)
        if (touches(v, 2)) sep_left.push_back(v);
    for (size_t v : right)
        if (touches(v, 1)) sep_right.push_back(v);
    for (size_t v : set) side[v] = 0;
    bool from_left = sep_left.size() <= sep_right.size();
    vector<size_t> sep = from_left ? sep_left : sep_right;
    vector<size_t> in_sep(sep);
    std::sort(in_sep.begin(), in_sep.end());
    auto rest = [&](const vector<size_t>& part) {
        vector<size_t> out;
        for (size_t v : part)
            if (!std::binary_search(in_sep.begin(), in_sep.end(), v)) out.push_back(v);
        return out;
    };
    if (from_left) {
        *left_out = rest(left);
        *right_out = right;
    } else {
        *left_out = left;
        *right_out = rest(right);
    }
    *sep_out = sep;
    return true;
}

// order.rs:19-52
vector<size_t> nested_dissection(const Csr& a, const vector<Vec3>& xyz) {
    if (a.n != xyz.size()) throw Error("1 point for each node");
    vector<size_t> order;
    order.reserve(a.n);
    vector<uint8_t> side(a.n, 0);
    struct Work {
        bool emit;
        vector<size_t> set;
    };
    vector<Work> stack;
    vector<size_t> all(a.n);
    for (size_t i = 0; i < a.n; ++i) all[i] = i;
    stack.push_back({false, std::move(all)});
    while (!stack.empty()) {
        Work w = std::move(stack.back());
        stack.pop_back();
        if (w.emit) {
            order.insert(order.end(), w.set.begin(), w.set.end());
            continue;
        }
        if (w.set.size() <= LEAF) {
            order.insert(order.end(), w.set.begin(), w.set.end());
            continue;
        }
        vector<size_t> left, right, sep;
        if (!split(a, w.set, xyz, side, &left, &right, &sep)) {
            order.insert(order.end(), w.set.begin(), w.set.end());
            continue;
        }
        stack.push_back({true, std::move(sep)});
        stack.push_back({false, std::move(right)});
        stack.push_back({false, std::move(left)});
    }
    return order;
}

// ------------------------------------------------------------------ symbolic.rs
// symbolic.rs:195-215
static vector<size_t> etree(const Csr& a, const vector<size_t>& order,
                            const vector<size_t>& iorder) {
    size_t n = a.n;
    vector<size_t> parent(n, NONE), ancestor(n, NONE);
    for (size_t k = 0; k < n; ++k) {
        size_t old = order[k];
        for (size_t e = a.ptr[old]; e < a.ptr[old + 1]; ++e) {
            size_t i = iorder[a.idx[e]];
            while (i != NONE && i < k) {
                size_t next = ancestor[i];
                ancestor[i] = k;
                if (next == NONE) parent[i] = k;
                i = next;
            }
        }
    }
    return parent;
}

// symbolic.rs:218-245
static vector<size_t> postorder(const vector<size_t>& parent) {
    size_t n = parent.size();
    vector<size_t> head(n, NONE), next(n, NONE);
    for (size_t j = n; j-- > 0;)
        if (parent[j] != NONE) {
            next[j] = head[parent[j]];
            head[parent[j]] = j;
        }
    vector<size_t> post;
    post.reserve(n);
    vector<size_t> stack;
    for (size_t root = 0; root < n; ++root) {
        if (parent[root] != NONE) continue;
        stack.push_back(root);
        while (!stack.empty()) {
            size_t top = stack.back();
            size_t child = head[top];
            if (child == NONE) {
                stack.pop_back();
                post.push_back(top);
            } else {
                head[top] = next[child];
                stack.push_back(child);
            }
        }
    }
    return post;
}

// symbolic.rs:249-266
static vector<size_t> column_counts(const Csr& a, const vector<size_t>& perm,
                                    const vector<size_t>& iperm, const vector<size_t>& parent) {
    size_t n = a.n;
    vector<size_t> counts(n, 1), mark(n, NONE);
    for (size_t i = 0; i < n; ++i) {
        mark[i] = i;
        size_t old = perm[i];
        for (size_t e = a.ptr[old]; e < a.ptr[old + 1]; ++e) {
            size_t j = iperm[a.idx[e]];
            while (j < i && mark[j] != i) {
                counts[j] += 1;
                mark[j] = i;
                j = parent[j];
            }
        }
    }
    return counts;
}

// symbolic.rs:41-149
Symbolic analyse(const Csr& a, const vector<size_t>& order) {
    size_t n = a.n;
    if (order.size() != n) throw Error("the order has each column once");
    auto inverse = [n](const vector<size_t>& p) {
        vector<size_t> ip(n, 0);
        for (size_t k = 0; k < p.size(); ++k) ip[p[k]] = k;
        return ip;
    };
    vector<size_t> iorder = inverse(order);
    vector<size_t> parent0 = etree(a, order, iorder);
    vector<size_t> post = postorder(parent0);
    Symbolic s;
    s.n = n;
    s.perm.resize(n);
    for (size_t k = 0; k < n; ++k) s.perm[k] = order[post[k]];
    s.iperm = inverse(s.perm);
    vector<size_t> ipost = inverse(post);
    vector<size_t> parent(n);
    for (size_t k = 0; k < n; ++k) parent[k] = parent0[post[k]] == NONE ? NONE : ipost[parent0[post[k]]];
    vector<size_t> counts = column_counts(a, s.perm, s.iperm, parent);
    vector<size_t> nchild(n, 0);
    for (size_t p : parent)
        if (p != NONE) nchild[p] += 1;
    s.start.push_back(0);
    for (size_t j = 1; j < n; ++j) {
        bool joins = parent[j - 1] == j && counts[j - 1] == counts[j] + 1 && nchild[j] == 1;
        if (!joins) s.start.push_back(j);
    }
    s.start.push_back(n);
    size_t ns = s.start.size() - 1;
    vector<size_t> of_col(n, 0);
    for (size_t q = 0; q < ns; ++q)
        for (size_t j = s.start[q]; j < s.start[q + 1]; ++j) of_col[j] = q;
    s.parent.resize(ns);
    for (size_t q = 0; q < ns; ++q) {
        size_t p = parent[s.start[q + 1] - 1];
        s.parent[q] = p == NONE ? NONE : of_col[p];
    }
    s.children.assign(ns, 0);
    vector<vector<size_t>> kids(ns);
    for (size_t q = 0; q < ns; ++q)
        if (s.parent[q] != NONE) {
            s.children[s.parent[q]] += 1;
            kids[s.parent[q]].push_back(q);
        }
    s.rows_ptr.push_back(0);
    vector<size_t> mark(n, NONE);
    vector<uint32_t> list;
    for (size_t q = 0; q < ns; ++q) {
        list.clear();
        size_t first = s.start[q], end = s.start[q + 1];
        for (size_t j = first; j < end; ++j) {
            mark[j] = q;
            list.push_back((uint32_t)j);
        }
        for (size_t j = first; j < end; ++j) {
            size_t old = s.perm[j];
            for (size_t e = a.ptr[old]; e < a.ptr[old + 1]; ++e) {
                size_t i = s.iperm[a.idx[e]];
                if (i >= end && mark[i] != q) {
                    mark[i] = q;
                    list.push_back((uint32_t)i);
                }
            }
        }
        for (size_t c : kids[q])
            for (size_t t = s.rows_ptr[c]; t < s.rows_ptr[c + 1]; ++t) {
                size_t i = s.rows[t];
                if (i >= end && mark[i] != q) {
                    mark[i] = q;
                    list.push_back((uint32_t)i);
                }
            }
        std::sort(list.begin(), list.end());
        s.rows.insert(s.rows.end(), list.begin(), list.end());
        s.rows_ptr.push_back(s.rows.size());
    }
    return s;
}

// symbolic.rs:162-170
uint64_t Symbolic::entries() const {
    uint64_t total = 0;
    for (size_t q = 0; q < supernodes(); ++q) {
        uint64_t k = start[q + 1] - start[q], m = rows_ptr[q + 1] - rows_ptr[q];
        total += k * m - k * (k - 1) / 2;
    }
    return total;
}

// symbolic.rs:174-182
double Symbolic::flops() const {
    double total = 0;
    for (size_t q = 0; q < supernodes(); ++q) {
        size_t k = start[q + 1] - start[q], m = rows_ptr[q + 1] - rows_ptr[q];
        double part = 0;
        for (size_t j = 0; j < k; ++j) part += std::pow((double)(m - j), 2.0);
        total += part;
    }
    return total;
}

// ------------------------------------------------------------------ cholesky.rs
static const double PIVOT = 1e-10;  // cholesky.rs:22

// cholesky.rs:173-225. Returns the local column of a pivot that is not positive, or -1.
static long partial_cholesky(double* f, size_t m, size_t k, const double* diag) {
    for (size_t j = 0; j < k; ++j) {
        double* col = f + j * m;
        double d = col[j];
        if (!(d > PIVOT * std::fabs(diag[j]))) return (long)j;
        double l = std::sqrt(d);
        col[j] = l;
        double inv = 1.0 / l;
        for (size_t r = j + 1; r < m; ++r) col[r] *= inv;
        for (size_t c = j + 1; c < k; ++c) {
            double* target = f + c * m;
            double factor = col[c];
            for (size_t r = c; r < m; ++r) target[r] -= col[r] * factor;
        }
    }
    double* l = f;
    for (size_t c = k; c < m; ++c) {
        double* target = f + c * m;
        size_t p = 0;
        while (p + 4 <= k) {
            const double *c0 = l + p * m, *c1 = l + (p + 1) * m, *c2 = l + (p + 2) * m,
                         *c3 = l + (p + 3) * m;
            double f0 = c0[c], f1 = c1[c], f2 = c2[c], f3 = c3[c];
            for (size_t r = c; r < m; ++r)
                target[r] -= c0[r] * f0 + c1[r] * f1 + c2[r] * f2 + c3[r] * f3;
            p += 4;
        }
        while (p < k) {
            const double* c0 = l + p * m;
            double f0 = c0[c];
            for (size_t r = c; r < m; ++r) target[r] -= c0[r] * f0;
            p += 1;
        }
    }
    return -1;
}

// cholesky.rs:44-122
Cholesky factor(const Symbolic& sym, const Csr& a) {
    size_t n = sym.n, ns = sym.supernodes();
    Cholesky out;
    out.offset.reserve(ns + 1);
    out.offset.push_back(0);
    for (size_t s = 0; s < ns; ++s) {
        size_t k = sym.start[s + 1] - sym.start[s];
        size_t m = sym.rows_ptr[s + 1] - sym.rows_ptr[s];
        out.offset.push_back(out.offset[s] + k * m);
    }
    out.values.assign(out.offset[ns], 0.0);
    vector<size_t> pos(n, SIZE_MAX);
    struct Update {
        vector<uint32_t> rows;
        vector<double> values;
    };
    vector<Update> stack;
    vector<double> front, diag;
    for (size_t s = 0; s < ns; ++s) {
        const uint32_t* rows = sym.rows.data() + sym.rows_ptr[s];
        size_t first = sym.start[s], end = sym.start[s + 1];
        size_t m = sym.rows_ptr[s + 1] - sym.rows_ptr[s], k = end - first;
        for (size_t l = 0; l < m; ++l) pos[rows[l]] = l;
        front.assign(m * m, 0.0);
        diag.assign(k, 0.0);
        for (size_t j = first; j < end; ++j) {
            size_t old = sym.perm[j];
            size_t col = (j - first) * m;
            for (size_t e = a.ptr[old]; e < a.ptr[old + 1]; ++e) {
                size_t i = sym.iperm[a.idx[e]];
                if (i >= j) front[col + pos[i]] += a.val[e];
                if (i == j) diag[j - first] = a.val[e];
            }
        }
        for (size_t c = 0; c < sym.children[s]; ++c) {
            Update u = std::move(stack.back());
            stack.pop_back();
            size_t mu = u.rows.size();
            vector<size_t> at(mu);
            for (size_t t = 0; t < mu; ++t) at[t] = pos[u.rows[t]];
            for (size_t b = 0; b < mu; ++b) {
                size_t col = at[b] * m;
                const double* src = u.values.data() + b * mu;
                for (size_t q = b; q < mu; ++q) front[col + at[q]] += src[q];
            }
        }
        long bad = partial_cholesky(front.data(), m, k, diag.data());
        if (bad >= 0) {
            size_t column = sym.perm[first + (size_t)bad];
            char buf[320];
            std::snprintf(buf, sizeof buf,
                          "the matrix is not positive definite: the pivot of column %zu is 0 or "
                          "less to the precision of the arithmetic (its diagonal is %s)",
                          column, rust_lower_exp(diag[(size_t)bad], -1).c_str());
            throw Error(buf);
        }
        std::copy(front.begin(), front.begin() + k * m, out.values.begin() + out.offset[s]);
        if (m > k) {
            size_t mu = m - k;
            Update u;
            u.values.assign(mu * mu, 0.0);
            for (size_t b = 0; b < mu; ++b) {
                size_t src = (k + b) * m + k;
                for (size_t q = b; q < mu; ++q) u.values[b * mu + q] = front[src + q];
            }
            u.rows.assign(rows + k, rows + m);
            stack.push_back(std::move(u));
        }
        for (size_t l = 0; l < m; ++l) pos[rows[l]] = SIZE_MAX;
    }
    out.sym = sym;
    return out;
}

// cholesky.rs:125-160
void Cholesky::solve(double* b) const {
    size_t n = sym.n, ns = sym.supernodes();
    vector<double> y(n);
    for (size_t k = 0; k < n; ++k) y[k] = b[sym.perm[k]];
    for (size_t s = 0; s < ns; ++s) {
        const uint32_t* rows = sym.rows.data() + sym.rows_ptr[s];
        size_t first = sym.start[s], end = sym.start[s + 1];
        size_t m = sym.rows_ptr[s + 1] - sym.rows_ptr[s];
        const double* block = values.data() + offset[s];
        for (size_t j = 0; j < end - first; ++j) {
            const double* col = block + j * m;
            double v = y[first + j] / col[j];
            y[first + j] = v;
            for (size_t r = j + 1; r < m; ++r) y[rows[r]] -= col[r] * v;
        }
    }
    for (size_t s = ns; s-- > 0;) {
        const uint32_t* rows = sym.rows.data() + sym.rows_ptr[s];
        size_t first = sym.start[s], end = sym.start[s + 1];
        size_t m = sym.rows_ptr[s + 1] - sym.rows_ptr[s];
        const double* block = values.data() + offset[s];
        for (size_t j = end - first; j-- > 0;) {
            const double* col = block + j * m;
            double v = y[first + j];
            for (size_t r = j + 1; r < m; ++r) v -= col[r] * y[rows[r]];
            y[first + j] = v / col[j];
        }
    }
    for (size_t k = 0; k < n; ++k) b[sym.perm[k]] = y[k];
}

}  // namespace orc
