// Symbolic analysis of the sparse Cholesky factor (symbolic.hpp).
#include "symbolic.hpp"

#include <algorithm>

namespace femgpu {
namespace {

// The pattern of `a` renumbered: row k holds the new indices of the entries of old row
// order[k], increasing.
struct Pattern {
    std::vector<int64_t> ptr;
    std::vector<int64_t> idx;
};

Pattern renumber(const HostCsr& a, const std::vector<int64_t>& order,
                 const std::vector<int64_t>& inv) {
    const int64_t n = a.n;
    Pattern p;
    p.ptr.assign(n + 1, 0);
    for (int64_t k = 0; k < n; ++k) p.ptr[k + 1] = p.ptr[k] + (a.ptr[order[k] + 1] - a.ptr[order[k]]);
    p.idx.resize(p.ptr[n]);
    for (int64_t k = 0; k < n; ++k) {
        int64_t* out = p.idx.data() + p.ptr[k];
        int64_t c = 0;
        for (int64_t e = a.ptr[order[k]]; e < a.ptr[order[k] + 1]; ++e) out[c++] = inv[a.idx[e]];
        std::sort(out, out + c);
    }
    return p;
}

// Liu's elimination tree with path compression (each column's entries above the diagonal
// attach the roots of their subtrees to it).
std::vector<int64_t> etree(const Pattern& p, int64_t n) {
    std::vector<int64_t> parent(n, -1), root(n, -1);
    for (int64_t k = 0; k < n; ++k) {
        for (int64_t e = p.ptr[k]; e < p.ptr[k + 1]; ++e) {
            int64_t i = p.idx[e];
            while (i >= 0 && i < k) {
                const int64_t up = root[i];
                root[i] = k;
                if (up < 0) parent[i] = k;
                i = up;
            }
        }
    }
    return parent;
}

// A postorder of the forest (children visited in increasing order): post[k] = the node at k.
std::vector<int64_t> postorder(const std::vector<int64_t>& parent) {
    const int64_t n = (int64_t)parent.size();
    std::vector<int64_t> head(n, -1), next(n, -1);
    for (int64_t j = n - 1; j >= 0; --j)
        if (parent[j] >= 0) {
            next[j] = head[parent[j]];
            head[parent[j]] = j;
        }
    std::vector<int64_t> post;
    post.reserve(n);
    std::vector<int64_t> stack;
    for (int64_t r = 0; r < n; ++r) {
        if (parent[r] >= 0) continue;
        stack.push_back(r);
        while (!stack.empty()) {
            const int64_t v = stack.back();
            if (head[v] >= 0) {
                const int64_t c = head[v];
                head[v] = next[c];
                stack.push_back(c);
            } else {
                stack.pop_back();
                post.push_back(v);
            }
        }
    }
    return post;
}

// The column counts of L (with the diagonal): row i of L holds the nodes on the tree paths from
// the entries j < i of row i of the matrix up to i; each is counted once per row.
std::vector<int64_t> column_counts(const Pattern& p, const std::vector<int64_t>& parent) {
    const int64_t n = (int64_t)parent.size();
    std::vector<int64_t> count(n, 0), seen(n, -1);
    for (int64_t i = 0; i < n; ++i) {
        seen[i] = i;
        count[i] += 1;
        for (int64_t e = p.ptr[i]; e < p.ptr[i + 1]; ++e) {
            int64_t j = p.idx[e];
            if (j >= i) break;
            while (seen[j] != i) {
                seen[j] = i;
                count[j] += 1;
                j = parent[j];
            }
        }
    }
    return count;
}

struct Ordered {
    std::vector<int64_t> perm, iperm, parent, count;
    Pattern pat;
};

// The order postordered, with its tree and column counts.
Ordered order_and_count(const HostCsr& a, const std::vector<int64_t>& order) {
    const int64_t n = a.n;
    std::vector<int64_t> inv(n);
    for (int64_t k = 0; k < n; ++k) inv[order[k]] = k;
    Pattern p0 = renumber(a, order, inv);
    std::vector<int64_t> par0 = etree(p0, n);
    std::vector<int64_t> post = postorder(par0);
    std::vector<int64_t> ipost(n);
    for (int64_t k = 0; k < n; ++k) ipost[post[k]] = k;
    Ordered o;
    o.perm.resize(n);
    o.iperm.resize(n);
    o.parent.resize(n);
    for (int64_t k = 0; k < n; ++k) {
        o.perm[k] = order[post[k]];
        o.iperm[o.perm[k]] = k;
        o.parent[k] = par0[post[k]] < 0 ? -1 : ipost[par0[post[k]]];
    }
    o.pat = renumber(a, o.perm, o.iperm);
    o.count = column_counts(o.pat, o.parent);
    return o;
}

// Fundamental supernodes: column j continues the supernode of j - 1 when it is the parent of
// j - 1, j - 1 is its only child, and their counts differ by 1.
std::vector<int64_t> supernode_starts(const Ordered& o) {
    const int64_t n = (int64_t)o.parent.size();
    std::vector<int64_t> nchild(n, 0);
    for (int64_t j = 0; j < n; ++j)
        if (o.parent[j] >= 0) nchild[o.parent[j]] += 1;
    std::vector<int64_t> first{0};
    for (int64_t j = 1; j < n; ++j) {
        const bool joins =
            o.parent[j - 1] == j && nchild[j] == 1 && o.count[j - 1] == o.count[j] + 1;
        if (!joins) first.push_back(j);
    }
    first.push_back(n);
    return first;
}

void figures(const Ordered& o, const std::vector<int64_t>& first, uint64_t* entries,
             double* flops) {
    uint64_t e = 0;
    double f = 0.0;
    for (size_t s = 0; s + 1 < first.size(); ++s) {
        double fs = 0.0;
        for (int64_t j = first[s]; j < first[s + 1]; ++j) {
            const double c = (double)o.count[j];
            e += (uint64_t)o.count[j];
            fs += c * c;
        }
        f += fs;
    }
    *entries = e;
    *flops = f;
}

}  // namespace

void factor_figures(const HostCsr& a, const std::vector<int64_t>& order, uint64_t* entries,
                    double* flops) {
    Ordered o = order_and_count(a, order);
    figures(o, supernode_starts(o), entries, flops);
}

Supernodal analyse_factor(const HostCsr& a, const std::vector<int64_t>& order) {
    Ordered o = order_and_count(a, order);
    Supernodal S;
    S.n = a.n;
    S.first = supernode_starts(o);
    S.ns = (int64_t)S.first.size() - 1;
    figures(o, S.first, &S.entries, &S.flops);
    const int64_t n = a.n, ns = S.ns;
    std::vector<int64_t> of(n);
    for (int64_t s = 0; s < ns; ++s)
        for (int64_t j = S.first[s]; j < S.first[s + 1]; ++j) of[j] = s;
    S.parent.assign(ns, -1);
    for (int64_t s = 0; s < ns; ++s) {
        const int64_t p = o.parent[S.first[s + 1] - 1];
        S.parent[s] = p < 0 ? -1 : of[p];
    }
    // Children lists, then each supernode's rows: its columns, the matrix's entries below them
    // and its children's rows past its last column (each child's pattern is done first).
    std::vector<int64_t> head(ns, -1), next(ns, -1);
    for (int64_t s = ns - 1; s >= 0; --s)
        if (S.parent[s] >= 0) {
            next[s] = head[S.parent[s]];
            head[S.parent[s]] = s;
        }
    std::vector<int64_t> seen(n, -1);
    S.rows_ptr.assign(1, 0);
    std::vector<uint32_t> list;
    for (int64_t s = 0; s < ns; ++s) {
        const int64_t f = S.first[s], end = S.first[s + 1];
        list.clear();
        for (int64_t j = f; j < end; ++j) {
            seen[j] = s;
            list.push_back((uint32_t)j);
        }
        for (int64_t j = f; j < end; ++j)
            for (int64_t e = o.pat.ptr[j]; e < o.pat.ptr[j + 1]; ++e) {
                const int64_t i = o.pat.idx[e];
                if (i >= end && seen[i] != s) {
                    seen[i] = s;
                    list.push_back((uint32_t)i);
                }
            }
        for (int64_t c = head[s]; c >= 0; c = next[c])
            for (int64_t t = S.rows_ptr[c]; t < S.rows_ptr[c + 1]; ++t) {
                const int64_t i = S.rows[t];
                if (i >= end && seen[i] != s) {
                    seen[i] = s;
                    list.push_back((uint32_t)i);
                }
            }
        std::sort(list.begin() + (end - f), list.end());
        S.rows.insert(S.rows.end(), list.begin(), list.end());
        S.rows_ptr.push_back((int64_t)S.rows.size());
    }
    S.height.assign(ns, 0);
    for (int64_t s = 0; s < ns; ++s)
        if (S.parent[s] >= 0)
            S.height[S.parent[s]] = std::max(S.height[S.parent[s]], S.height[s] + 1);
    S.perm = std::move(o.perm);
    S.iperm = std::move(o.iperm);
    return S;
}

}  // namespace femgpu
