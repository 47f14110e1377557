// The reference's fill-reducing order (order.rs:19-179) on all host threads: nested dissection
// by coordinate bisection. A set of more than 64 nodes is cut at 5 quantiles (0.3 to 0.7) of its
// coordinates along each axis whose extent is not 0 (a cut at or below the lowest coordinate
// moves to the next higher one); the cut whose separator (the nodes of the smaller side that
// couple to the other side) divided by sqrt(2 x the smaller side's fraction of the set) is the
// least wins, ties to the first; the separator is taken from the side with fewer coupled nodes;
// the order is the left part's, then the right part's, then the separator.
//
// Design. The two parts of a split are independent, so they are ordered on separate threads
// while threads are free (their orders are concatenated in the reference's sequence, so the
// result does not depend on the threads), and the 15 trial cuts of a large set are evaluated in
// parallel. No per-node state is cleared between sets: a set stamps its nodes with its own
// number, and a node belongs to the set being cut when its stamp is the set's; the side of a
// node under a trial cut is read from its coordinate. So concurrent sets never see each other's
// marks, and trials need no marks of their own.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <future>
#include <thread>

#include "hierarchy.hpp"

namespace femgpu {
namespace {

constexpr size_t LEAF = 64;                                 // order.rs:15
constexpr double CUTS[5] = {0.3, 0.4, 0.5, 0.6, 0.7};       // order.rs:57
constexpr size_t PARALLEL_SET = 20000;    // a set at least this big orders its parts on 2 threads
constexpr size_t PARALLEL_TRIALS = 100000;  // ... and tries its cuts on several

struct Dissection {
    const HostCsr& a;
    const double* xyz;
    std::vector<std::atomic<uint64_t>> stamp;
    std::atomic<uint64_t> next{1};
    std::atomic<int> spare;  // threads that may still be started

    Dissection(const HostCsr& m, const double* p, int threads)
        : a(m), xyz(p), stamp(m.n), spare(threads - 1) {
        for (auto& s : stamp) s.store(0, std::memory_order_relaxed);
    }

    bool in(int64_t w, uint64_t id) const {
        return stamp[w].load(std::memory_order_relaxed) == id;
    }
    bool below(int64_t v, int axis, double cut) const { return xyz[3 * v + axis] < cut; }

    // The separator of the cut (the fewer of the coupled nodes of each side) and the smaller
    // side's size.
    std::pair<int64_t, int64_t> trial(const std::vector<int64_t>& set, uint64_t id, int axis,
                                      double cut) const {
        int64_t nleft = 0, sl = 0, sr = 0;
        for (int64_t v : set) {
            const bool left = below(v, axis, cut);
            nleft += left;
            bool coupled = false;
            for (int64_t e = a.ptr[v]; e < a.ptr[v + 1] && !coupled; ++e) {
                const int64_t w = a.idx[e];
                coupled = in(w, id) && below(w, axis, cut) != left;
            }
            if (coupled) (left ? sl : sr) += 1;
        }
        return {std::min(sl, sr), std::min(nleft, (int64_t)set.size() - nleft)};
    }

    struct Cut {
        int axis;
        double cut;
    };

    // The trial cuts of the set in the reference's sequence (axis, then quantile).
    std::vector<Cut> cuts(const std::vector<int64_t>& set) const {
        double lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
            lo[d] = INFINITY;
            hi[d] = -INFINITY;
        }
        for (int64_t v : set)
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::fmin(lo[d], xyz[3 * v + d]);
                hi[d] = std::fmax(hi[d], xyz[3 * v + d]);
            }
        std::vector<Cut> out;
        std::vector<double> c;
        for (int axis = 0; axis < 3; ++axis) {
            if (!(hi[axis] > lo[axis])) continue;
            c.resize(set.size());
            for (size_t k = 0; k < set.size(); ++k) c[k] = xyz[3 * set[k] + axis];
            std::sort(c.begin(), c.end());
            const bool has_above = c.back() > lo[axis];
            const double above =
                has_above ? *std::upper_bound(c.begin(), c.end(), lo[axis]) : lo[axis];
            for (double q : CUTS) {
                double at = c[std::min((size_t)((double)c.size() * q), c.size() - 1)];
                if (at <= lo[axis]) {
                    if (!has_above) continue;
                    at = above;
                }
                out.push_back({axis, at});
            }
        }
        return out;
    }

    // The order of `set` (its nodes stamped `id` by the caller).
    std::vector<int64_t> order(std::vector<int64_t> set, uint64_t id) {
        if (set.size() <= LEAF) return set;
        const std::vector<Cut> trials = cuts(set);
        if (trials.empty()) return set;
        std::vector<double> cost(trials.size());
        auto eval = [&](size_t t) {
            const auto sc = trial(set, id, trials[t].axis, trials[t].cut);
            cost[t] = (double)sc.first / std::sqrt(2.0 * (double)sc.second / (double)set.size());
        };
        if (set.size() >= PARALLEL_TRIALS && trials.size() > 1) {
            std::vector<std::thread> pool;
            for (size_t t = 1; t < trials.size(); ++t) pool.emplace_back(eval, t);
            eval(0);
            for (auto& th : pool) th.join();
        } else {
            for (size_t t = 0; t < trials.size(); ++t) eval(t);
        }
        size_t best = 0;
        for (size_t t = 1; t < trials.size(); ++t)
            if (cost[t] < cost[best]) best = t;
        const int axis = trials[best].axis;
        const double cut = trials[best].cut;
        // The two sides and each one's nodes coupled to the other; the separator is the side
        // with fewer of them (the left one on a tie).
        std::vector<int64_t> left, right, cl, cr;
        for (int64_t v : set) {
            const bool l = below(v, axis, cut);
            bool coupled = false;
            for (int64_t e = a.ptr[v]; e < a.ptr[v + 1] && !coupled; ++e) {
                const int64_t w = a.idx[e];
                coupled = in(w, id) && below(w, axis, cut) != l;
            }
            (l ? left : right).push_back(v);
            if (coupled) (l ? cl : cr).push_back(v);
        }
        const bool from_left = cl.size() <= cr.size();
        std::vector<int64_t>& sep = from_left ? cl : cr;
        std::vector<int64_t>& part = from_left ? left : right;
        {
            // The part without its separator nodes (both lists are in set order).
            std::vector<int64_t> rest;
            rest.reserve(part.size() - sep.size());
            size_t k = 0;
            for (int64_t v : part) {
                if (k < sep.size() && sep[k] == v)
                    ++k;
                else
                    rest.push_back(v);
            }
            part = std::move(rest);
        }
        const uint64_t idl = next.fetch_add(2), idr = idl + 1;
        for (int64_t v : left) stamp[v].store(idl, std::memory_order_relaxed);
        for (int64_t v : right) stamp[v].store(idr, std::memory_order_relaxed);
        std::vector<int64_t> ol, orr;
        if (set.size() >= PARALLEL_SET && spare.fetch_sub(1) > 0) {
            auto f = std::async(std::launch::async,
                                [this, &left, idl] { return order(std::move(left), idl); });
            orr = order(std::move(right), idr);
            ol = f.get();
            spare.fetch_add(1);
        } else {
            if (set.size() >= PARALLEL_SET) spare.fetch_add(1);
            ol = order(std::move(left), idl);
            orr = order(std::move(right), idr);
        }
        ol.insert(ol.end(), orr.begin(), orr.end());
        ol.insert(ol.end(), sep.begin(), sep.end());
        return ol;
    }
};

}  // namespace

std::vector<int64_t> nested_dissection(const HostCsr& a, const double* xyz) {
    Dissection d(a, xyz, host_threads());
    std::vector<int64_t> all(a.n);
    for (int64_t i = 0; i < a.n; ++i) all[i] = i;
    const uint64_t id = d.next.fetch_add(1);
    for (int64_t i = 0; i < a.n; ++i) d.stamp[i].store(id, std::memory_order_relaxed);
    return d.order(std::move(all), id);
}

}  // namespace femgpu
