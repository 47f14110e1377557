// Robust orientation and in-circle predicates of points in the plane (predicates.rs): the
// determinant in floating point, kept when an error bound decides its sign, else computed exactly
// with floating-point expansions (sums of non-overlapping doubles) and returned as the sum of its
// components. The sign is always the exact one.
//
// Method: J. R. Shewchuk, Adaptive precision floating-point arithmetic and fast robust geometric
// predicates, Discrete Comput. Geom. 18 (1997) 305-363: the first-stage error bounds, the exact
// sum and product of 2 doubles, and expansion growth, sum and scaling with zero elimination. Only
// the filter and the exact stage are used (no intermediate stages), as in predicates.rs:1-15.
//
// Built with -ffp-contract=off: every operation rounds once, as the reference's f64 arithmetic.
#pragma once
#include <cmath>
#include <vector>

namespace femgpu {
namespace pred {

constexpr double kEps = 1.1102230246251565e-16;  // 2^-53
constexpr double kSplit = 134217729.0;           // 2^27 + 1
constexpr double kOrientBound = (3.0 + 16.0 * kEps) * kEps;
constexpr double kCircleBound = (10.0 + 96.0 * kEps) * kEps;

using Expansion = std::vector<double>;

// a + b = hi + lo exactly (Knuth).
inline void sum2(double a, double b, double& hi, double& lo) {
    hi = a + b;
    const double bv = hi - a, av = hi - bv;
    lo = (a - av) + (b - bv);
}

// a - b = hi + lo exactly.
inline void diff2(double a, double b, double& hi, double& lo) {
    hi = a - b;
    const double bv = a - hi, av = hi + bv;
    lo = (a - av) + (bv - b);
}

// Dekker's split of a into 2 non-overlapping halves of at most 26 significant bits.
inline void halves(double a, double& hi, double& lo) {
    const double c = kSplit * a, big = c - a;
    hi = c - big;
    lo = a - hi;
}

// a * b = hi + lo exactly (Dekker / Veltkamp).
inline void prod2(double a, double b, double& hi, double& lo) {
    hi = a * b;
    double ah, al, bh, bl;
    halves(a, ah, al);
    halves(b, bh, bl);
    const double e1 = hi - ah * bh, e2 = e1 - al * bh, e3 = e2 - ah * bl;
    lo = al * bl - e3;
}

// e + b, e an expansion in increasing magnitude; zero components dropped.
inline Expansion grow(const Expansion& e, double b) {
    Expansion h;
    h.reserve(e.size() + 1);
    double q = b;
    for (double x : e) {
        double s, t;
        sum2(q, x, s, t);
        q = s;
        if (t != 0.0) h.push_back(t);
    }
    if (q != 0.0 || h.empty()) h.push_back(q);
    return h;
}

// e + f: each non-zero component of f grown into e in turn; an empty result is {0}.
inline Expansion add(const Expansion& e, const Expansion& f) {
    Expansion h = e;
    for (double x : f)
        if (x != 0.0) h = grow(h, x);
    if (h.empty()) h.push_back(0.0);
    return h;
}

// e * b; zero components dropped.
inline Expansion scale(const Expansion& e, double b) {
    Expansion h;
    if (e.empty()) return h;
    h.reserve(2 * e.size());
    double q, t;
    prod2(e[0], b, q, t);
    if (t != 0.0) h.push_back(t);
    for (size_t i = 1; i < e.size(); ++i) {
        double p1, p0, s, u;
        prod2(e[i], b, p1, p0);
        sum2(q, p0, s, u);
        if (u != 0.0) h.push_back(u);
        double r, v;
        sum2(p1, s, r, v);  // |p1| >= |s| is not guaranteed: the exact sum either way
        if (v != 0.0) h.push_back(v);
        q = r;
    }
    if (q != 0.0 || h.empty()) h.push_back(q);
    return h;
}

// e * f: from {0}, the sum over the non-zero components of f of e scaled by each.
inline Expansion mul(const Expansion& e, const Expansion& f) {
    Expansion h{0.0};
    for (double x : f)
        if (x != 0.0) h = add(h, scale(e, x));
    return h;
}

// The sum of the components, smallest first: the expansion's value to about 1 rounding.
inline double value(const Expansion& e) {
    double q = 0.0;
    for (double x : e) q += x;
    return q;
}

inline Expansion neg(Expansion e) {
    for (double& x : e) x = -x;
    return e;
}

// Positive when a, b, c turn counterclockwise, negative clockwise, 0 on 1 line; twice the signed
// area when the filter decides (predicates.rs:17-51).
inline double orient2d(const double* a, const double* b, const double* c) {
    const double left = (a[0] - c[0]) * (b[1] - c[1]);
    const double right = (a[1] - c[1]) * (b[0] - c[0]);
    const double det = left - right;
    double sum;
    if (left > 0.0) {
        if (right <= 0.0) return det;
        sum = left + right;
    } else if (left < 0.0) {
        if (right >= 0.0) return det;
        sum = -left - right;
    } else {
        return det;
    }
    if (std::fabs(det) >= kOrientBound * sum) return det;
    // a0 b1 - a0 c1 + b0 c1 - b0 a1 + c0 a1 - c0 b1, each product exact.
    const double terms[6][2] = {{a[0], b[1]}, {-a[0], c[1]}, {b[0], c[1]},
                                {-b[0], a[1]}, {c[0], a[1]}, {-c[0], b[1]}};
    Expansion e;
    for (const auto& t : terms) {
        double hi, lo;
        prod2(t[0], t[1], hi, lo);
        e = add(e, Expansion{lo, hi});
    }
    return value(e);
}

// Positive when d is inside the circle through a, b, c (counterclockwise), negative outside, 0 on
// it (predicates.rs:53-91).
inline double incircle(const double* a, const double* b, const double* c, const double* d) {
    const double adx = a[0] - d[0], ady = a[1] - d[1];
    const double bdx = b[0] - d[0], bdy = b[1] - d[1];
    const double cdx = c[0] - d[0], cdy = c[1] - d[1];
    const double bc = bdx * cdy - cdx * bdy;
    const double ca = cdx * ady - adx * cdy;
    const double ab = adx * bdy - bdx * ady;
    const double al = adx * adx + ady * ady;
    const double bl = bdx * bdx + bdy * bdy;
    const double cl = cdx * cdx + cdy * cdy;
    const double det = al * bc + bl * ca + cl * ab;
    const double perm = (std::fabs(bdx * cdy) + std::fabs(cdx * bdy)) * al +
                        (std::fabs(cdx * ady) + std::fabs(adx * cdy)) * bl +
                        (std::fabs(adx * bdy) + std::fabs(bdx * ady)) * cl;
    if (std::fabs(det) > kCircleBound * perm) return det;
    auto dif = [](double p, double q) {
        double hi, lo;
        diff2(p, q, hi, lo);
        return Expansion{lo, hi};
    };
    const Expansion ax = dif(a[0], d[0]), ay = dif(a[1], d[1]);
    const Expansion bx = dif(b[0], d[0]), by = dif(b[1], d[1]);
    const Expansion cx = dif(c[0], d[0]), cy = dif(c[1], d[1]);
    auto cross = [](const Expansion& px, const Expansion& py, const Expansion& qx,
                    const Expansion& qy) { return add(mul(px, qy), neg(mul(qx, py))); };
    auto lift = [](const Expansion& x, const Expansion& y) { return add(mul(x, x), mul(y, y)); };
    const Expansion t1 = mul(lift(ax, ay), cross(bx, by, cx, cy));
    const Expansion t2 = mul(lift(bx, by), cross(cx, cy, ax, ay));
    const Expansion t3 = mul(lift(cx, cy), cross(ax, ay, bx, by));
    return value(add(add(t1, t2), t3));
}

}  // namespace pred
}  // namespace femgpu
