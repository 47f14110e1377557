// The host steps of the prism mesh (prism.rs, grid.rs): the footprints' outlines and their
// triangle mesh, and the graded planes of the extrusion axis. Built with -ffp-contract=off so that
// each operation rounds once, as the reference's f64 arithmetic does.
#include "prism.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>

#include "rust_format.hpp"

namespace femgpu {
namespace {

constexpr size_t kMinCircleSegments = 64;  // prism.rs:51
constexpr double kPi = 3.141592653589793;
const char* const kAxis[3] = {"x", "y", "z"};

[[noreturn]] void fail(const std::string& text) { throw std::runtime_error(text); }

bool total_less(double a, double b) {
    int64_t x, y;
    std::memcpy(&x, &a, 8);
    std::memcpy(&y, &b, 8);
    x ^= (int64_t)(((uint64_t)(x >> 63)) >> 1);
    y ^= (int64_t)(((uint64_t)(y >> 63)) >> 1);
    return x < y;
}

// The coordinates across axis `axis`: the next 2 axes in the order x, y, z, x (prism.rs:54-56).
P2 across(int axis, const double* p) { return {p[(axis + 1) % 3], p[(axis + 2) % 3]}; }

// Even-odd point in polygon (prism.rs:90-102).
bool inside(const std::vector<P2>& c, P2 p) {
    bool odd = false;
    const size_t n = c.size();
    for (size_t k = 0; k < n; ++k) {
        const P2 a = c[k], b = c[(k + 1) % n];
        if ((a[1] > p[1]) != (b[1] > p[1]) &&
            p[0] < a[0] + (p[1] - a[1]) / (b[1] - a[1]) * (b[0] - a[0]))
            odd = !odd;
    }
    return odd;
}

// More corners on each side longer than `max` (prism.rs:529-544).
std::vector<P2> densify(const std::vector<P2>& c, double max) {
    std::vector<P2> out;
    const size_t m = c.size();
    for (size_t k = 0; k < m; ++k) {
        const P2 a = c[k], b = c[(k + 1) % m];
        size_t n = 1;
        if (std::isfinite(max)) {
            const double dx = b[0] - a[0], dy = b[1] - a[1];
            n = std::max<size_t>((size_t)std::ceil(std::sqrt(dx * dx + dy * dy) / max), 1);
        }
        for (size_t i = 0; i < n; ++i) {
            const double t = (double)i / (double)n;
            out.push_back({a[0] + t * (b[0] - a[0]), a[1] + t * (b[1] - a[1])});
        }
    }
    return out;
}

// The planes of an axis from the size function: in interval i the size is the smaller of
// target[i] and at_key[k] + slope |x - key[k]| over the key planes k; each interval's cells are
// equal steps of the integral of 1 / h, by the trapezoid rule on 400 samples (grid.rs:487-518).
std::vector<double> place(const std::vector<double>& keys, const std::vector<double>& target,
                          const std::vector<double>& at_key, double slope) {
    auto h = [&](double x, size_t i) {
        double v = target[i];
        for (size_t k = 0; k < keys.size(); ++k) v = std::min(v, at_key[k] + slope * std::fabs(x - keys[k]));
        return v;
    };
    std::vector<double> planes{keys[0]};
    constexpr size_t samples = 400;
    std::vector<double> phi(samples + 1);
    for (size_t i = 0; i + 1 < keys.size(); ++i) {
        const double a = keys[i], b = keys[i + 1];
        const double step = (b - a) / (double)samples;
        phi[0] = 0.0;
        for (size_t s = 0; s < samples; ++s) {
            const double x0 = a + (double)s * step, x1 = a + (double)(s + 1) * step;
            phi[s + 1] = phi[s] + 0.5 * step * (1.0 / h(x0, i) + 1.0 / h(x1, i));
        }
        const double total = phi[samples];
        const double whole = std::ceil(total - 1e-6);
        const size_t cells = whole < 1.0 ? 1 : (size_t)whole;
        for (size_t c = 1; c < cells; ++c) {
            const double want = total * (double)c / (double)cells;
            size_t s = (size_t)(std::lower_bound(phi.begin(), phi.end(), want) - phi.begin());
            s = std::min(std::max<size_t>(s, 1), samples);
            const double f = (want - phi[s - 1]) / (phi[s] - phi[s - 1]);
            planes.push_back(a + ((double)s - 1.0 + f) * step);
        }
        planes.push_back(b);
    }
    return planes;
}

}  // namespace

std::vector<P2> outline_corners(const Outline& o, double max_cell) {
    if (!o.circle) return o.corners;
    size_t n = std::max((size_t)std::ceil(2.0 * kPi * o.radius / max_cell), kMinCircleSegments);
    n = (n + 3) / 4 * 4;
    std::vector<P2> out(n);
    for (size_t k = 0; k < n; ++k) {
        const double a = 2.0 * kPi * (double)k / (double)n;
        out[k] = {o.centre[0] + o.radius * std::cos(a), o.centre[1] + o.radius * std::sin(a)};
    }
    return out;
}

double plane_tol(const std::vector<double>& p) {
    return 1e-9 * std::max(std::fabs(p.back() - p.front()), std::numeric_limits<double>::min());
}

std::vector<double> axis_planes(const std::vector<Part>& parts, int d, const Spacing& spacing,
                                const std::vector<double>& extra) {
    std::vector<double> keys;
    for (const Part& p : parts) {
        keys.push_back(p.lo[d]);
        keys.push_back(p.hi[d]);
    }
    keys.insert(keys.end(), extra.begin(), extra.end());
    std::stable_sort(keys.begin(), keys.end(), total_less);
    const double t = plane_tol(keys);
    {
        std::vector<double> kept;
        for (double k : keys)
            if (kept.empty() || !(std::fabs(k - kept.back()) <= t)) kept.push_back(k);
        keys.swap(kept);
    }
    // The target size of each interval: max_cell, and min_cells through each part over it.
    std::vector<double> target(keys.size() - 1);
    for (size_t i = 0; i + 1 < keys.size(); ++i) {
        double v = spacing.max_cell;
        for (const Part& p : parts)
            if (p.lo[d] <= keys[i] + t && p.hi[d] >= keys[i + 1] - t)
                v = std::min(v, (p.hi[d] - p.lo[d]) / (double)spacing.min_cells);
        target[i] = v;
    }
    // The size at each key plane: the smaller target of its 2 intervals, lowered where 2 cells
    // side by side break the growth limit.
    std::vector<double> at_key(keys.size());
    for (size_t k = 0; k < keys.size(); ++k) {
        const double left = k > 0 ? target[k - 1] : INFINITY;
        const double right = k < target.size() ? target[k] : INFINITY;
        at_key[k] = std::min(left, right);
    }
    const double slope = 0.5 * (spacing.max_growth - 1.0);
    for (int round = 0; round < 60; ++round) {
        const std::vector<double> planes = place(keys, target, at_key, slope);
        std::vector<double> cells(planes.size() - 1);
        for (size_t c = 0; c + 1 < planes.size(); ++c) cells[c] = planes[c + 1] - planes[c];
        bool fixed = false;
        for (size_t c = 0; c + 1 < cells.size(); ++c) {
            const double small = cells[c] < cells[c + 1] ? cells[c] : cells[c + 1];
            const double large = cells[c] < cells[c + 1] ? cells[c + 1] : cells[c];
            if (large > spacing.max_growth * small * (1.0 + 1e-9)) {
                // The key plane next to the large cell gets a smaller size.
                const double x = planes[c + 1];
                size_t k = 0;
                while (k < keys.size() && keys[k] < x - t) ++k;
                k = std::min(k, keys.size() - 1);
                const size_t near3[3] = {k > 0 ? k - 1 : 0, k, std::min(k + 1, keys.size() - 1)};
                for (size_t q : near3) {
                    const bool near = std::fabs(keys[q] - x) <= 2.0 * large;
                    if (near && at_key[q] > small * 1.0001) {
                        at_key[q] = small;
                        fixed = true;
                    }
                }
            }
        }
        if (!fixed) return planes;
    }
    fail(std::string("the ") + kAxis[d] + " grid planes break the growth limit max_growth = " +
         rust_display(spacing.max_growth) +
         ": use a larger max_growth or a smaller max_cell");
}

Flat footprints(const std::vector<Part>& parts, int axis, Size2 size,
                const std::vector<double>& surface, bool periodic) {
    std::vector<P2> points;
    std::vector<std::array<uint32_t, 2>> segments;
    Flat flat;
    // The outline (first) and the holes of each part, as polygons.
    std::vector<std::vector<std::vector<P2>>> polygons;
    for (size_t k = 0; k < parts.size(); ++k) {
        const Part& p = parts[k];
        if (!(std::isfinite(p.lo[axis]) && std::isfinite(p.hi[axis]) && p.lo[axis] < p.hi[axis]))
            fail("part " + p.name + ": its " + kAxis[axis] +
                 " range must be 2 finite numbers, the first smaller");
        Footprint fp;
        if (p.has_footprint) {
            fp = p.footprint;
        } else {
            const P2 lo = across(axis, p.lo), hi = across(axis, p.hi);
            if (!(lo[0] < hi[0] && lo[1] < hi[1]))
                fail("part " + p.name + ": each range must have the first number smaller");
            fp.outline.corners = {lo, {hi[0], lo[1]}, hi, {lo[0], hi[1]}};
        }
        std::vector<std::vector<P2>> rings;
        for (size_t r = 0; r <= fp.holes.size(); ++r) {
            const Outline& o = r == 0 ? fp.outline : fp.holes[r - 1];
            std::vector<P2> corners;
            if (o.circle) {
                if (!(std::isfinite(o.radius) && o.radius > 0.0 && std::isfinite(o.centre[0]) &&
                      std::isfinite(o.centre[1])))
                    fail("part " + p.name + ": a circle needs a finite centre and a radius above 0");
                corners = outline_corners(o, std::min(size.max_size, surface[k]));
            } else {
                bool finite = true;
                for (const P2& c : o.corners) finite = finite && std::isfinite(c[0]) && std::isfinite(c[1]);
                if (o.corners.size() < 3 || !finite)
                    fail("part " + p.name +
                         ": a polygon needs 3 or more corners with finite coordinates");
                corners = densify(o.corners, surface[k]);
            }
            double area = 0.0;
            for (size_t c = 0; c < corners.size(); ++c) {
                const P2 a = corners[c], b = corners[(c + 1) % corners.size()];
                area += a[0] * b[1] - b[0] * a[1];
            }
            if (area == 0.0) fail("part " + p.name + ": an outline has no area");
            uint32_t circle = 0xffffffffu;
            if (o.circle) {
                flat.circles.push_back({o.centre, o.radius});
                circle = (uint32_t)flat.circles.size() - 1;
            }
            const uint32_t base = (uint32_t)points.size(), n = (uint32_t)corners.size();
            points.insert(points.end(), corners.begin(), corners.end());
            for (uint32_t c = 0; c < n; ++c) {
                segments.push_back({base + c, base + (c + 1) % n});
                flat.segment_circle.push_back(circle);
            }
            rings.push_back(std::move(corners));
        }
        polygons.push_back(std::move(rings));
    }
    // The parts that hold a point, highest priority first (the later part first at equal
    // priority), interned as labels in the order first met.
    auto classify = [&](P2 x) -> uint32_t {
        std::vector<uint32_t> list;
        for (uint32_t k = 0; k < (uint32_t)parts.size(); ++k) {
            const auto& rings = polygons[k];
            bool in = inside(rings[0], x);
            for (size_t h = 1; in && h < rings.size(); ++h)
                if (inside(rings[h], x)) in = false;
            if (in) list.push_back(k);
        }
        if (list.empty()) return kOutside;
        std::stable_sort(list.begin(), list.end(), [&](uint32_t a, uint32_t b) {
            if (parts[a].priority != parts[b].priority) return parts[a].priority > parts[b].priority;
            return a > b;
        });
        for (size_t c = 0; c < flat.covers.size(); ++c)
            if (flat.covers[c] == list) return (uint32_t)c;
        flat.covers.push_back(list);
        return (uint32_t)flat.covers.size() - 1;
    };
    flat.mesh = quality_mesh(points, segments, size, classify, periodic);
    return flat;
}

}  // namespace femgpu
