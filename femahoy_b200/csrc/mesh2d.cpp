// The quality triangle mesh of the footprints (mesh2d.rs). Host code: see mesh2d.hpp.
#include "mesh2d.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <limits>
#include <stdexcept>
#include <string>
#include <unordered_map>

#include "predicates.hpp"
#include "rust_format.hpp"

namespace femgpu {
namespace {

constexpr uint32_t NONE = 0xffffffffu;
constexpr double kRatio = 1.4142135623730951;  // sqrt 2 (mesh2d.rs:53)
constexpr size_t kMaxVertices = 4000000;       // mesh2d.rs:60
constexpr int kPeriodicRounds = 50;            // mesh2d.rs:112

[[noreturn]] void fail(const std::string& text) { throw std::runtime_error(text); }

double dist(P2 a, P2 b) {
    const double dx = a[0] - b[0], dy = a[1] - b[1];
    return std::sqrt(dx * dx + dy * dy);
}

// The total order of doubles (negative zero before positive zero), as f64::total_cmp.
bool tless(double a, double b) {
    int64_t x, y;
    std::memcpy(&x, &a, 8);
    std::memcpy(&y, &b, 8);
    x ^= (int64_t)(((uint64_t)(x >> 63)) >> 1);
    y ^= (int64_t)(((uint64_t)(y >> 63)) >> 1);
    return x < y;
}

double orient(P2 a, P2 b, P2 c) { return pred::orient2d(a.data(), b.data(), c.data()); }
double incircle(P2 a, P2 b, P2 c, P2 d) {
    return pred::incircle(a.data(), b.data(), c.data(), d.data());
}

// A segment after the clean: its ends and the input segments that hold it.
struct Piece {
    std::array<uint32_t, 2> ends;
    std::vector<uint32_t> origin;
};

// True when point v is on the segment `ends`, strictly between its ends, within tol.
bool on_segment(const std::vector<P2>& pts, std::array<uint32_t, 2> ends, uint32_t v, double tol) {
    const P2 a = pts[ends[0]], b = pts[ends[1]], p = pts[v];
    const double len2 = (b[0] - a[0]) * (b[0] - a[0]) + (b[1] - a[1]) * (b[1] - a[1]);
    const double s = ((p[0] - a[0]) * (b[0] - a[0]) + (p[1] - a[1]) * (b[1] - a[1])) / len2;
    if (!(s > 0.0 && s < 1.0)) return false;
    const P2 foot{a[0] + s * (b[0] - a[0]), a[1] + s * (b[1] - a[1])};
    return dist(foot, p) <= tol && dist(p, a) > tol && dist(p, b) > tol;
}

// Merge points within 1e-9 of the bounding box's diagonal, then split each segment at the points
// on it and at its crossings, up to 8 passes, and merge pieces on the same 2 points
// (mesh2d.rs:175-322).
void clean(const std::vector<P2>& points, const std::vector<std::array<uint32_t, 2>>& segs,
           std::vector<P2>* out_pts, std::vector<Piece>* out_pieces) {
    P2 lo{INFINITY, INFINITY}, hi{-INFINITY, -INFINITY};
    for (const P2& p : points)
        for (int d = 0; d < 2; ++d) {
            lo[d] = std::min(lo[d], p[d]);
            hi[d] = std::max(hi[d], p[d]);
        }
    const double tol = 1e-9 * std::max(dist(lo, hi), std::numeric_limits<double>::min());
    std::vector<P2>& pts = *out_pts;
    pts.clear();
    std::vector<size_t> order(points.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return tless(points[a][0], points[b][0]); });
    std::vector<uint32_t> map(points.size(), NONE);
    for (size_t k = 0; k < order.size(); ++k) {
        const size_t i = order[k];
        if (map[i] != NONE) continue;
        map[i] = (uint32_t)pts.size();
        for (size_t q = k + 1; q < order.size(); ++q) {
            const size_t j = order[q];
            if (points[j][0] - points[i][0] > tol) break;
            if (map[j] == NONE && dist(points[i], points[j]) <= tol) map[j] = (uint32_t)pts.size();
        }
        pts.push_back(points[i]);
    }
    std::vector<Piece> pieces;
    for (size_t k = 0; k < segs.size(); ++k) {
        Piece p{{map[segs[k][0]], map[segs[k][1]]}, {(uint32_t)k}};
        if (p.ends[0] != p.ends[1]) pieces.push_back(std::move(p));
    }
    for (int pass = 0; pass < 8; ++pass) {
        std::vector<std::vector<uint32_t>> cuts(pieces.size());
        bool changed = false;
        auto box = [&](const Piece& p, P2* blo, P2* bhi) {
            const P2 a = pts[p.ends[0]], b = pts[p.ends[1]];
            *blo = {std::min(a[0], b[0]), std::min(a[1], b[1])};
            *bhi = {std::max(a[0], b[0]), std::max(a[1], b[1])};
        };
        std::vector<size_t> by_x(pieces.size());
        for (size_t i = 0; i < by_x.size(); ++i) by_x[i] = i;
        std::stable_sort(by_x.begin(), by_x.end(), [&](size_t a, size_t b) {
            P2 al, ah, bl, bh;
            box(pieces[a], &al, &ah);
            box(pieces[b], &bl, &bh);
            return tless(al[0], bl[0]);
        });
        std::vector<P2> fresh;
        for (size_t k = 0; k < by_x.size(); ++k) {
            const size_t i = by_x[k];
            P2 ilo, ihi;
            box(pieces[i], &ilo, &ihi);
            for (size_t q = k + 1; q < by_x.size(); ++q) {
                const size_t j = by_x[q];
                P2 jlo, jhi;
                box(pieces[j], &jlo, &jhi);
                if (jlo[0] > ihi[0] + tol) break;
                if (jlo[1] > ihi[1] + tol || jhi[1] < ilo[1] - tol) continue;
                const uint32_t a = pieces[i].ends[0], b = pieces[i].ends[1];
                const uint32_t c = pieces[j].ends[0], d = pieces[j].ends[1];
                // An end of 1 segment inside the other.
                const struct {
                    size_t s;
                    std::array<uint32_t, 2> ends, other;
                } pairs[2] = {{i, {a, b}, {c, d}}, {j, {c, d}, {a, b}}};
                for (const auto& pr : pairs)
                    for (uint32_t v : pr.other)
                        if (v != pr.ends[0] && v != pr.ends[1] && on_segment(pts, pr.ends, v, tol)) {
                            cuts[pr.s].push_back(v);
                            changed = true;
                        }
                if (c == a || c == b || d == a || d == b) continue;
                const P2 pa = pts[a], pb = pts[b], pc = pts[c], pd = pts[d];
                const double o1 = orient(pa, pb, pc), o2 = orient(pa, pb, pd);
                const double o3 = orient(pc, pd, pa), o4 = orient(pc, pd, pb);
                if (o1 * o2 < 0.0 && o3 * o4 < 0.0) {
                    // A proper crossing, at the parameter o1 / (o1 - o2) along c-d.
                    const double s = o1 / (o1 - o2);
                    const P2 x{pc[0] + s * (pd[0] - pc[0]), pc[1] + s * (pd[1] - pc[1])};
                    uint32_t v = NONE;
                    for (size_t f = 0; f < fresh.size(); ++f)
                        if (dist(fresh[f], x) <= tol) {
                            v = (uint32_t)(pts.size() + f);
                            break;
                        }
                    if (v == NONE) {
                        fresh.push_back(x);
                        v = (uint32_t)(pts.size() + fresh.size() - 1);
                    }
                    cuts[i].push_back(v);
                    cuts[j].push_back(v);
                    changed = true;
                }
            }
        }
        pts.insert(pts.end(), fresh.begin(), fresh.end());
        if (!changed) break;
        std::vector<Piece> next;
        for (size_t k = 0; k < pieces.size(); ++k) {
            const Piece& p = pieces[k];
            const P2 a = pts[p.ends[0]], b = pts[p.ends[1]];
            auto along = [&](uint32_t v) {
                const P2 q = pts[v];
                return (q[0] - a[0]) * (b[0] - a[0]) + (q[1] - a[1]) * (b[1] - a[1]);
            };
            std::vector<uint32_t> cut = cuts[k];
            std::stable_sort(cut.begin(), cut.end(),
                             [&](uint32_t x, uint32_t y) { return tless(along(x), along(y)); });
            cut.erase(std::unique(cut.begin(), cut.end()), cut.end());
            cut.push_back(p.ends[1]);
            uint32_t prev = p.ends[0];
            for (uint32_t v : cut)
                if (v != prev) {
                    next.push_back(Piece{{prev, v}, p.origin});
                    prev = v;
                }
        }
        pieces = std::move(next);
    }
    // Pieces on the same 2 points are 1 piece with the input segments of each.
    std::unordered_map<uint64_t, size_t> merged;
    std::vector<Piece>& out = *out_pieces;
    out.clear();
    for (Piece& p : pieces) {
        const uint64_t key = ((uint64_t)std::min(p.ends[0], p.ends[1]) << 32) |
                             std::max(p.ends[0], p.ends[1]);
        auto it = merged.find(key);
        if (it != merged.end()) {
            for (uint32_t o : p.origin) {
                auto& og = out[it->second].origin;
                if (std::find(og.begin(), og.end(), o) == og.end()) og.push_back(o);
            }
        } else {
            merged.emplace(key, out.size());
            out.push_back(std::move(p));
        }
    }
}


// A triangle: its points counterclockwise, the triangle across the edge opposite each point (NONE
// at the hull) and the segment piece on that edge (NONE: none), and its region's label.
struct Tri {
    std::array<uint32_t, 3> v, n, seg;
    uint32_t label;
};

// Where a point lies: inside triangle t, on the edge opposite point i of t, or at vertex v.
struct Where {
    enum Kind { INSIDE, EDGE, VERTEX } kind;
    size_t t;
    int i;
    uint32_t v;
};

struct QueuedPiece {
    uint32_t a, b, piece;
    bool force;  // split even when nothing encroaches it
};

struct QueuedTri {
    size_t t;
    std::array<uint32_t, 3> v;
};

// The triangulation under refinement (mesh2d.rs:358-1233).
class Triangulation {
   public:
    std::vector<P2> pts;
    std::vector<double> size;        // the target size at each point
    std::vector<uint32_t> on_piece;  // the piece a point split, or NONE
    size_t inputs = 0;               // points after the clean; the next 3 are the outer triangle
    std::vector<Tri> tris;
    std::vector<uint32_t> at;  // a triangle of each point
    std::vector<std::array<uint32_t, 2>> piece_ends;
    std::vector<std::vector<uint32_t>> piece_origin;
    double max_size = 0, growth = 0;
    size_t last = 0;

    Triangulation(const std::vector<P2>& in, Size2 sz) {
        P2 lo{INFINITY, INFINITY}, hi{-INFINITY, -INFINITY};
        for (const P2& p : in)
            for (int d = 0; d < 2; ++d) {
                lo[d] = std::min(lo[d], p[d]);
                hi[d] = std::max(hi[d], p[d]);
            }
        const P2 c{0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1])};
        const double r = 100.0 * std::max(dist(lo, hi), sz.max_size);
        const size_t n = in.size();
        pts = in;
        pts.push_back({c[0] - 2.0 * r, c[1] - r});
        pts.push_back({c[0] + 2.0 * r, c[1] - r});
        pts.push_back({c[0], c[1] + 2.0 * r});
        size.assign(n + 3, sz.max_size);
        on_piece.assign(n + 3, NONE);
        inputs = n;
        tris.push_back(Tri{{(uint32_t)n, (uint32_t)n + 1, (uint32_t)n + 2}, {NONE, NONE, NONE},
                           {NONE, NONE, NONE}, kOutside});
        at.assign(n + 3, 0);
        max_size = sz.max_size;
        growth = sz.max_growth - 1.0;
        // Insertion in the order of x (then y), so that each walk is short.
        std::vector<size_t> order(n);
        for (size_t i = 0; i < n; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            if (tless(in[a][0], in[b][0])) return true;
            if (tless(in[b][0], in[a][0])) return false;
            return tless(in[a][1], in[b][1]);
        });
        for (size_t i : order) {
            const Where w = locate(pts[i], last);
            if (w.kind == Where::INSIDE)
                split_triangle(w.t, (uint32_t)i);
            else if (w.kind == Where::EDGE)
                split_edge(w.t, w.i, (uint32_t)i);
            else
                fail("the clean merged equal points");
        }
    }

    P2 p(uint32_t v) const { return pts[v]; }

    int index_of(size_t t, uint32_t v) const {
        for (int k = 0; k < 3; ++k)
            if (tris[t].v[k] == v) return k;
        fail("a point of the triangle");
    }

    int edge_to(size_t t, uint32_t other) const {
        for (int k = 0; k < 3; ++k)
            if (tris[t].n[k] == other) return k;
        fail("a neighbour");
    }

    void repoint(uint32_t n, uint32_t old, uint32_t now) {
        if (n != NONE) tris[n].n[edge_to(n, old)] = now;
    }

    void set_at(size_t t) {
        for (uint32_t v : tris[t].v) at[v] = (uint32_t)t;
    }

    // The triangle, edge or point that holds q, by a visibility walk from `start` whose first
    // edge tried at each step comes from a linear congruential sequence (mesh2d.rs:468-506).
    Where locate(P2 q, size_t start) {
        size_t t = start;
        uint64_t turn = 0;
        const size_t limit = 4 * tris.size() + 100;
        for (size_t step = 0; step < limit; ++step) {
            const Tri tri = tris[t];
            turn = turn * 1103515245ull + 12345ull;
            const uint64_t first = (turn >> 16) % 3;
            bool moved = false;
            for (int k = 0; k < 3; ++k) {
                const int i = (int)((first + k) % 3);
                if (orient(p(tri.v[(i + 1) % 3]), p(tri.v[(i + 2) % 3]), q) < 0.0) {
                    if (tri.n[i] == NONE) fail("a point is outside the outer triangle");
                    t = tri.n[i];
                    moved = true;
                    break;
                }
            }
            if (moved) continue;
            last = t;
            int zero[3], nz = 0;
            for (int i = 0; i < 3; ++i)
                if (orient(p(tri.v[(i + 1) % 3]), p(tri.v[(i + 2) % 3]), q) == 0.0) zero[nz++] = i;
            if (nz == 0) return Where{Where::INSIDE, t, 0, 0};
            if (nz == 1) return Where{Where::EDGE, t, zero[0], 0};
            uint32_t v = tri.v[0];
            for (uint32_t x : tri.v)
                if (p(x) == q) {
                    v = x;
                    break;
                }
            return Where{Where::VERTEX, t, 0, v};
        }
        fail("the walk to a point did not end");
    }

    // Point v inside triangle t: 3 triangles, then flips to the Delaunay triangulation.
    void split_triangle(size_t t, uint32_t v) {
        const Tri old = tris[t];
        const uint32_t a = old.v[0], b = old.v[1], c = old.v[2];
        const uint32_t t1 = (uint32_t)tris.size(), t2 = t1 + 1, tu = (uint32_t)t;
        tris[t] = Tri{{v, b, c}, {old.n[0], t1, t2}, {old.seg[0], NONE, NONE}, old.label};
        tris.push_back(Tri{{v, c, a}, {old.n[1], t2, tu}, {old.seg[1], NONE, NONE}, old.label});
        tris.push_back(Tri{{v, a, b}, {old.n[2], tu, t1}, {old.seg[2], NONE, NONE}, old.label});
        repoint(old.n[1], tu, t1);
        repoint(old.n[2], tu, t2);
        set_at(t);
        set_at(t1);
        set_at(t2);
        legalize({{t, 0}, {t1, 0}, {t2, 0}});
    }

    // Point v on the edge opposite point i of t; on a segment both halves keep the segment.
    void split_edge(size_t t, int i, uint32_t v) {
        const Tri old = tris[t];
        const uint32_t a = old.v[i], b = old.v[(i + 1) % 3], c = old.v[(i + 2) % 3];
        const uint32_t seg = old.seg[i];
        const uint32_t t_a = old.n[(i + 1) % 3], s_a = old.seg[(i + 1) % 3];  // edge c-a
        const uint32_t t_b = old.n[(i + 2) % 3], s_b = old.seg[(i + 2) % 3];  // edge a-b
        const uint32_t n = old.n[i];
        const uint32_t t3 = (uint32_t)tris.size(), tu = (uint32_t)t;
        if (n == NONE) {
            tris[t] = Tri{{a, b, v}, {NONE, t3, t_b}, {seg, NONE, s_b}, old.label};
            tris.push_back(Tri{{a, v, c}, {NONE, t_a, tu}, {seg, s_a, NONE}, old.label});
            repoint(t_a, tu, t3);
            set_at(t);
            set_at(t3);
            legalize({{t, 2}, {t3, 1}});
            return;
        }
        const Tri on = tris[n];
        const int j = edge_to(n, tu);
        const uint32_t d = on.v[j];
        const uint32_t n_d = on.n[(j + 2) % 3], sn_d = on.seg[(j + 2) % 3];  // edge d-c
        const uint32_t n_c = on.n[(j + 1) % 3], sn_c = on.seg[(j + 1) % 3];  // edge b-d
        const uint32_t t4 = t3 + 1;
        tris[t] = Tri{{a, b, v}, {t4, t3, t_b}, {seg, NONE, s_b}, old.label};
        tris.push_back(Tri{{a, v, c}, {n, t_a, tu}, {seg, s_a, NONE}, old.label});
        tris[n] = Tri{{d, c, v}, {t3, t4, n_d}, {seg, NONE, sn_d}, on.label};
        tris.push_back(Tri{{d, v, b}, {tu, n_c, n}, {seg, sn_c, NONE}, on.label});
        repoint(t_a, tu, t3);
        repoint(n_c, n, t4);
        set_at(t);
        set_at(t3);
        set_at(n);
        set_at(t4);
        legalize({{t, 2}, {t3, 1}, {n, 2}, {t4, 1}});
    }

    // Flip each stacked edge (opposite point i of t, the new point) whose other triangle has its
    // far point inside the circumcircle; segments are never flipped (Lawson).
    void legalize(std::vector<std::pair<size_t, int>> stack) {
        while (!stack.empty()) {
            const auto [t, i] = stack.back();
            stack.pop_back();
            const Tri tri = tris[t];
            const uint32_t n = tri.n[i];
            if (n == NONE || tri.seg[i] != NONE) continue;
            const int j = edge_to(n, (uint32_t)t);
            const uint32_t d = tris[n].v[j];
            if (incircle(p(tri.v[0]), p(tri.v[1]), p(tri.v[2]), p(d)) > 0.0) {
                flip(t, i);
                stack.push_back({t, 0});
                stack.push_back({n, 0});
            }
        }
    }

    // Flip the edge opposite point i of t: t becomes (a, b, d), its neighbour (a, d, c).
    void flip(size_t t, int i) {
        const Tri tri = tris[t];
        const uint32_t a = tri.v[i], b = tri.v[(i + 1) % 3], c = tri.v[(i + 2) % 3];
        const uint32_t t_a = tri.n[(i + 1) % 3], s_a = tri.seg[(i + 1) % 3];  // edge c-a
        const uint32_t t_b = tri.n[(i + 2) % 3], s_b = tri.seg[(i + 2) % 3];  // edge a-b
        const uint32_t n = tri.n[i];
        const Tri on = tris[n];
        const int j = edge_to(n, (uint32_t)t);
        const uint32_t d = on.v[j];
        const uint32_t n_c = on.n[(j + 1) % 3], sn_c = on.seg[(j + 1) % 3];  // edge b-d
        const uint32_t n_d = on.n[(j + 2) % 3], sn_d = on.seg[(j + 2) % 3];  // edge d-c
        tris[t] = Tri{{a, b, d}, {n_c, n, t_b}, {sn_c, NONE, s_b}, tri.label};
        tris[n] = Tri{{a, d, c}, {n_d, t_a, (uint32_t)t}, {sn_d, s_a, NONE}, on.label};
        repoint(n_c, n, (uint32_t)t);
        repoint(t_a, (uint32_t)t, n);
        set_at(t);
        set_at(n);
    }

    // The triangle and local index of edge a-b, turning around a both ways (a may be on the hull).
    bool find_edge(uint32_t a, uint32_t b, size_t* ft, int* fi) const {
        const size_t start = at[a];
        for (int dir = 1; dir <= 2; ++dir) {
            size_t t = start;
            for (int step = 0; step < 10000; ++step) {
                const int k = index_of(t, a);
                const Tri& tri = tris[t];
                if (tri.v[(k + 1) % 3] == b) {
                    *ft = t;
                    *fi = (k + 2) % 3;
                    return true;
                }
                if (tri.v[(k + 2) % 3] == b) {
                    *ft = t;
                    *fi = (k + 1) % 3;
                    return true;
                }
                const uint32_t next = tri.n[(k + dir) % 3];
                if (next == NONE || next == start) break;
                t = next;
            }
        }
        return false;
    }

    // The split point of piece a-b: its middle, or a power-of-2 distance from an input point at
    // 1 end (concentric shells), kept within a quarter and 3 quarters.
    P2 split_point(uint32_t a, uint32_t b) const {
        const P2 pa = p(a), pb = p(b);
        const double len = dist(pa, pb);
        const bool ia = a < inputs, ib = b < inputs;
        if (ia != ib) {
            const P2 from = ia ? pa : pb, to = ia ? pb : pa;
            const double d = std::pow(2.0, std::round(std::log2(0.5 * len)));
            const double s = std::min(std::max(d / len, 0.25), 0.75);
            return {from[0] + s * (to[0] - from[0]), from[1] + s * (to[1] - from[1])};
        }
        return {0.5 * (pa[0] + pb[0]), 0.5 * (pa[1] + pb[1])};
    }

    // The size at a new point q from the points `near`: the graded field, at most max_size.
    double size_at(P2 q, const uint32_t* near, int count) const {
        double h = max_size;
        for (int k = 0; k < count; ++k)
            h = std::min(h, size[near[k]] + growth * dist(q, p(near[k])));
        return h;
    }

    uint32_t add_point(P2 q, double h, uint32_t piece) {
        if (pts.size() >= kMaxVertices)
            fail("the 2D mesh needs more than " + std::to_string(kMaxVertices) +
                 " points: use a larger max_cell, or remove a very small detail of an outline");
        pts.push_back(q);
        size.push_back(h);
        on_piece.push_back(piece);
        at.push_back(0);
        return (uint32_t)pts.size() - 1;
    }

    // Split piece a-b of segment `piece` (an edge) at its split point.
    uint32_t split_piece(uint32_t a, uint32_t b, uint32_t piece) {
        size_t t;
        int i;
        if (!find_edge(a, b, &t, &i)) fail("a piece of a segment is an edge");
        const P2 m = split_point(a, b);
        const uint32_t ab[2] = {a, b};
        const uint32_t v = add_point(m, size_at(m, ab, 2), piece);
        split_edge(t, i, v);
        return v;
    }

    // Make each segment a chain of edges by splitting the ones that are not edges, then mark the
    // edges of the segments fixed (mesh2d.rs:746-787).
    void recover() {
        std::vector<std::array<uint32_t, 3>> queue;
        for (size_t k = 0; k < piece_ends.size(); ++k)
            queue.push_back({piece_ends[k][0], piece_ends[k][1], (uint32_t)k});
        while (!queue.empty()) {
            const auto [a, b, piece] = queue.back();
            queue.pop_back();
            size_t t;
            int i;
            if (find_edge(a, b, &t, &i)) {
                tris[t].seg[i] = piece;
                const uint32_t n = tris[t].n[i];
                if (n != NONE) tris[n].seg[edge_to(n, (uint32_t)t)] = piece;
                continue;
            }
            const P2 m = split_point(a, b);
            const Where w = locate(m, at[a]);
            const uint32_t ab[2] = {a, b};
            uint32_t v;
            if (w.kind == Where::VERTEX) {
                v = w.v;
            } else {
                v = add_point(m, size_at(m, ab, 2), piece);
                if (w.kind == Where::INSIDE)
                    split_triangle(w.t, v);
                else
                    split_edge(w.t, w.i, v);
            }
            if (v == a || v == b) fail("2 segments of the outlines are too close to mesh");
            queue.push_back({a, v, piece});
            queue.push_back({v, b, piece});
        }
    }

    double area2(size_t t) const {
        const Tri& tri = tris[t];
        return orient(p(tri.v[0]), p(tri.v[1]), p(tri.v[2]));
    }

    // Each region bounded by segments takes the label of the centroid of its largest triangle (the
    // last of equal ones); a region touching the outer triangle is outside (mesh2d.rs:789-834).
    void label_regions(const std::function<uint32_t(P2)>& classify) {
        std::vector<uint32_t> region(tris.size(), NONE);
        for (size_t start = 0; start < tris.size(); ++start) {
            if (region[start] != NONE) continue;
            std::vector<size_t> members{start};
            region[start] = (uint32_t)start;
            for (size_t k = 0; k < members.size(); ++k) {
                const Tri tri = tris[members[k]];
                for (int i = 0; i < 3; ++i) {
                    const uint32_t n = tri.n[i];
                    if (n != NONE && tri.seg[i] == NONE && region[n] == NONE) {
                        region[n] = (uint32_t)start;
                        members.push_back(n);
                    }
                }
            }
            bool outer = false;
            for (size_t t : members)
                for (uint32_t v : tris[t].v)
                    if (v >= inputs && v < inputs + 3) outer = true;
            uint32_t label = kOutside;
            if (!outer) {
                size_t big = members[0];
                double best = area2(big);
                for (size_t k = 1; k < members.size(); ++k) {
                    const double a = area2(members[k]);
                    if (!tless(a, best)) {  // ties go to the later triangle
                        best = a;
                        big = members[k];
                    }
                }
                const P2 a = p(tris[big].v[0]), b = p(tris[big].v[1]), c = p(tris[big].v[2]);
                label = classify({(a[0] + b[0] + c[0]) / 3.0, (a[1] + b[1] + c[1]) / 3.0});
            }
            for (size_t t : members) tris[t].label = label;
        }
    }

    // The circumcentre of t and its squared circumradius (mesh2d.rs:837-849).
    void circumcentre(size_t t, P2* centre, double* r2) const {
        const P2 a = p(tris[t].v[0]), b = p(tris[t].v[1]), c = p(tris[t].v[2]);
        const double bx = b[0] - a[0], by = b[1] - a[1];
        const double cx = c[0] - a[0], cy = c[1] - a[1];
        const double d = 2.0 * orient({0.0, 0.0}, {bx, by}, {cx, cy});
        const double b2 = bx * bx + by * by, c2 = cx * cx + cy * cy;
        const double ux = (cy * b2 - by * c2) / d, uy = (bx * c2 - cx * b2) / d;
        *centre = {a[0] + ux, a[1] + uy};
        *r2 = ux * ux + uy * uy;
    }

    // A labelled triangle that is too large for the size field, or skinny (circumradius over
    // shortest edge above sqrt 2) unless its short edge joins 2 segments meeting below 60 degrees.
    bool bad(size_t t) const {
        const Tri& tri = tris[t];
        if (tri.label == kOutside) return false;
        P2 q[3];
        for (int k = 0; k < 3; ++k) q[k] = p(tri.v[k]);
        double len2[3];
        for (int i = 0; i < 3; ++i) {
            const P2 a = q[(i + 1) % 3], b = q[(i + 2) % 3];
            len2[i] = (a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]);
        }
        int shortest = 0;
        for (int i = 1; i < 3; ++i)
            if (tless(len2[i], len2[shortest])) shortest = i;
        P2 centre;
        double r2;
        circumcentre(t, &centre, &r2);
        const P2 g{(q[0][0] + q[1][0] + q[2][0]) / 3.0, (q[0][1] + q[1][1] + q[2][1]) / 3.0};
        const double h = size_at(g, tri.v.data(), 3);
        if (3.0 * r2 > h * h) return true;
        if (r2 <= kRatio * kRatio * len2[shortest]) return false;
        return !small_angle_between(tri.v[(shortest + 1) % 3], tri.v[(shortest + 2) % 3]);
    }

    // True when u and w are on 2 pieces that share an input point where they meet at an angle
    // below 60 degrees.
    bool small_angle_between(uint32_t u, uint32_t w) const {
        const uint32_t pu = on_piece[u], pw = on_piece[w];
        if (pu == NONE || pw == NONE || pu == pw) return false;
        const auto eu = piece_ends[pu], ew = piece_ends[pw];
        for (uint32_t z : eu) {
            if (ew[0] != z && ew[1] != z) continue;
            const P2 pz = p(z);
            const P2 x = p(eu[0] == z ? eu[1] : eu[0]), y = p(ew[0] == z ? ew[1] : ew[0]);
            const double vx0 = x[0] - pz[0], vx1 = x[1] - pz[1];
            const double vy0 = y[0] - pz[0], vy1 = y[1] - pz[1];
            const double cosine =
                (vx0 * vy0 + vx1 * vy1) / (std::hypot(vx0, vx1) * std::hypot(vy0, vy1));
            return cosine > 0.5;
        }
        return false;
    }

    // Piece opposite point i of t is encroached when the far point of a labelled triangle beside
    // it lies inside its diametral circle.
    bool encroached(size_t t, int i) const {
        auto check = [&](size_t s, int k) {
            const Tri& tri = tris[s];
            if (tri.label == kOutside) return false;
            const P2 a = p(tri.v[(k + 1) % 3]), b = p(tri.v[(k + 2) % 3]), c = p(tri.v[k]);
            return (a[0] - c[0]) * (b[0] - c[0]) + (a[1] - c[1]) * (b[1] - c[1]) < 0.0;
        };
        if (check(t, i)) return true;
        const uint32_t n = tris[t].n[i];
        return n != NONE && check(n, edge_to(n, (uint32_t)t));
    }

    // The triangle that holds c, by a straight walk from the centroid of t; `hit` is set, with the
    // triangle and edge, when the walk meets a segment first (mesh2d.rs:924-967).
    Where walk(size_t t, P2 c, bool* hit) const {
        const P2 q0 = p(tris[t].v[0]), q1 = p(tris[t].v[1]), q2 = p(tris[t].v[2]);
        const P2 s{(q0[0] + q1[0] + q2[0]) / 3.0, (q0[1] + q1[1] + q2[1]) / 3.0};
        uint32_t from = NONE;
        *hit = false;
        for (size_t step = 0; step < tris.size() + 10; ++step) {
            const Tri& tri = tris[t];
            double o[3];
            for (int i = 0; i < 3; ++i) o[i] = orient(p(tri.v[(i + 1) % 3]), p(tri.v[(i + 2) % 3]), c);
            if (o[0] >= 0.0 && o[1] >= 0.0 && o[2] >= 0.0) {
                int zero[3], nz = 0;
                for (int i = 0; i < 3; ++i)
                    if (o[i] == 0.0) zero[nz++] = i;
                if (nz == 0) return Where{Where::INSIDE, t, 0, 0};
                if (nz == 1) return Where{Where::EDGE, t, zero[0], 0};
                return Where{Where::VERTEX, t, 0, tri.v[3 - zero[0] - zero[1]]};
            }
            // The exit edge: c beyond it and the line s-c passing between its 2 points.
            int exit = -1;
            for (int i = 0; i < 3 && exit < 0; ++i) {
                if (!(o[i] < 0.0 && tri.n[i] != from)) continue;
                const double a = orient(s, c, p(tri.v[(i + 1) % 3]));
                const double b = orient(s, c, p(tri.v[(i + 2) % 3]));
                if (a * b <= 0.0) exit = i;
            }
            for (int i = 0; i < 3 && exit < 0; ++i)
                if (o[i] < 0.0) exit = i;
            if (tri.seg[exit] != NONE) {
                *hit = true;
                return Where{Where::EDGE, t, exit, 0};
            }
            if (tri.n[exit] == NONE) fail("a circumcentre is outside the outer triangle");
            from = (uint32_t)t;
            t = tri.n[exit];
        }
        fail("the walk to a circumcentre did not end");
    }

    // The pieces on the edges of the cavity of c (the triangles from t whose circumcircle holds
    // it) whose diametral circle holds c.
    std::vector<std::array<uint32_t, 3>> encroached_by(size_t t, P2 c) const {
        std::vector<size_t> seen{t};
        std::vector<std::array<uint32_t, 3>> out;
        for (size_t k = 0; k < seen.size(); ++k) {
            const Tri tri = tris[seen[k]];
            for (int i = 0; i < 3; ++i) {
                const uint32_t a = tri.v[(i + 1) % 3], b = tri.v[(i + 2) % 3];
                if (tri.seg[i] != NONE) {
                    const P2 pa = p(a), pb = p(b);
                    if ((pa[0] - c[0]) * (pb[0] - c[0]) + (pa[1] - c[1]) * (pb[1] - c[1]) < 0.0)
                        out.push_back({a, b, tri.seg[i]});
                    continue;
                }
                const uint32_t n = tri.n[i];
                if (n == NONE || std::find(seen.begin(), seen.end(), (size_t)n) != seen.end())
                    continue;
                const Tri& nt = tris[n];
                if (incircle(p(nt.v[0]), p(nt.v[1]), p(nt.v[2]), c) > 0.0) seen.push_back(n);
            }
        }
        return out;
    }

    // The triangles around point v, turning 1 way and, at the hull, the other way too.
    std::vector<size_t> star(uint32_t v) const {
        const size_t start = at[v];
        std::vector<size_t> out{start};
        for (int dir = 1; dir <= 2; ++dir) {
            size_t t = start;
            for (;;) {
                const int k = index_of(t, v);
                const uint32_t next = tris[t].n[(k + dir) % 3];
                if (next == NONE) break;
                if (next == start) return out;
                t = next;
                out.push_back(t);
            }
        }
        return out;
    }

    void after_insert(uint32_t v, std::deque<QueuedPiece>& pieces, std::deque<QueuedTri>& badq) {
        for (size_t t : star(v)) {
            const Tri tri = tris[t];
            if (bad(t)) badq.push_back({t, tri.v});
            for (int i = 0; i < 3; ++i)
                if (tri.seg[i] != NONE && encroached(t, i))
                    pieces.push_back({tri.v[(i + 1) % 3], tri.v[(i + 2) % 3], tri.seg[i], false});
        }
    }

    // Ruppert refinement of the labelled regions: encroached pieces first, then bad triangles
    // by their circumcentres, each in the order queued (mesh2d.rs:1022-1097).
    void refine() {
        std::deque<QueuedPiece> pieces;
        std::deque<QueuedTri> badq;
        for (size_t t = 0; t < tris.size(); ++t) {
            for (int i = 0; i < 3; ++i) {
                const Tri tri = tris[t];
                const uint32_t a = tri.v[(i + 1) % 3], b = tri.v[(i + 2) % 3];
                if (tri.seg[i] != NONE && a < b && encroached(t, i))
                    pieces.push_back({a, b, tri.seg[i], false});
            }
            if (bad(t)) badq.push_back({t, tris[t].v});
        }
        for (;;) {
            if (!pieces.empty()) {
                const QueuedPiece q = pieces.front();
                pieces.pop_front();
                size_t t;
                int i;
                if (!find_edge(q.a, q.b, &t, &i)) continue;
                if (tris[t].seg[i] == NONE || !(q.force || encroached(t, i))) continue;
                const uint32_t v = split_piece(q.a, q.b, q.piece);
                after_insert(v, pieces, badq);
                continue;
            }
            if (badq.empty()) break;
            const QueuedTri bt = badq.front();
            badq.pop_front();
            if (tris[bt.t].v != bt.v || !bad(bt.t)) continue;
            P2 c;
            double r2;
            circumcentre(bt.t, &c, &r2);
            bool hit;
            const Where w = walk(bt.t, c, &hit);
            if (hit || (w.kind == Where::EDGE && tris[w.t].seg[w.i] != NONE)) {
                // The circumcentre lies beyond a segment, or on one: split that piece instead.
                const Tri& s = tris[w.t];
                pieces.push_back({s.v[(w.i + 1) % 3], s.v[(w.i + 2) % 3], s.seg[w.i], true});
                badq.push_back(bt);
                continue;
            }
            if (w.kind == Where::VERTEX) continue;
            const auto list = encroached_by(w.t, c);
            if (!list.empty()) {
                for (const auto& e : list) pieces.push_back({e[0], e[1], e[2], true});
                badq.push_back(bt);
                continue;
            }
            const uint32_t fresh = add_point(c, size_at(c, bt.v.data(), 3), NONE);
            if (w.kind == Where::INSIDE)
                split_triangle(w.t, fresh);
            else
                split_edge(w.t, w.i, fresh);
            after_insert(fresh, pieces, badq);
        }
    }

    // The pieces on the line u[d] = at: their ends and the piece.
    std::vector<std::array<uint32_t, 3>> pieces_on(int d, double line, double tol) const {
        std::vector<std::array<uint32_t, 3>> out;
        for (const Tri& tri : tris)
            for (int i = 0; i < 3; ++i) {
                const uint32_t a = tri.v[(i + 1) % 3], b = tri.v[(i + 2) % 3];
                if (tri.seg[i] != NONE && a < b && std::fabs(p(a)[d] - line) <= tol &&
                    std::fabs(p(b)[d] - line) <= tol)
                    out.push_back({a, b, tri.seg[i]});
            }
        return out;
    }

    // Each vertex on a piece on 1 side of the inputs' bounding box gets a partner at the same
    // place on the opposite side (a split of the piece there); returns the new vertices
    // (mesh2d.rs:1136-1197).
    size_t match_sides() {
        P2 lo{INFINITY, INFINITY}, hi{-INFINITY, -INFINITY};
        for (size_t k = 0; k < inputs; ++k)
            for (int d = 0; d < 2; ++d) {
                lo[d] = std::min(lo[d], pts[k][d]);
                hi[d] = std::max(hi[d], pts[k][d]);
            }
        const double tol = 1e-9 * std::max(dist(lo, hi), std::numeric_limits<double>::min());
        size_t added = 0;
        for (int d = 0; d < 2; ++d) {
            const int o = 1 - d;
            auto length = [&](const std::vector<std::array<uint32_t, 3>>& list) {
                double sum = 0.0;
                for (const auto& e : list) sum += std::fabs(p(e[0])[o] - p(e[1])[o]);
                return sum;
            };
            const double low = length(pieces_on(d, lo[d], tol));
            const double high = length(pieces_on(d, hi[d], tol));
            if (std::fabs(low - high) > 1e-6 * (hi[o] - lo[o])) {
                const char* u = d == 0 ? "a" : "b";
                fail(std::string("the outlines on the 2 sides ") + u + " = " + rust_display(lo[d]) +
                     " and " + u + " = " + rust_display(hi[d]) +
                     " of the cell do not match: the parts must touch the 2 sides along the same "
                     "ranges, so that copies of the cell side by side fill the space");
            }
            const double ends[2][2] = {{lo[d], hi[d]}, {hi[d], lo[d]}};
            for (const auto& fr : ends) {
                const auto src = pieces_on(d, fr[0], tol);
                auto dst = pieces_on(d, fr[1], tol);
                std::vector<double> want;
                for (const auto& e : src) {
                    want.push_back(p(e[0])[o]);
                    want.push_back(p(e[1])[o]);
                }
                std::stable_sort(want.begin(), want.end(), tless);
                std::vector<double> kept;
                for (double w : want)
                    if (kept.empty() || !(std::fabs(w - kept.back()) <= tol)) kept.push_back(w);
                for (double c : kept) {
                    size_t k = dst.size();
                    for (size_t q = 0; q < dst.size(); ++q) {
                        const double pa = p(dst[q][0])[o], pb = p(dst[q][1])[o];
                        if (std::min(pa, pb) + tol < c && c < std::max(pa, pb) - tol) {
                            k = q;
                            break;
                        }
                    }
                    if (k == dst.size()) continue;
                    const auto [a, b, piece] = dst[k];
                    P2 m{0.0, 0.0};
                    m[d] = p(a)[d];
                    m[o] = c;
                    size_t t;
                    int i;
                    if (!find_edge(a, b, &t, &i)) fail("a piece of a segment is an edge");
                    const uint32_t ab[2] = {a, b};
                    const uint32_t v = add_point(m, size_at(m, ab, 2), piece);
                    split_edge(t, i, v);
                    dst[k] = {a, v, piece};
                    dst.push_back({v, b, piece});
                    ++added;
                }
            }
        }
        return added;
    }

    // The labelled triangles on the points they use, numbered in first use.
    Mesh2 output() const {
        Mesh2 m;
        std::vector<uint32_t> map(pts.size(), NONE), number(tris.size(), NONE);
        uint32_t kept = 0;
        for (size_t t = 0; t < tris.size(); ++t)
            if (tris[t].label != kOutside) number[t] = kept++;
        for (const Tri& tri : tris) {
            if (tri.label == kOutside) continue;
            m.across.push_back({tri.n[0] == NONE ? NONE : number[tri.n[0]],
                                tri.n[1] == NONE ? NONE : number[tri.n[1]],
                                tri.n[2] == NONE ? NONE : number[tri.n[2]]});
            std::array<uint32_t, 3> v;
            for (int k = 0; k < 3; ++k) {
                if (map[tri.v[k]] == NONE) {
                    map[tri.v[k]] = (uint32_t)m.points.size();
                    m.points.push_back(pts[tri.v[k]]);
                }
                v[k] = map[tri.v[k]];
            }
            for (int i = 0; i < 3; ++i)
                if (tri.seg[i] != NONE) {
                    const uint32_t a = v[(i + 1) % 3], b = v[(i + 2) % 3];
                    m.segments[{std::min(a, b), std::max(a, b)}] = piece_origin[tri.seg[i]];
                }
            m.triangles.push_back(v);
            m.label.push_back(tri.label);
        }
        return m;
    }
};

}  // namespace

Mesh2 quality_mesh(const std::vector<P2>& points, const std::vector<std::array<uint32_t, 2>>& segs,
                   Size2 size, const std::function<uint32_t(P2)>& classify, bool periodic) {
    if (!(size.max_size > 0.0 && std::isfinite(size.max_size)))
        fail("the largest cell size must be a number above 0");
    if (!(size.max_growth > 1.0 && std::isfinite(size.max_growth)))
        fail("max_growth must be a number above 1");
    for (const P2& q : points)
        if (!std::isfinite(q[0]) || !std::isfinite(q[1]))
            fail("each point of an outline must have finite coordinates");
    std::vector<P2> pts;
    std::vector<Piece> pieces;
    clean(points, segs, &pts, &pieces);
    if (pieces.empty()) fail("the outlines have no segment");
    Triangulation t(pts, size);
    for (const Piece& pc : pieces) {
        const double len = dist(pts[pc.ends[0]], pts[pc.ends[1]]);
        for (uint32_t v : pc.ends) t.size[v] = std::min(t.size[v], len);
        t.piece_ends.push_back(pc.ends);
        t.piece_origin.push_back(pc.origin);
    }
    t.recover();
    t.label_regions(classify);
    t.refine();
    if (periodic) {
        int rounds = 0;
        while (t.match_sides() > 0) {
            if (++rounds > kPeriodicRounds)
                fail("the periodic 2D mesh did not settle in " + std::to_string(kPeriodicRounds) +
                     " rounds: use a larger max_cell or a larger max_growth");
            t.refine();
        }
    }
    return t.output();
}

}  // namespace femgpu
