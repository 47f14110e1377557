"""The host steps of the prism mesh, on the CPU: the quality triangle mesh (mesh2d.rs, checked
with the reference's own properties from crates/fem/tests/mesh2d.rs, in exact arithmetic), the
prism split (tests/tet.rs:89-140) and the graded planes of an axis (grid.rs:418-484, bit-exact
with the oracle, and grid.rs:548-612's properties)."""
from __future__ import annotations

import itertools
import math
from fractions import Fraction

import numpy as np
import pytest

from femahoy_b200 import prism as P
from femahoy_b200._lib import FemError
from oracle import prism as O


# ------------------------------------------------------------------ helpers (tests/mesh2d.rs)

def loops(polygons):
    """The points and segments of closed polygons (tests/mesh2d.rs:10-22)."""
    pts, segs = [], []
    for poly in polygons:
        base = len(pts)
        pts.extend(poly)
        segs.extend((base + k, base + (k + 1) % len(poly)) for k in range(len(poly)))
    return np.array(pts, dtype=np.float64), np.array(segs, dtype=np.uint32)


def circle(c, r, n):
    return [(c[0] + r * math.cos(2 * math.pi * k / n), c[1] + r * math.sin(2 * math.pi * k / n))
            for k in range(n)]


def area(poly):
    return 0.5 * abs(sum(poly[k][0] * poly[(k + 1) % len(poly)][1]
                         - poly[(k + 1) % len(poly)][0] * poly[k][1] for k in range(len(poly))))


def tri_area(m, t):
    a, b, c = m.points[m.triangles[t]]
    return 0.5 * ((b[0] - a[0]) * (c[1] - a[1]) - (c[0] - a[0]) * (b[1] - a[1]))


def min_angle(m, t):
    p = m.points[m.triangles[t]]
    out = 180.0
    for i in range(3):
        u, v = p[(i + 1) % 3] - p[i], p[(i + 2) % 3] - p[i]
        c = np.dot(u, v) / (np.linalg.norm(u) * np.linalg.norm(v))
        out = min(out, math.degrees(math.acos(max(-1.0, min(1.0, c)))))
    return out


def exact_incircle(a, b, c, d):
    a, b, c, d = ([Fraction(x) for x in p] for p in (a, b, c, d))
    rows = [(p[0] - d[0], p[1] - d[1]) for p in (a, b, c)]
    m = [(x, y, x * x + y * y) for x, y in rows]
    return (m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2])
            - m[0][1] * (m[1][0] * m[2][2] - m[2][0] * m[1][2])
            + m[0][2] * (m[1][0] * m[2][1] - m[2][0] * m[1][1]))


def exact_orient(a, b, c):
    a, b, c = ([Fraction(x) for x in p] for p in (a, b, c))
    return (a[0] - c[0]) * (b[1] - c[1]) - (a[1] - c[1]) * (b[0] - c[0])


def check(m):
    """tests/mesh2d.rs:78-103: counterclockwise triangles, each edge in at most 2 triangles, and
    each edge not on a segment locally Delaunay, all in exact arithmetic; also the across table
    agrees with the edges."""
    P_ = m.points
    edges = {}
    for t, tri in enumerate(m.triangles):
        assert exact_orient(*P_[tri]) > 0, f"triangle {t} is not counterclockwise"
        for i in range(3):
            e = tuple(sorted((int(tri[(i + 1) % 3]), int(tri[(i + 2) % 3]))))
            edges.setdefault(e, []).append((t, i))
    for e, lst in edges.items():
        assert len(lst) <= 2, f"edge {e} has {len(lst)} triangles"
        if len(lst) == 2:
            (t0, i0), (t1, i1) = lst
            assert m.across[t0, i0] == t1 and m.across[t1, i1] == t0
            if e not in m.segments:
                a, b, c = P_[m.triangles[t0]]
                d = P_[m.triangles[t1][i1]]
                assert exact_incircle(a, b, c, d) <= 0, f"edge {e} is not Delaunay"
        else:
            t0, i0 = lst[0]
            assert m.across[t0, i0] == P.OUTSIDE


def size(max_size):
    return P.Size(max_size, 1.3)


def in_poly(poly, x):
    return O.inside(poly, x)


# ------------------------------------------------------------------ mesh2d (tests/mesh2d.rs)

def test_a_square_has_the_angle_bound_and_its_area():
    sq = [(0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0)]
    p, s = loops([sq])
    m = P.mesh2d(p, s, size(0.1), lambda x: 0 if in_poly(sq, x) else P.OUTSIDE)
    check(m)
    total = sum(tri_area(m, t) for t in range(len(m.triangles)))
    assert abs(total - 1.0) < 1e-12
    assert min(min_angle(m, t) for t in range(len(m.triangles))) >= P.MIN_ANGLE
    for tri in m.triangles:
        for i in range(3):
            a, b = m.points[tri[i]], m.points[tri[(i + 1) % 3]]
            assert math.hypot(*(a - b)) < 0.1 * 1.5


def test_a_plate_with_a_hole_is_graded_and_has_the_angle_bound():
    outer = [(0.0, 0.0), (4.0, 0.0), (4.0, 2.0), (0.0, 2.0)]
    hole = circle((1.0, 1.0), 0.3, 48)
    p, s = loops([outer, hole])
    m = P.mesh2d(p, s, size(0.5),
                 lambda x: 7 if in_poly(outer, x) and not in_poly(hole, x) else P.OUTSIDE)
    check(m)
    total = sum(tri_area(m, t) for t in range(len(m.triangles)))
    assert abs(total - (8.0 - area(hole))) < 1e-12
    assert (m.label == 7).all()
    assert min(min_angle(m, t) for t in range(len(m.triangles))) >= P.MIN_ANGLE

    def mean_edge(pred):
        vals = [math.sqrt(tri_area(m, t)) for t, tri in enumerate(m.triangles)
                if pred(m.points[tri].mean(axis=0))]
        return sum(vals) / len(vals)

    near = mean_edge(lambda c: math.hypot(c[0] - 1.0, c[1] - 1.0) < 0.45)
    far = mean_edge(lambda c: c[0] > 3.5)
    assert far > 3.0 * near


def test_crossing_outlines_give_regions_with_the_right_areas():
    a = [(0.0, 0.0), (2.0, 0.0), (2.0, 2.0), (0.0, 2.0)]
    b = [(1.0, 1.0), (3.0, 1.0), (3.0, 3.0), (1.0, 3.0)]
    c = [(0.5, 0.0), (1.5, 0.0), (1.0, 2.5)]
    p, s = loops([a, b, c])

    def classify(x):
        bits = int(in_poly(a, x)) | int(in_poly(b, x)) << 1 | int(in_poly(c, x)) << 2
        return P.OUTSIDE if bits == 0 else bits

    m = P.mesh2d(p, s, size(0.25), classify)
    check(m)
    by = {}
    for t in range(len(m.triangles)):
        by[int(m.label[t])] = by.get(int(m.label[t]), 0.0) + tri_area(m, t)
    tip_left = 0.5 * 0.2 * 0.5 * 0.5
    assert abs(sum(by.values()) - (7.0 + tip_left)) < 1e-9
    for bit, want in ((1, 4.0), (2, 4.0), (4, area(c))):
        assert abs(sum(v for l, v in by.items() if l & bit) - want) < 1e-9
    assert min(min_angle(m, t) for t in range(len(m.triangles))) > 5.0
    # The crossings are edges of the mesh held by both input segments.
    assert any(len(v) == 2 for v in m.segments.values())


def test_a_small_input_angle_does_not_stop_the_refinement_from_ending():
    t = math.radians(5.0)
    wedge = [(0.0, 0.0), (1.0, 0.0), (math.cos(t), math.sin(t))]
    p, s = loops([wedge])
    m = P.mesh2d(p, s, size(0.05), lambda x: 0 if in_poly(wedge, x) else P.OUTSIDE)
    check(m)
    total = sum(tri_area(m, k) for k in range(len(m.triangles)))
    assert abs(total - area(wedge)) < 1e-12
    for k in range(len(m.triangles)):
        if min_angle(m, k) < P.MIN_ANGLE:
            r = max(math.hypot(*q) for q in m.points[m.triangles[k]])
            assert r < 0.5, f"a skinny triangle far from the tip, at r = {r}"


def test_a_periodic_mesh_has_matching_sides():
    """mesh2d.rs:1136-1197: each vertex on a side of the bounding box has a partner on the
    opposite side; a unit cell with an off-centre hole."""
    cell = [(0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0)]
    hole = circle((0.4, 0.55), 0.2, 32)
    p, s = loops([cell, hole])
    m = P.periodic_mesh2d(p, s, size(0.2),
                          lambda x: 0 if in_poly(cell, x) and not in_poly(hole, x) else P.OUTSIDE)
    check(m)
    for d in range(2):
        o = 1 - d
        lo = sorted(q[o] for q in m.points if abs(q[d]) <= 1e-12)
        hi = sorted(q[o] for q in m.points if abs(q[d] - 1.0) <= 1e-12)
        assert len(lo) == len(hi) and np.allclose(lo, hi, atol=1e-12)


def test_mesh2d_refuses_bad_sizes_and_empty_outlines_with_the_reference_texts():
    sq = [(0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0)]
    p, s = loops([sq])
    cls = lambda x: 0  # noqa: E731
    for sz, text in ((P.Size(0.0, 1.3), "the largest cell size must be a number above 0"),
                     (P.Size(0.1, 1.0), "max_growth must be a number above 1")):
        with pytest.raises(FemError, match=text):
            P.mesh2d(p, s, sz, cls)
    with pytest.raises(FemError, match="the outlines have no segment"):
        P.mesh2d(p, np.zeros((0, 2), np.uint32), size(0.1), cls)
    bad = p.copy()
    bad[0, 0] = math.nan
    with pytest.raises(FemError, match="each point of an outline must have finite coordinates"):
        P.mesh2d(bad, s, size(0.1), cls)


# ------------------------------------------------------------------ split_prism (tests/tet.rs)

def _tet_volume(p):
    return O.volume(p)


def test_each_prism_split_fills_the_prism_and_cuts_each_face_at_its_smallest_corner():
    corners = [(0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0),
               (0.0, 0.0, 1.0), (1.0, 0.0, 1.0), (0.0, 1.0, 1.0)]
    quads = [(0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5)]
    count = 0
    for g in itertools.permutations(range(6)):
        count += 1
        tets = P.split_prism(g)
        assert tets == O.split_prism(g)
        total = sum(abs(_tet_volume([corners[k] for k in t])) for t in tets)
        assert abs(total - 0.5) < 1e-12, g
        for q in quads:
            mn = min(q, key=lambda k: g[k])
            opposite = q[(q.index(mn) + 2) % 4]
            assert any(mn in t and opposite in t for t in tets), (g, q)
    assert count == 720


# ------------------------------------------------------------------ planes (grid.rs)

def _part(name, lo, hi, material=0, priority=0):
    return P.Part(name, material, priority, lo, hi)


def _ratios(p):
    d = np.diff(p)
    return max([1.0] + [max(a, b) / min(a, b) for a, b in zip(d[:-1], d[1:])])


SPACING = P.Spacing(1.0, 1.3, 2)


def test_each_part_face_is_a_plane_and_the_cells_grow_at_most_by_the_limit():
    parts = [_part("block", (0.0, 0.0, 0.0), (10.0, 10.0, 5.0)),
             _part("layer", (2.0, 3.0, 5.0), (7.0, 6.0, 5.01), material=1)]
    for d in range(3):
        planes = P.axis_planes(parts, d, SPACING)
        ref = O.axis_planes([(p.lo, p.hi) for p in parts], d, (1.0, 1.3, 2))
        assert planes.tolist() == ref
        for p in parts:
            for x in (p.lo[d], p.hi[d]):
                assert np.abs(planes - x).min() < 1e-12
        assert _ratios(planes) <= 1.3 + 1e-9
        assert np.diff(planes).max() <= 1.0 + 1e-12
    z = P.axis_planes(parts, 2, SPACING)
    assert ((z > 5.0 + 1e-9) & (z < 5.01 - 1e-9)).sum() >= 1


def test_random_parts_keep_the_growth_limit_and_equal_the_oracle():
    seed = 12345
    mask = (1 << 64) - 1

    def nxt():
        nonlocal seed
        seed = (seed * 6364136223846793005 + 1442695040888963407) & mask
        return (seed >> 11) / float(1 << 53)

    for _ in range(30):
        parts = []
        for i in range(5):
            lo = tuple(10.0 * nxt() for _ in range(3))
            hi = tuple(lo[d] + 0.01 + 5.0 * nxt() ** 3 for d in range(3))
            parts.append(_part(f"p{i}", lo, hi))
        for d in range(3):
            planes = P.axis_planes(parts, d, SPACING)
            assert _ratios(planes) <= 1.3 + 1e-9
            assert planes.tolist() == O.axis_planes([(p.lo, p.hi) for p in parts], d,
                                                    (1.0, 1.3, 2))


def test_axis_planes_with_extra_keys_equal_the_oracle():
    parts = [_part("a", (0.0, 0.0, 0.0), (3.0, 2.0, 0.2)), _part("b", (2.0, 0.5, 0.2),
                                                                (2.8, 1.5, 0.5))]
    sp = P.Spacing(0.2, 1.3, 2)
    for d in range(3):
        got = P.axis_planes(parts, d, sp, extra=[0.7, 1.1])
        assert got.tolist() == O.axis_planes([(p.lo, p.hi) for p in parts], d, (0.2, 1.3, 2),
                                             [0.7, 1.1])


# ------------------------------------------------------------------ the box grid's oracle (grid.rs)

def test_box_grid_oracle_passes_the_reference_tests():
    """oracle/grid.py against grid.rs:548-642: the higher priority holds the overlap, the same
    priority with other materials is refused, the faces of a box cover its surface."""
    from oracle import grid as OG
    sp = (1.0, 1.3, 2)
    parts = [("a", 0, 0, (0.0,) * 3, (2.0,) * 3), ("b", 1, 1, (1.0,) * 3, (3.0,) * 3)]
    planes, part = OG.build(parts, sp)
    nx, ny = len(planes[0]) - 1, len(planes[1]) - 1

    def cell_at(x):
        i = [int(np.searchsorted(planes[d], x[d]) - 1) for d in range(3)]
        return i[0] + nx * (i[1] + ny * i[2])

    assert part[cell_at((1.5, 1.5, 1.5))] == 1 and part[cell_at((0.5, 0.5, 0.5))] == 0
    assert part[cell_at((2.5, 0.5, 0.5))] == OG.VOID
    with pytest.raises(ValueError, match="same priority"):
        OG.build([("a", 0, 0, (0.0,) * 3, (2.0,) * 3), ("b", 1, 0, (1.0,) * 3, (3.0,) * 3)], sp)
    planes, part = OG.build([("a", 0, 0, (0.0,) * 3, (2.0, 3.0, 4.0))], sp)
    n = [len(p) - 1 for p in planes]
    area = 0.0
    for cell, side in OG.faces(planes, part):
        c = (cell % n[0], (cell // n[0]) % n[1], cell // (n[0] * n[1]))
        size = [planes[d][c[d] + 1] - planes[d][c[d]] for d in range(3)]
        area += np.prod([size[d] for d in range(3) if d != side // 2])
    assert abs(area - 2.0 * (6.0 + 8.0 + 12.0)) < 1e-9
    points, ijk, cells, cell_of, mpart = OG.number(planes, part)
    assert len(points) == (n[0] + 1) * (n[1] + 1) * (n[2] + 1) and len(cells) == len(part)


def test_prism_mesh_refuses_bad_parts_with_the_reference_texts_before_any_device_work():
    """prism.rs:197-200, 404-481, 224-240: the host steps run first, so these refusals need no
    GPU; each text is the reference's."""
    sp = P.Spacing(0.2, 1.3, 2)
    poly = lambda c: P.Footprint(P.Outline.polygon(c), [])  # noqa: E731
    sq = [(0, 0), (1, 0), (1, 1), (0, 1)]
    cases = [
        ([], sp, "the model has no part"),
        ([P.Part("a", 0, 0, (0, 0, 0), (1, 1, 1))], P.Spacing(float("inf"), 1.3, 2),
         "max_cell must be a number above 0"),
        ([P.Part("c", 0, 0, (0, 0, 1), (1, 1, 1))], sp,
         "part c: its z range must be 2 finite numbers, the first smaller"),
        ([P.Part("b", 0, 0, (1, 0, 0), (1, 1, 1))], sp,
         "part b: each range must have the first number smaller"),
        ([P.Part("p", 0, 0, (0, 0, 0), (0, 0, 1), poly([(0, 0), (1, 0)]))], sp,
         "part p: a polygon needs 3 or more corners with finite coordinates"),
        ([P.Part("q", 0, 0, (0, 0, 0), (0, 0, 1),
                 P.Footprint(P.Outline.circle((0, 0), 0.0), []))], sp,
         "part q: a circle needs a finite centre and a radius above 0"),
        ([P.Part("z", 0, 0, (0, 0, 0), (0, 0, 1), poly([(0, 0), (1, 1), (2, 2)]))], sp,
         "part z: an outline has no area"),
        ([P.Part("a", 0, 0, (0, 0, 0), (0, 0, 1), poly(sq)),
          P.Part("b", 1, 0, (0, 0, 0), (0, 0, 1), poly([(0.5, 0.5), (2, 0.5), (2, 2), (0.5, 2)]))],
         sp, "parts a and b overlap with the same priority and other materials: give the part "
             "that must hold the overlap a higher priority"),
    ]
    for parts, spacing, text in cases:
        with pytest.raises(FemError) as e:
            P.mesh(parts, 2, spacing, 10**9, "")
        assert str(e.value) == text


def test_box_grid_refuses_bad_parts_and_spacings_before_any_device_work():
    """grid.rs:119-143 and 473-481: the checks and the planes run on the host first, so these
    refusals need no GPU; each text is the reference's."""
    from femahoy_b200 import grid as G
    a = P.Part("a", 0, 0, (0.0,) * 3, (1.0,) * 3)
    cases = [
        ([], P.Spacing(1.0, 1.3, 2), "the model has no part"),
        ([a], P.Spacing(0.0, 1.3, 2), "max_cell must be a number above 0"),
        ([a], P.Spacing(0.5, 1.0, 2), "max_growth must be a number above 1"),
        ([a], P.Spacing(0.5, 1.3, 0), "min_cells must be 1 or more"),
        ([P.Part("bad", 0, 0, (0.0, 1.0, 0.0), (1.0, 1.0, 1.0))], P.Spacing(1.0, 1.3, 2),
         "part bad: its y range must be 2 finite numbers, the first smaller"),
    ]
    for parts, sp, text in cases:
        with pytest.raises(FemError) as e:
            G.build(parts, sp)
        assert str(e.value) == text
