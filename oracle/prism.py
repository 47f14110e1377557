"""CPU oracle of the prism mesh (TEST INFRASTRUCTURE ONLY): a plain-Python restatement of
femahoy's crates/fem/src/prism.rs (the footprints' outlines and labels, the extrusion into
tetrahedra, the boundary faces) and grid.rs axis_planes, in the reference's sequential order.

Only the tests use it, as the checker of ``femahoy_b200.prism`` (whose extrusion runs on the
device, by a different scheme: first-use ranks from atomics and prefix sums, faces from the
prisms' neighbours). The 2D quality mesh itself (mesh2d.rs) is not restated here: the tests feed
the same triangle mesh to both sides and check it against the reference's own properties
(tests/mesh2d.rs). Pinned by the reference's known answers: every one of the 720 corner orders
of split_prism fills the prism and cuts each face at its smallest corner (tests/tet.rs:89-140),
the extruded mesh of a plate with a hole and a lid is conforming with the parts' volumes and a
closed surface (tests/tet.rs:142-214), and the planes keep each part face and the growth limit
(grid.rs:548-612).
"""
from __future__ import annotations

import math

OUTSIDE = 0xFFFFFFFF
NONE = 0xFFFFFFFF
MIN_CIRCLE_SEGMENTS = 64  # prism.rs:51


def across(axis, p):
    """prism.rs:54-56."""
    return (p[(axis + 1) % 3], p[(axis + 2) % 3])


def point(axis, uv, w):
    """prism.rs:58-64."""
    p = [0.0, 0.0, 0.0]
    p[axis] = w
    p[(axis + 1) % 3] = uv[0]
    p[(axis + 2) % 3] = uv[1]
    return p


def circle_corners(centre, radius, max_cell):
    """Outline::corners of a circle (prism.rs:71-88)."""
    n = max(int(math.ceil(2.0 * math.pi * radius / max_cell)), MIN_CIRCLE_SEGMENTS)
    n = (n + 3) // 4 * 4
    out = []
    for k in range(n):
        a = 2.0 * math.pi * k / n
        out.append((centre[0] + radius * math.cos(a), centre[1] + radius * math.sin(a)))
    return out


def inside(corners, p):
    """Even-odd rule (prism.rs:90-102)."""
    odd = False
    n = len(corners)
    for k in range(n):
        a, b = corners[k], corners[(k + 1) % n]
        if (a[1] > p[1]) != (b[1] > p[1]) and \
                p[0] < a[0] + (p[1] - a[1]) / (b[1] - a[1]) * (b[0] - a[0]):
            odd = not odd
    return odd


def densify(corners, mx):
    """prism.rs:529-544."""
    out = []
    m = len(corners)
    for k in range(m):
        a, b = corners[k], corners[(k + 1) % m]
        n = max(int(math.ceil(math.sqrt((b[0] - a[0]) ** 2 + (b[1] - a[1]) ** 2) / mx)), 1) \
            if math.isfinite(mx) else 1
        for i in range(n):
            t = i / n
            out.append((a[0] + t * (b[0] - a[0]), a[1] + t * (b[1] - a[1])))
    return out


# ------------------------------------------------------------------ planes (grid.rs:413-518)

def tol(p):
    return 1e-9 * max(abs(p[-1] - p[0]), 2.2250738585072014e-308)


def place(keys, target, at_key, slope):
    def h(x, i):
        v = target[i]
        for k, s in zip(keys, at_key):
            v = min(v, s + slope * abs(x - k))
        return v

    planes = [keys[0]]
    samples = 400
    for i in range(len(keys) - 1):
        a, b = keys[i], keys[i + 1]
        step = (b - a) / samples
        phi = [0.0] * (samples + 1)
        for s in range(samples):
            x0, x1 = a + s * step, a + (s + 1) * step
            phi[s + 1] = phi[s] + 0.5 * step * (1.0 / h(x0, i) + 1.0 / h(x1, i))
        total = phi[samples]
        cells = max(int(math.ceil(total - 1e-6)), 1)
        for c in range(1, cells):
            want = total * c / cells
            s = 0
            while s < len(phi) and phi[s] < want:
                s += 1
            s = min(max(s, 1), samples)
            f = (want - phi[s - 1]) / (phi[s] - phi[s - 1])
            planes.append(a + (s - 1.0 + f) * step)
        planes.append(b)
    return planes


def axis_planes(parts, d, spacing, extra=()):
    """parts: (lo, hi) pairs of 3-tuples; spacing: (max_cell, max_growth, min_cells)."""
    max_cell, max_growth, min_cells = spacing
    keys = sorted([v for lo, hi in parts for v in (lo[d], hi[d])] + list(extra))
    t = tol(keys)
    kept = []
    for k in keys:
        if not kept or not abs(k - kept[-1]) <= t:
            kept.append(k)
    keys = kept
    target = []
    for i in range(len(keys) - 1):
        v = max_cell
        for lo, hi in parts:
            if lo[d] <= keys[i] + t and hi[d] >= keys[i + 1] - t:
                v = min(v, (hi[d] - lo[d]) / min_cells)
        target.append(v)
    at_key = [min(target[k - 1] if k > 0 else math.inf,
                  target[k] if k < len(target) else math.inf) for k in range(len(keys))]
    slope = 0.5 * (max_growth - 1.0)
    for _ in range(60):
        planes = place(keys, target, at_key, slope)
        cells = [planes[c + 1] - planes[c] for c in range(len(planes) - 1)]
        fixed = False
        for c in range(len(cells) - 1):
            w0, w1 = cells[c], cells[c + 1]
            small, large = (w0, w1) if w0 < w1 else (w1, w0)
            if large > max_growth * small * (1.0 + 1e-9):
                x = planes[c + 1]
                k = 0
                while k < len(keys) and keys[k] < x - t:
                    k += 1
                k = min(k, len(keys) - 1)
                for q in (max(k - 1, 0), k, min(k + 1, len(keys) - 1)):
                    if abs(keys[q] - x) <= 2.0 * large and at_key[q] > small * 1.0001:
                        at_key[q] = small
                        fixed = True
        if not fixed:
            return planes
    raise ValueError("growth limit")


# ------------------------------------------------------------------ footprints (prism.rs:397-527)

def footprint_inputs(parts, axis, max_size):
    """The points, segments, segment circles, circles and a classify (with its covers list) of
    the footprints of `parts`: each part is (name, material, priority, lo, hi, footprint) with
    footprint None or (outline, holes), an outline ('polygon', corners) or ('circle', centre,
    radius). The outline of each part first, then its holes, as prism.rs:414-509."""
    points, segments, segment_circle, circles, polygons = [], [], [], [], []
    for p in parts:
        name, material, priority, lo, hi, fp = p
        if fp is None:
            a, b = across(axis, lo), across(axis, hi)
            fp = (("polygon", [a, (b[0], a[1]), b, (a[0], b[1])]), [])
        rings = []
        for o in [fp[0]] + list(fp[1]):
            if o[0] == "circle":
                corners = circle_corners(o[1], o[2], min(max_size, math.inf))
                circles.append((tuple(o[1]), o[2]))
                circle = len(circles) - 1
            else:
                corners = densify([tuple(c) for c in o[1]], math.inf)
                circle = NONE
            base, n = len(points), len(corners)
            points.extend(corners)
            for k in range(n):
                segments.append((base + k, base + (k + 1) % n))
                segment_circle.append(circle)
            rings.append(corners)
        polygons.append((rings[0], rings[1:]))
    covers = []

    def classify(x):
        lst = [k for k in range(len(parts))
               if inside(polygons[k][0], x) and not any(inside(h, x) for h in polygons[k][1])]
        if not lst:
            return OUTSIDE
        lst.sort(key=lambda k: (-parts[k][2], -k))
        if lst in covers:
            return covers.index(lst)
        covers.append(lst)
        return len(covers) - 1

    return points, segments, segment_circle, circles, classify, covers


# ------------------------------------------------------------------ extrusion (prism.rs:216-379)

ROTATE = [[0, 1, 2, 3, 4, 5], [1, 2, 0, 4, 5, 3], [2, 0, 1, 5, 3, 4],
          [3, 5, 4, 0, 2, 1], [4, 3, 5, 1, 0, 2], [5, 4, 3, 2, 1, 0]]


def split_prism(g):
    """prism.rs:144-154."""
    m = min(range(6), key=lambda k: g[k])
    r = ROTATE[m]
    if min(g[r[1]], g[r[5]]) < min(g[r[2]], g[r[4]]):
        t = [[0, 1, 2, 5], [0, 1, 5, 4], [0, 4, 5, 3]]
    else:
        t = [[0, 1, 2, 4], [0, 4, 2, 5], [0, 4, 5, 3]]
    return [[r[k] for k in tet] for tet in t]


def volume(p):
    """prism.rs:156-162, in its operation order."""
    a = [p[1][i] - p[0][i] for i in range(3)]
    b = [p[2][i] - p[0][i] for i in range(3)]
    c = [p[3][i] - p[0][i] for i in range(3)]
    return (a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0])
            + a[2] * (b[0] * c[1] - b[1] * c[0])) / 6.0


def extrude(parts, axis, planes, flat_points, triangles, label, covers, segments_of_edge,
            segment_circle, max_points, hollow=()):
    """prism.rs:216-379 from the 2D mesh: returns (points, tets, part, faces) with faces
    (nodes, tet, beyond, circles) sorted by (tet, nodes); raises ValueError with the reference's
    texts (the refusal as 'refusal')."""
    is_hollow = lambda p: p < len(hollow) and bool(hollow[p])  # noqa: E731
    t = tol(planes)
    layers = len(planes) - 1
    part_of = [NONE] * (len(covers) * layers)
    for l, lst in enumerate(covers):
        for k in range(layers):
            z0, z1 = planes[k], planes[k + 1]
            holds = lambda p: parts[p][3][axis] <= z0 + t and parts[p][4][axis] >= z1 - t  # noqa
            first = next((p for p in lst if holds(p)), None)
            if first is None:
                continue
            for p in lst:
                if p != first and holds(p) and parts[p][2] == parts[first][2] and \
                        parts[p][1] != parts[first][1]:
                    raise ValueError(f"parts {parts[p][0]} and {parts[first][0]} overlap with the "
                                     "same priority and other materials: give the part that must "
                                     "hold the overlap a higher priority")
            part_of[l * layers + k] = first
    nv = len(flat_points)
    number = {}
    pts, tets, part = [], [], []
    for tri, lab in zip(triangles, label):
        for k in range(layers):
            p = part_of[lab * layers + k]
            if p == NONE:
                continue
            g = [(k + c // 3) * nv + int(tri[c % 3]) for c in range(6)]
            node = []
            for c in range(6):
                if g[c] not in number:
                    number[g[c]] = len(pts)
                    pts.append(point(axis, flat_points[int(tri[c % 3])], planes[k + c // 3]))
                    if len(pts) > max_points:
                        raise ValueError("refusal")
                node.append(number[g[c]])
            for local in split_prism(g):
                tet = [node[c] for c in local]
                if volume([pts[v] for v in tet]) < 0.0:
                    tet[2], tet[3] = tet[3], tet[2]
                tets.append(tet)
                part.append(p)
    if not any(not is_hollow(p) for p in part):
        raise ValueError("the parts hold no volume")
    seen = {}
    for e, tet in enumerate(tets):
        for f in ((1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1)):
            nodes = tuple(tet[k] for k in f)
            seen.setdefault(tuple(sorted(nodes)), []).append((e, nodes))
    outer = []
    for v in seen.values():
        solid = [x for x in v if not is_hollow(part[x[0]])]
        if len(solid) == 1 and len(v) == 1:
            outer.append((solid[0][0], solid[0][1], NONE))
        elif len(solid) == 1 and len(v) == 2:
            other = next(x for x in v if x[0] != solid[0][0])
            outer.append((solid[0][0], solid[0][1], part[other[0]]))
    flat_of = [0] * len(pts)
    for slot, n in number.items():
        flat_of[n] = slot % nv
    tet_of, point_of = {}, {}
    kept_pts, kept_tets, kept_part = [], [], []
    for e, tet in enumerate(tets):
        if is_hollow(part[e]):
            continue
        tet_of[e] = len(kept_tets)
        row = []
        for v in tet:
            if v not in point_of:
                point_of[v] = len(kept_pts)
                kept_pts.append(pts[v])
            row.append(point_of[v])
        kept_tets.append(row)
        kept_part.append(part[e])
    faces = []
    for tet, nodes, beyond in outer:
        fl = sorted(set(flat_of[n] for n in nodes))
        circles = []
        if len(fl) == 2:
            circles = sorted(set(segment_circle[k] for k in segments_of_edge.get((fl[0], fl[1]), [])
                                 if segment_circle[k] != NONE))
        faces.append((tuple(point_of[v] for v in nodes), tet_of[tet], beyond, circles))
    faces.sort(key=lambda f: (f[1], f[0]))
    return kept_pts, kept_tets, kept_part, faces
