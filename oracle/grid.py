"""CPU oracle of the box grid (TEST INFRASTRUCTURE ONLY): a plain-Python restatement of
femahoy's crates/fem/src/grid.rs Grid::build (:119-154), assign (:292-330), faces (:234-254)
and heat.rs:1165-1210 number, in the reference's sequential order. Only the tests use it, as
the checker of ``femahoy_b200.grid``. Pinned by the reference's known answers (grid.rs:548-642:
the part faces on planes and the growth limit, the higher priority holding an overlap and the
"same priority" refusal, the faces of a box covering its surface)."""
from __future__ import annotations

from . import prism as _p

VOID = 0xFFFFFFFF


def _partition_point(a, pred):
    k = 0
    while k < len(a) and pred(a[k]):
        k += 1
    return k


def build(parts, spacing, extra=((), (), ())):
    """parts: (name, material, priority, lo, hi); spacing: (max_cell, max_growth, min_cells).
    Returns (planes, part per cell); raises ValueError with the reference's texts."""
    if not parts:
        raise ValueError("the model has no part")
    planes = [_p.axis_planes([(p[3], p[4]) for p in parts], d, spacing, extra[d])
              for d in range(3)]
    nx, ny, nz = (len(planes[d]) - 1 for d in range(3))
    best = [None] * (nx * ny * nz)
    for index, p in enumerate(parts):
        rng = []
        for d in range(3):
            t = _p.tol(planes[d])
            rng.append((_partition_point(planes[d], lambda x: x < p[3][d] - t),
                        _partition_point(planes[d], lambda x: x < p[4][d] - t)))
        for k in range(*rng[2]):
            for j in range(*rng[1]):
                for i in range(*rng[0]):
                    cell = i + nx * (j + ny * k)
                    other = best[cell]
                    if other is not None and parts[other][2] > p[2]:
                        continue
                    if other is not None and parts[other][2] == p[2] and \
                            parts[other][1] != p[1]:
                        x = [0.5 * (planes[d][c] + planes[d][c + 1])
                             for d, c in enumerate((i, j, k))]
                        raise ValueError(f"parts {parts[other][0]} and {p[0]} overlap at "
                                         f"{tuple(x)} with the same priority")
                    best[cell] = index
    return planes, [VOID if b is None else b for b in best]


CORNERS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]


def number(planes, part):
    """heat.rs:1165-1210: (points, ijk, cells, cell_of, mesh part)."""
    nx, ny, nz = (len(planes[d]) - 1 for d in range(3))
    num = {}
    ijk, cells, cell_of = [], [], []
    for cell in range(len(part)):
        if part[cell] == VOID:
            continue
        c = (cell % nx, (cell // nx) % ny, cell // (nx * ny))
        row = []
        for o in CORNERS:
            g = (c[0] + o[0], c[1] + o[1], c[2] + o[2])
            key = g[0] + (nx + 1) * (g[1] + (ny + 1) * g[2])
            if key not in num:
                num[key] = len(ijk)
                ijk.append(g)
            row.append(num[key])
        cells.append(row)
        cell_of.append(cell)
    points = [[planes[d][g[d]] for d in range(3)] for g in ijk]
    return points, ijk, cells, cell_of, [part[c] for c in cell_of]


def faces(planes, part):
    """grid.rs:234-254: (cell, side) with side in x-, x+, y-, y+, z-, z+ order."""
    n = [len(planes[d]) - 1 for d in range(3)]
    out = []
    for cell in range(len(part)):
        if part[cell] == VOID:
            continue
        c = [cell % n[0], (cell // n[0]) % n[1], cell // (n[0] * n[1])]
        for s in range(6):
            d, positive = s // 2, s % 2 == 1
            m = list(c)
            m[d] += 1 if positive else -1
            if m[d] < 0 or m[d] >= n[d] or part[m[0] + n[0] * (m[1] + n[1] * m[2])] == VOID:
                out.append((cell, s))
    return out
