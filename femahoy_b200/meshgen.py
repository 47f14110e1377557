"""Seeded synthetic inputs for the solve path: structured box meshes of Kuhn tetrahedra and the
loads and supports of the benchmark problems.

The reference meshes its parts by extruding a 2D Delaunay mesh into prisms cut into 3 tets
(crates/fem/src/prism.rs:144-170). The benchmark problems instead use a box of nx x ny x nz
hexahedra, each split into the 6 Kuhn tetrahedra that share its (0,0,0)-(1,1,1) diagonal, one
per permutation of the axes. Node (i, j, k) is number i + (nx+1) (j + (ny+1) k). A tetrahedron
of an odd permutation has its 2nd and 3rd nodes swapped so that every volume is positive, as
crates/fem/src/tet10.rs:70-74 assumes.

Loads follow the reference's consistent loads: a uniform volume source gives V/4 to each corner
(crates/fem/src/heat.rs:410-424), a face traction on a linear triangle A/3 to each corner, and
on a quadratic triangle A/3 to each edge point and 0 to each corner
(crates/fem/src/elastic_tet.rs:248-262).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# The 6 axis permutations of the Kuhn split, in lexicographic order.
PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
# crates/fem/src/tet10.rs:38: the corners of each edge point of a 10-node tetrahedron.
EDGES = np.array([[0, 1], [1, 2], [0, 2], [0, 3], [1, 3], [2, 3]])
# The 4 faces of a tetrahedron (local corners).
FACES = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])


@dataclass
class BoxMesh:
    """A box of nx x ny x nz cells of sides L, split into Kuhn tetrahedra."""

    dims: tuple
    lengths: tuple
    points: np.ndarray  # (n, 3) float64
    tets: np.ndarray  # (6 cells, 4) uint32
    ijk: np.ndarray  # (n, 3) uint32: the grid point of each node
    planes: list = field(default_factory=list)  # 3 arrays of plane coordinates

    @property
    def n(self):
        return len(self.points)


def box(nx, ny, nz, lengths=(1.0, 1.0, 1.0)) -> BoxMesh:
    """The Kuhn tetrahedra of a box grid (6 per cell, in cell order then PERMS order)."""
    lx, ly, lz = (float(v) for v in lengths)
    planes = [lx * np.arange(nx + 1) / nx, ly * np.arange(ny + 1) / ny,
              lz * np.arange(nz + 1) / nz]
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1),
                          indexing="ij")
    ijk = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.uint32)
    points = np.stack([planes[0][ijk[:, 0]], planes[1][ijk[:, 1]], planes[2][ijk[:, 2]]],
                      axis=1)
    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()

    def node(di, dj, dk):
        return (ci + di) + (nx + 1) * ((cj + dj) + (ny + 1) * (ck + dk))

    tets = np.empty((ci.size, 6, 4), dtype=np.int64)
    for t, perm in enumerate(PERMS):
        v = [np.zeros(3, dtype=int)]
        for ax in perm:
            nxt = v[-1].copy()
            nxt[ax] += 1
            v.append(nxt)
        ids = [node(*c) for c in v]
        odd = perm in [(0, 2, 1), (1, 0, 2), (2, 1, 0)]
        if odd:
            ids[1], ids[2] = ids[2], ids[1]
        for c in range(4):
            tets[:, t, c] = ids[c]
    return BoxMesh(dims=(nx, ny, nz), lengths=(lx, ly, lz), points=points,
                   tets=tets.reshape(-1, 4).astype(np.uint32), ijk=ijk, planes=planes)


def boundary_faces(mesh: BoxMesh, axis: int, side: int):
    """The faces of the tetrahedra on the plane ``axis`` = 0 (side 0) or its last plane
    (side 1): (tet index, local face index) pairs, in tetrahedron order."""
    target = 0 if side == 0 else mesh.dims[axis]
    on = mesh.ijk[:, axis] == target
    flags = on[mesh.tets]  # (T, 4)
    out_t, out_f = [], []
    for f, corners in enumerate(FACES):
        hit = flags[:, corners].all(axis=1)
        t = np.nonzero(hit)[0]
        out_t.append(t)
        out_f.append(np.full(t.size, f))
    t = np.concatenate(out_t)
    f = np.concatenate(out_f)
    order = np.lexsort((f, t))
    return t[order], f[order]


def face_area(points, tri):
    """The area of each triangle ``tri`` (F, 3) of node numbers."""
    a, b, c = points[tri[:, 0]], points[tri[:, 1]], points[tri[:, 2]]
    return 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1)


@dataclass
class Problem:
    """A discretized problem before the solve: the elements, material data per element, the
    fixed unknowns with their values, the load and the grid point of each unknown."""

    kind: str  # "p1_heat", "p1_elastic", "p2_elastic"
    mesh: BoxMesh
    nodes: np.ndarray  # element nodes: (T, 4) corners or (T, 10) points
    coef: np.ndarray  # (T, 3) conductivities or (T, 2) E and nu
    n_points: int  # number of points (corners + edge points for P2)
    comps: int
    fixed: np.ndarray  # bool per unknown
    values: np.ndarray  # fixed value per unknown (0 where free)
    load: np.ndarray  # per unknown
    edges: np.ndarray | None = None  # P2: the corners of each edge point
    xyz: np.ndarray | None = None  # the coordinates of all points
    seed: int | None = None

    @property
    def n_unknowns(self):
        return self.n_points * self.comps

    @property
    def free(self):
        return np.nonzero(~self.fixed)[0].astype(np.int64)


def heat_cube(n=128, seed=1234, source=1.0) -> Problem:
    """P1 heat conduction in the unit cube of n^3 cells: conductivity exp(N(0, 1)) per
    tetrahedron (numpy PCG64, ``seed``), T = 1 on x = 0 and T = 0 on x = 1, a uniform volume
    source lumped V/4 to each corner."""
    mesh = box(n, n, n)
    rng = np.random.default_rng(seed)
    k = np.exp(rng.standard_normal(len(mesh.tets)))
    coef = np.repeat(k[:, None], 3, axis=1)
    fixed = (mesh.ijk[:, 0] == 0) | (mesh.ijk[:, 0] == n)
    values = np.where(mesh.ijk[:, 0] == 0, 1.0, 0.0)
    values[~fixed] = 0.0
    vol = tet_volumes(mesh.points, mesh.tets)
    load = np.zeros(mesh.n)
    np.add.at(load, mesh.tets.ravel(), np.repeat(source * vol / 4.0, 4))
    return Problem("p1_heat", mesh, mesh.tets, coef, mesh.n, 1, fixed, values, load,
                   xyz=mesh.points, seed=seed)


# The corners of a box cell in VTK order: (0,0,0), (1,0,0), (1,1,0), (0,1,0), (0,0,1), (1,0,1),
# (1,1,1), (0,1,1).
HEX_BITS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]


def box_cells(mesh):
    """The box cells of a BoxMesh's grid (nx ny nz, in grid order), 8 corners each in VTK order,
    as the reference's grid meshes (crates/fem/src/heat.rs:804-826)."""
    nx, ny, nz = mesh.dims
    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    cols = [(ci + a) + (nx + 1) * ((cj + b) + (ny + 1) * (ck + c)) for a, b, c in HEX_BITS]
    return np.stack(cols, axis=1).astype(np.uint32)


def heat_cube_hex(n=64, seed=1234, source=1.0) -> "Problem":
    """P1 heat conduction on the box cells of the unit cube (the reference's box-grid heat
    model): conductivity exp(N(0, 1)) per cell (numpy PCG64, ``seed``), T = 1 on x = 0 and
    T = 0 on x = 1, a uniform volume source lumped V/8 to each corner (heat.rs:417-423)."""
    mesh = box(n, n, n)
    cells = box_cells(mesh)
    rng = np.random.default_rng(seed)
    k = np.exp(rng.standard_normal(len(cells)))
    coef = np.repeat(k[:, None], 3, axis=1)
    fixed = (mesh.ijk[:, 0] == 0) | (mesh.ijk[:, 0] == n)
    values = np.where(mesh.ijk[:, 0] == 0, 1.0, 0.0)
    values[~fixed] = 0.0
    p = mesh.points
    vol = np.prod(p[cells[:, 6]] - p[cells[:, 0]], axis=1)
    load = np.zeros(mesh.n)
    for c in range(8):
        np.add.at(load, cells[:, c], source * vol / 8.0)
    return Problem("hex_heat", mesh, cells, coef, mesh.n, 1, fixed, values, load,
                   xyz=mesh.points, seed=seed)


def orthotropic(e, nu=None, g=None):
    """The 9 constants (Ex, Ey, Ez, nu_xy, nu_xz, nu_yz, G_xy, G_xz, G_yz) of a material with its
    axes on x, y and z (crates/fem/src/hex.rs:47-55); with one modulus and one ratio, the
    isotropic material (hex.rs:57-65: G = E / (2 (1 + nu)))."""
    if np.isscalar(e):
        return np.array([e] * 3 + [nu] * 3 + [e / (2.0 * (1.0 + nu))] * 3, dtype=np.float64)
    return np.concatenate([np.asarray(e, float), np.asarray(nu, float), np.asarray(g, float)])


def graded_planes(n, length, grade):
    """n cells over ``length`` whose widths grow geometrically, the last ``grade`` times the
    first."""
    if n < 2 or grade == 1.0:
        return length * np.arange(n + 1) / n
    w = grade ** (np.arange(n) / (n - 1))
    return np.concatenate([[0.0], np.cumsum(w)]) * (length / w.sum())


def hex_cantilever(nx=24, ny=2, nz=2, length=6.0, width=0.5, depth=0.5, e=1000.0, nu=0.3,
                   load=-1.0, grade=1.0, seed=None) -> Problem:
    """A cantilever of box cells (the reference's box-grid elastic model, elastic.rs:352-391):
    every unknown fixed at x = 0, a total force ``load`` along z on the face x = ``length``
    (each face cell gives a quarter of its share to each of its 4 corners). ``grade`` makes the
    cells along x and z grow geometrically (last / first = grade); with ``seed``, about half the
    cells (numpy PCG64) take an orthotropic material (E, E/2, E/4; 0.25, 0.3, 0.35; G = 0.3 E,
    0.25 E, 0.2 E) in place of the isotropic (e, nu)."""
    mesh = box(nx, ny, nz, (length, width, depth))
    mesh.planes[0] = graded_planes(nx, length, grade)
    mesh.planes[2] = graded_planes(nz, depth, grade)
    for d in range(3):
        mesh.points[:, d] = mesh.planes[d][mesh.ijk[:, d]]
    cells = box_cells(mesh)
    coef = np.tile(orthotropic(e, nu), (len(cells), 1))
    if seed is not None:
        pick = np.random.default_rng(seed).random(len(cells)) < 0.5
        coef[pick] = orthotropic([e, e / 2.0, e / 4.0], [0.25, 0.3, 0.35],
                                 [0.3 * e, 0.25 * e, 0.2 * e])
    n = mesh.n
    fixed = np.repeat(mesh.ijk[:, 0] == 0, 3)
    force = np.zeros(3 * n)
    ci = np.arange(len(cells)) % nx
    end = cells[ci == nx - 1]
    p = mesh.points
    area = (p[end[:, 2], 1] - p[end[:, 1], 1]) * (p[end[:, 5], 2] - p[end[:, 1], 2])
    share = load * area / (width * depth) / 4.0
    for c in (1, 2, 5, 6):  # the corners on the cell's x = high face
        np.add.at(force, 3 * end[:, c].astype(np.int64) + 2, share)
    return Problem("hex_elastic", mesh, cells, coef, n, 3, fixed, np.zeros(3 * n), force,
                   xyz=mesh.points, seed=seed)


def hex_classes(prob):
    """The element classes of the box cells of ``prob``: (origin (C, 3) the lowest grid point
    of each cell, cls (C,) its class, keys (K, 12) the 3 sides and 9 material constants of each
    class). Cells whose 12 numbers are equal bit for bit share a class (and a matrix)."""
    cells = prob.nodes
    p = prob.xyz
    keys = np.concatenate([p[cells[:, 6]] - p[cells[:, 0]], prob.coef], axis=1)
    raw = np.ascontiguousarray(keys).view(np.dtype((np.void, 96))).ravel()
    _, first, cls = np.unique(raw, return_index=True, return_inverse=True)
    return (prob.mesh.ijk[cells[:, 0]].astype(np.uint32), cls.astype(np.uint32).ravel(),
            keys[first])


def extruded(npoints=300, layers=8, height=1.0, seed=0):
    """A footprint mesh extruded in layers, as the reference's prism meshes are (prism.rs): an
    unstructured triangulation (scipy Delaunay of jittered points in the unit square) extruded
    into ``layers`` wedges, each split into 3 tetrahedra by the lowest-index rule (shared quad
    faces split alike). Returns (xyz, tets): the corner points lie on z planes but not on x or
    y planes."""
    from scipy.spatial import Delaunay
    rng = np.random.default_rng(seed)
    m = int(np.ceil(np.sqrt(npoints)))
    g = (np.stack(np.meshgrid(np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 2)
         + 0.5) / m
    inner = (g > 0.6 / m).all(axis=1) & (g < 1 - 0.6 / m).all(axis=1)
    g[inner] += rng.uniform(-0.3 / m, 0.3 / m, size=(inner.sum(), 2))
    tri = Delaunay(g).simplices
    n2 = len(g)
    z = height * np.arange(layers + 1) / layers
    xyz = np.column_stack([np.tile(g, (layers + 1, 1)), np.repeat(z, n2)])
    tets = []
    for k in range(layers):
        for t in tri:
            a, b, c = sorted(int(v) for v in t)
            lo = [a + k * n2, b + k * n2, c + k * n2]
            hi = [v + n2 for v in lo]
            tets += [[lo[0], lo[1], lo[2], hi[2]], [lo[0], lo[1], hi[1], hi[2]],
                     [lo[0], hi[0], hi[1], hi[2]]]
    tets = np.asarray(tets, dtype=np.uint32)
    # Positive orientation (the assembly takes |volume| from the gradients either way).
    p = xyz[tets]
    neg = np.linalg.det(p[:, 1:] - p[:, :1]) < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    return xyz, tets


def level_of(xyz, free, comps=3):
    """The grid level of the free unknowns of points that need not fill a grid: the distinct
    coordinates of each axis are the planes."""
    planes = [np.unique(xyz[:, d]) for d in range(3)]
    node = free // comps
    pts = np.stack([np.searchsorted(planes[d], xyz[node, d]) for d in range(3)],
                   axis=1).astype(np.uint32)
    return planes, pts, (free % comps).astype(np.uint8)


def lumped_capacity(mesh, capacity=1.0, cells=None):
    """crates/fem/src/heat.rs:413-423: each corner of a cell takes capacity V / per (4 corners
    of a tetrahedron, or 8 of a box cell given as ``cells``), summed over the cells in order and
    then their corners, as the reference's loop."""
    if cells is None:
        cells, vol = mesh.tets, tet_volumes(mesh.points, mesh.tets)
    else:
        p = mesh.points
        vol = np.prod(p[cells[:, 6]] - p[cells[:, 0]], axis=1)
    per = cells.shape[1]
    out = np.zeros(mesh.n)
    np.add.at(out, cells.ravel(), np.repeat(capacity * vol / per, per))
    return out


def tet_volumes(points, tets):
    p = points[tets]
    e = p[:, 1:, :] - p[:, :1, :]
    return np.linalg.det(e) / 6.0


def cantilever_p1(dims=(40, 4, 4), lengths=(100.0, 10.0, 10.0), e=210e3, nu=0.3,
                  pressure=1.0) -> Problem:
    """P1 elasticity of a cantilever (mm, MPa): all unknowns fixed at x = 0, a uniform
    pressure on the top face z = Lz (traction -pressure along z), A/3 to each corner."""
    mesh = box(*dims, lengths)
    n = mesh.n
    coef = np.tile(np.array([e, nu]), (len(mesh.tets), 1))
    fixed = np.repeat(mesh.ijk[:, 0] == 0, 3)
    values = np.zeros(3 * n)
    load = np.zeros(3 * n)
    t, f = boundary_faces(mesh, 2, 1)
    tri = mesh.tets[t][np.arange(len(t))[:, None], FACES[f]]
    area = face_area(mesh.points, tri)
    np.add.at(load, 3 * tri.ravel().astype(np.int64) + 2, np.repeat(-pressure * area / 3.0, 3))
    return Problem("p1_elastic", mesh, mesh.tets, coef, n, 3, fixed, values, load,
                   xyz=mesh.points)


def random_cantilever_p1(rng, lo=(10, 1, 1), hi=(80, 8, 8), nrhs=16, cell=2.5):
    """One member of the batched workload: a P1 cantilever whose cell counts are log-uniform
    between ``lo`` and ``hi``, E uniform in [50, 250] GPa, nu in [0.25, 0.35], clamped at x = 0,
    with ``nrhs`` random top-face traction load cases (components uniform in [-1, 1] MPa)."""
    dims = tuple(int(round(np.exp(rng.uniform(np.log(a), np.log(b))))) for a, b in zip(lo, hi))
    e = rng.uniform(50e3, 250e3)
    nu = rng.uniform(0.25, 0.35)
    lengths = tuple(cell * d for d in dims)
    mesh = box(*dims, lengths)
    n = mesh.n
    coef = np.tile(np.array([e, nu]), (len(mesh.tets), 1))
    fixed = np.repeat(mesh.ijk[:, 0] == 0, 3)
    t, f = boundary_faces(mesh, 2, 1)
    tri = mesh.tets[t][np.arange(len(t))[:, None], FACES[f]]
    area = face_area(mesh.points, tri)
    loads = np.zeros((nrhs, 3 * n))
    for r in range(nrhs):
        trac = rng.uniform(-1.0, 1.0, size=3)
        for d in range(3):
            np.add.at(loads[r], 3 * tri.ravel().astype(np.int64) + d,
                      np.repeat(trac[d] * area / 3.0, 3))
    prob = Problem("p1_elastic", mesh, mesh.tets, coef, n, 3, fixed, np.zeros(3 * n),
                   loads[0], xyz=mesh.points)
    return prob, loads


def beam_p2(edges, tets10, dims=(200, 20, 20), lengths=(200.0, 20.0, 20.0), e=70e3, nu=0.33,
            seed=1234, mesh=None) -> Problem:
    """P2 elasticity of a box beam clamped at x = 0 with a random traction on x = L: each
    boundary face has its own traction with components uniform in [-1, 1] MPa (numpy PCG64,
    ``seed``), A/3 to each of its 3 edge points. ``edges``/``tets10`` are the quadratic mesh of
    the box's tetrahedra (crates/fem/src/tet10.rs:244-272)."""
    mesh = mesh if mesh is not None else box(*dims, lengths)
    nc = mesh.n
    npts = nc + len(edges)
    mid = 0.5 * (mesh.points[edges[:, 0]] + mesh.points[edges[:, 1]])
    xyz = np.concatenate([mesh.points, mid])
    coef = np.tile(np.array([e, nu]), (len(mesh.tets), 1))
    # A point is on x = 0 when its corners are (a corner itself, or both corners of its edge).
    on0 = np.concatenate([mesh.ijk[:, 0] == 0,
                          (mesh.ijk[edges[:, 0], 0] == 0) & (mesh.ijk[edges[:, 1], 0] == 0)])
    fixed = np.repeat(on0, 3)
    values = np.zeros(3 * npts)
    load = np.zeros(3 * npts)
    t, f = boundary_faces(mesh, 0, 1)
    rng = np.random.default_rng(seed)
    trac = rng.uniform(-1.0, 1.0, size=(len(t), 3))
    tri = mesh.tets[t][np.arange(len(t))[:, None], FACES[f]]
    area = face_area(mesh.points, tri)
    # The edge points of each face: the edges of the tetrahedron between the face's corners.
    local = FACES[f]  # (F, 3) local corners
    pairs = [(0, 1), (1, 2), (2, 0)]
    for a, b in pairs:
        la, lb = local[:, a], local[:, b]
        lo_, hi_ = np.minimum(la, lb), np.maximum(la, lb)
        k = np.full(len(t), -1)
        for ei, (p0, p1) in enumerate(EDGES):
            k[(lo_ == p0) & (hi_ == p1)] = ei
        ep = tets10[t, 4 + k].astype(np.int64)
        for d in range(3):
            np.add.at(load, 3 * ep + d, trac[:, d] * area / 3.0)
    return Problem("p2_elastic", mesh, tets10, coef, npts, 3, fixed, values, load,
                   edges=edges, xyz=xyz, seed=seed)


def grid_unknowns(prob: Problem):
    """The grid level of the free unknowns of a P1 problem (crates/fem/src/multigrid.rs:55-59):
    the planes of each axis, and the grid point and component of each free unknown."""
    free = prob.free
    node = free // prob.comps
    comp = (free % prob.comps).astype(np.uint8)
    return prob.mesh.planes, prob.mesh.ijk[node].astype(np.uint32), comp
