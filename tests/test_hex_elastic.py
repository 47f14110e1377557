"""Elasticity on the box cells of the grid: the 8-node hex with 9 incompatible modes condensed
(crates/fem/src/hex.rs:218-311), assembled as elastic.rs:386-391 does for the box-grid models.

CPU: the oracle's element against the reference's own unit tests of it (hex.rs:443-526: the
stiffness is symmetric, a rigid motion has no force, one cell holds a pure bending field with
the exact energy) and a cantilever of box cells against beam theory. GPU: the device assembly bit
for bit against the oracle, and the grid multigrid solve against the oracle's direct solution."""
import numpy as np
import pytest

import oracle
from femahoy_b200 import meshgen as mg

SIZE = np.array([2.0, 0.5, 0.1])  # hex.rs:402


def nodal(f, size=SIZE):
    """hex.rs:453-460: the corner displacements of the field f of the position."""
    u = np.empty(24)
    for n, b in enumerate(mg.HEX_BITS):
        u[3 * n:3 * n + 3] = f(np.asarray(b, float) * size)
    return u


def test_oracle_hex_stiffness_is_symmetric_and_rigid_motions_have_no_force():
    """hex.rs:462-489 (the strain check of the rigid motions needs the recovery, not built)."""
    k = oracle.hex8_stiffness(SIZE, oracle.orthotropic(200.0, 0.3))
    assert np.all(np.abs(k - k.T) <= 1e-12 * np.maximum(np.abs(k), 1.0))
    motions = [lambda x: [1.0, 0.0, 0.0], lambda x: [0.0, 1.0, 0.0], lambda x: [0.0, 0.0, 1.0],
               lambda x: [-x[1], x[0], 0.0], lambda x: [0.0, -x[2], x[1]],
               lambda x: [x[2], 0.0, -x[0]]]
    scale = np.abs(k).max()
    for m in motions:
        f = k @ nodal(m)
        assert np.abs(f).max() < 1e-12 * scale


def test_oracle_rigid_motions_have_no_strain():
    """hex.rs:485-488: the strain of a rigid motion at a point inside the cell is 0."""
    c = oracle.orthotropic(200.0, 0.3)
    for f in [lambda x: [1.0, 0.0, 0.0], lambda x: [-x[1], x[0], 0.0],
              lambda x: [0.0, -x[2], x[1]], lambda x: [x[2], 0.0, -x[0]]]:
        e, _ = oracle.hex8_strain_stress(SIZE, c, [0.3, -0.2, 0.7], nodal(f), np.zeros(8),
                                         alpha=[1e-5] * 3)
        assert np.abs(e).max() < 1e-12


def test_oracle_uniform_strain_gives_the_exact_stress():
    """hex.rs:491-519: a uniform strain field gives e0 and D e0 at each Gauss point, and a
    uniform temperature change with no displacement gives -D alpha dT."""
    c = oracle.orthotropic(200.0, 0.3)
    normal, shear = oracle.isotropic(200.0, 0.3)
    alpha = [1e-5, 2e-5, 3e-5]
    e0 = np.array([1e-3, -2e-3, 0.5e-3, 4e-4, -3e-4, 2e-4])
    u = nodal(lambda x: [e0[0] * x[0] + e0[5] * x[1], e0[1] * x[1] + e0[3] * x[2],
                         e0[2] * x[2] + e0[4] * x[0]])
    want = np.concatenate([normal @ e0[:3], shear * e0[3:]])
    p = 1.0 / np.sqrt(3.0)
    for b in mg.HEX_BITS:
        xi = np.where(np.asarray(b) == 1, p, -p)
        e, s = oracle.hex8_strain_stress(SIZE, c, xi, u, np.zeros(8), alpha=alpha)
        assert np.abs(e - e0).max() < 1e-15
        assert np.abs(s - want).max() < 1e-12
    _, s = oracle.hex8_strain_stress(SIZE, c, [0.1, 0.2, 0.3], np.zeros(24), np.full(8, 10.0),
                                     alpha=alpha)
    assert np.abs(s[:3] + normal @ np.asarray(alpha) * 10.0).max() < 1e-12


def test_oracle_box_recovery_of_a_uniform_strain():
    """elastic.rs:615-660 on graded box cells of 1 material: the mean strain and stress at each
    point of a uniform strain field are e0 (tensor components) and D e0."""
    c = mg.hex_cantilever(nx=5, ny=3, nz=4, grade=1.5)
    e0 = np.array([1e-3, -2e-3, 0.5e-3, 4e-4, -3e-4, 2e-4])
    x = c.xyz
    u = np.stack([e0[0] * x[:, 0] + e0[5] * x[:, 1], e0[1] * x[:, 1] + e0[3] * x[:, 2],
                  e0[2] * x[:, 2] + e0[4] * x[:, 0]], axis=1).ravel()
    r = oracle.recover(c.xyz, c.nodes, c.coef, u, hex=True)
    normal, shear = oracle.isotropic(1000.0, 0.3)
    sig = np.concatenate([normal @ e0[:3], shear * e0[3:]])
    assert np.abs(r["strain"] - [e0[0], e0[1], e0[2], e0[5] / 2, e0[3] / 2, e0[4] / 2]).max() < 1e-15
    assert np.abs(r["stress"] - [sig[0], sig[1], sig[2], sig[5], sig[3], sig[4]]).max() < 1e-12
    assert r["peaks"][0].element >= 0


def test_oracle_one_cell_bends_with_the_exact_curvature():
    """hex.rs:521-545: u^T K u equals E I kappa^2 L for the pure bending field (nu = 0)."""
    e, kappa = 1000.0, 1e-3
    k = oracle.hex8_stiffness(SIZE, oracle.orthotropic(e, 0.0))
    u = nodal(lambda x: [-kappa * x[0] * (x[2] - SIZE[2] / 2.0), 0.0, kappa * x[0] ** 2 / 2.0])
    ku = u @ (k @ u)
    exact = e * SIZE[1] * SIZE[2] ** 3 / 12.0 * kappa ** 2 * SIZE[0]
    assert abs(ku - exact) < 1e-9 * exact


def test_oracle_orthotropic_box_cell_rejects_unstable_materials():
    with pytest.raises(oracle.OracleError, match="no stable material"):
        oracle.hex8_stiffness(SIZE, oracle.orthotropic(1.0, 0.5))
    with pytest.raises(oracle.OracleError, match="moduli must be above 0"):
        oracle.hex8_stiffness(SIZE, oracle.orthotropic([1.0, -1.0, 1.0], [0.3] * 3, [1.0] * 3))


def test_oracle_box_cantilever_matches_beam_theory():
    """A cantilever of box cells, 2 cells through the depth: the incompatible modes hold the
    bending, so the tip deflection is near P L^3 / (3 E I) (the plain trilinear hex locks far
    below it). Clamped at x = 0, a tip load on x = L."""
    c = mg.hex_cantilever(nx=24, ny=2, nz=2, length=6.0, width=0.5, depth=0.5, load=-1.0)
    k = oracle.pattern(3 * c.mesh.n, oracle.dof_elements(c.nodes))
    k.assemble(6, c.xyz, c.nodes, c.coef)
    a = k.submatrix(c.free)
    rhs = k.reduced_rhs(c.load, c.values, c.free)
    x, _ = oracle.direct_solve(a, c.xyz[c.free // 3], rhs)
    u = np.zeros(3 * c.mesh.n)
    u[c.free] = x
    tip = (c.mesh.ijk[:, 0] == 24)
    w = u[3 * np.nonzero(tip)[0] + 2].mean()
    e, i = 1000.0, 0.5 * 0.5 ** 3 / 12.0
    beam = -1.0 * 6.0 ** 3 / (3.0 * e * i)
    assert 0.97 < w / beam < 1.05


def class_table(c):
    """The cells of a box-cell problem for the cell-based coarse matrices: (origin, class,
    the oracle's matrix of each class)."""
    origin, cls, keys = mg.hex_classes(c)
    return origin, cls, np.stack([oracle.hex8_stiffness(k[:3], k[3:]) for k in keys])


def dense(csr):
    ptr, idx, val = csr.arrays()
    a = np.zeros((len(ptr) - 1, len(ptr) - 1))
    for i in range(len(ptr) - 1):
        a[i, idx[ptr[i]:ptr[i + 1]]] = val[ptr[i]:ptr[i + 1]]
    return a


def test_oracle_coarse_cell_is_the_condensed_product_and_bends_exactly():
    """multigrid.rs:458-681 on 1 coarse cell of 2 x 2 x 2 fine cells, every unknown free: the
    coarse matrix is T^T K T of the coarse cell's 8 corner and 9 mode fields at the fine
    corners (formed here in numpy) with the modes condensed; it has no force for a rigid
    motion, and it holds a pure bending field with the exact energy, as 1 cell does."""
    size = (2.0, 0.5, 0.1)
    c = mg.hex_cantilever(nx=2, ny=2, nz=2, length=size[0], width=size[1], depth=size[2],
                          e=1000.0, nu=0.0)
    n = c.mesh.n
    k = oracle.pattern(3 * n, oracle.dof_elements(c.nodes))
    k.assemble(6, c.xyz, c.nodes, c.coef)
    free = np.arange(3 * n)
    ac, cp, cc = oracle.by_cells(k, c.mesh.planes, c.mesh.ijk[free // 3].astype(np.uint32),
                                 (free % 3).astype(np.uint8), class_table(c))
    corner = [tuple(b) for b in mg.HEX_BITS]
    perm = np.array([3 * corner.index(tuple(int(v) for v in p)) + q for p, q in zip(cp, cc)])
    got = np.zeros((24, 24))
    got[np.ix_(perm, perm)] = dense(ac)
    xi = 2.0 * c.xyz / np.asarray(size) - 1.0
    t = np.zeros((3 * n, 33))
    for m, b in enumerate(mg.HEX_BITS):
        f = np.prod([np.where(b[d], 0.5 * (1 + xi[:, d]), 0.5 * (1 - xi[:, d]))
                     for d in range(3)], axis=0)
        for q in range(3):
            t[q::3, 3 * m + q] = f
    for d in range(3):
        for q in range(3):
            t[q::3, 24 + 3 * d + q] = 1.0 - xi[:, d] ** 2
    kc = t.T @ dense(k) @ t
    want = kc[:24, :24] - kc[:24, 24:] @ np.linalg.solve(kc[24:, 24:], kc[24:, :24])
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    assert np.abs(got - got.T).max() <= 1e-13 * np.abs(got).max()
    corners = np.asarray(mg.HEX_BITS, float) * np.asarray(size)
    for f in [lambda x: [1.0, 0.0, 0.0], lambda x: [0.0, 1.0, 0.0], lambda x: [0.0, 0.0, 1.0],
              lambda x: [-x[1], x[0], 0.0], lambda x: [0.0, -x[2], x[1]],
              lambda x: [x[2], 0.0, -x[0]]]:
        u = np.concatenate([f(x) for x in corners])
        assert np.abs(got @ u).max() < 1e-12 * np.abs(got).max()
    kappa = 1e-3
    u = np.concatenate([[-kappa * x[0] * (x[2] - size[2] / 2.0), 0.0, kappa * x[0] ** 2 / 2.0]
                        for x in corners])
    exact = 1000.0 * size[1] * size[2] ** 3 / 12.0 * kappa ** 2 * size[0]
    assert abs(u @ got @ u - exact) < 1e-9 * exact


def test_oracle_cell_multigrid_solves_the_cantilever():
    """multigrid.rs:84-139 with cells: every coarse level from the cells of the one above; PCG
    with it reaches the direct solution."""
    c = mg.hex_cantilever(nx=48, ny=6, nz=6, length=6.0, width=0.75, depth=0.75, load=-1.0,
                          grade=1.1, seed=3)
    k = oracle.pattern(3 * c.mesh.n, oracle.dof_elements(c.nodes))
    k.assemble(6, c.xyz, c.nodes, c.coef)
    a = k.submatrix(c.free)
    rhs = k.reduced_rhs(c.load, c.values, c.free)
    planes, pts, comp = mg.grid_unknowns(c)
    s = oracle.Solver(a, "grid", planes=planes, points=pts, comp=comp, method="multigrid",
                      cells=class_table(c))
    assert len(s.levels()) >= 2
    x, it, res = s.solve(rhs, tol=1e-10)
    xd, _ = oracle.direct_solve(a, c.xyz[c.free // 3], rhs)
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)


@pytest.mark.gpu
def test_gpu_box_cell_elastic_assembly_is_bit_identical():
    """Graded cells of 2 materials (isotropic and orthotropic) in the x and z directions: the
    element classes differ, and each entry is the sum in cell order."""
    import femahoy_b200 as fg
    c = mg.hex_cantilever(nx=10, ny=3, nz=4, length=3.0, width=0.6, depth=0.4, load=-1.0,
                          grade=1.3, seed=7)
    K = fg.Csr.assemble(fg.HEX8_ELASTIC, c.xyz, c.nodes, c.coef)
    Ko = oracle.pattern(3 * c.mesh.n, oracle.dof_elements(c.nodes))
    Ko.assemble(6, c.xyz, c.nodes, c.coef)
    for a, b in zip(K.arrays(), Ko.arrays()):
        assert np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.gpu
def test_gpu_box_cell_elastic_rejects_bad_materials():
    import femahoy_b200 as fg
    c = mg.hex_cantilever(nx=2, ny=1, nz=1)
    coef = c.coef.copy()
    coef[1] = oracle.orthotropic(1.0, 0.5)
    with pytest.raises(fg.FemError, match="no stable material"):
        fg.Csr.assemble(fg.HEX8_ELASTIC, c.xyz, c.nodes, coef)
    coef[1] = oracle.orthotropic(-1.0, 0.3)
    with pytest.raises(fg.FemError, match="moduli must be above 0"):
        fg.Csr.assemble(fg.HEX8_ELASTIC, c.xyz, c.nodes, coef)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_box_cantilever_solves(precision):
    """PCG with the grid V-cycle on a box-cell cantilever against the oracle's direct solution
    (1e-8 relative) and its own true residual."""
    import femahoy_b200 as fg
    c = mg.hex_cantilever(nx=48, ny=6, nz=6, length=6.0, width=0.75, depth=0.75, load=-1.0,
                          grade=1.1, seed=3)
    K = fg.Csr.assemble(fg.HEX8_ELASTIC, c.xyz, c.nodes, c.coef)
    A = K.submatrix(c.free)
    rhs = fg.reduced_rhs(K, c.load, c.values, c.free)
    planes, pts, comp = mg.grid_unknowns(c)
    s = fg.Solver(A, fg.Unknowns.Grid(fg.Level(planes, pts, comp)), fg.Method.Multigrid,
                  precision=precision,
                  options=fg.Options(precision=precision, coarsest=600)).with_tol(1e-10)
    assert s.levels()[0] == A.n and len(s.levels()) >= 2
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.true_residual <= 1.2e-10
    Ko = oracle.pattern(3 * c.mesh.n, oracle.dof_elements(c.nodes))
    Ko.assemble(6, c.xyz, c.nodes, c.coef)
    xd, _ = oracle.direct_solve(Ko.submatrix(c.free), c.xyz[c.free // 3],
                                Ko.reduced_rhs(c.load, c.values, c.free))
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)


def cells_of(c, fg):
    """The device's cells of a box-cell problem: the class matrices from femgpu_hex_elements."""
    origin, cls, keys = mg.hex_classes(c)
    return fg.Cells(origin, cls, fg.hex_elements(keys)), keys


@pytest.mark.gpu
def test_gpu_hex_elements_are_bit_identical():
    import femahoy_b200 as fg
    c = mg.hex_cantilever(nx=6, ny=2, nz=3, grade=1.4, seed=11)
    cells, keys = cells_of(c, fg)
    want = np.stack([oracle.hex8_stiffness(k[:3], k[3:]) for k in keys])
    assert np.array_equal(cells.matrices.view(np.uint64), want.view(np.uint64))
    with pytest.raises(fg.FemError, match="side not above 0"):
        bad = keys[:1].copy()
        bad[0, 1] = 0.0
        fg.hex_elements(bad)


def _kept_planes(p):
    """multigrid.rs:341-346: every other plane and the last (axes of more than 2 planes)."""
    p = np.asarray(p)
    if len(p) <= 2:
        return p
    k = list(range(0, len(p), 2))
    if k[-1] != len(p) - 1:
        k.append(len(p) - 1)
    return p[k]


def _to_grid_order(so, planes, pts, comp, level):
    """The oracle's matrix of `level` (its unknowns in first-sight order, multigrid.rs:329-452)
    renumbered in grid order (z, y, x, component), and the grid points in that order."""
    import scipy.sparse as sp
    pl, p_, c_ = [np.asarray(x) for x in planes], pts, comp
    for l in range(level):
        _, p_, c_ = oracle.coarsen(so.level_matrix(l), pl, p_, c_)
        pl = [_kept_planes(x) for x in pl]
    comps = int(c_.max()) + 1
    key = c_.astype(np.int64) + comps * (p_[:, 0].astype(np.int64) + len(pl[0]) * (
        p_[:, 1].astype(np.int64) + len(pl[1]) * p_[:, 2].astype(np.int64)))
    o = np.argsort(key, kind="stable")
    ptr, idx, val = so.level_matrix(level).arrays()
    m = sp.csr_matrix((val, idx, ptr), shape=(len(ptr) - 1,) * 2)[o][:, o].tocsr()
    m.sort_indices()
    return m, p_[o], c_[o]


@pytest.mark.gpu
@pytest.mark.parametrize("level", [1, 2])
def test_gpu_coarse_matrices_against_the_oracle(level):
    """multigrid.rs:329-681 on a graded cantilever of 2 materials: the device's coarsening (grid
    order) reaches the oracle's coarse unknowns; the coarse matrices from the cells (host
    threads, level 2 formed from level 1's cells) equal the oracle's bit for bit, and the
    device's Galerkin products P^T A P (coarsen.cu, summed in its own order) equal the oracle's
    to rounding."""
    import femahoy_b200 as fg
    c = mg.hex_cantilever(nx=64, ny=8, nz=12, length=8.0, width=1.0, depth=1.5, load=-1.0,
                          grade=1.3, seed=9)
    K = fg.Csr.assemble(fg.HEX8_ELASTIC, c.xyz, c.nodes, c.coef)
    A = K.submatrix(c.free)
    planes, pts, comp = mg.grid_unknowns(c)
    cells, _ = cells_of(c, fg)
    ptr, idx, val, gp, gc = fg.coarse_matrix(A, fg.Unknowns.Grid(fg.Level(planes, pts, comp)),
                                             level, cells)
    Ko = oracle.pattern(3 * c.mesh.n, oracle.dof_elements(c.nodes))
    Ko.assemble(6, c.xyz, c.nodes, c.coef)
    so = oracle.Solver(Ko.submatrix(c.free), "grid", planes=planes, points=pts, comp=comp,
                       method="multigrid", cells=class_table(c))
    want, wp, wc = _to_grid_order(so, planes, pts, comp, level)
    assert np.array_equal(gp, wp) and np.array_equal(gc, wc)
    assert np.array_equal(ptr, want.indptr) and np.array_equal(idx, want.indices)
    assert np.array_equal(val.view(np.uint64), want.data.view(np.uint64))
    # The Galerkin form through the same entry, against the oracle's P^T A P.
    ptr, idx, val, gp, gc = fg.coarse_matrix(A, fg.Unknowns.Grid(fg.Level(planes, pts, comp)),
                                             level)
    sg = oracle.Solver(Ko.submatrix(c.free), "grid", planes=planes, points=pts, comp=comp,
                       method="multigrid")
    want, wp, wc = _to_grid_order(sg, planes, pts, comp, level)
    assert np.array_equal(gp, wp) and np.array_equal(gc, wc)
    assert np.array_equal(ptr, want.indptr) and np.array_equal(idx, want.indices)
    rows = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
    scale = np.maximum.reduceat(np.abs(want.data), ptr[:-1])[rows]
    assert np.all(np.abs(val - want.data) <= 1e-12 * scale)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_box_cantilever_solves_with_cells(precision):
    """PCG with the cell-based V-cycle (the reference's box-grid elastic solver) against the
    oracle's direct solution (1e-8 relative) and its own true residual."""
    import femahoy_b200 as fg
    c = mg.hex_cantilever(nx=48, ny=6, nz=6, length=6.0, width=0.75, depth=0.75, load=-1.0,
                          grade=1.1, seed=3)
    K = fg.Csr.assemble(fg.HEX8_ELASTIC, c.xyz, c.nodes, c.coef)
    A = K.submatrix(c.free)
    rhs = fg.reduced_rhs(K, c.load, c.values, c.free)
    planes, pts, comp = mg.grid_unknowns(c)
    cells, _ = cells_of(c, fg)
    s = fg.Solver(A, fg.Unknowns.Grid(fg.Level(planes, pts, comp)), fg.Method.Multigrid,
                  cells=cells, precision=precision,
                  options=fg.Options(precision=precision, coarsest=600)).with_tol(1e-10)
    assert len(s.levels()) >= 2
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.true_residual <= 1.2e-10
    Ko = oracle.pattern(3 * c.mesh.n, oracle.dof_elements(c.nodes))
    Ko.assemble(6, c.xyz, c.nodes, c.coef)
    xd, _ = oracle.direct_solve(Ko.submatrix(c.free), c.xyz[c.free // 3],
                                Ko.reduced_rhs(c.load, c.values, c.free))
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)


def hex_recovery_case(seed=4, nparts=3):
    """A graded cantilever of 2 materials with a random displacement, a random temperature
    change, expansion per cell, parts and a few singular points."""
    c = mg.hex_cantilever(nx=7, ny=3, nz=4, grade=1.4, seed=seed)
    rng = np.random.default_rng(seed)
    n, nel = c.mesh.n, len(c.nodes)
    return {"xyz": c.xyz, "hexes": c.nodes, "coef": c.coef,
            "expansion": rng.uniform(1e-6, 3e-5, size=(nel, 3)),
            "part": rng.integers(0, nparts, size=nel).astype(np.uint32), "nparts": nparts,
            "singular": (rng.random(n) < 0.05).astype(np.uint8),
            "u": rng.standard_normal(3 * n) * 1e-3, "dtemp": rng.standard_normal(n) * 10.0}


def test_oracle_box_recovery_peaks_follow_the_loop():
    """elastic.rs:636-650: the peak of each part is the first strict maximum over the visits in
    loop order (cell, then corner), and the regular peak the same over the visits that touch no
    singular point; checked against a numpy walk of the oracle's own per-visit values."""
    c = hex_recovery_case()
    r = oracle.recover(c["xyz"], c["hexes"], c["coef"], c["u"], expansion=c["expansion"],
                       dtemp=c["dtemp"], part=c["part"], nparts=c["nparts"],
                       singular=c["singular"], hex=True)
    best = [(-np.inf, -1, -1)] * c["nparts"]
    reg = [(-np.inf, -1, -1)] * c["nparts"]
    seen = [False] * c["nparts"]
    for e, nodes in enumerate(c["hexes"]):
        size = c["xyz"][nodes[6]] - c["xyz"][nodes[0]]
        ue = c["u"].reshape(-1, 3)[nodes].ravel()
        near = bool(c["singular"][nodes].any())
        p = c["part"][e]
        for k, b in enumerate(mg.HEX_BITS):
            xi = np.where(np.asarray(b) == 1, 1.0, -1.0)
            _, s = oracle.hex8_strain_stress(size, c["coef"][e], xi, ue, c["dtemp"][nodes],
                                             alpha=c["expansion"][e])
            s = [s[0], s[1], s[2], s[5], s[3], s[4]]
            vm = np.sqrt(0.5 * ((s[0] - s[1]) ** 2 + (s[1] - s[2]) ** 2 + (s[2] - s[0]) ** 2)
                         + 3.0 * (s[3] ** 2 + s[4] ** 2 + s[5] ** 2))
            if vm > best[p][0]:
                best[p] = (vm, e, k)
            if not (near or c["singular"][nodes[k]]) and (not seen[p] or vm > reg[p][0]):
                seen[p] = True
                reg[p] = (vm, e, k)
    for p, pk in enumerate(r["peaks"]):
        assert (pk.element, pk.local) == best[p][1:] and abs(pk.mises - best[p][0]) <= 1e-9 * best[p][0]
        assert (pk.regular_element, pk.regular_local) == reg[p][1:]


def box_recovery_parity(c):
    from femahoy_b200.recover import Recovery
    ref = oracle.recover(c["xyz"], c["hexes"], c["coef"], c["u"], expansion=c["expansion"],
                         dtemp=c["dtemp"], part=c["part"], nparts=c["nparts"],
                         singular=c["singular"], hex=True)
    rec = Recovery(c["xyz"], c["hexes"], c["coef"], expansion=c["expansion"], part=c["part"],
                   nparts=c["nparts"], singular=c["singular"], hex=True)
    got = rec.run(c["u"], c["dtemp"])
    for key in ("stress", "strain", "mises"):
        assert np.array_equal(np.asarray(got[key]).view(np.uint64), ref[key].view(np.uint64)), key
    scale = np.nanmax(np.abs(ref["stress"]))
    assert np.allclose(got["principal"], ref["principal"], rtol=0, atol=1e-12 * scale,
                       equal_nan=True)
    return ref, got


@pytest.mark.gpu
def test_gpu_box_recovery_ties_and_nan():
    """All displacements 0 (every strain 0, ties: the first visit wins), then a NaN displacement
    at a corner: the strains of its cells are NaN at every corner, as the reference's sums over
    the 11 functions make them (a zero gradient times NaN is NaN)."""
    c = hex_recovery_case(seed=9)
    c["u"] = np.zeros_like(c["u"])
    c["dtemp"] = np.zeros_like(c["dtemp"])
    box_recovery_parity(c)
    c["u"][3 * int(c["hexes"][5, 2]) + 1] = np.nan
    ref, _ = box_recovery_parity(c)
    assert np.isnan(ref["strain"][c["hexes"][5, 0]]).any()


@pytest.mark.gpu
def test_gpu_box_recovery_is_bit_identical_to_the_oracle():
    """elastic.rs:615-660 on the device against the oracle: stress, strain and von Mises bit for
    bit, the principal stresses to 1e-12 of the largest stress (acos, cos), the peaks equal."""
    from femahoy_b200.recover import Recovery
    c = hex_recovery_case()
    ref, got = box_recovery_parity(c)
    for g, o in zip(got["peaks"], ref["peaks"]):
        assert (g.element, g.local, g.point, int(g.singular), g.regular_element, g.regular_local,
                g.regular_point) == (o.element, o.local, o.point, int(o.singular),
                                     o.regular_element, o.regular_local, o.regular_point)
        assert np.array_equal(np.array([g.mises, g.regular_mises]).view(np.uint64),
                              np.array([o.mises, o.regular_mises]).view(np.uint64))
    # Without the optional arrays: 1 part, no expansion, no temperature.
    ref = oracle.recover(c["xyz"], c["hexes"], c["coef"], c["u"], hex=True)
    got = Recovery(c["xyz"], c["hexes"], c["coef"], hex=True).run(c["u"])
    assert np.array_equal(got["stress"].view(np.uint64), ref["stress"].view(np.uint64))


def test_oracle_thermal_load_of_a_cell_is_its_free_expansion():
    """hex.rs:222-297: the load of a uniform temperature change dT equals K times the free
    thermal expansion (alpha_d dT x_d along each axis), which has no stress; with an
    orthotropic material and an expansion per axis."""
    c = oracle.orthotropic([200.0, 120.0, 90.0], [0.25, 0.3, 0.35], [70.0, 60.0, 50.0])
    alpha = np.array([1e-5, 2e-5, 3e-5])
    k, load, _, _ = oracle.hex8_element(SIZE, c, alpha)
    dt = 7.0
    u = nodal(lambda x: list(alpha * dt * np.asarray(x)))
    f = load @ np.full(8, dt)
    assert np.abs(k @ u - f).max() <= 1e-12 * np.abs(f).max()


def test_oracle_box_loads_sum_the_cells():
    """elastic.rs:386-405 over graded cells: with no temperature the forces are the volume
    terms (an eighth of its cell's at each corner), summing to accel times the volume; with a
    uniform temperature on a free body of 1 material they equal K times the free expansion."""
    c = mg.hex_cantilever(nx=4, ny=2, nz=3, grade=1.4)
    nel = len(c.nodes)
    accel = np.tile([0.0, -2.0, -9.81], (nel, 1))
    f = oracle.hex_loads(c.xyz, c.nodes, c.coef, accel=accel)
    vol = np.prod(c.xyz[c.nodes[:, 6]] - c.xyz[c.nodes[:, 0]], axis=1).sum()
    assert np.allclose(f.reshape(-1, 3).sum(axis=0), [0.0, -2.0 * vol, -9.81 * vol], rtol=1e-13)
    alpha = np.tile([1e-5, 1e-5, 1e-5], (nel, 1))
    dt = np.full(c.mesh.n, 5.0)
    f = oracle.hex_loads(c.xyz, c.nodes, c.coef, expansion=alpha, dtemp=dt)
    k = oracle.pattern(3 * c.mesh.n, oracle.dof_elements(c.nodes))
    k.assemble(6, c.xyz, c.nodes, c.coef)
    u = (1e-5 * 5.0 * c.xyz).ravel()
    assert np.abs(dense(k) @ u - f).max() <= 1e-12 * np.abs(f).max()


@pytest.mark.gpu
def test_gpu_box_loads_are_bit_identical():
    """elastic.rs:386-405 on the device against the oracle: graded cells, 2 materials, an
    expansion per cell, a random temperature change and volume forces."""
    from femahoy_b200.recover import hex_loads
    c = hex_recovery_case(seed=6)
    nel = len(c["hexes"])
    accel = np.random.default_rng(2).standard_normal((nel, 3))
    ref = oracle.hex_loads(c["xyz"], c["hexes"], c["coef"], expansion=c["expansion"],
                           accel=accel, dtemp=c["dtemp"])
    got = hex_loads(c["xyz"], c["hexes"], c["coef"], expansion=c["expansion"], accel=accel,
                    dtemp=c["dtemp"])
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
    ref = oracle.hex_loads(c["xyz"], c["hexes"], c["coef"], accel=accel)
    got = hex_loads(c["xyz"], c["hexes"], c["coef"], accel=accel)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))


def test_oracle_box_mass_is_the_integral_of_the_corner_functions():
    """hex.rs:408-431: each entry is the 2-point Gauss integral of rho N_i N_j (exact for the
    trilinear functions), 0 between components, and the entries sum to 3 times the mass."""
    m = oracle.hex8_mass(SIZE, 7.0)
    jac = np.prod(SIZE) / 8.0
    p = 1.0 / np.sqrt(3.0)

    def shape(xi):
        return np.array([np.prod([0.5 * (1 + xi[d]) if b[d] else 0.5 * (1 - xi[d])
                                  for d in range(3)]) for b in mg.HEX_BITS])
    gauss = [np.where(np.asarray(b) == 1, p, -p) for b in mg.HEX_BITS]
    for i in range(8):
        for j in range(8):
            exact = sum(7.0 * shape(x)[i] * shape(x)[j] * jac for x in gauss)
            assert abs(m[3 * i, 3 * j] - exact) < 1e-14
            assert m[3 * i, 3 * j + 1] == 0.0
    assert abs(m.sum() - 3.0 * 7.0 * 8.0 * jac) < 1e-12


@pytest.mark.gpu
def test_gpu_box_mass_is_bit_identical():
    import femahoy_b200 as fg
    c = mg.hex_cantilever(nx=6, ny=2, nz=3, grade=1.3, seed=5)
    rho = np.random.default_rng(1).uniform(1.0, 8.0, len(c.nodes))
    M = fg.Csr.assemble(fg.HEX8_MASS, c.xyz, c.nodes, rho)
    Mo = oracle.pattern(3 * c.n_points, oracle.dof_elements(c.nodes))
    Mo.assemble(7, c.xyz, c.nodes, rho)
    for a, b in zip(M.arrays(), Mo.arrays()):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    sizes = c.xyz[c.nodes[:4, 6]] - c.xyz[c.nodes[:4, 0]]
    got = fg.hex_mass(sizes, rho[:4])
    for e in range(4):
        assert np.array_equal(got[e].view(np.uint64), oracle.hex8_mass(sizes[e], rho[e]).view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_box_modes_match_the_oracle(precision):
    """modes.rs:355-420: the 6 lowest modes of a clamped box-cell cantilever by the device's
    subspace iteration, its PCG preconditioned by the V-cycle whose coarse matrices come from the
    cells of K - shift M, against the oracle's subspace iteration (its direct solver):
    eigenvalues to 1e-8."""
    import femahoy_b200 as fg
    from femahoy_b200.modes import modes
    c = mg.hex_cantilever(nx=40, ny=4, nz=4, length=8.0, width=0.8, depth=0.8, grade=1.1, seed=2)
    rho = np.where(c.coef[:, 1] == c.coef[:, 0], 7.8e-9, 2.7e-9)  # isotropic: steel
    Kf = fg.Csr.assemble(fg.HEX8_ELASTIC, c.xyz, c.nodes, c.coef).submatrix(c.free)
    Mf = fg.Csr.assemble(fg.HEX8_MASS, c.xyz, c.nodes, rho).submatrix(c.free)
    origin, cls, keys = mg.hex_classes(c)
    first = np.array([np.nonzero(cls == k)[0][0] for k in range(len(keys))])
    cells = fg.Cells(origin, cls, fg.hex_elements(keys), fg.hex_mass(keys[:, :3], rho[first]))
    planes, pts, comp = mg.grid_unknowns(c)
    u = fg.Unknowns.Grid(fg.Level(planes, pts, comp))
    opts = fg.Options(precision=precision, coarsest=300)
    values, vecs, st = modes(Kf, Mf, 6, u, fg.Method.Multigrid, options=opts, cells=cells)
    ko = oracle.Csr.from_arrays(Kf.n, *Kf.arrays())
    mo = oracle.Csr.from_arrays(Mf.n, *Mf.arrays())
    ptr, idx, val = ko.arrays()
    a = oracle.Csr.from_arrays(ko.n, ptr, idx, val - st.shift * mo.arrays()[2])

    def solve(b, x0):
        x, _ = oracle.direct_solve(a, c.xyz[c.free // 3], b)
        return x

    ov, _, _ = oracle.subspace(ko, mo, st.shift, 6, solve)
    assert np.abs(values - ov).max() <= 1e-8 * ov.max()


@pytest.mark.gpu
def test_gpu_box_cell_errors():
    """The box-cell kinds assemble by rows only; a cell with a side not above 0 is refused; the
    cells of a solver must lie inside the planes; coarsening past the grid is refused."""
    import femahoy_b200 as fg
    c = mg.hex_cantilever(nx=4, ny=2, nz=2)
    for kind, coef in ((fg.HEX8_ELASTIC, c.coef), (fg.HEX8_MASS, np.ones(len(c.nodes)))):
        with pytest.raises(fg.FemError, match="assemble by rows"):
            fg.Csr.assemble(kind, c.xyz, c.nodes, coef, mode=fg.COLOUR)
    flipped = c.nodes[:, [6, 7, 4, 5, 2, 3, 0, 1]]  # corner 6 below corner 0
    with pytest.raises(fg.FemError, match="side not above 0"):
        fg.Csr.assemble(fg.HEX8_ELASTIC, c.xyz, flipped, c.coef)
    K = fg.Csr.assemble(fg.HEX8_ELASTIC, c.xyz, c.nodes, c.coef)
    A = K.submatrix(c.free)
    planes, pts, comp = mg.grid_unknowns(c)
    u = fg.Unknowns.Grid(fg.Level(planes, pts, comp))
    cells, _ = cells_of(c, fg)
    bad = fg.Cells(cells.origin + np.array([10, 0, 0], np.uint32), cells.cls, cells.matrices)
    with pytest.raises(fg.FemError, match="past the planes"):
        fg.Solver(A, u, fg.Method.Multigrid, cells=bad)
    with pytest.raises(fg.FemError, match="does not coarsen"):
        fg.coarse_matrix(A, u, 5, cells)


def test_extruded_mesh_is_conforming_with_points_on_z_planes():
    """meshgen.extruded: positive volumes summing to the footprint's area times the height,
    every triangular face shared by at most 2 tetrahedra (the wedges' quad faces split alike),
    and the corner points on the layers' z planes but not on x planes."""
    xyz, tets = mg.extruded(npoints=80, layers=3, height=2.0, seed=1)
    p = xyz[tets]
    vol = np.linalg.det(p[:, 1:] - p[:, :1]) / 6.0
    assert vol.min() > 0.0
    foot = np.unique(xyz[:, :2], axis=0)
    lo, hi = foot.min(axis=0), foot.max(axis=0)
    assert abs(vol.sum() - np.prod(hi - lo) * 2.0) < 1e-12
    faces = np.sort(np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]],
                                    tets[:, [1, 2, 3]]]), axis=1)
    _, count = np.unique(faces, axis=0, return_counts=True)
    assert count.max() == 2
    planes, pts, comp = mg.level_of(xyz, np.arange(3 * len(xyz)))
    assert len(planes[2]) == 4 and len(planes[0]) > 10
    assert np.allclose(planes[2][pts[:, 2]], xyz[np.arange(3 * len(xyz)) // 3, 2])
