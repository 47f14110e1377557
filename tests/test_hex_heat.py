"""Heat on the box cells of the grid (heat.rs:804-826 with the conduction matrix of
heat.rs:1246-1273): the reference's box-grid heat model.

CPU: the oracle's element (symmetric, zero row sums) and the reference's layered-wall test
(tests/heat.rs:112-128: the interface temperatures and the heat flow of a layered wall are
exact). GPU: the device assembly bit for bit against the oracle, and the solve."""
import numpy as np
import pytest

import oracle
from femahoy_b200 import meshgen as mg


def layered_wall(layers=((0.5, 1.0), (0.25, 0.05), (1.0, 2.0)), cells=(4, 2, 8), ny=2, nz=2):
    """A wall along x of layers (thickness, conductivity), cells[i] box cells through layer i,
    T = 100 on x = 0 and 0 on the far face, no source: 1D heat flow."""
    xs = [0.0]
    ks = []
    for (t, k), c in zip(layers, cells):
        for j in range(c):
            xs.append(xs[-1] + t / c)
            ks.append(k)
    nx = len(ks)
    mesh = mg.box(nx, ny, nz, (1.0, 1.0, 1.0))
    x = np.asarray(xs)
    mesh.points[:, 0] = x[mesh.ijk[:, 0]]
    mesh.planes[0] = x
    hexes = mg.box_cells(mesh)
    ci = np.arange(len(hexes)) % nx
    coef = np.repeat(np.asarray(ks)[ci][:, None], 3, axis=1)
    fixed = (mesh.ijk[:, 0] == 0) | (mesh.ijk[:, 0] == nx)
    values = np.where(mesh.ijk[:, 0] == 0, 100.0, 0.0)
    free = np.nonzero(~fixed)[0].astype(np.int64)
    resist = sum(t / k for t, k in layers)
    q = 100.0 / resist
    exact = np.empty(nx + 1)
    exact[0] = 100.0
    for i in range(nx):
        exact[i + 1] = exact[i] - q * (x[i + 1] - x[i]) / ks[i]
    return mesh, hexes, coef, values, free, exact[mesh.ijk[:, 0]]


def test_oracle_box_cell_conduction_is_symmetric_with_zero_row_sums():
    mesh = mg.box(1, 1, 1, (0.3, 0.7, 1.1))
    k = oracle.pattern(8, mg.box_cells(mesh))
    k.assemble(5, mesh.points, mg.box_cells(mesh), np.array([[1.5, 2.0, 0.5]]))
    ptr, idx, val = k.arrays()
    a = np.zeros((8, 8))
    for i in range(8):
        a[i, idx[ptr[i]:ptr[i + 1]]] = val[ptr[i]:ptr[i + 1]]
    assert np.allclose(a, a.T, rtol=0, atol=1e-15)
    assert np.abs(a.sum(axis=1)).max() < 1e-14


def test_oracle_layered_wall_is_exact():
    """tests/heat.rs:112-128: trilinear box cells hold the piecewise-linear 1D solution."""
    mesh, hexes, coef, values, free, exact = layered_wall()
    k = oracle.pattern(mesh.n, hexes)
    k.assemble(5, mesh.points, hexes, coef)
    a = k.submatrix(free)
    rhs = k.reduced_rhs(np.zeros(mesh.n), values, free)
    x, _ = oracle.direct_solve(a, mesh.points[free], rhs)
    assert np.abs(x - exact[free]).max() < 1e-10


@pytest.mark.gpu
def test_gpu_box_cell_assembly_is_bit_identical():
    import femahoy_b200 as fg
    h = mg.heat_cube_hex(12, seed=3)
    K = fg.Csr.assemble(fg.HEX8_HEAT, h.xyz, h.nodes, h.coef)
    Ko = oracle.pattern(h.n_points, h.nodes)
    Ko.assemble(5, h.xyz, h.nodes, h.coef)
    for a, b in zip(K.arrays(), Ko.arrays()):
        assert np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_box_cell_heat_solves(precision):
    """The layered wall (exact to 1e-8 of 100) and a 24^3 lognormal cube against the oracle's
    direct solution (1e-8), by PCG with the grid's V-cycle."""
    import femahoy_b200 as fg
    mesh, hexes, coef, values, free, exact = layered_wall(cells=(8, 4, 16), ny=8, nz=8)
    K = fg.Csr.assemble(fg.HEX8_HEAT, mesh.points, hexes, coef)
    A = K.submatrix(free)
    rhs = fg.reduced_rhs(K, np.zeros(mesh.n), values, free)
    lv = fg.Level(mesh.planes, mesh.ijk[free].astype(np.uint32),
                  np.zeros(len(free), np.uint8))
    s = fg.Solver(A, fg.Unknowns.Grid(lv), fg.Method.Multigrid, precision=precision,
                  options=fg.Options(precision=precision, coarsest=64)).with_tol(1e-12)
    x = np.zeros(A.n)
    s.solve(rhs, x)
    assert np.abs(x - exact[free]).max() < 1e-8 * 100.0
    h = mg.heat_cube_hex(24, seed=5)
    K = fg.Csr.assemble(fg.HEX8_HEAT, h.xyz, h.nodes, h.coef)
    A = K.submatrix(h.free)
    rhs = fg.reduced_rhs(K, h.load, h.values, h.free)
    planes, pts, comp = mg.grid_unknowns(h)
    s = fg.Solver(A, fg.Unknowns.Grid(fg.Level(planes, pts, comp)), fg.Method.Multigrid,
                  precision=precision).with_tol(1e-10)
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.true_residual <= 1.2e-10
    Ko = oracle.pattern(h.n_points, h.nodes)
    Ko.assemble(5, h.xyz, h.nodes, h.coef)
    xd, _ = oracle.direct_solve(Ko.submatrix(h.free), h.xyz[h.free],
                                Ko.reduced_rhs(h.load, h.values, h.free))
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
