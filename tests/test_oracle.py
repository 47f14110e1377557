"""The oracle against the reference's own known answers (its unit tests), and the analytic
identities its integration tests check. CPU only."""
import re

import numpy as np
import pytest

import oracle
from femahoy_b200 import meshgen as mg


def laplacian(n):
    """cholesky.rs:234-258: the shifted 5-point Laplacian of an n x n grid."""
    ids = lambda i, j: i + n * j
    elements = []
    for j in range(n):
        for i in range(n):
            if i + 1 < n:
                elements.append([ids(i, j), ids(i + 1, j)])
            if j + 1 < n:
                elements.append([ids(i, j), ids(i, j + 1)])
    a = oracle.pattern(n * n, np.array(elements))
    for e in elements:
        a.add_element(e, [1.0, -1.0, -1.0, 1.0])
    ptr, idx, val = a.arrays()
    for i in range(n * n):
        k = ptr[i] + np.searchsorted(idx[ptr[i]:ptr[i + 1]], i)
        val[k] += 0.01
    a = oracle.Csr.from_arrays(n * n, ptr, idx, val)
    xyz = np.array([[k % n, k // n, 0.0] for k in range(n * n)], dtype=float)
    return a, xyz


def test_pattern_of_two_elements():
    """sparse.rs:299-305"""
    a = oracle.pattern(3, np.array([[0, 1], [1, 2]]))
    ptr, idx, _ = a.arrays()
    assert ptr.tolist() == [0, 2, 5, 7]
    assert idx.tolist() == [0, 1, 0, 1, 2, 1, 2]


def test_galerkin_of_1d_laplacian():
    """sparse.rs:307-324"""
    el = np.array([[0, 1], [1, 2]])
    a = oracle.pattern(3, el)
    for e in el:
        a.add_element(e, [1.0, -1.0, -1.0, 1.0])
    p = oracle.Rect.from_arrays(3, 2, [0, 1, 3, 4], [0, 0, 1, 1], [1.0, 0.5, 0.5, 1.0])
    c = p.galerkin(a)
    _, idx, val = c.arrays()
    assert idx.tolist() == [0, 1, 0, 1]
    assert val.tolist() == [0.5, -0.5, -0.5, 0.5]


def test_factor_solves_grid_laplacian():
    """cholesky.rs:260-279"""
    a, xyz = laplacian(40)
    x = np.sin(np.arange(a.n) * 0.37)
    b = a.mul(x)
    sol, entries = oracle.direct_solve(a, xyz, b)
    assert np.abs(sol - x).max() < 1e-9
    assert entries < 40_000


def test_singular_matrix_is_an_error():
    """cholesky.rs:281-293"""
    a, xyz = laplacian(10)
    ptr, idx, val = a.arrays()
    for i in range(a.n):
        k = ptr[i] + np.searchsorted(idx[ptr[i]:ptr[i + 1]], i)
        val[k] -= 0.01
    a = oracle.Csr.from_arrays(a.n, ptr, idx, val)
    with pytest.raises(oracle.OracleError) as e:
        oracle.direct_solve(a, xyz, np.ones(a.n))
    assert "not positive definite" in str(e.value) or "singular" in str(e.value)


def test_order_is_permutation_with_middle_last():
    """order.rs:186-197"""
    n = 200
    el = np.array([[i, i + 1] for i in range(n - 1)])
    a = oracle.pattern(n, el)
    xyz = np.array([[i, 0.0, 0.0] for i in range(n)])
    order = oracle.nested_dissection(a, xyz)
    assert sorted(order.tolist()) == list(range(n))
    assert order[-1] == 99


def test_pattern_counts_of_the_benchmark_meshes():
    """The nnz of the structured Kuhn meshes: config 1's scalar and operator patterns."""
    p = mg.cantilever_p1()
    assert p.mesh.n == 1025 and len(p.mesh.tets) == 3840
    k = oracle.pattern(p.mesh.n, p.nodes)
    assert k.shape == (1025, 12097)
    k3 = oracle.pattern(3 * p.mesh.n, oracle.dof_elements(p.nodes))
    assert k3.shape == (3075, 108873)
    assert len(p.free) == 3000


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_element_matrices_are_symmetric_and_rigid_motions_are_free(kind):
    """hex.rs:400-552's identities on the tetrahedra: a symmetric element matrix, no force
    from a rigid motion (heat: a constant field)."""
    rng = np.random.default_rng(3)
    p = np.array([[0, 0, 0], [2.0, 0.1, 0], [0.3, 1.5, 0.2], [0.1, 0.4, 0.9]])
    p = p + 0.05 * rng.standard_normal(p.shape)
    if kind == 0:
        ke = oracle.element_matrix(0, p, [1.0, 2.0, 3.0])
        assert np.allclose(ke, ke.T, rtol=0, atol=1e-14 * np.abs(ke).max())
        assert np.abs(ke @ np.ones(4)).max() < 1e-13 * np.abs(ke).max()
        return
    ke = oracle.element_matrix(kind, p, [210e3, 0.3])
    assert np.allclose(ke, ke.T, rtol=0, atol=1e-12 * np.abs(ke).max())
    pts = p if kind == 1 else np.concatenate(
        [p, 0.5 * (p[mg.EDGES[:, 0]] + p[mg.EDGES[:, 1]])])
    w = np.array([0.3, -0.2, 0.5])
    for u in [np.tile([1.0, 0, 0], len(pts)), np.tile([0, 1.0, 0], len(pts)),
              np.cross(w, pts).ravel()]:
        assert np.abs(ke @ u).max() < 1e-9 * np.abs(ke).max()


def test_linear_field_is_exact_on_tetrahedra():
    """fem-tests/tet.rs:219 on the Kuhn mesh: with no source and T fixed at 1 on x = 0 and 0 on
    x = 1, the temperature is 1 - x at every node, by direct and by PCG-MG."""
    h = mg.heat_cube(8, source=0.0)
    h.coef[:] = 2.5
    k = oracle.pattern(h.n_points, h.nodes)
    k.assemble(0, h.xyz, h.nodes, h.coef)
    a = k.submatrix(h.free)
    rhs = k.reduced_rhs(h.load, h.values, h.free)
    exact = 1.0 - h.xyz[h.free, 0]
    xd, _ = oracle.direct_solve(a, h.xyz[h.free], rhs)
    assert np.abs(xd - exact).max() < 1e-12
    planes, pts, comp = mg.grid_unknowns(h)
    s = oracle.Solver(a, "grid", planes=planes, points=pts, comp=comp, method="multigrid")
    x, it, res = s.solve(rhs, tol=1e-12)
    assert np.abs(x - exact).max() < 1e-10


def test_direct_and_multigrid_agree_on_heat():
    """fem-tests/heat.rs:130 on a lognormal 16^3 cube: |T_direct - T_mg| < 1e-6."""
    h = mg.heat_cube(16)
    k = oracle.pattern(h.n_points, h.nodes)
    k.assemble(0, h.xyz, h.nodes, h.coef)
    a = k.submatrix(h.free)
    rhs = k.reduced_rhs(h.load, h.values, h.free)
    planes, pts, comp = mg.grid_unknowns(h)
    s = oracle.Solver(a, "grid", planes=planes, points=pts, comp=comp, method="multigrid")
    assert s.levels()[0] == a.n and len(s.levels()) > 1
    x, it, res = s.solve(rhs)
    xd, _ = oracle.direct_solve(a, h.xyz[h.free], rhs)
    assert np.abs(x - xd).max() < 1e-6
    assert res <= 1e-10


def test_direct_and_p_multigrid_agree_on_p2():
    """fem-tests/elastic_tet.rs:236: |u_direct - u_pmg| < 1e-8 max|u| on a small P2 beam."""
    m = mg.box(8, 2, 2, (40.0, 10.0, 10.0))
    edges, t10 = oracle.quadratic(m.points, m.tets)
    prob = mg.beam_p2(edges, t10, mesh=m)
    k = oracle.pattern(3 * prob.n_points, oracle.dof_elements(prob.nodes))
    k.assemble(2, prob.xyz, prob.nodes, prob.coef)
    free = prob.free
    a = k.submatrix(free)
    rhs = k.reduced_rhs(prob.load, prob.values, free)
    p, cxyz = oracle.prolongation(prob.xyz, m.n, edges, free)
    s = oracle.Solver(a, "quadratic", xyz=prob.xyz[free // 3], p=p, coarse=cxyz,
                      method="multigrid")
    x, it, res = s.solve(rhs)
    xd, _ = oracle.direct_solve(a, prob.xyz[free // 3], rhs)
    scale = np.abs(xd).max()
    assert np.abs(x - xd).max() < 1e-8 * scale
    assert it > 0


def test_pcg_reports_non_convergence_and_cancel():
    """multigrid.rs:729-735: the error texts of too few iterations and of a cancel."""
    h = mg.heat_cube(16)
    k = oracle.pattern(h.n_points, h.nodes)
    k.assemble(0, h.xyz, h.nodes, h.coef)
    a = k.submatrix(h.free)
    rhs = k.reduced_rhs(h.load, h.values, h.free)
    planes, pts, comp = mg.grid_unknowns(h)
    s = oracle.Solver(a, "grid", planes=planes, points=pts, comp=comp, method="multigrid")
    with pytest.raises(oracle.OracleError) as e:
        s.solve(rhs, max_iter=1)
    assert re.fullmatch(r"conjugate gradients did not converge: the residual is "
                        r"[1-9]\.[0-9]{2}e-?[1-9][0-9]* after 1 iterations", str(e.value))

    with pytest.raises(oracle.OracleError, match="^cancelled$"):
        s.solve(rhs, cancel=True)


def test_quadratic_numbers_edges_in_first_seen_order():
    """tet10.rs:244-272: the edge points of the first tetrahedron are the first edges, in
    EDGES order; each edge of the mesh appears once."""
    m = mg.box(3, 2, 2)
    edges, t10 = oracle.quadratic(m.points, m.tets)
    assert t10[0, 4:].tolist() == list(range(m.n, m.n + 6))
    keys = {tuple(e) for e in edges.tolist()}
    assert len(keys) == len(edges)
    # Euler: a Kuhn box has (nx+1)(ny+1)(nz+1) + edges - faces + cells = 1 (V - E + F - C).
    assert all(a < b for a, b in edges.tolist())


def test_colouring_separates_elements_that_share_a_node():
    m = mg.box(6, 5, 4)
    col, nc = oracle.colour(m.n, m.tets)
    assert col.max() + 1 == nc
    for c in range(nc):
        nodes = m.tets[col == c].ravel()
        assert len(np.unique(nodes)) == len(nodes)


def test_orthotropic_with_equal_constants_is_the_isotropic_element():
    """hex.rs:58-64: Orthotropic::isotropic is the orthotropic law with E, nu and
    G = E / (2 (1 + nu)) on every axis: the same 30 x 30 element, bit for bit."""
    p = np.array([[0.0, 0.0, 0.0], [2.0, 0.1, 0.0], [0.3, 1.5, 0.2], [0.1, 0.4, 0.9]])
    e, nu = 70e3, 0.33
    g = e / (2.0 * (1.0 + nu))
    iso = oracle.element_matrix(2, p, np.array([e, nu]))
    ortho = oracle.element_matrix(4, p, np.array([e, e, e, nu, nu, nu, g, g, g]))
    assert np.array_equal(iso, ortho)


def test_pivot_text_is_the_references():
    """cholesky.rs:92-97: the diagonal in Rust's "{:e}" form (shortest digits, bare exponent)."""
    a = oracle.Csr.from_arrays(1, np.array([0, 1]), np.array([0], np.uint32),
                               np.array([-2.5e-3]))
    with pytest.raises(oracle.OracleError) as e:
        oracle.direct_solve(a, np.zeros((1, 3)), np.ones(1))
    assert str(e.value) == ("the matrix is not positive definite: the pivot of column 0 is 0 or "
                            "less to the precision of the arithmetic (its diagonal is -2.5e-3)")
