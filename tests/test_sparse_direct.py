"""The device's sparse multifrontal Cholesky (the direct method above 4,096 unknowns) against the
oracle's multifrontal factor (cholesky.rs:44-167 in the order of order.rs).

The reference picks its direct solver for P2 models up to DIRECT_UNKNOWNS = 30,000 unknowns
(elastic_tet.rs:52-56) and for flat models up to DIRECT_ENTRIES = 2.5e8 factor entries
(elastic_tet.rs:58-63, elastic.rs:264-275), where its multigrid does not converge. The device
factor solves those systems itself. Its accuracy is the factorization's: the same factor summed
in another order, so the solutions agree to the conditioning of each system (the oracle's own
solve leaves |b - A x| / |b| = 1.2e-10 on the 50 x 5 x 5 P2 beam and 4e-9 on the flat plate
below, and one refinement step moves its solution by 1.7e-11 on the beam). The bounds below
are those floors: the true residual and the distance to the oracle's solution.
"""
import numpy as np
import pytest

import femahoy_b200 as fg
import oracle
from femahoy_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _rel(x, y):
    return float(np.linalg.norm(x - y) / np.linalg.norm(y))


def _p2_system(dims, lengths):
    m = mg.box(*dims, lengths)
    q = fg.Quadratic.new(m.points, m.tets)
    prob = mg.beam_p2(q.edges, q.tets, dims=dims, lengths=lengths, mesh=m, seed=7)
    K = fg.Csr.assemble(fg.P2_ELASTIC, prob.xyz, prob.nodes, prob.coef)
    A = K.submatrix(prob.free)
    rhs = fg.reduced_rhs(K, prob.load, prob.values, prob.free)
    Ko = oracle.pattern(prob.n_unknowns, oracle.dof_elements(prob.nodes))
    Ko.assemble(2, prob.xyz, prob.nodes, prob.coef)
    Ao = Ko.submatrix(prob.free)
    xyz = prob.xyz[prob.free // 3]
    P, coarse = fg.prolongation(prob.xyz, m.n, q.edges, prob.free)
    return A, rhs, Ao, xyz, fg.Unknowns.Quadratic(xyz, P, coarse)


def test_p2_beam_direct_matches_the_oracles_factor():
    """Config 3's problem at 50 x 5 x 5 cells (36,300 unknowns): the direct method."""
    A, rhs, Ao, xyz, u = _p2_system((50, 5, 5), (250.0, 25.0, 25.0))
    s = fg.Solver(A, u, fg.Method.Direct)
    assert s.method() == fg.Method.Direct
    assert "sparse multifrontal factor" in s.describe()
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    xd, _ = oracle.direct_solve(Ao, xyz, rhs)
    assert st.iterations == 0 and st.true_residual <= 1e-10
    assert _rel(x, xd) <= 1e-10


def test_heat_direct_matches_the_oracles_factor():
    h = mg.heat_cube(24)
    K = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    A = K.submatrix(h.free)
    rhs = fg.reduced_rhs(K, h.load, h.values, h.free)
    Ko = oracle.pattern(h.n_points, h.nodes)
    Ko.assemble(0, h.xyz, h.nodes, h.coef)
    planes, pts, comp = mg.grid_unknowns(h)
    s = fg.Solver(A, fg.Unknowns.Grid(fg.Level(planes, pts, comp)), fg.Method.Direct)
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    xd, _ = oracle.direct_solve(Ko.submatrix(h.free), h.xyz[h.free], rhs)
    assert st.true_residual < 1e-13
    assert _rel(x, xd) <= 1e-12
    # The solver is reused across right sides (the factor stays on the device).
    y = np.zeros(A.n)
    s.solve(2.0 * rhs, y)
    assert _rel(y, 2.0 * xd) <= 1e-12


def test_flat_p2_plate_takes_the_sparse_factor():
    """A flat P2 plate (cells 9 wide and 1 high, above the reference's MULTIGRID_ASPECT of 8,
    elastic_tet.rs:58-63): Crossover::Flops {inf, DIRECT_ENTRIES, flat} chooses the direct
    method (elastic_tet.rs:301-307), which the device factors itself (6,300 unknowns)."""
    A, rhs, Ao, xyz, u = _p2_system((10, 10, 2), (90.0, 90.0, 2.0))
    assert A.n > 4096
    s = fg.Solver(A, u, None, fg.Crossover.Flops(float("inf"), 250_000_000, True))
    assert s.method() == fg.Method.Direct
    assert "sparse multifrontal factor" in s.describe()
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    xd, _ = oracle.direct_solve(Ao, xyz, rhs)
    assert st.true_residual <= 1e-8
    assert _rel(x, xd) <= 1e-8


def test_singular_matrix_text_equals_the_oracles():
    """cholesky.rs:92-97 through the sparse factor: a heat matrix with no fixed point is singular
    (its constant vector), and the first pivot that fails is the oracle's."""
    h = mg.heat_cube(18)
    K = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    assert K.n > 4096
    u = fg.Unknowns.Grid(fg.Level(h.mesh.planes, h.mesh.ijk, np.zeros(h.n_points, np.uint8)))
    with pytest.raises(fg.FemError) as e:
        fg.Solver(K, u, fg.Method.Direct)
    Ko = oracle.pattern(h.n_points, h.nodes)
    Ko.assemble(0, h.xyz, h.nodes, h.coef)
    with pytest.raises(oracle.OracleError) as eo:
        oracle.direct_solve(Ko, h.xyz, np.ones(h.n_points))
    assert e.value.code == 3
    assert str(e.value) == str(eo.value)
