"""Parity at the benchmark's own tolerance, 1e-8: the device solution against the oracle's.

The reference solves with PCG and its multigrid V-cycle (multigrid.rs:692-753) and stops when
the recurrence residual |r| / |b| is at most the tolerance. At the same tolerance, two solvers
with different preconditioners reach solutions that differ by about the tolerance. These tests
solve the heat cube at 64^3 (262,144 unknowns: 8 times smaller than the 128^3 benchmark, the
same generator, seed and lognormal conductivity) and the P2 beam at 50 x 5 x 5 cells (config 3's
problem, 36,300 unknowns) to 1e-8, and check the relative L2 difference against:

- the oracle's PCG-MG (the reference's algorithm: line Gauss-Seidel, coarse Cholesky) at the
  same tolerance 1e-8;
- the oracle's converged solution: its multifrontal Cholesky (cholesky.rs:44-167) where that is
  cheap (the beam), else its PCG-MG run on to 1e-12 (the cube, whose sparse factor is too large
  for a test).

Tolerance of the checks: 1e-8 relative L2, the north star's bar for solutions at 1e-8.
"""
import numpy as np
import pytest

import femahoy_b200 as fg
import oracle
from femahoy_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

TOL = 1e-8
BAR = 1e-8


def _rel(x, y):
    return float(np.linalg.norm(x - y) / np.linalg.norm(y))


@pytest.fixture(scope="module")
def heat64():
    h = mg.heat_cube(64, seed=1234)
    K = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    A = K.submatrix(h.free)
    rhs = fg.reduced_rhs(K, h.load, h.values, h.free)
    del K
    Ko = oracle.pattern(h.n_points, h.nodes)
    Ko.assemble(0, h.xyz, h.nodes, h.coef)
    Ao = Ko.submatrix(h.free)
    planes, pts, comp = mg.grid_unknowns(h)
    so = oracle.Solver(Ao, "grid", planes=planes, points=pts, comp=comp, method="multigrid")
    x8, it8, _ = so.solve(rhs, tol=TOL)
    x12, _, res12 = so.solve(rhs, x=x8, tol=1e-12)
    assert res12 <= 1e-12
    unknowns = fg.Unknowns.Grid(fg.Level(planes, pts, comp))
    return A, rhs, unknowns, x8, x12, it8


@pytest.mark.parametrize("precision", [fg.FP64, fg.MIXED])
def test_heat64_at_tol_1e8_matches_oracle(heat64, precision):
    A, rhs, unknowns, x8, x12, _ = heat64
    s = fg.Solver(A, unknowns, fg.Method.Multigrid, precision=precision).with_tol(TOL)
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.residual <= TOL and st.true_residual <= TOL
    assert _rel(x, x12) <= BAR, "against the oracle's converged solution"
    assert _rel(x, x8) <= BAR, "against the oracle's PCG-MG at the same tolerance"


@pytest.fixture(scope="module")
def beam50():
    m = mg.box(50, 5, 5, (250.0, 25.0, 25.0))
    q = fg.Quadratic.new(m.points, m.tets)
    prob = mg.beam_p2(q.edges, q.tets, dims=(50, 5, 5), lengths=(250.0, 25.0, 25.0), mesh=m,
                      seed=1234)
    K = fg.Csr.assemble(fg.P2_ELASTIC, prob.xyz, prob.nodes, prob.coef)
    A = K.submatrix(prob.free)
    rhs = fg.reduced_rhs(K, prob.load, prob.values, prob.free)
    del K
    Ko = oracle.pattern(prob.n_unknowns, oracle.dof_elements(prob.nodes))
    Ko.assemble(2, prob.xyz, prob.nodes, prob.coef)
    Ao = Ko.submatrix(prob.free)
    xyz = prob.xyz[prob.free // 3]
    xd, _ = oracle.direct_solve(Ao, xyz, rhs)
    P, coarse = fg.prolongation(prob.xyz, m.n, q.edges, prob.free)
    Po = oracle.Rect.from_arrays(P.rows, P.cols, P.ptr, P.idx, P.val)
    so = oracle.Solver(Ao, "quadratic", xyz=xyz, p=Po, coarse=coarse, method="multigrid")
    x8, _, _ = so.solve(rhs, tol=TOL)
    unknowns = fg.Unknowns.Quadratic(xyz, P, coarse)
    return A, rhs, unknowns, xd, x8


@pytest.mark.parametrize("precision", [fg.FP64, fg.MIXED])
def test_p2_beam_50x5x5_at_tol_1e8_matches_oracle(beam50, precision):
    A, rhs, unknowns, xd, x8 = beam50
    s = fg.Solver(A, unknowns, fg.Method.Multigrid, precision=precision).with_tol(TOL)
    assert len(s.levels()) >= 2
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.residual <= TOL and st.true_residual <= TOL
    assert _rel(x, xd) <= BAR, "against the oracle's multifrontal Cholesky"
    assert _rel(x, x8) <= BAR, "against the oracle's p-multigrid PCG at the same tolerance"
