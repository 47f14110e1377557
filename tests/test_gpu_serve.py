"""The server of solve requests: a request's result is the same alone and in a concurrent mix,
the budget evicts the least recently used idle solver, and errors come back per ticket."""
import numpy as np
import pytest

import femahoy_b200 as fg
from femahoy_b200 import meshgen as mg
from femahoy_b200.serve import Server

pytestmark = pytest.mark.gpu


def _heat(n, seed, precision=fg.MIXED):
    h = mg.heat_cube(n, seed=seed)
    K = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    A = K.submatrix(h.free)
    rhs = fg.reduced_rhs(K, h.load, h.values, h.free)
    planes, pts, comp = mg.grid_unknowns(h)
    u = fg.Unknowns.Grid(fg.Level(planes, pts, comp))
    return A, u, rhs


def _elastic(dims):
    p = mg.cantilever_p1(dims=dims, lengths=tuple(2.5 * d for d in dims))
    K = fg.Csr.assemble(fg.P1_ELASTIC, p.xyz, p.nodes, p.coef)
    A = K.submatrix(p.free)
    rhs = fg.reduced_rhs(K, p.load, p.values, p.free)
    planes, pts, comp = mg.grid_unknowns(p)
    return A, fg.Unknowns.Grid(fg.Level(planes, pts, comp)), rhs


def _solver(A, u):
    return fg.Solver(A, u, fg.Method.Multigrid, precision=fg.MIXED).with_tol(1e-9)


def test_results_are_the_same_alone_and_in_the_mix():
    """Each solver's sums run in a fixed order on its own stream, so a request's solution is bit
    for bit the one it has alone, whatever runs beside it."""
    problems = {1: _heat(20, 1), 2: _heat(28, 2), 3: _heat(12, 3), 4: _elastic((24, 4, 4))}
    alone = {}
    for key, (A, u, rhs) in problems.items():
        x = np.zeros(A.n)
        _solver(A, u).solve(rhs, x)
        alone[key] = x
    server = Server(slots=3, budget_bytes=8 << 30)
    for key, (A, u, _) in problems.items():
        server.put(key, _solver(A, u))
    rng = np.random.default_rng(0)
    order = rng.permutation(np.repeat(list(problems), 4))
    tickets = [(k, server.submit(int(k), problems[k][2])) for k in order]
    for k, t in tickets:
        x, st, latency = server.wait(t)
        assert st.true_residual <= 1e-9
        assert latency > 0
        assert np.array_equal(x.view(np.uint64), alone[k].view(np.uint64))


def test_budget_evicts_the_least_recently_used_idle_solver():
    a = _heat(12, 4)
    s1 = _solver(a[0], a[1])
    need = s1.device_bytes()
    server = Server(slots=2, budget_bytes=int(2.5 * need))
    server.put(10, s1)
    server.put(11, _solver(a[0], a[1]))
    server.wait(server.submit(10, a[2]))  # 10 is now the most recently used
    server.reserve(need)                  # room for a third: 11 goes
    assert server.has(10) and not server.has(11)
    server.put(12, _solver(a[0], a[1]))
    assert server.resident_count == 2
    assert server.resident_bytes <= int(2.5 * need)


def test_a_failed_solve_reports_on_its_ticket():
    A, u, rhs = _heat(12, 5)
    server = Server(slots=1, budget_bytes=4 << 30)
    server.put(7, _solver(A, u).with_max_iter(1))
    with pytest.raises(fg.FemError, match="did not converge"):
        server.wait(server.submit(7, rhs))
    with pytest.raises(fg.FemError):
        server.submit(99, rhs)  # no such key
