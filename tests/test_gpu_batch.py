"""The batched solver: every (system, right side) pair against the oracle's FP64 direct solve
(the reference's multifrontal Cholesky), the reference's PCG stopping rules per pair, and the
batch's own reporting."""
import numpy as np
import pytest

import femahoy_b200 as fg
import oracle
from femahoy_b200 import meshgen as mg
from femahoy_b200.batch import Batch

pytestmark = pytest.mark.gpu


def _member(rng, hi=(30, 4, 4), nrhs=4):
    """A random cantilever of the batched workload: its device matrix, right sides (rows, nrhs)
    and grid unknowns."""
    p, loads = mg.random_cantilever_p1(rng, hi=hi, nrhs=nrhs)
    K = fg.Csr.assemble(fg.P1_ELASTIC, p.xyz, p.nodes, p.coef)
    A = K.submatrix(p.free)
    rhs = np.stack([fg.reduced_rhs(K, loads[r], p.values, p.free) for r in range(nrhs)], axis=1)
    planes, pts, comp = mg.grid_unknowns(p)
    return p, A, rhs, fg.Unknowns.Grid(fg.Level(planes, pts, comp))


def _oracle_matrix(p):
    Ko = oracle.pattern(p.n_unknowns, oracle.dof_elements(p.nodes))
    Ko.assemble(1, p.xyz, p.nodes, p.coef)
    return Ko.submatrix(p.free)


def _direct(p, rhs):
    Ao = _oracle_matrix(p)
    return np.stack([oracle.direct_solve(Ao, p.xyz[p.free // 3], rhs[:, r])[0]
                     for r in range(rhs.shape[1])], axis=1)


def _residuals(p, rhs, x):
    """|b - A x| / |b| of each right side with the oracle's matrix, on the CPU."""
    Ao = _oracle_matrix(p)
    return [np.linalg.norm(rhs[:, r] - Ao.mul(x[:, r])) / np.linalg.norm(rhs[:, r])
            for r in range(rhs.shape[1])]


def _rel(x, y):
    return np.linalg.norm(x - y) / np.linalg.norm(y)


def _batch(members, nrhs, precision=fg.MIXED, coarsest=0):
    return Batch([m[1] for m in members], [m[3] for m in members], nrhs, precision=precision,
                 options=fg.Options(precision=precision, coarsest=coarsest))


@pytest.mark.parametrize("precision", [fg.MIXED, fg.FP64])
def test_every_pair_matches_the_direct_solve(precision):
    """At 1e-10 (these cantilevers have condition numbers up to 2e6, and the FP64 direct
    solution itself leaves |b - A x| / |b| up to 3e-11, so 1e-10 is near the attainable floor):
    each pair's residual recomputed on the CPU with the oracle's matrix, and its distance to
    the direct solution. Deepest levels of at most 256 unknowns, so every member runs a real
    multigrid cycle."""
    rng = np.random.default_rng(11)
    members = [_member(rng) for _ in range(10)]
    b = _batch(members, 4, precision, coarsest=256).with_tol(1e-10)
    assert len(b.levels()) >= 2
    xs, st = b.solve([m[2] for m in members])
    # The stopping test is the reference's, on the recurrence residual (multigrid.rs:721-723);
    # the true residual may sit a rounding drift above it.
    assert st.not_converged == 0
    assert st.max_residual <= 1e-10
    assert st.max_true_residual <= 1.2e-10
    it, truth, res, status = b.segments()
    assert (status == 0).all() and (res <= 1e-10).all() and (it >= 1).all()
    for (p, _, rhs, _), x in zip(members, xs):
        assert max(_residuals(p, rhs, x)) <= 1.2e-10
        xd = _direct(p, rhs)
        for r in range(4):
            assert _rel(x[:, r], xd[:, r]) <= 1e-6


def test_sixteen_right_sides_of_the_batched_workload():
    """Members drawn as in the batched workload (10x1x1 to 80x8x8 cells, 16 load cases) at
    1e-8, every pair's true residual within tolerance, 3 members against the direct solve."""
    rng = np.random.default_rng(5)
    members = [_member(rng, hi=(80, 8, 8), nrhs=16) for _ in range(24)]
    b = _batch(members, 16).with_tol(1e-8)
    xs, st = b.solve([m[2] for m in members])
    assert st.not_converged == 0
    assert st.max_true_residual <= 1e-8
    assert st.max_iterations < 40
    for k in (0, 7, 23):
        p, _, rhs, _ = members[k]
        assert max(_residuals(p, rhs, xs[k])) <= 1.2e-8
        assert _rel(xs[k], _direct(p, rhs)) <= 1e-4


def test_one_right_side_and_a_single_level():
    """nrhs = 1, and systems at or below `coarsest`: the cycle is the dense solve. In FP32 that
    inverse cuts the residual by about cond x 6e-8 per iteration (cond near 1e5 here), so the
    FP64 outer loop takes a few iterations to reach 1e-10."""
    rng = np.random.default_rng(2)
    members = [_member(rng, hi=(12, 2, 2), nrhs=1) for _ in range(5)]
    b = _batch(members, 1, coarsest=4096).with_tol(1e-10)
    assert len(b.levels()) == 1
    xs, st = b.solve([m[2] for m in members])
    assert st.max_iterations <= 6
    for (p, _, rhs, _), x in zip(members, xs):
        assert _rel(x, _direct(p, rhs)) <= 1e-8


def test_a_zero_right_side_gives_zero_without_iterating():
    """multigrid.rs:704-711, per pair."""
    rng = np.random.default_rng(3)
    members = [_member(rng) for _ in range(3)]
    rhs = [m[2].copy() for m in members]
    rhs[1][:, 2] = 0.0
    b = _batch(members, 4, coarsest=256).with_tol(1e-10)
    x0 = b.pack([np.ones_like(r) for r in rhs])
    x, st = b.solve_packed(b.pack(rhs), x0)
    xs = b.unpack(x)
    assert np.array_equal(xs[1][:, 2], np.zeros(len(xs[1])))
    it, truth, _, status = b.segments()
    assert it[1, 2] == 0 and status[1, 2] == 0
    assert st.max_true_residual <= 1.2e-10


def test_the_iteration_limit_names_the_pair():
    rng = np.random.default_rng(4)
    members = [_member(rng) for _ in range(3)]
    b = _batch(members, 4, coarsest=256).with_tol(1e-14).with_max_iter(2)
    with pytest.raises(fg.FemError, match="system 0, right side 0: conjugate gradients did not "
                                          "converge: the residual is .* after 2 iterations"):
        b.solve([m[2] for m in members])
    it, _, _, status = b.segments()
    assert (status == 1).all() and (it == 2).all()


def test_results_do_not_depend_on_the_run():
    """Fixed-order sums: 2 solves of the same batch are bit for bit the same."""
    rng = np.random.default_rng(6)
    members = [_member(rng, hi=(40, 6, 6)) for _ in range(6)]
    b = _batch(members, 4).with_tol(1e-10)
    rhs = [m[2] for m in members]
    x1, _ = b.solve(rhs)
    x2, _ = b.solve(rhs)
    for a, c in zip(x1, x2):
        assert np.array_equal(a.view(np.uint64), c.view(np.uint64))


def test_a_batch_takes_grid_unknowns_only():
    rng = np.random.default_rng(7)
    p, A, rhs, grid = _member(rng)
    with pytest.raises(fg.FemError, match="multigrid needs the box grid"):
        Batch([A], [fg.Unknowns.Points(p.xyz[p.free // 3])], 4)
    with pytest.raises(fg.FemError, match="1, 4 or 16 right sides"):
        Batch([A], [grid], 3)
