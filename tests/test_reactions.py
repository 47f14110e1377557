"""Reactions of a solved elastic model (elastic::reactions, crates/fem/src/elastic.rs:772-839).

The oracle is pinned by the reference's force balance (elastic.rs:20-22: the applied loads plus
the reactions sum to 0 to the precision of the solve) and by a pure-Python restatement of the
loop on a small model; the device is checked bit for bit against the oracle.
"""
import numpy as np
import pytest

import femahoy_b200 as fg
import oracle
from femahoy_b200 import meshgen as mg


def _solved_cantilever():
    """Config 1's cantilever solved by the oracle's multifrontal Cholesky: the full stiffness,
    the full displacement and load, the clamp mask."""
    p = mg.cantilever_p1(dims=(12, 2, 2), lengths=(30.0, 5.0, 5.0))
    Ko = oracle.pattern(p.n_unknowns, oracle.dof_elements(p.nodes))
    Ko.assemble(1, p.xyz, p.nodes, p.coef)
    Ao = Ko.submatrix(p.free)
    rhs = Ko.reduced_rhs(p.load, p.values, p.free)
    x, _ = oracle.direct_solve(Ao, p.xyz[p.free // 3], rhs)
    u = p.values.astype(np.float64).copy()
    u[p.free] = x
    return p, Ko, u


def _python_reactions(K, u, force, fixed, owner, nloads, applied, gross):
    """elastic.rs:786-831 line by line in Python floats."""
    ptr, idx, val = K.arrays()
    ku = []
    for i in range(K.n):
        s = 0.0
        for k in range(ptr[i], ptr[i + 1]):
            s += float(val[k]) * float(u[idx[k]])
        ku.append(s)
    total = [float(a) for a in applied]
    lf = [[0.0, 0.0, 0.0] for _ in range(nloads)]
    for i in range(K.n):
        if fixed[i]:
            r = ku[i] - float(force[i])
            total[i % 3] += r
            gross += abs(r)
            if owner[i] < nloads:
                lf[owner[i]][i % 3] += r
    m = 0.0
    for t in total:
        m = max(m, abs(t))
    return np.array(lf), np.array(total), gross, (m / gross if gross > 0 else 0.0)


def test_oracle_reactions_balance_the_applied_loads():
    """elastic.rs:20-22: the clamp's reaction balances the applied load; the imbalance is at the
    precision of the direct solve."""
    p, Ko, u = _solved_cantilever()
    fixed = p.fixed.astype(np.uint8)
    owner = np.zeros(p.n_unknowns, np.uint32)
    applied = np.array([p.load[c::3].sum() for c in range(3)])
    gross = float(np.abs(p.load).sum())
    lf, total, g, imb = oracle.reactions(Ko, u, p.load, fixed, owner, 1, applied, gross)
    assert imb < 1e-10
    assert np.allclose(lf[0], -applied, rtol=1e-9, atol=1e-9 * g)
    assert np.abs(total).max() <= 1e-10 * g


def test_oracle_reactions_equal_the_python_loop():
    p, Ko, u = _solved_cantilever()
    rng = np.random.default_rng(3)
    fixed = (rng.random(p.n_unknowns) < 0.3).astype(np.uint8)
    owner = rng.integers(0, 4, p.n_unknowns).astype(np.uint32)  # 3 loads, owner 3 is none
    force = rng.standard_normal(p.n_unknowns)
    applied = rng.standard_normal(3)
    got = oracle.reactions(Ko, u, force, fixed, owner, 3, applied, 1.5)
    ref = _python_reactions(Ko, u, force, fixed, owner, 3, applied, 1.5)
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
    assert got[2] == ref[2] and got[3] == ref[3]


@pytest.mark.gpu
def test_device_reactions_are_bit_identical_with_the_oracle():
    p, Ko, u = _solved_cantilever()
    K = fg.Csr.assemble(fg.P1_ELASTIC, p.xyz, p.nodes, p.coef)
    cases = []
    fixed = p.fixed.astype(np.uint8)
    cases.append((u, p.load, fixed, np.zeros(p.n_unknowns, np.uint32), 1,
                  np.array([p.load[c::3].sum() for c in range(3)]), float(np.abs(p.load).sum())))
    rng = np.random.default_rng(11)
    for nloads in (3, 40):
        fx = (rng.random(p.n_unknowns) < 0.4).astype(np.uint8)
        ow = rng.integers(0, nloads + 2, p.n_unknowns).astype(np.uint32)  # some past nloads
        uu = rng.standard_normal(p.n_unknowns)
        ff = rng.standard_normal(p.n_unknowns)
        cases.append((uu, ff, fx, ow, nloads, rng.standard_normal(3), 0.25))
    # No fixed unknown at all, and a NaN displacement.
    cases.append((u, p.load, np.zeros(p.n_unknowns, np.uint8), np.zeros(p.n_unknowns, np.uint32),
                  1, np.ones(3), 2.0))
    un = u.copy()
    un[5] = np.nan
    cases.append((un, p.load, fixed, np.zeros(p.n_unknowns, np.uint32), 1, np.zeros(3), 0.0))
    for uu, ff, fx, ow, nl, ap, g0 in cases:
        got = fg.reactions(K, uu, ff, fx, ow, nl, ap, g0)
        lf, tot, g, imb = oracle.reactions(Ko, uu, ff, fx, ow, nl, ap, g0)
        assert np.array_equal(got.load_force.view(np.uint64), lf.view(np.uint64))
        assert np.array_equal(got.total.view(np.uint64), tot.view(np.uint64))
        assert np.array_equal(np.float64(got.gross).view(np.uint64), np.float64(g).view(np.uint64))
        assert np.array_equal(np.float64(got.imbalance).view(np.uint64),
                              np.float64(imb).view(np.uint64))


@pytest.mark.gpu
def test_device_solve_then_reactions_balance():
    """The device's own solve of the cantilever, then its reactions: the balance holds to the
    solve's tolerance."""
    p = mg.cantilever_p1(dims=(12, 2, 2), lengths=(30.0, 5.0, 5.0))
    K = fg.Csr.assemble(fg.P1_ELASTIC, p.xyz, p.nodes, p.coef)
    A = K.submatrix(p.free)
    rhs = fg.reduced_rhs(K, p.load, p.values, p.free)
    s = fg.Solver(A, fg.Unknowns.Points(p.xyz[p.free // 3]))
    x = np.zeros(A.n)
    s.solve(rhs, x)
    u = p.values.astype(np.float64).copy()
    u[p.free] = x
    applied = np.array([p.load[c::3].sum() for c in range(3)])
    r = fg.reactions(K, u, p.load, p.fixed, np.zeros(p.n_unknowns, np.uint32), 1, applied,
                     float(np.abs(p.load).sum()))
    assert r.imbalance < 1e-10
    assert np.allclose(r.load_force[0], -applied, rtol=1e-9, atol=1e-9 * r.gross)
