"""Transient heat (heat.rs:686-733): backward Euler with the lumped capacity.

CPU: the oracle's loop against the reference's own transient test (tests/heat.rs:244-264: a
transient ends at the steady state with its energy balance, and heats up in its first steps).
GPU: the device loop against the oracle's, frame by frame, with the direct solver (1e-12) and
with multigrid (1e-8), in FP64 and in the mixed form."""
import ctypes

import numpy as np
import pytest

import oracle
from femahoy_b200 import meshgen as mg


def problem(n, seed=2):
    h = mg.heat_cube(n, seed=seed)
    k = oracle.pattern(h.n_points, h.nodes)
    k.assemble(0, h.xyz, h.nodes, h.coef)
    cap = mg.lumped_capacity(h.mesh, capacity=4.0)
    return h, k, cap


def oracle_solver(h, method):
    planes, pts, comp = mg.grid_unknowns(h)
    return lambda a: oracle.Solver(a, "grid", planes=planes, points=pts, comp=comp,
                                   method=method)


def imbalance(e, load):
    """stored - sum(load) - fixed: the free rows' residual summed (K has zero column sums)."""
    return abs(e[0] - load.sum() - e[1]) / e[2]


def test_oracle_transient_ends_at_the_steady_state_with_its_energy_balance():
    h, k, cap = problem(6)
    free = h.free
    frames, energies, _ = oracle.transient(k, cap, 0.05, free, h.load, h.values, 200,
                                           oracle_solver(h, "direct"), output_every=20)
    assert len(frames) == 10
    # The steady state: the reduced system of K alone.
    a = k.submatrix(free)
    xs, _ = oracle.direct_solve(a, h.xyz[free], k.reduced_rhs(h.load, h.values, free))
    assert np.abs(frames[-1][free] - xs).max() < 1e-6 * np.abs(xs).max()
    for e in energies:
        assert imbalance(e, h.load) < 1e-9
    # In the first steps the body stores heat.
    first, _, _ = oracle.transient(k, cap, 0.05, free, h.load, h.values, 1,
                                   oracle_solver(h, "direct"))
    assert first[0][free].max() > 0
    _, e1, _ = oracle.transient(k, cap, 0.05, free, h.load, h.values, 1,
                                oracle_solver(h, "direct"))
    assert e1[0][0] > 0


def test_oracle_transient_right_side_matches_its_definition():
    """heat.rs:1219-1244 with the capacity term, restated in numpy."""
    h, k, cap = problem(4)
    free = h.free
    rng = np.random.default_rng(1)
    t = rng.standard_normal(h.n_points)
    dt = 0.3
    ptr, idx, val = k.arrays()
    kf = oracle.Csr.from_arrays(k.n, ptr, idx, val)
    kf.add_capacity(cap, dt)
    got = kf.reduced_rhs_transient(h.load, t, free, cap, dt)
    fptr, fidx, fval = kf.arrays()
    isfree = np.zeros(h.n_points, bool)
    isfree[free] = True
    for q, i in enumerate(free):
        r = h.load[i] + cap[i] / dt * t[i]
        for e in range(fptr[i], fptr[i + 1]):
            if not isfree[fidx[e]]:
                r -= fval[e] * t[fidx[e]]
        assert got[q] == r


# ------------------------------------------------------------------ the device loop


def gpu_run(h, cap, dt, steps, every, method, precision, kind=None):
    import femahoy_b200 as fg
    from femahoy_b200.transient import Transient
    K = fg.Csr.assemble(fg.P1_HEAT if kind is None else kind, h.xyz, h.nodes, h.coef)
    planes, pts, comp = mg.grid_unknowns(h)
    u = fg.Unknowns.Grid(fg.Level(planes, pts, comp))
    m = fg.Method.Direct if method == "direct" else fg.Method.Multigrid
    # coarsest 1000: a real V-cycle below the 4,335 free points of the 16^3 cube.
    tr = Transient(K, cap, dt, h.free, u, m,
                   options=fg.Options(precision=precision, coarsest=1000))
    return tr, tr.run(steps, h.load, h.values, output_every=every)


@pytest.mark.gpu
@pytest.mark.parametrize("method,precision,tol", [("direct", 0, 1e-12), ("multigrid", 0, 1e-8),
                                                  ("multigrid", 1, 1e-8)])
def test_gpu_transient_matches_the_oracle(method, precision, tol):
    h, k, cap = problem(16)
    dt, steps, every = 0.02, 12, 4
    _, (frames, energies, t, st) = gpu_run(h, cap, dt, steps, every, method, precision)
    of, oe, _ = oracle.transient(k, cap, dt, h.free, h.load, h.values, steps,
                                 oracle_solver(h, method), output_every=every)
    assert len(frames) == len(of) == 3
    for g, o in zip(frames, of):
        assert np.abs(g - o).max() <= tol * np.abs(o).max()
    for g, o in zip(energies, oe):
        assert abs(g.stored - o[0]) <= tol * o[2] and abs(g.fixed - o[1]) <= tol * o[2]
        assert abs(g.gross - o[2]) <= tol * o[2]
        assert imbalance((g.stored, g.fixed, g.gross), h.load) < 1e-8
    assert np.array_equal(t, frames[-1])
    assert st.iterations >= (steps if method == "multigrid" else 0)


@pytest.mark.gpu
def test_gpu_transient_reaches_the_steady_state():
    import femahoy_b200 as fg
    h, k, cap = problem(12)
    tr, (frames, energies, t, st) = gpu_run(h, cap, 0.5, 60, 30, "multigrid", 1)
    free = h.free
    xs, _ = oracle.direct_solve(k.submatrix(free), h.xyz[free],
                                k.reduced_rhs(h.load, h.values, free))
    assert np.abs(t[free] - xs).max() < 1e-6 * np.abs(xs).max()
    assert "multigrid" in tr.solver.describe() or tr.solver.method() == fg.Method.Multigrid


@pytest.mark.gpu
def test_gpu_transient_cancelled():
    import femahoy_b200 as fg
    from femahoy_b200.transient import Transient
    h, _, cap = problem(8)
    K = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    planes, pts, comp = mg.grid_unknowns(h)
    tr = Transient(K, cap, 0.1, h.free, fg.Unknowns.Grid(fg.Level(planes, pts, comp)))
    with pytest.raises(fg.FemError) as e:
        tr.run(5, h.load, h.values, cancelled=ctypes.c_int(1))
    assert str(e.value) == "cancelled" and e.value.code == 1
    with pytest.raises(fg.FemError) as e:
        Transient(K, cap, 0.0, h.free, fg.Unknowns.Grid(fg.Level(planes, pts, comp)))
    assert "time step" in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_transient_on_box_cells_matches_the_oracle(precision):
    """The box grid's transient heat (heat.rs:413-423 with 8 corners per cell, 686-733): the
    device loop on hex8 conduction cells against the oracle's, multigrid, to 1e-8."""
    import femahoy_b200 as fg
    h = mg.heat_cube_hex(14, seed=3)
    k = oracle.pattern(h.n_points, h.nodes)
    k.assemble(5, h.xyz, h.nodes, h.coef)
    cap = mg.lumped_capacity(h.mesh, capacity=3.0, cells=h.nodes)
    dt, steps, every = 0.02, 8, 4
    _, (frames, energies, _, _) = gpu_run(h, cap, dt, steps, every, "multigrid", precision,
                                          kind=fg.HEX8_HEAT)
    of, oe, _ = oracle.transient(k, cap, dt, h.free, h.load, h.values, steps,
                                 oracle_solver(h, "multigrid"), output_every=every)
    for g, o in zip(frames, of):
        assert np.abs(g - o).max() <= 1e-8 * np.abs(o).max()
    for g, o in zip(energies, oe):
        assert abs(g.stored - o[0]) <= 1e-8 * o[2]
