"""The device solver against the oracle's FP64 direct solve (the reference's multifrontal
Cholesky) and against the reference's PCG semantics and error texts."""
import ctypes
import re

import numpy as np
import pytest

import femahoy_b200 as fg
import oracle
from femahoy_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _system(prob):
    """The device matrix of the free unknowns, the right side, and the oracle's."""
    kind = {"p1_heat": 0, "p1_elastic": 1, "p2_elastic": 2}[prob.kind]
    K = fg.Csr.assemble(kind, prob.xyz, prob.nodes, prob.coef)
    A = K.submatrix(prob.free)
    rhs = fg.reduced_rhs(K, prob.load, prob.values, prob.free)
    nodes = prob.nodes if kind == 0 else oracle.dof_elements(prob.nodes)
    Ko = oracle.pattern(prob.n_unknowns, nodes)
    Ko.assemble(kind, prob.xyz, prob.nodes, prob.coef)
    Ao = Ko.submatrix(prob.free)
    return A, rhs, Ao


def _grid(prob):
    planes, pts, comp = mg.grid_unknowns(prob)
    return fg.Unknowns.Grid(fg.Level(planes, pts, comp))


def _rel(x, y):
    return np.linalg.norm(x - y) / np.linalg.norm(y)


def test_cantilever_fp64_pcg_multigrid():
    """Config 1: P1 cantilever, 3,000 free unknowns, plain FP64 PCG + MG at 1e-10. The grid is at
    the coarsest size, so the cycle is the coarse solve (multigrid.rs:94)."""
    p = mg.cantilever_p1()
    A, rhs, Ao = _system(p)
    s = fg.Solver(A, _grid(p), fg.Method.Multigrid).with_tol(1e-10)
    assert s.method() == fg.Method.Multigrid
    assert s.levels() == [3000]
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    xd, _ = oracle.direct_solve(Ao, p.xyz[p.free // 3], rhs)
    assert st.residual <= 1e-10
    assert st.true_residual <= 1e-10
    assert _rel(x, xd) <= 1e-8
    assert 1 <= st.iterations <= 5


@pytest.mark.parametrize("precision", [fg.FP64, fg.MIXED])
def test_heat_multigrid_matches_direct(precision):
    """Config 2's problem at 24^3: lognormal conductivity; |x - x_chol| / |x_chol| <= 1e-8."""
    h = mg.heat_cube(24)
    A, rhs, Ao = _system(h)
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=precision).with_tol(1e-10)
    assert len(s.levels()) >= 2
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    xd, _ = oracle.direct_solve(Ao, h.xyz[h.free], rhs)
    assert st.true_residual <= 1e-10
    assert _rel(x, xd) <= 1e-8
    assert st.iterations < 60


def test_heat_oracle_pcg_agrees_at_tolerance():
    """The reference's own PCG-MG (line Gauss-Seidel) and the device solve reach the same
    temperatures at the same tolerance, within 1e-8 relative."""
    h = mg.heat_cube(16)
    A, rhs, Ao = _system(h)
    planes, pts, comp = mg.grid_unknowns(h)
    so = oracle.Solver(Ao, "grid", planes=planes, points=pts, comp=comp, method="multigrid")
    xo, _, _ = so.solve(rhs, tol=1e-10)
    for precision in (fg.FP64, fg.MIXED):
        s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=precision).with_tol(1e-10)
        x = np.zeros(A.n)
        s.solve(rhs, x)
        assert _rel(x, xo) <= 1e-8


def test_p2_p_multigrid_matches_direct():
    """Config 3's problem on a 16 x 4 x 4 beam: p-multigrid P2 -> P1, then geometric levels."""
    m = mg.box(16, 4, 4, (80.0, 20.0, 20.0))
    q = fg.Quadratic.new(m.points, m.tets)
    prob = mg.beam_p2(q.edges, q.tets, mesh=m)
    A, rhs, Ao = _system(prob)
    free = prob.free
    P, coarse = fg.prolongation(prob.xyz, m.n, q.edges, free)
    u = fg.Unknowns.Quadratic(prob.xyz[free // 3], P, coarse)
    for precision in (fg.FP64, fg.MIXED):
        s = fg.Solver(A, u, fg.Method.Multigrid, precision=precision, options=fg.Options(
            precision=precision, coarsest=200)).with_tol(1e-10)
        assert len(s.levels()) >= 3
        x = np.zeros(A.n)
        st = s.solve(rhs, x)
        xd, _ = oracle.direct_solve(Ao, prob.xyz[free // 3], rhs)
        assert st.true_residual <= 1e-10
        assert np.abs(x - xd).max() <= 1e-8 * np.abs(xd).max()


def test_direct_method_matches_oracle():
    h = mg.heat_cube(10)
    A, rhs, Ao = _system(h)
    s = fg.Solver(A, _grid(h))  # Crossover::Unknowns(3000) picks the direct solver
    assert s.method() == fg.Method.Direct
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    xd, _ = oracle.direct_solve(Ao, h.xyz[h.free], rhs)
    assert st.iterations == 0
    assert st.residual < 1e-12
    assert _rel(x, xd) < 1e-12


def test_points_refuse_multigrid():
    h = mg.heat_cube(4)
    A, _, _ = _system(h)
    with pytest.raises(fg.FemError, match="^multigrid needs the box grid"):
        fg.Solver(A, fg.Unknowns.Points(h.xyz[h.free]), fg.Method.Multigrid)


def test_not_converged_and_cancelled_texts():
    """multigrid.rs:729-737 through the device loop (on the reference's coarsest size, 3000, so
    that the cycle is not the exact dense solve)."""
    h = mg.heat_cube(16)
    A, rhs, _ = _system(h)
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid,
                  options=fg.Options(coarsest=3000)).with_max_iter(1)
    assert len(s.levels()) >= 2
    # Rust's "{residual:.2e}": 2 digits after the point, the exponent a bare integer (1.23e-5).
    with pytest.raises(fg.FemError) as e:
        s.solve(rhs, np.zeros(A.n))
    assert re.fullmatch(r"conjugate gradients did not converge: the residual is "
                        r"[1-9]\.[0-9]{2}e-?[1-9][0-9]* after 1 iterations", str(e.value)), str(e.value)
    # From x = 0 the first residual is |b| / |b| = 1: the whole text is known.
    s.with_max_iter(0)
    with pytest.raises(fg.FemError) as e:
        s.solve(rhs, np.zeros(A.n))
    assert str(e.value) == ("conjugate gradients did not converge: the residual is 1.00e0 after "
                            "0 iterations")
    s.with_max_iter(500)
    flag = ctypes.c_int(1)
    with pytest.raises(fg.FemError) as e:
        s.solve(rhs, np.zeros(A.n), cancelled=flag)
    assert str(e.value) == "cancelled" and e.value.code == 1


def test_zero_right_side_gives_zero():
    """multigrid.rs:704-711: |b| = 0 gives x = 0 and 0 iterations."""
    h = mg.heat_cube(8)
    A, _, _ = _system(h)
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid)
    x = np.ones(A.n)
    st = s.solve(np.zeros(A.n), x)
    assert st.iterations == 0 and not x.any()


def test_singular_matrix_is_not_positive_definite():
    """cholesky.rs:281-293 on the direct path of the device."""
    h = mg.heat_cube(4)
    K = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)  # no fixed points: singular
    planes = h.mesh.planes
    u = fg.Unknowns.Grid(fg.Level(planes, h.mesh.ijk, np.zeros(h.n_points, np.uint8)))
    with pytest.raises(fg.FemError, match="not positive definite"):
        fg.Solver(K, u, fg.Method.Direct)


def test_pivot_text_is_the_references():
    """cholesky.rs:92-97 writes the diagonal with Rust's "{:e}": the shortest digits that read
    back, the exponent a bare integer."""
    A = fg.Csr.from_arrays(1, np.array([0, 1]), np.array([0], np.uint32), np.array([-2.5e-3]))
    with pytest.raises(fg.FemError) as e:
        fg.Solver(A, fg.Unknowns.Points(np.zeros((1, 3))), fg.Method.Direct)
    assert str(e.value) == ("the matrix is not positive definite: the pivot of column 0 is 0 or "
                            "less to the precision of the arithmetic (its diagonal is -2.5e-3)")


def test_solver_reuse_across_right_sides():
    """A solver solves many right sides (solve.rs:1-5); the start value is honoured."""
    h = mg.heat_cube(16)
    A, rhs, Ao = _system(h)
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=fg.MIXED).with_tol(1e-10)
    xs = []
    for k in range(3):
        x = np.zeros(A.n)
        s.solve(rhs * (k + 1), x)
        xs.append(x)
    assert _rel(xs[1], 2 * xs[0]) < 1e-9 and _rel(xs[2], 3 * xs[0]) < 1e-9
    x = xs[0].copy()
    st = s.solve(rhs, x)
    assert st.iterations == 0


def test_cancel_during_the_device_loop():
    """A flag raised by another host thread while the device runs the PCG loop ends the solve
    with "cancelled" before the iteration limit (multigrid.rs:735, polled each iteration)."""
    import threading
    import time

    h = mg.heat_cube(48)
    A, rhs, _ = _system(h)
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid)
    s.solve(rhs, np.zeros(A.n))  # builds the loop graph
    s.with_tol(1e-300).with_max_iter(100000)
    flag = ctypes.c_int(0)
    timer = threading.Timer(0.05, lambda: setattr(flag, "value", 1))
    timer.start()
    t0 = time.perf_counter()
    with pytest.raises(fg.FemError) as e:
        s.solve(rhs, np.zeros(A.n), cancelled=flag)
    timer.cancel()
    assert str(e.value) == "cancelled"
    assert time.perf_counter() - t0 < 30.0


def test_nan_right_side_breaks_down_with_an_error():
    """A NaN in the right side stops the device loop at once instead of running to max_iter."""
    h = mg.heat_cube(8)
    A, rhs, _ = _system(h)
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid)
    bad = rhs.copy()
    bad[3] = np.nan
    with pytest.raises(fg.FemError):
        s.solve(bad, np.zeros(A.n))


@pytest.mark.parametrize("kind", ["heat", "elastic"])
@pytest.mark.parametrize("precision", [fg.FP64, fg.MIXED])
def test_fused_coarse_levels_give_the_same_bits(kind, precision):
    """The small levels run as 1 cooperative kernel (the same row functions as the separate
    kernels): the solution is bit for bit the one of the separate launches, for stencil levels
    (heat) and SELL levels (elasticity)."""
    if kind == "heat":
        p = mg.heat_cube(40, seed=7)
    else:
        p = mg.cantilever_p1(dims=(48, 8, 8), lengths=(120.0, 20.0, 20.0))
    A, rhs, _ = _system(p)
    xs, its = [], []
    # Elasticity in scalar SELL form (the fused kernel reads stencils and SELL; 3x3-block levels
    # keep separate launches).
    fmt = 0 if kind == "heat" else 1
    for tail in (65536, 0):
        s = fg.Solver(A, _grid(p), fg.Method.Multigrid, precision=precision,
                      options=fg.Options(precision=precision, tail=tail, coarsest=200,
                                         format=fmt, degree=2))
        s = s.with_tol(1e-10)
        assert ("cooperative kernel" in s.describe()) == (tail > 0)
        x = np.zeros(A.n)
        st = s.solve(rhs, x)
        assert st.true_residual <= 1e-10
        xs.append(x)
        its.append(st.iterations)
    assert its[0] == its[1]
    assert np.array_equal(xs[0].view(np.uint64), xs[1].view(np.uint64))


@pytest.mark.parametrize("precision", [fg.FP64, fg.MIXED])
def test_programmatic_launches_give_the_same_bits(precision):
    """Each kernel of the loop waits on the device for the one before it, so the launches that
    may start early compute what the plain stream-ordered launches compute, bit for bit."""
    h = mg.heat_cube(32, seed=3)
    A, rhs, _ = _system(h)
    xs = []
    for launch in (0, 1):
        s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=precision,
                      options=fg.Options(precision=precision, launch=launch)).with_tol(1e-10)
        x = np.zeros(A.n)
        st = s.solve(rhs, x)
        assert st.true_residual <= 1e-10
        xs.append(x)
    assert np.array_equal(xs[0].view(np.uint64), xs[1].view(np.uint64))


@pytest.mark.parametrize("precision", [fg.MIXED])
def test_tile_kernels_give_the_same_bits(precision):
    """The finest FP32 stencil steps and residuals with each tile's own arrays brought into
    shared memory by bulk copies compute what the direct kernels compute, bit for bit (a level of
    180,000 rows: enough tiles to fill the GPU)."""
    h = mg.heat_cube(56, seed=5)
    A, rhs, _ = _system(h)
    xs, its = [], []
    for tiles in (1, 2):
        s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=precision,
                      options=fg.Options(precision=precision, tiles=tiles)).with_tol(1e-10)
        assert ("bulk-copied tiles" in s.describe()) == (tiles == 2)
        x = np.zeros(A.n)
        st = s.solve(rhs, x)
        assert st.true_residual <= 1e-10
        xs.append(x)
        its.append(st.iterations)
    assert its[0] == its[1]
    assert np.array_equal(xs[0].view(np.uint64), xs[1].view(np.uint64))


@pytest.mark.parametrize("precision", [fg.MIXED, fg.FP64])
def test_stencil_kernels_give_the_same_bits(precision):
    """Every stencil product kernel (K at run time, K at compile time, 2 rows per thread,
    marching planes with all gathers from shared memory) sums each row in the same order, so the
    solves are the same bits whichever the autotuner picks (the 56^3 cube: levels of 180,000,
    24,000 and 3,400 rows, K = 8 and 14)."""
    h = mg.heat_cube(56, seed=5)
    A, rhs, _ = _system(h)
    xs, its = [], []
    for kernel, text in ((1, "loop"), (2, "unrolled"), (3, "2 rows per thread"),
                         (4, "marching planes")):
        s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=precision,
                      options=fg.Options(precision=precision, stencil=kernel, tiles=1,
                                         degree=2)).with_tol(1e-10)
        assert text in s.describe()
        x = np.zeros(A.n)
        st = s.solve(rhs, x)
        assert st.true_residual <= 1e-10
        xs.append(x)
        its.append(st.iterations)
    assert len(set(its)) == 1
    for x in xs[1:]:
        assert np.array_equal(xs[0].view(np.uint64), x.view(np.uint64))


def test_fp16_stencil_coefficients_solve_to_the_same_tolerance():
    """The mixed form with the stencil levels' coefficients in FP16 (scaled by each level's
    largest): the V-cycle changes by about 2^-11 relative, and flexible CG still reaches the
    tolerance on the true FP64 residual in at most 1 more iteration. The FP64 form ignores the
    option."""
    h = mg.heat_cube(32, seed=3)
    A, rhs, _ = _system(h)
    its = {}
    for values in (1, 2):
        s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=fg.MIXED,
                      options=fg.Options(precision=fg.MIXED, values=values)).with_tol(1e-10)
        assert ("fp16" in s.describe()) == (values == 2)
        x = np.zeros(A.n)
        st = s.solve(rhs, x)
        assert st.true_residual <= 1.2e-10
        its[values] = st.iterations
    assert its[2] <= its[1] + 1
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=fg.FP64,
                  options=fg.Options(precision=fg.FP64, values=2))
    assert "fp16" not in s.describe()


@pytest.mark.parametrize("precision", [fg.FP64, fg.MIXED])
def test_fourth_kind_chebyshev_smoother(precision):
    """The fourth-kind Chebyshev smoother (Lottes 2023; the same kernels, other coefficients)
    solves the lognormal heat cube to the tolerance, to the oracle's direct solution."""
    h = mg.heat_cube(24, seed=11)
    A, rhs, Ao = _system(h)
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=precision,
                  options=fg.Options(precision=precision, smoother=4, coarsest=1000,
                                     degree=2)).with_tol(1e-10)
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.true_residual <= 1.2e-10
    xd, _ = oracle.direct_solve(Ao, h.xyz[h.free], rhs)
    assert _rel(x, xd) <= 1e-8


@pytest.mark.parametrize("precision", [fg.MIXED, fg.FP64])
def test_cluster_legs_give_the_same_bits(precision):
    """The small levels' legs as thread-block cluster launches (cluster barriers between the
    steps, coherent loads of what the launch wrote) compute what the separate launches compute,
    bit for bit (the 56^3 cube: levels of 24,000 and 3,400 rows take the cluster legs)."""
    h = mg.heat_cube(56, seed=5)
    A, rhs, _ = _system(h)
    xs, its = [], []
    for cluster in (0, 1):
        s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=precision,
                      options=fg.Options(precision=precision, cluster=cluster,
                                         degree=2)).with_tol(1e-10)
        assert ("legs as clusters" in s.describe()) == (cluster == 1)
        x = np.zeros(A.n)
        st = s.solve(rhs, x)
        assert st.true_residual <= 1.2e-10
        xs.append(x)
        its.append(st.iterations)
    assert its[0] == its[1]
    assert np.array_equal(xs[0].view(np.uint64), xs[1].view(np.uint64))


def test_fp16_coarsest_inverse_solves_to_the_same_tolerance():
    """The mixed form with the coarsest level's dense inverse in FP16 (scaled by its largest
    entry; the product sums in FP32): the coarse correction changes by about 2^-11 relative, and
    flexible CG still reaches the tolerance on the true FP64 residual in at most 1 more
    iteration, near the oracle's direct solution. The FP64 form ignores the option."""
    h = mg.heat_cube(40, seed=7)
    A, rhs, Ao = _system(h)
    its, xs = {}, {}
    for values in (1, 3):
        s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=fg.MIXED,
                      options=fg.Options(precision=fg.MIXED, values=values,
                                         coarsest=3000)).with_tol(1e-10)
        x = np.zeros(A.n)
        st = s.solve(rhs, x)
        assert st.true_residual <= 1.2e-10
        its[values] = st.iterations
        xs[values] = x
    assert its[3] <= its[1] + 1
    assert _rel(xs[3], xs[1]) <= 1e-8
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=fg.FP64,
                  options=fg.Options(precision=fg.FP64, values=3)).with_tol(1e-10)
    x = np.zeros(A.n)
    assert s.solve(rhs, x).true_residual <= 1.2e-10


@pytest.mark.parametrize("precision", [fg.FP64, fg.MIXED])
def test_block_operators_match_sell_for_elasticity(precision):
    """Elasticity levels in 3x3-block form (each node's 3 rows share their block columns) solve
    to the same solution as in scalar SELL form, both against the direct oracle."""
    p = mg.cantilever_p1(dims=(48, 8, 8), lengths=(120.0, 20.0, 20.0))
    A, rhs, Ao = _system(p)
    xd, _ = oracle.direct_solve(Ao, p.xyz[p.free // 3], rhs)
    for fmt in (0, 1):
        s = fg.Solver(A, _grid(p), fg.Method.Multigrid, precision=precision,
                      options=fg.Options(precision=precision, coarsest=200, format=fmt))
        s = s.with_tol(1e-10)
        assert ("3x3-block" in s.describe()) == (fmt == 0)
        x = np.zeros(A.n)
        st = s.solve(rhs, x)
        assert st.true_residual <= 1.2e-10
        assert _rel(x, xd) <= 1e-6


@pytest.mark.parametrize("precision", [fg.FP64, fg.MIXED])
def test_solve_from_zero_equals_solve_with_a_zero_start(precision):
    """femgpu_solver_solve_zero (x written only) gives the bits of femgpu_solver_solve from a
    zero start value, whatever the output array held before."""
    h = mg.heat_cube(20, seed=7)
    A, rhs, _ = _system(h)
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=precision).with_tol(1e-10)
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    y = np.full(A.n, np.nan)
    sz = s.solve_zero(rhs, y)
    assert np.array_equal(x.view(np.uint64), y.view(np.uint64))
    assert (st.iterations, st.residual) == (sz.iterations, sz.residual)


def _symbolic_cases():
    h = mg.heat_cube(10, seed=4)
    c = mg.hex_cantilever(nx=24, ny=3, nz=4, grade=1.2, seed=1)
    return [("heat", h, 0), ("box cells", c, 6)]


@pytest.mark.parametrize("case", [0, 1])
def test_symbolic_counts_equal_the_oracle(case):
    """order.rs + symbolic.rs restated in the library: the factor's entries and flops in the
    nested dissection order equal the oracle's (flops bit for bit)."""
    name, prob, kind = _symbolic_cases()[case]
    K = fg.Csr.assemble(kind, prob.xyz, prob.nodes, prob.coef)
    A = K.submatrix(prob.free)
    e, f = fg.symbolic_counts(A, _grid(prob))
    nodes = prob.nodes if kind == 0 else oracle.dof_elements(prob.nodes)
    Ko = oracle.pattern(prob.n_unknowns, nodes)
    Ko.assemble(kind, prob.xyz, prob.nodes, prob.coef)
    planes, pts, comp = mg.grid_unknowns(prob)
    xyz = np.stack([planes[d][pts[:, d]] for d in range(3)], axis=1)
    eo, fo = oracle.symbolic_counts(Ko.submatrix(prob.free), xyz)
    assert e == eo and np.float64(f).view(np.uint64) == np.float64(fo).view(np.uint64), (name, e, eo)


def test_flops_crossover_chooses_as_the_reference():
    """solve.rs:160-172 with the box-grid elastic rule Flops{1.5e5, 2.5e8, flat} (elastic.rs:537):
    the library's method equals the oracle's for a small beam (direct, 1,480 flops per unknown),
    a thick one (multigrid, 1.8e5) and the same thick one called flat (direct)."""
    cases = [(mg.hex_cantilever(nx=6, ny=2, nz=2), False),
             (mg.hex_cantilever(nx=16, ny=14, nz=14), False),
             (mg.hex_cantilever(nx=16, ny=14, nz=14), True)]
    seen = set()
    for c, flat in cases:
        K = fg.Csr.assemble(fg.HEX8_ELASTIC, c.xyz, c.nodes, c.coef)
        A = K.submatrix(c.free)
        s = fg.Solver(A, _grid(c), None, fg.Crossover.Flops(1.5e5, 250_000_000, flat))
        Ko = oracle.pattern(3 * c.n_points, oracle.dof_elements(c.nodes))
        Ko.assemble(6, c.xyz, c.nodes, c.coef)
        planes, pts, comp = mg.grid_unknowns(c)
        so = oracle.Solver(Ko.submatrix(c.free), "grid", planes=planes, points=pts, comp=comp,
                           crossover=("flops", 1.5e5, 250_000_000, flat))
        assert s.method().name.lower() == so.method(), (A.n, flat)
        seen.add(so.method())
    assert seen == {"direct", "multigrid"}


@pytest.mark.parametrize("precision", [fg.FP64, fg.MIXED])
def test_extruded_mesh_with_z_coarsening(precision):
    """A footprint mesh extruded in layers (the shape of the reference's prism meshes): its points
    lie on z planes but not on x or y planes. With only z coarsened (axes = 4) the V-cycle halves
    the layers down to the dense coarse solve; the PCG solution equals the oracle's direct one."""
    xyz, tets = mg.extruded(npoints=300, layers=8, seed=3)
    n = len(xyz)
    coef = np.tile([1000.0, 0.3], (len(tets), 1))
    fixed = np.repeat(xyz[:, 2] == 0.0, 3)
    free = np.nonzero(~fixed)[0].astype(np.int64)
    load = np.zeros(3 * n)
    load[3 * np.nonzero(xyz[:, 2] == 1.0)[0] + 0] = 1e-3
    K = fg.Csr.assemble(fg.P1_ELASTIC, xyz, tets, coef)
    A = K.submatrix(free)
    rhs = fg.reduced_rhs(K, load, np.zeros(3 * n), free)
    planes, pts, comp = mg.level_of(xyz, free)
    s = fg.Solver(A, fg.Unknowns.Grid(fg.Level(planes, pts, comp)), fg.Method.Multigrid,
                  precision=precision,
                  options=fg.Options(precision=precision, axes=4, coarsest=2000)).with_tol(1e-10)
    assert len(s.levels()) >= 2 and s.levels()[-1] < s.levels()[0]
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.true_residual <= 1.2e-10
    Ko = oracle.pattern(3 * n, oracle.dof_elements(tets))
    Ko.assemble(1, xyz, tets, coef)
    xd, _ = oracle.direct_solve(Ko.submatrix(free), xyz[free // 3],
                                Ko.reduced_rhs(load, np.zeros(3 * n), free))
    assert _rel(x, xd) <= 1e-8


@pytest.mark.parametrize("precision", [fg.FP64, fg.MIXED])
def test_extruded_mesh_with_a_sparse_coarsest_level(precision):
    """A footprint too large for the dense coarse solve: the z-only coarsening stops at 2 planes
    of 3,025 points (18,150 unknowns, above the dense inverse's 16,384), and that level takes the
    sparse multifrontal factor, as the reference's coarsest level always does
    (multigrid.rs:124-131). The PCG solution equals the oracle's direct one."""
    xyz, tets = mg.extruded(npoints=3025, layers=4, seed=7)
    n = len(xyz)
    coef = np.tile([1000.0, 0.3], (len(tets), 1))
    fixed = np.repeat(xyz[:, 2] == 0.0, 3)
    free = np.nonzero(~fixed)[0].astype(np.int64)
    load = np.zeros(3 * n)
    load[3 * np.nonzero(xyz[:, 2] == 1.0)[0] + 2] = -1e-3
    K = fg.Csr.assemble(fg.P1_ELASTIC, xyz, tets, coef)
    A = K.submatrix(free)
    rhs = fg.reduced_rhs(K, load, np.zeros(3 * n), free)
    planes, pts, comp = mg.level_of(xyz, free)
    s = fg.Solver(A, fg.Unknowns.Grid(fg.Level(planes, pts, comp)), fg.Method.Multigrid,
                  precision=precision,
                  options=fg.Options(precision=precision, axes=4, coarsest=2000)).with_tol(1e-10)
    assert s.levels()[-1] == 18150 and "sparse multifrontal factor" in s.describe()
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.true_residual <= 1.2e-10
    Ko = oracle.pattern(3 * n, oracle.dof_elements(tets))
    Ko.assemble(1, xyz, tets, coef)
    xd, _ = oracle.direct_solve(Ko.submatrix(free), xyz[free // 3],
                                Ko.reduced_rhs(load, np.zeros(3 * n), free))
    assert _rel(x, xd) <= 1e-8


def test_extruded_p2_mesh_with_z_coarsening():
    """P2 elasticity on the extruded footprint (the reference's prism meshes carry P2 tets,
    elastic_tet.rs): p-multigrid to the P1 corners, then z-only geometric levels; the solution
    equals the oracle's direct one."""
    xyz, tets = mg.extruded(npoints=100, layers=6, seed=5)
    q = fg.Quadratic.new(xyz, tets)
    n = len(q.points)
    coef = np.tile([1000.0, 0.3], (len(q.tets), 1))
    fixed = np.repeat(q.points[:, 2] == 0.0, 3)
    free = np.nonzero(~fixed)[0].astype(np.int64)
    load = np.zeros(3 * n)
    load[3 * np.nonzero(q.points[:, 2] == 1.0)[0] + 1] = 1e-3
    K = fg.Csr.assemble(fg.P2_ELASTIC, q.points, q.tets, coef)
    A = K.submatrix(free)
    rhs = fg.reduced_rhs(K, load, np.zeros(3 * n), free)
    P, coarse = fg.prolongation(q.points, len(xyz), q.edges, free)
    u = fg.Unknowns.Quadratic(q.points[free // 3], P, coarse)
    s = fg.Solver(A, u, fg.Method.Multigrid,
                  options=fg.Options(axes=4, coarsest=1000)).with_tol(1e-10)
    assert len(s.levels()) >= 3
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.true_residual <= 1.2e-10
    Ko = oracle.pattern(3 * n, oracle.dof_elements(q.tets))
    Ko.assemble(2, q.points, q.tets, coef)
    xd, _ = oracle.direct_solve(Ko.submatrix(free), q.points[free // 3],
                                Ko.reduced_rhs(load, np.zeros(3 * n), free))
    assert _rel(x, xd) <= 1e-8


def test_bounded_wait_runs_out_and_the_solver_stays_usable():
    """The stencil tile kernels wait on mbarriers for their bulk copies, each wait bounded. With
    a limit of 0 polls every such wait runs out at once: the solve must end with
    FEMGPU_ERR_TIMEOUT and its text instead of hanging, and the same handle must solve normally
    once the default limit is back."""
    h = mg.heat_cube(64)
    A, rhs, _ = _system(h)
    s = fg.Solver(A, _grid(h), fg.Method.Multigrid, precision=fg.MIXED,
                  options=fg.Options(precision=fg.MIXED, tiles=2)).with_tol(1e-8)
    assert "bulk" in s.describe(), s.describe()
    x = np.zeros(A.n)
    s.solve(rhs, x)
    lib = fg.lib()
    assert lib.femgpu_solver_set_wait_limit(s.handle, 0) == 0
    with pytest.raises(fg.FemError) as e:
        s.solve(rhs, np.zeros(A.n))
    assert e.value.code == 10
    assert str(e.value) == ("a bulk copy of a stencil tile did not complete within its wait "
                            "limit")
    assert lib.femgpu_solver_set_wait_limit(s.handle, 4194304) == 0
    y = np.zeros(A.n)
    st = s.solve(rhs, y)
    assert st.true_residual <= 1e-8
    assert np.array_equal(x, y)


@pytest.mark.parametrize("level", [1, 2])
def test_heat_coarse_levels_against_the_oracle(level):
    """The device's plane coarsening with the operator weights of a scalar (multigrid.rs:386-401)
    and its Galerkin products P^T A P, on the lognormal heat cube: the coarse unknowns are the
    oracle's (renumbered in grid order) and the coarse matrices agree to rounding."""
    from test_hex_elastic import _to_grid_order
    h = mg.heat_cube(40)
    A, _, Ao = _system(h)
    planes, pts, comp = mg.grid_unknowns(h)
    ptr, idx, val, gp, gc = fg.coarse_matrix(A, _grid(h), level)
    so = oracle.Solver(Ao, "grid", planes=planes, points=pts, comp=comp, method="multigrid",
                       crossover=("unknowns", 0))
    want, wp, wc = _to_grid_order(so, planes, pts, comp, level)
    assert np.array_equal(gp, wp) and np.array_equal(gc, wc)
    assert np.array_equal(ptr, want.indptr) and np.array_equal(idx, want.indices)
    rows = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
    scale = np.maximum.reduceat(np.abs(want.data), ptr[:-1])[rows]
    assert np.all(np.abs(val - want.data) <= 1e-12 * scale)
