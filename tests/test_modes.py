"""Modes: shift-invert subspace iteration with Rayleigh-Ritz (eigen.rs:81-177, modes.rs:
180-216) and the P2 consistent mass (tet10.rs:173-212).

CPU: the oracle against the reference's own unit tests of eigen.rs (the Jacobi method on the
second difference matrix, M-orthonormal vectors of the generalized problem, the modes of a free
chain) and the mass against its exact integrals (tet10.rs:302-338)."""
import numpy as np
import pytest

import oracle


def second_difference(n):
    a = np.zeros((n, n))
    for i in range(n):
        a[i, i] = 2.0
        if i + 1 < n:
            a[i, i + 1] = a[i + 1, i] = -1.0
    return a


def test_oracle_jacobi_finds_the_eigenvalues_of_the_second_difference():
    """eigen.rs:339-363"""
    n = 7
    a = second_difference(n)
    values, v = oracle.dense_jacobi(a)
    for k in range(n):
        exact = 2.0 - 2.0 * np.cos((k + 1) * np.pi / (n + 1))
        assert abs(values[k] - exact) < 1e-13
        assert np.abs(a @ v[:, k] - values[k] * v[:, k]).max() < 1e-12


def generalized_case(n=5):
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    k = 1.0 / (1.0 + i + j) + 3.0 * (i == j)
    m = np.where(i == j, 1e4 ** (i % 2), 0.1)
    return k, m


def test_oracle_generalized_gives_m_orthonormal_vectors():
    """eigen.rs:365-402"""
    k, m = generalized_case()
    values, q = oracle.dense_generalized(k, m)
    assert np.abs(q.T @ m @ q - np.eye(5)).max() < 1e-10
    for a in range(5):
        kq, mq = k @ q[:, a], m @ q[:, a]
        assert np.all(np.abs(kq - values[a] * mq) < 1e-9 * np.maximum(np.abs(kq), 1e-3))
    assert np.all(np.diff(values) >= 0)


def free_chain(n=40):
    kk = oracle.pattern(n, np.array([[i, i + 1] for i in range(n - 1)]))
    for i in range(n - 1):
        kk.add_element([i, i + 1], [1.0, -1.0, -1.0, 1.0])
    mm = oracle.pattern(n, np.array([[i, i + 1] for i in range(n - 1)]))
    for i in range(n):
        mm.add_element([i], [1.0])
    return kk, mm


def test_oracle_subspace_finds_the_modes_of_a_free_chain():
    """eigen.rs:404-452: lambda_k = 2 - 2 cos(k pi / n), the 0 mode included, shift -0.01."""
    n, shift, count = 40, -0.01, 6
    kk, mm = free_chain(n)
    kd = np.zeros((n, n))
    ptr, idx, val = kk.arrays()
    for i in range(n):
        for e in range(ptr[i], ptr[i + 1]):
            kd[i, idx[e]] = val[e]
    a = kd - shift * np.eye(n)
    values, v = oracle.dense_jacobi(a)

    def solve(b, x0):
        return v @ ((v.T @ b) / values)

    lam, vecs, its = oracle.subspace(kk, mm, shift, count, solve)
    for j in range(count):
        exact = 2.0 - 2.0 * np.cos(j * np.pi / n)
        assert abs(lam[j] - exact) < 1e-10, (j, lam[j], exact)
    assert 1 < its < oracle.EIGEN_MAX_ITER


def test_oracle_p2_mass_is_the_exact_integral_of_the_functions():
    """tet10.rs:302-338: each entry is rho times the exact integral of N_i N_j."""
    from math import factorial
    p = np.array([[0.0, 0.0, 0.0], [2.0, 0.1, 0.0], [0.3, 1.5, 0.2], [0.1, 0.4, 0.9]])
    m = oracle.element_matrix(3, p, np.array([3.0]))
    _, vol = oracle.tet_gradients(p)
    edges = [(0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3)]

    def terms(i):
        unit = lambda k, q: tuple(q if c == k else 0 for c in range(4))
        if i < 4:
            return [(2.0, unit(i, 2)), (-1.0, unit(i, 1))]
        a, b = edges[i - 4]
        return [(4.0, tuple(int(c in (a, b)) for c in range(4)))]

    for i in range(10):
        for j in range(10):
            exact = 0.0
            for ci, ei in terms(i):
                for cj, ej in terms(j):
                    e = [x + y for x, y in zip(ei, ej)]
                    num = np.prod([factorial(q) for q in e])
                    exact += ci * cj * 6.0 * vol * num / factorial(sum(e) + 3)
            assert abs(m.reshape(30, 30)[3 * i, 3 * j] - 3.0 * exact) < 1e-12
            assert m.reshape(30, 30)[3 * i, 3 * j + 1] == 0.0


# ------------------------------------------------------------------ the library


@pytest.mark.gpu
def test_library_dense_generalized_matches_the_oracle():
    """The library's Rayleigh-Ritz solver (on the device: the reference's scaled Cholesky
    reduction, then the parallel Jacobi method) against the oracle's cyclic Jacobi (eigen.rs:183-331)
    on eigen.rs:365-402's matrices, on random pairs up to the largest subspace (p = 128) and on a
    pair with a repeated eigenvalue: the eigenvalues to 1e-12 of the largest, Q^T M Q = I and
    K Q = M Q diag(values) to 1e-10, and each vector of a simple eigenvalue equal to the oracle's up
    to its sign."""
    from femahoy_b200.modes import dense_generalized
    rng = np.random.default_rng(4)
    cases = [generalized_case()]
    for n in (12, 37, 128):
        a = rng.standard_normal((n, n))
        b = rng.standard_normal((n, n))
        cases.append((a + a.T, b @ b.T + n * np.eye(n)))
    cases.append((np.diag([1.0, 2.0, 2.0, 3.0, 5.0]), np.eye(5)))
    for k, m in cases:
        v1, q1 = dense_generalized(k, m)
        v2, q2 = oracle.dense_generalized(k, m)
        scale = np.abs(v2).max()
        assert np.abs(v1 - v2).max() <= 1e-12 * scale
        assert np.abs(q1.T @ m @ q1 - np.eye(len(v1))).max() <= 1e-10
        assert np.abs(k @ q1 - (m @ q1) * v1).max() <= 1e-10 * scale
        gap = np.minimum(np.abs(np.diff(v2, prepend=-np.inf)), np.abs(np.diff(v2, append=np.inf)))
        for j in np.nonzero(gap > 1e-6 * scale)[0]:
            sign = np.sign(q1[:, j] @ m @ q2[:, j])
            assert np.abs(sign * q1[:, j] - q2[:, j]).max() <= 1e-8 * np.abs(q2[:, j]).max()


def p2_model(dims=(8, 2, 2), lengths=(80.0, 10.0, 10.0)):
    from femahoy_b200 import meshgen as mg
    box = mg.box(*dims, lengths)
    edges, t10 = oracle.quadratic(box.points, box.tets)
    prob = mg.beam_p2(edges, t10, mesh=box)
    density = np.full(len(t10), 2.7e-9)  # aluminium, t/mm^3
    return box, edges, t10, prob, density


@pytest.mark.gpu
def test_gpu_p2_mass_assembly_is_bit_identical():
    import femahoy_b200 as fg
    _, _, t10, prob, density = p2_model()
    Mg = fg.Csr.assemble(fg.P2_MASS, prob.xyz, t10, density)
    Mo = oracle.pattern(3 * prob.n_points, oracle.dof_elements(t10))
    Mo.assemble(3, prob.xyz, t10, density)
    for g, o in zip(Mg.arrays(), Mo.arrays()):
        assert np.array_equal(np.asarray(g), np.asarray(o))


@pytest.mark.gpu
def test_gpu_modes_of_a_free_chain():
    """eigen.rs:404-452 on the device: 6 modes of a free chain of 40 masses, 0 mode included,
    with the direct solver: lambda_k = 2 - 2 cos(k pi / n) to 1e-10."""
    import femahoy_b200 as fg
    from femahoy_b200.modes import modes
    n = 40
    kk, mm = free_chain(n)
    K = fg.Csr.from_arrays(n, *kk.arrays())
    M = fg.Csr.from_arrays(n, *mm.arrays())
    u = fg.Unknowns.Points(np.column_stack([np.arange(n), np.zeros(n), np.zeros(n)]))
    values, vecs, st = modes(K, M, 6, u, fg.Method.Direct, shift=-0.01)
    for j in range(6):
        assert abs(values[j] - (2.0 - 2.0 * np.cos(j * np.pi / n))) < 1e-10
    ptr, idx, val = mm.arrays()
    assert np.abs(vecs @ vecs.T - np.eye(6)).max() < 1e-10  # M = I


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_modes_of_a_p2_beam_match_the_oracle(precision):
    """The 6 lowest modes of a free-clamped P2 beam: the device's subspace iteration (p-multigrid
    PCG, FP64 and mixed) against the oracle's (its direct solver), eigenvalues to 1e-8."""
    import femahoy_b200 as fg
    from femahoy_b200.modes import modes
    box, edges, t10, prob, density = p2_model()
    free = prob.free
    Kf = fg.Csr.assemble(fg.P2_ELASTIC, prob.xyz, t10, prob.coef).submatrix(free)
    Mf = fg.Csr.assemble(fg.P2_MASS, prob.xyz, t10, density).submatrix(free)
    P, coarse = fg.prolongation(prob.xyz, box.n, edges, free)
    u = fg.Unknowns.Quadratic(prob.xyz[free // 3], P, coarse)
    opts = fg.Options(precision=precision, coarsest=200)
    values, vecs, st = modes(Kf, Mf, 6, u, fg.Method.Multigrid, options=opts)
    ko = oracle.Csr.from_arrays(Kf.n, *Kf.arrays())
    mo = oracle.Csr.from_arrays(Mf.n, *Mf.arrays())
    kd = np.array([v for v in Kf.diagonal()])
    md = np.array([v for v in Mf.diagonal()])
    shift = -oracle.MODES_SHIFT * np.sum(kd / md) / len(kd)
    assert abs(st.shift - shift) <= 1e-12 * abs(shift)
    ptr, idx, val = ko.arrays()
    a = oracle.Csr.from_arrays(ko.n, ptr, idx, val - st.shift * mo.arrays()[2])

    def solve(b, x0):
        x, _ = oracle.direct_solve(a, prob.xyz[free // 3], b)
        return x

    ov, _, _ = oracle.subspace(ko, mo, st.shift, 6, solve)
    assert np.abs(values - ov).max() <= 1e-8 * ov.max()
    assert st.iterations > 1 and st.solves == st.iterations * 14
