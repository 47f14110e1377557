"""multigrid::pcg (multigrid.rs:692-753) with the caller's preconditioner: the oracle's restatement
on the CPU (convergence, the texts of its failures, b = 0), and the library's femgpu_pcg /
femgpu_pcg_device against it on the GPU (the same iterations, the solution to rounding, the same
texts, the solver's V-cycle as a device preconditioner)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import femahoy_b200 as fg
import oracle
from femahoy_b200 import _lib as L
from femahoy_b200 import meshgen as mg


def _laplacian(n):
    """The 1D Laplacian with a shifted diagonal (cholesky.rs:234-258's matrix family)."""
    ptr, idx, val = [0], [], []
    for i in range(n):
        for j, v in ((i - 1, -1.0), (i, 2.0 + 0.01 * (i % 7)), (i + 1, -1.0)):
            if 0 <= j < n:
                idx.append(j)
                val.append(v)
        ptr.append(len(idx))
    return np.array(ptr, np.int64), np.array(idx, np.uint32), np.array(val)


def _heat(k=10, seed=2):
    return mg.heat_cube(k, seed=seed)


def test_oracle_pcg_converges_and_fails_with_the_reference_texts():
    ptr, idx, val = _laplacian(200)
    a = oracle.Csr.from_arrays(200, ptr, idx, val)
    rng = np.random.default_rng(0)
    b = rng.standard_normal(200)
    diag = val[[np.nonzero(idx[ptr[i]:ptr[i + 1]] == i)[0][0] + ptr[i] for i in range(200)]]

    def jacobi(r, z):
        z[:] = r / diag

    x = np.zeros(200)
    it, res = oracle.pcg(a, b, x, jacobi, 1e-10, 500)
    A = np.zeros((200, 200))
    for i in range(200):
        A[i, idx[ptr[i]:ptr[i + 1]]] = val[ptr[i]:ptr[i + 1]]
    assert res <= 1e-10 and 0 < it <= 200
    assert np.linalg.norm(x - np.linalg.solve(A, b)) <= 1e-8 * np.linalg.norm(x)
    with pytest.raises(oracle.OracleError,
                       match=r"^conjugate gradients did not converge: the residual is "
                             r"\d\.\d\de-\d+ after 3 iterations$"):
        oracle.pcg(a, b, np.zeros(200), jacobi, 1e-10, 3)
    with pytest.raises(oracle.OracleError, match="^cancelled$"):
        oracle.pcg(a, b, np.zeros(200), None, 1e-10, 500, cancel=C.c_int(1))
    x = np.ones(200)
    assert oracle.pcg(a, np.zeros(200), x, jacobi) == (0, 0.0)
    assert not x.any()


@pytest.mark.gpu
def test_pcg_with_a_host_preconditioner_equals_the_oracle():
    """A 3D heat cube's reduced system, Jacobi from a numpy callback, from a nonzero start value:
    the iterations equal the oracle's and the solution agrees to rounding."""
    h = _heat(14)
    K = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    A = K.submatrix(h.free)
    b = fg.reduced_rhs(K, h.load, h.values, h.free)
    Ao = oracle.Csr.from_arrays(A.n, *A.arrays())
    ptr, idx, val = A.arrays()
    d = np.array([val[ptr[i] + np.nonzero(idx[ptr[i]:ptr[i + 1]] == i)[0][0]]
                  for i in range(A.n)])

    def jacobi(r, z):
        z[:] = r / d

    x0 = np.linspace(0.0, 1.0, A.n)
    x = x0.copy()
    c = fg.pcg(A, b, x, jacobi, 1e-10, 500)
    xo = x0.copy()
    it, res = oracle.pcg(Ao, b, xo, jacobi, 1e-10, 500)
    assert c.iterations == it and c.residual <= 1e-10
    assert abs(c.residual - res) <= 1e-3 * res
    assert np.linalg.norm(x - xo) <= 1e-9 * np.linalg.norm(xo)


@pytest.mark.gpu
def test_pcg_failures_carry_the_reference_texts_and_keep_the_last_iterate():
    ptr, idx, val = _laplacian(300)
    A = fg.Csr.from_arrays(300, ptr, idx, val)
    Ao = oracle.Csr.from_arrays(300, ptr, idx, val)
    b = np.random.default_rng(4).standard_normal(300)
    x = np.zeros(300)
    with pytest.raises(fg.FemError) as e:
        fg.pcg(A, b, x, None, 1e-10, 5)
    xo = np.zeros(300)
    with pytest.raises(oracle.OracleError) as eo:
        oracle.pcg(Ao, b, xo, None, 1e-10, 5)
    assert e.value.code == L.NOT_CONVERGED and str(e.value) == str(eo.value)
    assert np.linalg.norm(x - xo) <= 1e-12 * np.linalg.norm(xo) and x.any()
    with pytest.raises(fg.FemError, match="^cancelled$") as e:
        fg.pcg(A, b, np.zeros(300), None, 1e-10, 500, cancelled=C.c_int(1))
    assert e.value.code == L.CANCELLED
    x = np.ones(300)
    c = fg.pcg(A, np.zeros(300), x)
    assert (c.iterations, c.residual) == (0, 0.0) and not x.any()


@pytest.mark.gpu
def test_pcg_device_with_the_solver_v_cycle_as_preconditioner():
    """femgpu_pcg_device on device vectors with the solver's own V-cycle
    (femgpu_solver_precondition_device, on the solver's stream) as the preconditioner: a few
    iterations to 1e-10, and the solution is the oracle's direct one to 1e-8."""
    torch = pytest.importorskip("torch")
    h = _heat(16)
    K = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    A = K.submatrix(h.free)
    b = fg.reduced_rhs(K, h.load, h.values, h.free)
    planes, pts, comp = mg.grid_unknowns(h)
    s = fg.Solver(A, fg.Unknowns.Grid(fg.Level(planes, pts, comp)), fg.Method.Multigrid,
                  options=fg.Options(precision=fg.FP64))
    db = torch.tensor(b, dtype=torch.float64, device="cuda")
    dx = torch.zeros_like(db)
    torch.cuda.synchronize()

    def vcycle(r, z, n, stream, ctx):
        L.check(L.lib().femgpu_solver_precondition_device(s.handle, C.c_void_p(r),
                                                          C.c_void_p(z)))

    cb = L.PRECONDITION_DEVICE_FN(vcycle)
    out = L.Convergence_t()
    L.check(L.lib().femgpu_pcg_device(A.handle, C.c_void_p(db.data_ptr()),
                                      C.c_void_p(dx.data_ptr()), cb, None, 1e-10, 500, None,
                                      None, C.byref(out)))
    x = dx.cpu().numpy()
    assert out.residual <= 1e-10 and 0 < out.iterations < 40
    xd, _ = oracle.direct_solve(oracle.Csr.from_arrays(A.n, *A.arrays()), h.xyz[h.free], b)
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
