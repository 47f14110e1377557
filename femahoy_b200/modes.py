"""Modes (include/femgpu.h ``femgpu_modes``): the lowest eigenpairs of K x = lambda M x by
shift-invert subspace iteration with Rayleigh-Ritz, crates/fem/src/eigen.rs:81-177 as
crates/fem/src/modes.rs:180-216 runs it, with (K - shift M) solved by this library's solver.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .solve import Crossover, Options, unknowns_c


@dataclass
class ModesStats:
    iterations: int
    solves: int
    pcg_iterations: int
    shift: float
    seconds: float


def modes(k, m, count, unknowns, method=None, crossover: Crossover | None = None, *,
          shift=None, precision=L.FP64, options: Options | None = None, vectors=True,
          cancel=None, cells=None):
    """The ``count`` lowest eigenpairs of the free submatrices ``k`` and ``m`` (Csr, the same
    pattern): (values, vectors (count, n) or None, ModesStats). ``shift`` None is
    modes.rs:186-191's default. ``cells`` (a Cells with its ``mass``): the box grid's modes
    (modes.rs:355-420), the solver's coarse matrices from the cells of K - shift M."""
    n = k.n
    keep = []
    u = unknowns_c(unknowns, keep)
    crossover = crossover or Crossover.Unknowns(16384)
    opts = options or Options(precision=precision)
    cr, oc = crossover._c(), opts._c()
    values = np.empty(count)
    vecs = np.empty((count, n)) if vectors else None
    st = L.ModesStats_t()
    mth = -1 if method is None else int(method)
    flag = C.byref(cancel) if isinstance(cancel, C.c_int) else None
    cc = C.byref(cells._c(keep)) if cells is not None else None
    L.check(L.lib().femgpu_modes_cells(k.handle, m.handle, count,
                                       float("nan") if shift is None else float(shift),
                                       C.byref(u), mth, C.byref(cr), C.byref(oc), cc, flag,
                                       L.ptr(values), L.ptr(vecs), C.byref(st)))
    return values, vecs, ModesStats(st.iterations, st.solves, st.pcg_iterations, st.shift,
                                    st.seconds)


def dense_generalized(k, m):
    """eigen.rs:183-269 on the device (the parallel Jacobi method after the reference's scaled
    Cholesky reduction): (values ascending, Q) with Q^T M Q = I."""
    k = L.arr(k, np.float64)
    m = L.arr(m, np.float64)
    n = k.shape[0]
    values, q = np.empty(n), np.empty((n, n))
    L.check(L.lib().femgpu_dense_generalized(L.ptr(k), L.ptr(m), n, L.ptr(values), L.ptr(q)))
    return values, q
