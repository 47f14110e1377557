"""Rect (sparse.rs:196-293) and Csr::diagonal (sparse.rs:88-93) on the device, against the
oracle: P x and P^T x bit for bit, the Galerkin product P^T A P with the same pattern and its
entries to rounding, the diagonal exactly; on the p-multigrid prolongation of a P2 box and a
random rectangular matrix with empty rows and columns."""
from __future__ import annotations

import numpy as np
import pytest

import femahoy_b200 as fg
import oracle
from femahoy_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _p2_problem():
    box = mg.box(4, 3, 5)
    q = fg.Quadratic.new(box.points, box.tets)
    n = len(q.points)
    coef = np.tile([1000.0, 0.3], (len(q.tets), 1))
    fixed = np.repeat(q.points[:, 0] == 0.0, 3)
    free = np.nonzero(~fixed)[0].astype(np.int64)
    K = fg.Csr.assemble(fg.P2_ELASTIC, q.points, q.tets, coef).submatrix(free)
    P, _ = fg.prolongation(q.points, len(box.points), q.edges, free)
    return K, P, n


def _random_rect(rows, cols, rng):
    ptr, idx, val = [0], [], []
    for i in range(rows):
        k = 0 if i % 7 == 3 else int(rng.integers(1, 6))
        cs = np.sort(rng.choice(cols - 2, size=min(k, cols - 2), replace=False))
        idx += cs.tolist()
        val += rng.standard_normal(len(cs)).tolist()
        ptr.append(len(idx))
    return fg.Rect(rows, cols, np.array(ptr, np.int64), np.array(idx, np.uint32), np.array(val))


def test_rect_products_are_the_oracles_bit_for_bit():
    rng = np.random.default_rng(7)
    K, P, _ = _p2_problem()
    for R in (P, _random_rect(300, 120, rng)):
        Ro = oracle.Rect.from_arrays(R.rows, R.cols, R.ptr, R.idx, R.val)
        x = rng.standard_normal(R.cols)
        y = rng.standard_normal(R.rows)
        assert np.array_equal(R.mul(x), Ro.mul(x))
        assert np.array_equal(R.mul_transpose(y), Ro.mul_transpose(y))
        # Twice on the same handle (the transpose is kept).
        assert np.array_equal(R.mul_transpose(2.0 * y), Ro.mul_transpose(2.0 * y))


def test_galerkin_and_diagonal_equal_the_oracle():
    K, P, _ = _p2_problem()
    Ko = oracle.Csr.from_arrays(K.n, *K.arrays())
    Po = oracle.Rect.from_arrays(P.rows, P.cols, P.ptr, P.idx, P.val)
    G = P.galerkin(K)
    Go = Po.galerkin(Ko)
    (gp, gi, gv), (op, oi, ov) = G.arrays(), Go.arrays()
    assert np.array_equal(gp, op) and np.array_equal(gi, oi)
    assert np.abs(gv - ov).max() <= 1e-13 * np.abs(ov).max()
    d = K.diagonal()
    ptr, idx, val = K.arrays()
    want = np.array([val[ptr[i]:ptr[i + 1]][idx[ptr[i]:ptr[i + 1]] == i].sum()
                     for i in range(K.n)])
    assert np.array_equal(d, want)


def test_rect_refuses_bad_arrays():
    bad = fg.Rect(2, 3, np.array([0, 2, 1], np.int64), np.array([0, 1], np.uint32),
                  np.ones(2))
    with pytest.raises(fg.FemError, match="the row pointers must not decrease"):
        bad.mul(np.ones(3))
    bad = fg.Rect(1, 3, np.array([0, 1], np.int64), np.array([5], np.uint32), np.ones(1))
    with pytest.raises(fg.FemError, match="a column past the columns"):
        bad.mul(np.ones(3))
