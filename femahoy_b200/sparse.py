"""The sparse matrices of the path (crates/fem/src/sparse.rs), held on the device.

``Csr`` mirrors sparse.rs:12-135: ``Csr.pattern`` (sparse.rs:22), the whole element loop of
``add_element`` as one device assembly (sparse.rs:75, called by heat.rs:920-927 and
elastic_tet.rs:183-193), ``submatrix`` (sparse.rs:108) and ``mul`` (sparse.rs:96). ``Rect``
(sparse.rs:202) is the host form of a prolongation.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


class Csr:
    """A square CSR matrix with both triangles, on the device (sparse.rs:12-17)."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            L.lib().femgpu_csr_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    # ---------------------------------------------------------------- construction
    @classmethod
    def pattern(cls, n, elements):
        """sparse.rs:22-65: the pattern of the elements (rows of ``elements``), values 0."""
        e = L.arr(elements, np.uint32)
        h = C.c_void_p()
        L.check(L.lib().femgpu_pattern(n, e.shape[0], e.shape[1], L.ptr(e), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, n, ptr, idx, val):
        """The device copy of host CSR arrays."""
        p, i, v = L.arr(ptr, np.int64), L.arr(idx, np.uint32), L.arr(val, np.float64)
        h = C.c_void_p()
        L.check(L.lib().femgpu_csr_upload(n, L.ptr(p), L.ptr(i), L.ptr(v), C.byref(h)))
        return cls(h.value)

    @classmethod
    def assemble(cls, kind, points, nodes, coef, mode=L.GATHER):
        """Csr::pattern + Csr::add_element over every element on the device. ``kind``:
        femahoy_b200.P1_HEAT (``coef`` (T, 3) conductivities), P1_ELASTIC or P2_ELASTIC
        (``coef`` (T, 2) E and nu; unknown 3 node + component), P2_MASS (``coef`` (T,) the
        density), P2_ELASTIC_ORTHO (``coef`` (T, 9) orthotropic constants), HEX8_HEAT (box
        cells, ``coef`` (T, 3) conductivities) or HEX8_ELASTIC (box cells with incompatible
        modes, ``coef`` (T, 9) orthotropic constants). ``mode`` GATHER gives the reference's
        values bit for bit; COLOUR scatters colour by colour (P1 and P2 elasticity, P1 heat)."""
        x = L.arr(points, np.float64)
        e = L.arr(nodes, np.uint32)
        c = L.arr(coef, np.float64)
        h = C.c_void_p()
        L.check(L.lib().femgpu_assemble(kind, mode, x.shape[0], L.ptr(x), e.shape[0], L.ptr(e),
                                        L.ptr(c), C.byref(h)))
        return cls(h.value)

    # ---------------------------------------------------------------- queries
    @property
    def shape(self):
        n, nnz = C.c_size_t(), C.c_size_t()
        L.check(L.lib().femgpu_csr_info(self._h, C.byref(n), C.byref(nnz)))
        return n.value, nnz.value

    @property
    def n(self):
        return self.shape[0]

    def arrays(self):
        """(ptr, idx, val) on the host."""
        n, nnz = self.shape
        ptr = np.empty(n + 1, np.int64)
        idx = np.empty(nnz, np.uint32)
        val = np.empty(nnz, np.float64)
        L.check(L.lib().femgpu_csr_download(self._h, L.ptr(ptr), L.ptr(idx), L.ptr(val)))
        return ptr, idx, val

    @property
    def ptr(self):
        return self.arrays()[0]

    @property
    def idx(self):
        return self.arrays()[1]

    @property
    def val(self):
        return self.arrays()[2]

    # ---------------------------------------------------------------- operations
    def submatrix(self, keep):
        """sparse.rs:108-135: the rows and columns ``keep``, in that order."""
        k = L.arr(keep, np.int64)
        h = C.c_void_p()
        L.check(L.lib().femgpu_csr_submatrix(self._h, L.ptr(k), len(k), C.byref(h)))
        return Csr(h.value)

    def mul(self, x):
        """sparse.rs:96-105: y = A x."""
        x = L.arr(x, np.float64)
        y = np.empty(self.n)
        L.check(L.lib().femgpu_csr_mul(self._h, L.ptr(x), L.ptr(y)))
        return y

    def diagonal(self):
        """sparse.rs:89-93, on the device."""
        d = np.empty(self.n)
        L.check(L.lib().femgpu_csr_diagonal(self._h, L.ptr(d)))
        return d


@dataclass
class Rect:
    """sparse.rs:202-208: a rectangular CSR matrix on the host (a prolongation)."""

    rows: int
    cols: int
    ptr: np.ndarray
    idx: np.ndarray
    val: np.ndarray

    def _device(self):
        """The device copy (femgpu_rect), made on first use and kept with the arrays."""
        h = self.__dict__.get("_handle")
        if h is None:
            ptr, idx, val = (L.arr(self.ptr, np.int64), L.arr(self.idx, np.uint32),
                             L.arr(self.val, np.float64))
            out = C.c_void_p()
            L.check(L.lib().femgpu_rect_upload(int(self.rows), int(self.cols), L.ptr(ptr),
                                               L.ptr(idx), L.ptr(val), C.byref(out)))
            h = _RectHandle(out.value)
            self.__dict__["_handle"] = h
        return h.h

    def mul(self, x):
        """sparse.rs:212-220: y = P x on the device, each row summed in the reference's order."""
        x = L.arr(x, np.float64)
        y = np.empty(self.rows)
        L.check(L.lib().femgpu_rect_mul(self._device(), L.ptr(x), L.ptr(y)))
        return y

    def mul_transpose(self, x):
        """sparse.rs:223-230: y = P^T x on the device, each entry summed in the reference's
        order (increasing row of P)."""
        x = L.arr(x, np.float64)
        y = np.empty(self.cols)
        L.check(L.lib().femgpu_rect_mul_transpose(self._device(), L.ptr(x), L.ptr(y)))
        return y

    def galerkin(self, a: "Csr") -> "Csr":
        """sparse.rs:233-292: P^T A P on the device (the reference's pattern; its entries to
        rounding)."""
        out = C.c_void_p()
        L.check(L.lib().femgpu_rect_galerkin(self._device(), a.handle, C.byref(out)))
        return Csr(out.value)


class _RectHandle:
    """Frees a femgpu_rect with its owner."""

    def __init__(self, h):
        self.h = h

    def __del__(self):
        h, self.h = self.h, None
        if h:
            L.lib().femgpu_rect_free(h)


def colour(n, elements):
    """The colour of each element for the colour-ordered scatter (no reference counterpart):
    elements sharing a node differ. Returns (colours, number of colours)."""
    e = L.arr(elements, np.uint32)
    out = np.empty(e.shape[0], np.uint32)
    nc = C.c_int()
    L.check(L.lib().femgpu_colour(n, e.shape[0], e.shape[1], L.ptr(e), L.ptr(out), C.byref(nc)))
    return out, nc.value
