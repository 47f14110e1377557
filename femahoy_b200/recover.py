"""Post-solve recovery of P2 elasticity (include/femgpu.h ``femgpu_recovery_*``): the strain and
the stress at the 10 points of each cell, their mean at each point, the von Mises and principal
stresses of the means, and the peak von Mises stress of each part, as the loop of
crates/fem/src/elastic_tet.rs:367-427 and elastic_tet.rs:482-483.

``Recovery(xyz, tets10, coef)`` keeps the mesh side on the device (a record of constants per
cell and the cells of each point); ``run(u)`` recovers from the full displacement (3 values per
point). Stress order xx, yy, zz, xy, yz, xz; strain as tensor components in the same order.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass
class Peak:
    """The reference's ``Peak`` of 1 part (crates/fem/src/elastic.rs:186-195), with the cell
    and the point of each value. ``regular_element`` -1 is ``None``."""
    mises: float
    element: int
    local: int
    point: int
    singular: bool
    regular_mises: float
    regular_element: int
    regular_local: int
    regular_point: int

    @classmethod
    def of(cls, p):
        return cls(p.mises, p.element, p.local, p.point, bool(p.singular), p.regular_mises,
                   p.regular_element, p.regular_local, p.regular_point)


@dataclass
class Reactions:
    """The result of ``reactions``: the force of each load (the reference's ``Reaction::force``
    for a fixed face set, its ``point_force`` for a point support), the applied forces plus the
    reactions per component, the gross magnitude of the forces and the imbalance."""
    load_force: np.ndarray
    total: np.ndarray
    gross: float
    imbalance: float


def reactions(k, u, force, fixed, owner, nloads, applied, gross=0.0) -> Reactions:
    """elastic::reactions (crates/fem/src/elastic.rs:772-839) on the device: r = K u - f at the
    fixed unknowns, summed per owner load, per component and in magnitude, in the reference's
    order. ``k`` the full stiffness (Csr), ``u`` and ``force`` full vectors, ``fixed`` a mask,
    ``owner`` the load that fixed each unknown, ``applied`` the 3 applied sums, ``gross`` the
    gross magnitude before the reactions."""
    n = k.n
    u = np.ascontiguousarray(u, dtype=np.float64)
    f = np.ascontiguousarray(force, dtype=np.float64)
    fx = np.ascontiguousarray(fixed, dtype=np.uint8)
    ow = np.ascontiguousarray(owner, dtype=np.uint32)
    ap = np.ascontiguousarray(applied, dtype=np.float64)
    if not (len(u) == len(f) == len(fx) == len(ow) == n) or ap.shape != (3,):
        raise ValueError("u, force, fixed and owner need 1 value per unknown, applied 3")
    lf = np.zeros((max(nloads, 1), 3))
    tot = np.zeros(3)
    g, imb = C.c_double(), C.c_double()
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    L.check(L.lib().femgpu_reactions(k._h, p(u), p(f), p(fx), p(ow), nloads, p(ap), gross,
                                     p(lf), p(tot), C.byref(g), C.byref(imb)))
    return Reactions(lf[:nloads].copy(), tot, g.value, imb.value)


def hex_loads(xyz, hexes, coef, *, expansion=None, accel=None, dtemp=None):
    """The forces of the box cells' loop (crates/fem/src/elastic.rs:386-405) on the device: the
    load of the corner temperature changes ``dtemp`` (1 per point) through each cell's expansion
    (3 per cell), plus ``accel`` (3 per cell: density times gravity plus the body force) times
    the volume / 8, summed over the cells in order. Returns 3 values per point."""
    xyz = L.arr(xyz, np.float64).reshape(-1, 3)
    hexes = L.arr(hexes, np.uint32).reshape(-1, 8)
    coef = L.arr(coef, np.float64).reshape(-1, 9)
    opt = lambda a, k: None if a is None else L.arr(a, np.float64).reshape(-1, k)
    exp, acc = opt(expansion, 3), opt(accel, 3)
    dt = None if dtemp is None else L.arr(dtemp, np.float64)
    force = np.empty(3 * len(xyz))
    L.check(L.lib().femgpu_hex_loads(len(xyz), L.ptr(xyz), len(hexes), L.ptr(hexes), L.ptr(coef),
                                     L.ptr(exp), L.ptr(acc), L.ptr(dt), L.ptr(force)))
    return force


class Recovery:
    """``hex=True``: the box grid's loop (crates/fem/src/elastic.rs:615-660) over box cells,
    ``tets10`` then holding the 8 corners of each cell (VTK order) and ``coef`` the 9
    orthotropic constants of each cell; the peaks' ``local`` is the corner."""

    def __init__(self, xyz, tets10, coef, *, expansion=None, part=None, nparts=1,
                 singular=None, hex=False):
        xyz = L.arr(xyz, np.float64).reshape(-1, 3)
        t10 = L.arr(tets10, np.uint32).reshape(-1, 8 if hex else 10)
        coef = L.arr(coef, np.float64).reshape(-1, 9 if hex else 2)
        exp = None if expansion is None else L.arr(expansion, np.float64).reshape(-1, 3)
        part = None if part is None else L.arr(part, np.uint32)
        sing = None if singular is None else L.arr(singular, np.uint8)
        h = C.c_void_p()
        new = L.lib().femgpu_recovery_new_hex if hex else L.lib().femgpu_recovery_new
        L.check(new(len(xyz), L.ptr(xyz), len(t10), L.ptr(t10), L.ptr(coef), L.ptr(exp),
                    L.ptr(part), nparts, L.ptr(sing), C.byref(h)))
        self._h = h.value
        self._free = L.lib().femgpu_recovery_free
        self.npoints = len(xyz)
        self.ncells = len(t10)
        self.nparts = nparts

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def run(self, u, dtemp=None, *, peaks=True, principal=True):
        """Host arrays in and out: a dict of stress (n, 6), strain (n, 6), mises (n,),
        principal (n, 3) or None, and peaks (a list of Peak, 1 per part) or None."""
        n = self.npoints
        u = L.arr(u, np.float64).reshape(-1)
        if len(u) != 3 * n:
            raise L.FemError(L.INVALID, "u holds 3 values per point")
        dt = None if dtemp is None else L.arr(dtemp, np.float64)
        stress, strain, mises = np.empty((n, 6)), np.empty((n, 6)), np.empty(n)
        pr = np.empty((n, 3)) if principal else None
        pk = (L.Peak_t * self.nparts)() if peaks else None
        L.check(L.lib().femgpu_recovery_run(self._h, L.ptr(u), L.ptr(dt), L.ptr(stress),
                                            L.ptr(strain), L.ptr(mises), L.ptr(pr),
                                            C.cast(pk, C.c_void_p) if peaks else None))
        return {"stress": stress, "strain": strain, "mises": mises, "principal": pr,
                "peaks": [Peak.of(p) for p in pk] if peaks else None}

    def probes(self, u, points, *, dtemp=None, temperature=None, names=None):
        """The probes (crates/fem/src/elastic_tet.rs:428-467) at ``points`` (P, 3): a dict of
        displacement (P, 3), stress (P, 6), mises (P,), temperature (P,) and hits (P,), the
        cells that share each point. ``temperature`` holds the absolute corner temperatures,
        ``dtemp`` their change (for the stress); ``names`` the probes' names for the error of a
        point in no cell."""
        n = self.npoints
        u = L.arr(u, np.float64).reshape(-1)
        if len(u) != 3 * n:
            raise L.FemError(L.INVALID, "u holds 3 values per point")
        pts = L.arr(points, np.float64).reshape(-1, 3)
        m = len(pts)
        dt = None if dtemp is None else L.arr(dtemp, np.float64)
        tp = None if temperature is None else L.arr(temperature, np.float64)
        nm = None
        if names is not None:
            enc = [x.encode() for x in names]
            nm = (C.c_char_p * m)(*enc)
        disp, stress, mises, temp = np.empty((m, 3)), np.empty((m, 6)), np.empty(m), np.empty(m)
        hits = np.empty(m, np.int64)
        L.check(L.lib().femgpu_recovery_probes(
            self._h, L.ptr(u), L.ptr(dt), L.ptr(tp), m, L.ptr(pts),
            C.cast(nm, C.c_void_p) if nm is not None else None, L.ptr(disp), L.ptr(stress),
            L.ptr(mises), L.ptr(temp), L.ptr(hits)))
        return {"displacement": disp, "stress": stress, "mises": mises, "temperature": temp,
                "hits": hits}

    def run_device(self, u, stress, strain, *, dtemp=None, mises=None, principal=None,
                   peaks=True):
        """Device buffers (torch CUDA float64 tensors, contiguous) in and out; returns the list
        of Peak or None. Returns when the results are written."""
        def dp(t):
            return None if t is None else C.c_void_p(t.data_ptr())
        pk = (L.Peak_t * self.nparts)() if peaks else None
        L.check(L.lib().femgpu_recovery_run_device(
            self._h, dp(u), dp(dtemp), dp(stress), dp(strain), dp(mises), dp(principal),
            C.cast(pk, C.c_void_p) if peaks else None))
        return [Peak.of(p) for p in pk] if peaks else None

    def last_time(self):
        """(ms, algorithmic bytes) of the recovery kernels of the last run (CUDA events)."""
        ms, by = C.c_double(), C.c_double()
        L.check(L.lib().femgpu_recovery_last_time(self._h, C.byref(ms), C.byref(by)))
        return ms.value, by.value

    def bytes(self):
        return int(L.lib().femgpu_recovery_bytes(self._h))
