"""CPU oracle of the fh-fem iterative solve path (TEST INFRASTRUCTURE ONLY).

A C++17 restatement of femahoy's crates/fem (sparse.rs, heat.rs tet kernels, tet10.rs,
hex.rs, multigrid.rs, pmultigrid.rs, order.rs, symbolic.rs, cholesky.rs, solve.rs), built
into ``liboracle.so`` by ``oracle/Makefile`` and loaded here with ctypes. Only the tests, the
smoke check and the CPU-baseline leg of ``bench.py`` use it, as the checker; the product
(``femahoy_b200`` / ``libfemgpu.so``) never imports it.

Parity is pinned by the reference's own unit-test known answers (sparse.rs:299-325,
cholesky.rs:260-293, order.rs:186-197, tet10.rs:302-338) ported in ``tests/test_oracle.py``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")


def build() -> str:
    """Compile liboracle.so with the committed Makefile (g++ only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def _load():
    if not os.path.exists(_SO):
        build()
    lib = C.CDLL(_SO)
    P, S, D, I = C.c_void_p, C.c_size_t, C.c_double, C.c_int
    sig = {
        "orc_pattern": (P, [S, P, S, I]),
        "orc_csr_import": (P, [S, P, P, P]),
        "orc_csr_info": (None, [P, P, P]),
        "orc_csr_export": (None, [P, P, P, P]),
        "orc_csr_free": (None, [P]),
        "orc_add_element": (I, [P, P, I, P, P, S]),
        "orc_mul": (None, [P, P, P]),
        "orc_set_threads": (None, [C.c_int]),
        "orc_submatrix": (P, [P, P, S]),
        "orc_reduced_rhs": (None, [P, P, P, P, S, P]),
        "orc_reactions": (None, [P, P, P, P, P, S, P, D, P, P, P, P]),
        "orc_probes": (C.c_long, [P, S, P, P, P, P, P, P, S, P, P, P, P, P, P]),
        "orc_tet_gradients": (None, [P, P, P]),
        "orc_isotropic": (I, [D, D, P, P, P, S]),
        "orc_element_matrix": (I, [I, P, P, P]),
        "orc_hex8_stiffness": (I, [P, P, P, P, S]),
        "orc_hex8_element": (I, [P, P, P, P, P, P, P, P, S]),
        "orc_hex8_strain_stress": (I, [P, P, P, P, P, P, P, P, P, S]),
        "orc_recover_hex": (I, [S, P, S, P, P, P, P, P, P, S, P, P, P, P, P, P, P, S]),
        "orc_hex_loads": (I, [S, P, S, P, P, P, P, P, P, P, S]),
        "orc_hex8_mass": (None, [P, D, P]),
        "orc_symbolic_counts": (None, [P, P, P, P]),
        "orc_assemble": (I, [P, I, P, P, S, P, P, S]),
        "orc_quadratic": (S, [P, S, P, S, P, P]),
        "orc_colour": (I, [S, P, S, I, P]),
        "orc_colour_priority": (C.c_uint32, [C.c_uint32]),
        "orc_rect_import": (P, [S, S, P, P, P]),
        "orc_rect_info": (None, [P, P, P, P]),
        "orc_rect_export": (None, [P, P, P, P]),
        "orc_rect_free": (None, [P]),
        "orc_rect_mul": (None, [P, P, P]),
        "orc_rect_mul_transpose": (None, [P, P, P]),
        "orc_galerkin": (P, [P, P]),
        "orc_coarsen": (P, [P, P, S, P, S, P, S, P, P, S, P, P, P]),
        "orc_by_cells": (P, [P, P, S, P, S, P, S, P, P, S, S, P, P, P, S, P, P, P]),
        "orc_prolongation": (P, [P, S, S, P, S, P, S, P, P]),
        "orc_nested_dissection": (None, [P, P, P]),
        "orc_direct_solve": (I, [P, P, P, P, P, S]),
        "orc_pcg": (I, [P, P, P, C.CFUNCTYPE(None, P, P, S, P), P, D, S, P, P, P, P, S]),
        "orc_solver_new": (P, [P, I, P, S, P, S, P, S, P, P, P, P, P, S, I, I, S, D,
                               C.c_uint64, I, S, P, P, P, S, P, S]),
        "orc_solver_level_matrix": (P, [P, S]),
        "orc_solver_free": (None, [P]),
        "orc_solver_method": (I, [P]),
        "orc_solver_levels": (S, [P]),
        "orc_solver_level_size": (S, [P, S]),
        "orc_solver_solve": (I, [P, P, P, D, S, P, P, P, P, S]),
        "orc_solver_precondition": (None, [P, P, P]),
        "orc_recover": (I, [S, P, S, P, P, P, P, P, P, S, P, P, P, P, P, P, P, S]),
        "orc_add_capacity": (I, [P, P, D, P, S]),
        "orc_dense_generalized": (I, [P, P, I, P, P, P, S]),
        "orc_dense_jacobi": (None, [P, I, P, P]),
        "orc_reduced_rhs_transient": (None, [P, P, P, P, S, P, D, P]),
        "orc_transient_energy": (None, [S, P, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = _load()


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OracleError(RuntimeError):
    """The reference's error text (its ``Err(String)``)."""


class Csr:
    """sparse.rs:12-17, held by the oracle library."""

    def __init__(self, handle):
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None):
            _lib.orc_csr_free(self.h)
            self.h = None

    @classmethod
    def from_arrays(cls, n, ptr, idx, val):
        ptr = np.ascontiguousarray(ptr, dtype=np.int64)
        idx = np.ascontiguousarray(idx, dtype=np.uint32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        return cls(_lib.orc_csr_import(n, _p(ptr), _p(idx), _p(val)))

    @property
    def shape(self):
        n, nnz = C.c_size_t(), C.c_size_t()
        _lib.orc_csr_info(self.h, C.byref(n), C.byref(nnz))
        return n.value, nnz.value

    @property
    def n(self):
        return self.shape[0]

    def arrays(self):
        n, nnz = self.shape
        ptr = np.empty(n + 1, np.int64)
        idx = np.empty(nnz, np.uint32)
        val = np.empty(nnz, np.float64)
        _lib.orc_csr_export(self.h, _p(ptr), _p(idx), _p(val))
        return ptr, idx, val

    def add_element(self, nodes, ke):
        nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
        ke = np.ascontiguousarray(ke, dtype=np.float64)
        err = C.create_string_buffer(512)
        if _lib.orc_add_element(self.h, _p(nodes), len(nodes), _p(ke), err, 512):
            raise OracleError(err.value.decode())

    def mul(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n)
        _lib.orc_mul(self.h, _p(x), _p(y))
        return y

    def submatrix(self, keep):
        keep = np.ascontiguousarray(keep, dtype=np.int64)
        return Csr(_lib.orc_submatrix(self.h, _p(keep), len(keep)))

    def reduced_rhs(self, load, t, free):
        load = np.ascontiguousarray(load, dtype=np.float64)
        t = np.ascontiguousarray(t, dtype=np.float64)
        free = np.ascontiguousarray(free, dtype=np.int64)
        out = np.empty(len(free))
        _lib.orc_reduced_rhs(self.h, _p(load), _p(t), _p(free), len(free), _p(out))
        return out

    def add_capacity(self, capacity, dt):
        """heat.rs:691-696: capacity / dt added to each diagonal entry, in place."""
        capacity = np.ascontiguousarray(capacity, dtype=np.float64)
        err = C.create_string_buffer(512)
        if _lib.orc_add_capacity(self.h, _p(capacity), dt, err, 512):
            raise OracleError(err.value.decode())

    def reduced_rhs_transient(self, load, t, free, capacity, dt):
        """heat.rs:1219-1244 with Some((capacity, dt))."""
        load = np.ascontiguousarray(load, dtype=np.float64)
        t = np.ascontiguousarray(t, dtype=np.float64)
        free = np.ascontiguousarray(free, dtype=np.int64)
        capacity = np.ascontiguousarray(capacity, dtype=np.float64)
        out = np.empty(len(free))
        _lib.orc_reduced_rhs_transient(self.h, _p(load), _p(t), _p(free), len(free),
                                       _p(capacity), dt, _p(out))
        return out

    def assemble(self, kind, xyz, nodes, coef):
        """Add every element, in increasing element order (heat.rs:920-927,
        elastic_tet.rs:183-193, modes.rs:470-476). kind 0 = P1 heat, 1 = P1 elasticity, 2 = P2
        elasticity (E, nu), 3 = P2 mass (density), 4 = P2 elasticity of an orthotropic material
        (E_x, E_y, E_z, nu_xy, nu_xz, nu_yz, G_xy, G_xz, G_yz), 5 = box cells of 8 corners in
        VTK order (the 3 conductivities)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
        coef = np.ascontiguousarray(coef, dtype=np.float64)
        err = C.create_string_buffer(512)
        if _lib.orc_assemble(self.h, kind, _p(xyz), _p(nodes), nodes.shape[0], _p(coef), err,
                             512):
            raise OracleError(err.value.decode())


def reactions(k: Csr, u, force, fixed, owner, nloads, applied, gross=0.0):
    """elastic.rs:772-839: (load_force (nloads, 3), total (3,), gross, imbalance)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    f = np.ascontiguousarray(force, dtype=np.float64)
    fx = np.ascontiguousarray(fixed, dtype=np.uint8)
    ow = np.ascontiguousarray(owner, dtype=np.uint32)
    ap = np.ascontiguousarray(applied, dtype=np.float64)
    lf = np.zeros((max(nloads, 1), 3))
    tot = np.zeros(3)
    g, imb = C.c_double(), C.c_double()
    _lib.orc_reactions(k.h, _p(u), _p(f), _p(fx), _p(ow), nloads, _p(ap), gross, _p(lf),
                       _p(tot), C.byref(g), C.byref(imb))
    return lf[:nloads], tot, g.value, imb.value


def probes(xyz, tets10, coef, u, points, *, expansion=None, dtemp=None, temperature=None):
    """elastic_tet.rs:428-467: (displacement (P, 3), stress (P, 6), mises (P,), temperature
    (P,), hits (P,)); raises OracleError for a probe in no cell."""
    f = lambda a, t=np.float64: None if a is None else np.ascontiguousarray(a, dtype=t)
    xyz_, t10, cf, uu, pts = f(xyz), f(tets10, np.uint32), f(coef), f(u), f(points)
    ex, dt, tp = f(expansion), f(dtemp), f(temperature)
    n = len(pts)
    dsp, st, ms, tv = np.zeros((n, 3)), np.zeros((n, 6)), np.zeros(n), np.zeros(n)
    hits = np.zeros(n, np.int64)
    bad = _lib.orc_probes(_p(xyz_), len(t10), _p(t10), _p(cf), _p(ex), _p(dt), _p(tp), _p(uu),
                          n, _p(pts), _p(dsp), _p(st), _p(ms), _p(tv), _p(hits))
    if bad >= 0:
        raise OracleError(f"probe {bad} is in no part")
    return dsp, st, ms, tv, hits


def set_threads(n):
    """Host threads of the restatement's matrix products and PCG dot products (1: the
    reference's single thread, the default)."""
    _lib.orc_set_threads(int(n))


def pattern(n, elements):
    """sparse.rs:22-65 for elements of equal size (rows of ``elements``)."""
    e = np.ascontiguousarray(elements, dtype=np.uint32)
    return Csr(_lib.orc_pattern(n, _p(e), e.shape[0], e.shape[1]))


def dof_elements(nodes):
    """The unknowns 3 node + component of each element (elastic_tet.rs:178-182)."""
    nodes = np.asarray(nodes, dtype=np.uint32)
    m = nodes.shape[1]
    return (3 * np.repeat(nodes, 3, axis=1) + np.tile(np.arange(3, dtype=np.uint32), m)).astype(
        np.uint32)


def tet_gradients(p):
    p = np.ascontiguousarray(p, dtype=np.float64).reshape(12)
    g = np.empty(12)
    v = C.c_double()
    _lib.orc_tet_gradients(_p(p), _p(g), C.byref(v))
    return g.reshape(4, 3), v.value


def element_matrix(kind, p, coef):
    p = np.ascontiguousarray(p, dtype=np.float64).reshape(12)
    coef = np.ascontiguousarray(coef, dtype=np.float64)
    m = {0: 4, 1: 12, 2: 30, 3: 30, 4: 30}[kind]
    ke = np.empty(m * m)
    _lib.orc_element_matrix(kind, _p(p), _p(coef), _p(ke))
    return ke.reshape(m, m)


def orthotropic(e, nu=None, g=None):
    """The 9 constants (Ex, Ey, Ez, nu_xy, nu_xz, nu_yz, G_xy, G_xz, G_yz) of an orthotropic
    material (hex.rs:47-55); with one modulus and a ratio, the isotropic material
    (hex.rs:57-65: G = E / (2 (1 + nu)))."""
    if np.isscalar(e):
        return np.array([e] * 3 + [nu] * 3 + [e / (2.0 * (1.0 + nu))] * 3)
    return np.concatenate([np.asarray(e, float), np.asarray(nu, float), np.asarray(g, float)])


def hex8_stiffness(size, c):
    """hex.rs:218-297: the 24 x 24 stiffness of the 8 corners (unknown 3 corner + component) of a
    box cell with the side lengths ``size``, its 9 incompatible modes condensed, for the
    orthotropic constants ``c`` (``orthotropic``)."""
    size = np.ascontiguousarray(size, dtype=np.float64).reshape(3)
    c = np.ascontiguousarray(c, dtype=np.float64).reshape(9)
    kc = np.empty(576)
    err = C.create_string_buffer(512)
    if _lib.orc_hex8_stiffness(_p(size), _p(c), _p(kc), err, 512):
        raise OracleError(err.value.decode())
    return kc.reshape(24, 24)


def isotropic(e, nu):
    normal = np.empty(9)
    shear = np.empty(3)
    err = C.create_string_buffer(512)
    if _lib.orc_isotropic(e, nu, _p(normal), _p(shear), err, 512):
        raise OracleError(err.value.decode())
    return normal.reshape(3, 3), shear


def quadratic(xyz, tets):
    """tet10.rs:244-272: (edges (E, 2), tets10 (T, 10))."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    tets = np.ascontiguousarray(tets, dtype=np.uint32)
    edges = np.empty((6 * len(tets), 2), np.uint32)
    t10 = np.empty((len(tets), 10), np.uint32)
    ne = _lib.orc_quadratic(_p(xyz), len(xyz), _p(tets), len(tets), _p(edges), _p(t10))
    return edges[:ne].copy(), t10


class Peak(C.Structure):
    """elastic_tet.rs:367-427 ``Peak`` of 1 part (the layout of ``femgpu_peak``)."""
    _fields_ = [("mises", C.c_double), ("element", C.c_int64), ("local", C.c_int32),
                ("point", C.c_uint32), ("singular", C.c_int32), ("pad", C.c_int32),
                ("regular_mises", C.c_double), ("regular_element", C.c_int64),
                ("regular_local", C.c_int32), ("regular_point", C.c_uint32)]


def hex8_element(size, c, alpha=(0.0, 0.0, 0.0)):
    """hex.rs:218-309: (k (24, 24), load (24, 8), mode_u (9, 24), mode_t (9, 8)) of a box
    cell."""
    size, c, alpha = (np.ascontiguousarray(v, dtype=np.float64) for v in (size, c, alpha))
    k, load, mu, mt = np.empty(576), np.empty(192), np.empty(216), np.empty(72)
    err = C.create_string_buffer(512)
    if _lib.orc_hex8_element(_p(size), _p(c), _p(alpha), _p(k), _p(load), _p(mu), _p(mt), err,
                             512):
        raise OracleError(err.value.decode())
    return k.reshape(24, 24), load.reshape(24, 8), mu.reshape(9, 24), mt.reshape(9, 8)


def symbolic_counts(a: Csr, xyz):
    """symbolic.rs:162-182 (entries, flops) of the factor of ``a`` in the nested dissection
    order of ``xyz`` (order.rs:19-198)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    e, f = C.c_uint64(), C.c_double()
    _lib.orc_symbolic_counts(a.h, _p(xyz), C.byref(e), C.byref(f))
    return e.value, f.value


def hex8_mass(size, density):
    """hex.rs:337-353: the 24 x 24 consistent mass of a box cell."""
    size = np.ascontiguousarray(size, dtype=np.float64)
    m = np.empty(576)
    _lib.orc_hex8_mass(_p(size), float(density), _p(m))
    return m.reshape(24, 24)


def hex_loads(xyz, hexes, coef, *, expansion=None, accel=None, dtemp=None):
    """elastic.rs:386-405: the thermal forces (load T) and the volume forces (accel, the
    density times gravity plus the body force per unit volume, per cell) of the box cells, summed
    over the cells in order: 3 values per point."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    hexes = np.ascontiguousarray(hexes, dtype=np.uint32)
    coef = np.ascontiguousarray(coef, dtype=np.float64)
    opt = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
    force = np.empty(3 * len(xyz))
    err = C.create_string_buffer(512)
    if _lib.orc_hex_loads(len(xyz), _p(xyz), len(hexes), _p(hexes), _p(coef),
                          _p(opt(expansion)), _p(opt(accel)), _p(opt(dtemp)), _p(force), err,
                          512):
        raise OracleError(err.value.decode())
    return force


def hex8_strain_stress(size, c, xi, u, t, alpha=(0.0, 0.0, 0.0)):
    """hex.rs:311-335: (engineering strain, stress), both xx, yy, zz, yz, xz, xy."""
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (size, c, alpha, xi, u, t)]
    e, s = np.empty(6), np.empty(6)
    err = C.create_string_buffer(512)
    if _lib.orc_hex8_strain_stress(*[_p(v) for v in a], _p(e), _p(s), err, 512):
        raise OracleError(err.value.decode())
    return e, s


def recover(xyz, tets10, coef, u, *, expansion=None, dtemp=None, part=None, nparts=1,
            singular=None, hex=False):
    """elastic_tet.rs:367-427 and 482-483: the mean strain and stress at each point of the
    quadratic mesh, their von Mises and principal stresses, and the peaks of each part. Returns a
    dict of arrays: stress (n, 6), strain (n, 6), mises (n,), principal (n, 3), peaks (list).
    ``hex``: the box grid's loop (elastic.rs:615-660) over box cells (``tets10`` then holds 8
    corners per cell and ``coef`` 9 orthotropic constants per cell)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    t10 = np.ascontiguousarray(tets10, dtype=np.uint32)
    coef = np.ascontiguousarray(coef, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    opt = lambda a, t: None if a is None else np.ascontiguousarray(a, dtype=t)
    expansion, dtemp = opt(expansion, np.float64), opt(dtemp, np.float64)
    part, singular = opt(part, np.uint32), opt(singular, np.uint8)
    n = len(xyz)
    stress, strain = np.empty((n, 6)), np.empty((n, 6))
    mises, principal = np.empty(n), np.empty((n, 3))
    peaks = (Peak * nparts)()
    err = C.create_string_buffer(512)
    fn = _lib.orc_recover_hex if hex else _lib.orc_recover
    st = fn(n, _p(xyz), len(t10), _p(t10), _p(coef), _p(expansion), _p(dtemp),
            _p(u), _p(part), nparts, _p(singular), _p(stress), _p(strain),
            _p(mises), _p(principal), C.cast(peaks, C.c_void_p), err, 512)
    if st:
        raise OracleError(err.value.decode())
    return {"stress": stress, "strain": strain, "mises": mises, "principal": principal,
            "peaks": list(peaks)}


def colour(n, elements):
    e = np.ascontiguousarray(elements, dtype=np.uint32)
    out = np.empty(e.shape[0], np.uint32)
    nc = _lib.orc_colour(n, _p(e), e.shape[0], e.shape[1], _p(out))
    return out, nc


class Rect:
    """sparse.rs:202-293, held by the oracle library."""

    def __init__(self, handle):
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None):
            _lib.orc_rect_free(self.h)
            self.h = None

    @classmethod
    def from_arrays(cls, rows, cols, ptr, idx, val):
        ptr = np.ascontiguousarray(ptr, dtype=np.int64)
        idx = np.ascontiguousarray(idx, dtype=np.uint32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        return cls(_lib.orc_rect_import(rows, cols, _p(ptr), _p(idx), _p(val)))

    @property
    def shape(self):
        r, c, nnz = C.c_size_t(), C.c_size_t(), C.c_size_t()
        _lib.orc_rect_info(self.h, C.byref(r), C.byref(c), C.byref(nnz))
        return r.value, c.value, nnz.value

    def arrays(self):
        r, _, nnz = self.shape
        ptr = np.empty(r + 1, np.int64)
        idx = np.empty(nnz, np.uint32)
        val = np.empty(nnz, np.float64)
        _lib.orc_rect_export(self.h, _p(ptr), _p(idx), _p(val))
        return ptr, idx, val

    def mul(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.shape[0])
        _lib.orc_rect_mul(self.h, _p(x), _p(y))
        return y

    def mul_transpose(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.shape[1])
        _lib.orc_rect_mul_transpose(self.h, _p(x), _p(y))
        return y

    def galerkin(self, a: Csr) -> Csr:
        return Csr(_lib.orc_galerkin(self.h, a.h))


def _level_args(planes, points, comp):
    px, py, pz = (np.ascontiguousarray(p, dtype=np.float64) for p in planes)
    pts = np.ascontiguousarray(points, dtype=np.uint32)
    cmp_ = np.ascontiguousarray(comp, dtype=np.uint8)
    return (px, py, pz, pts, cmp_)


def coarsen(a: Csr, planes, points, comp):
    """multigrid.rs:329-452: (P, coarse points, coarse comp) or None."""
    px, py, pz, pts, cmp_ = _level_args(planes, points, comp)
    n = len(pts)
    cp = np.empty((n, 3), np.uint32)
    cc = np.empty(n, np.uint8)
    cn = C.c_size_t()
    h = _lib.orc_coarsen(a.h, _p(px), len(px), _p(py), len(py), _p(pz), len(pz), _p(pts),
                         _p(cmp_), n, _p(cp), _p(cc), C.byref(cn))
    if not h:
        return None
    return Rect(h), cp[:cn.value].copy(), cc[:cn.value].copy()


def by_cells(a: Csr, planes, points, comp, cells):
    """multigrid.rs:458-608 after coarsen: (coarse matrix, coarse points, coarse comp) or None.
    ``cells`` as for Solver."""
    px, py, pz, pts, cmp_ = _level_args(planes, points, comp)
    n = len(pts)
    origin = np.ascontiguousarray(cells[0], dtype=np.uint32)
    cls = np.ascontiguousarray(cells[1], dtype=np.uint32)
    table = np.ascontiguousarray(cells[2], dtype=np.float64)
    cp = np.empty((n, 3), np.uint32)
    cc = np.empty(n, np.uint8)
    cn = C.c_size_t()
    h = _lib.orc_by_cells(a.h, _p(px), len(px), _p(py), len(py), _p(pz), len(pz), _p(pts),
                          _p(cmp_), n, len(origin), _p(origin), _p(cls), _p(table),
                          table.size // 576, _p(cp), _p(cc), C.byref(cn))
    if not h:
        return None
    return Csr(h), cp[:cn.value].copy(), cc[:cn.value].copy()


def prolongation(points, corners, edges, free):
    """pmultigrid.rs:104-151: (P, coarse xyz)."""
    pts = np.ascontiguousarray(points, dtype=np.float64)
    e = np.ascontiguousarray(edges, dtype=np.uint32)
    f = np.ascontiguousarray(free, dtype=np.int64)
    cxyz = np.empty((len(f), 3))
    nc = C.c_size_t()
    h = _lib.orc_prolongation(_p(pts), len(pts), corners, _p(e), len(e), _p(f), len(f),
                              _p(cxyz), C.byref(nc))
    return Rect(h), cxyz[:nc.value].copy()


def nested_dissection(a: Csr, xyz):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    out = np.empty(a.n, np.int64)
    _lib.orc_nested_dissection(a.h, _p(xyz), _p(out))
    return out


def direct_solve(a: Csr, xyz, b):
    """The FP64 direct oracle: nested dissection, symbolic analysis and the multifrontal
    Cholesky factor (order.rs, symbolic.rs, cholesky.rs). Returns (x, factor entries)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    x = np.array(b, dtype=np.float64, copy=True)
    entries = C.c_uint64()
    err = C.create_string_buffer(512)
    if _lib.orc_direct_solve(a.h, _p(xyz), _p(x), C.byref(entries), err, 512):
        raise OracleError(err.value.decode())
    return x, entries.value


_PRE = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)


def pcg(a: Csr, b, x, precondition=None, tol=1e-10, max_iter=500, cancel=None):
    """multigrid.rs:692-753: x (numpy, updated in place) from its start value; precondition(r,
    z) writes z = M^-1 r into the numpy array z (None: z = r). Returns (iterations, residual)."""
    b = np.ascontiguousarray(b, dtype=np.float64)

    def call(r, z, n, _ctx):
        zr = np.ctypeslib.as_array(C.cast(z, C.POINTER(C.c_double)), shape=(n,))
        rr = np.ctypeslib.as_array(C.cast(r, C.POINTER(C.c_double)), shape=(n,))
        precondition(rr.copy(), zr)

    cb = _PRE(call) if precondition is not None else _PRE()
    it, res = C.c_size_t(), C.c_double()
    err = C.create_string_buffer(512)
    flag = C.byref(cancel) if cancel is not None else None
    if _lib.orc_pcg(a.h, _p(b), _p(x), cb, None, tol, max_iter, flag, C.byref(it),
                    C.byref(res), err, 512):
        raise OracleError(err.value.decode())
    return it.value, res.value


class Solver:
    """solve.rs:58-250. ``kind``: 'grid' (planes, points, comp), 'points' (xyz) or
    'quadratic' (xyz, p: Rect, coarse xyz). ``method``: None, 'direct' or 'multigrid'."""

    def __init__(self, a: Csr, kind, *, planes=None, points=None, comp=None, xyz=None, p=None,
                 coarse=None, method=None, crossover=("unknowns", 3000), cells=None):
        """``cells`` (grid only, multigrid.rs:62-68): (origin (C, 3) the lowest grid point of
        each cell, cls (C,) its class, matrices (K, 24, 24) of the classes); the coarse
        matrices then come from the cells (multigrid.rs:458-608)."""
        err = C.create_string_buffer(512)
        nce = ncl = 0
        origin = cls = table = None
        if cells is not None:
            origin = np.ascontiguousarray(cells[0], dtype=np.uint32)
            cls = np.ascontiguousarray(cells[1], dtype=np.uint32)
            table = np.ascontiguousarray(cells[2], dtype=np.float64)
            nce, ncl = len(origin), table.size // 576
        k = {"grid": 0, "points": 1, "quadratic": 2}[kind]
        m = {None: -1, "direct": 0, "multigrid": 1}[method]
        px = py = pz = pts = cmp_ = xyz_ = cx = None
        nx = ny = nz = 0
        if k == 0:
            px, py, pz, pts, cmp_ = _level_args(planes, points, comp)
            nx, ny, nz = len(px), len(py), len(pz)
        if k >= 1:
            xyz_ = np.ascontiguousarray(xyz, dtype=np.float64)
        nc = 0
        if k == 2:
            cx = np.ascontiguousarray(coarse, dtype=np.float64)
            nc = len(cx)
        if crossover[0] == "unknowns":
            fr, un, fl, en, flat = 0, crossover[1], 0.0, 0, 0
        else:
            fr, un = 1, 0
            fl, en, flat = crossover[1], crossover[2], int(crossover[3])
        self.h = _lib.orc_solver_new(a.h, k, _p(px), nx, _p(py), ny, _p(pz), nz, _p(pts),
                                     _p(cmp_), _p(xyz_), p.h if p is not None else None, _p(cx),
                                     nc, m, fr, un, fl, en, flat, nce, _p(origin), _p(cls),
                                     _p(table), ncl, err, 512)
        if not self.h:
            raise OracleError(err.value.decode())
        self.n = a.n

    def __del__(self):
        if getattr(self, "h", None):
            _lib.orc_solver_free(self.h)
            self.h = None

    def method(self):
        return ["direct", "multigrid"][_lib.orc_solver_method(self.h)]

    def levels(self):
        return [_lib.orc_solver_level_size(self.h, i)
                for i in range(_lib.orc_solver_levels(self.h))]

    def level_matrix(self, level):
        """The matrix of multigrid level ``level`` (0 = the system's)."""
        h = _lib.orc_solver_level_matrix(self.h, level)
        if not h:
            raise OracleError(f"no multigrid level {level}")
        return Csr(h)

    def solve(self, b, x=None, tol=0.0, max_iter=0, cancel=None):
        """Returns (x, iterations, residual); raises OracleError with the reference text."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x is None else np.array(x, dtype=np.float64, copy=True)
        it, res = C.c_size_t(), C.c_double()
        err = C.create_string_buffer(512)
        flag = None
        if cancel is not None:
            flag = C.c_int(int(cancel))
        st = _lib.orc_solver_solve(self.h, _p(b), _p(x), tol, max_iter,
                                   C.byref(flag) if flag is not None else None, C.byref(it),
                                   C.byref(res), err, 512)
        if st:
            raise OracleError(err.value.decode())
        return x, it.value, res.value

    def precondition(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros(self.n)
        _lib.orc_solver_precondition(self.h, _p(r), _p(z))
        return z


def transient_energy(kt, rate, load, fixed):
    """heat.rs:535-547 for a transient step with no radiation, summed in point order: (stored,
    fixed, the sum of |rate| and |q| over the points)."""
    kt, rate, load = (np.ascontiguousarray(a, dtype=np.float64) for a in (kt, rate, load))
    fixed = np.ascontiguousarray(fixed, dtype=np.uint8)
    out = np.empty(3)
    _lib.orc_transient_energy(len(kt), _p(kt), _p(rate), _p(load), _p(fixed), _p(out))
    return tuple(out)


def transient(k, capacity, dt, free, load, t0, steps, make_solver, output_every=1, tol=1e-10):
    """heat.rs:686-733: backward Euler with the lumped capacity. ``k`` is the full conductivity
    matrix (a Csr), ``make_solver(a)`` the solver of the free unknowns of K + C/dt. Returns the
    temperatures and the energies (stored, fixed, |rate| + |q| summed) of the steps s with
    s % output_every == 0 or s == steps, and the PCG iterations of all steps."""
    n = k.n
    ptr, idx, val = k.arrays()
    a_full = Csr.from_arrays(n, ptr, idx, val)
    a_full.add_capacity(capacity, dt)
    solver = make_solver(a_full.submatrix(free))
    capacity = np.asarray(capacity, dtype=np.float64)
    t = np.array(t0, dtype=np.float64, copy=True)
    x = t[free].copy()
    fixed = np.ones(n, np.uint8)
    fixed[free] = 0
    frames, energies, iterations = [], [], 0
    for s in range(1, steps + 1):
        previous = t.copy()
        rhs = a_full.reduced_rhs_transient(load, t, free, capacity, dt)
        x, it, _ = solver.solve(rhs, x, tol=tol)
        iterations += it
        t[free] = x
        kt = k.mul(t)
        rate = capacity * (t - previous) / dt
        if s % max(output_every, 1) == 0 or s == steps:
            frames.append(t.copy())
            energies.append(transient_energy(kt, rate, load, fixed))
    return frames, energies, iterations


def dense_jacobi(a):
    """eigen.rs:274-331: (ascending eigenvalues, eigenvectors as columns) of a symmetric matrix."""
    a = np.array(a, dtype=np.float64, copy=True)
    n = a.shape[0]
    values, v = np.empty(n), np.empty((n, n))
    _lib.orc_dense_jacobi(_p(a), n, _p(values), _p(v))
    return values, v


def dense_generalized(k, m):
    """eigen.rs:183-269: K q = lambda M q, ascending, with Q^T M Q = I."""
    k = np.ascontiguousarray(k, dtype=np.float64)
    m = np.ascontiguousarray(m, dtype=np.float64)
    n = k.shape[0]
    values, q = np.empty(n), np.empty((n, n))
    err = C.create_string_buffer(512)
    if _lib.orc_dense_generalized(_p(k), _p(m), n, _p(values), _p(q), err, 512):
        raise OracleError(err.value.decode())
    return values, q


EIGEN_TOL = 1e-6   # eigen.rs:34
EIGEN_MAX_ITER = 120  # eigen.rs:40
MODES_SHIFT = 1e-8  # modes.rs:93


def subspace_vectors(n, count):
    """eigen.rs:48-50"""
    return min(max(2 * count, count + 8), n)


def start_vectors(mdiag, p):
    """eigen.rs:96-113: the diagonal of M, then xorshift vectors (seed 0x9e3779b97f4a7c15)."""
    n = len(mdiag)
    x = np.empty((p, n))
    x[0] = mdiag
    seed = 0x9E3779B97F4A7C15
    mask = (1 << 64) - 1
    for j in range(1, p):
        for i in range(n):
            seed ^= (seed << 13) & mask
            seed ^= seed >> 7
            seed ^= (seed << 17) & mask
            x[j, i] = (seed >> 11) / float(1 << 53) - 0.5
    return x


def subspace(k, m, shift, count, solve):
    """eigen.rs:81-177 with ``k``, ``m`` oracle Csr and ``solve(b, x0) -> x`` the solve of
    (K - shift M) x = b from the start value x0. Returns (values, vectors (count, n),
    iterations)."""
    n = k.n
    if count == 0 or count > n:
        raise OracleError(f"the model has {n} unknowns, so it has 1 to {n} modes, not {count}")
    p = subspace_vectors(n, count)
    ptr, idx, val = m.arrays()
    mdiag = np.zeros(n)
    for i in range(n):
        for e in range(ptr[i], ptr[i + 1]):
            if idx[e] == i:
                mdiag[i] = val[e]
    x = start_vectors(mdiag, p)
    mu = None
    for iteration in range(1, EIGEN_MAX_ITER + 1):
        y = np.stack([m.mul(x[j]) for j in range(p)])
        bar = np.stack([solve(y[j], x[j] / mu[j] if mu is not None else np.zeros(n))
                        for j in range(p)])
        mb = np.stack([m.mul(bar[j]) for j in range(p)])
        kr = 0.5 * (bar @ y.T + (bar @ y.T).T)
        mr = bar @ mb.T  # eigen.rs:140-146 forms i <= j and mirrors it
        mr = np.triu(mr) + np.triu(mr, 1).T
        converged = iteration > 1 and all(
            np.sqrt(max(1.0 - kr[i, i] ** 2 / mr[i, i], 0.0)) <= EIGEN_TOL for i in range(count))
        mu, q = dense_generalized(kr, mr)
        x = q.T @ bar
        if converged:
            return mu[:count] + shift, x[:count], iteration
    raise OracleError(f"the subspace iteration did not converge in {EIGEN_MAX_ITER} iterations:"
                      " ask for fewer modes")

