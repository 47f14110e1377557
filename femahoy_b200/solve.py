"""The linear solver of a model (crates/fem/src/solve.rs) on the device.

``Solver(a, unknowns, method, crossover)`` and ``Solver.solve(b, x, cancelled)`` keep the
reference's arguments, defaults, errors and reuse across right sides; ``Unknowns.Grid``,
``Unknowns.Points`` and ``Unknowns.Quadratic`` are solve.rs:64-77; ``Level`` is
multigrid.rs:55-59; ``Crossover`` solve.rs:28-39; ``Method`` solve.rs:47-50; ``Stats``
solve.rs:81-86. The extra keyword ``precision`` picks the plain FP64 form or the mixed form
(FP32 V-cycle inside FP64 flexible CG).
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .sparse import Csr, Rect

STEADY_DIRECT_LIMIT = 3_000  # solve.rs:18
TRANSIENT_DIRECT_LIMIT = 40_000  # solve.rs:24
PCG_TOL = 1e-10  # solve.rs:42
PCG_MAX_ITER = 500  # solve.rs:43


class Method(enum.IntEnum):
    """solve.rs:47-50"""

    Direct = 0
    Multigrid = 1


class Crossover:
    """solve.rs:28-39"""

    def __init__(self, rule, unknowns=0, flops=0.0, entries=0, flat=False):
        self.rule, self.unknowns, self.flops, self.entries, self.flat = (rule, unknowns, flops,
                                                                          entries, flat)

    @classmethod
    def Unknowns(cls, n):
        return cls(0, unknowns=n)

    @classmethod
    def Flops(cls, flops, entries, flat):
        return cls(1, flops=flops, entries=entries, flat=flat)

    def _c(self):
        return L.Crossover_t(self.rule, self.unknowns, self.flops, self.entries, int(self.flat))


@dataclass
class Level:
    """multigrid.rs:55-59: the planes of each axis, and the grid point and the component of
    each unknown."""

    planes: list
    points: np.ndarray  # (n, 3) uint32
    comp: np.ndarray  # (n,) uint8


@dataclass
class Unknowns:
    """solve.rs:64-77"""

    kind: int
    level: Level | None = None
    points: np.ndarray | None = None
    p: Rect | None = None
    coarse: np.ndarray | None = None
    coarse_comp: np.ndarray | None = None

    @classmethod
    def Grid(cls, level: Level):
        return cls(0, level=level)

    @classmethod
    def Points(cls, xyz):
        return cls(1, points=np.asarray(xyz, dtype=np.float64))

    @classmethod
    def Quadratic(cls, points, p: Rect, coarse, coarse_comp=None):
        return cls(2, points=np.asarray(points, dtype=np.float64), p=p,
                   coarse=np.asarray(coarse, dtype=np.float64), coarse_comp=coarse_comp)


@dataclass
class Stats:
    """solve.rs:81-86: the PCG iterations (0 for the direct solver) and |b - A x| / |b| by the
    reference's definition (the recurrence residual of PCG). ``true_residual`` is recomputed in
    FP64 on the device; ``seconds`` is the device time of the solve."""

    iterations: int
    residual: float
    true_residual: float = 0.0
    seconds: float = 0.0
    launches: int = 0


@dataclass
class Options:
    """This library's own knobs; zeros choose the defaults."""

    precision: int = L.FP64
    degree: int = 0
    lower: float = 0.0
    sell_c: int = 0
    coarsest: int = 0
    max_levels: int = 0
    graph: int = 0
    format: int = 0  # 0: stencil where the level allows it, else SELL-C; 1: SELL-C only
    tail: int = 0    # > 0: levels of at most this many rows run as 1 fused kernel (0: none)
    launch: int = 0  # 0: programmatic dependent launch in the PCG loop; 1: plain launches
    values: int = 0  # mixed form: 0 default, 1 FP32, 2 FP16 stencils, 3 FP16 coarsest inverse
    tiles: int = 0   # finest FP32 stencil steps from bulk-copied tiles: 0 tuned, 1 off, 2 on
    axes: int = 0    # the axes the coarsening halves (bits x 1, y 2, z 4; 0: all)
    stencil: int = 0  # stencil kernel: 0 tuned, 1 runtime K, 2 compile-time K, 3 2 rows, 4 march
    smoother: int = 0  # Chebyshev polynomial: 0 the default, 1 the first kind, 4 the fourth
    cluster: int = 0  # small levels: 1 each leg as 1 cluster launch, 0 a launch per step
    l2: int = 0      # 1: the coarsest inverse persisting in L2
    upper: float = 0.0  # Chebyshev interval upper end over lambda_max (0: 1.1)

    def _c(self):
        return L.Options_t(self.precision, self.degree, self.lower, self.sell_c, 0, self.coarsest,
                           self.max_levels, self.graph, self.format, self.tail, self.launch,
                           self.values, self.tiles, self.axes, self.stencil, self.smoother,
                           self.cluster, self.l2, self.upper)


def unknowns_c(unknowns: "Unknowns", keep: list) -> L.Unknowns_t:
    """The femgpu_unknowns of ``unknowns``; the arrays it points into are appended to ``keep``,
    which must outlive the call that reads it."""
    u = L.Unknowns_t()
    u.kind = unknowns.kind
    if unknowns.kind == 0:
        lv = unknowns.level
        planes = [L.arr(p, np.float64) for p in lv.planes]
        pts = L.arr(lv.points, np.uint32).reshape(-1, 3)
        comp = L.arr(lv.comp, np.uint8)
        keep += planes + [pts, comp]
        for d in range(3):
            u.planes[d] = planes[d].ctypes.data
            u.nplanes[d] = len(planes[d])
        u.points = pts.ctypes.data
        u.comp = comp.ctypes.data
    else:
        xyz = L.arr(unknowns.points, np.float64).reshape(-1, 3)
        keep.append(xyz)
        u.xyz = xyz.ctypes.data
    if unknowns.kind == 2:
        p = unknowns.p
        pp, pi, pv = L.arr(p.ptr, np.int64), L.arr(p.idx, np.uint32), L.arr(p.val, np.float64)
        cx = L.arr(unknowns.coarse, np.float64).reshape(-1, 3)
        keep += [pp, pi, pv, cx]
        u.p_cols = p.cols
        u.p_ptr, u.p_idx, u.p_val = pp.ctypes.data, pi.ctypes.data, pv.ctypes.data
        u.coarse_xyz = cx.ctypes.data
        if unknowns.coarse_comp is not None:
            cc = L.arr(unknowns.coarse_comp, np.uint8)
            keep.append(cc)
            u.coarse_comp = cc.ctypes.data
    return u


@dataclass
class Cells:
    """multigrid.rs:62-68: the box cells of a displacement model on grid unknowns, each by its
    lowest grid point ``origin`` (C, 3) and the class ``cls`` (C,) of its 24 x 24 matrix among
    ``matrices`` (K, 24, 24) (unknown 3 n + c for corner n in VTK order)."""

    origin: np.ndarray
    cls: np.ndarray
    matrices: np.ndarray
    mass: np.ndarray | None = None  # the classes' consistent masses, for the modes

    def _c(self, keep):
        o = L.arr(self.origin, np.uint32).reshape(-1, 3)
        c = L.arr(self.cls, np.uint32).ravel()
        m = L.arr(self.matrices, np.float64).reshape(-1, 576)
        w = None if self.mass is None else L.arr(self.mass, np.float64).reshape(-1, 576)
        keep += [o, c, m, w]
        return L.Cells_t(len(o), o.ctypes.data, c.ctypes.data, m.ctypes.data, len(m),
                         None if w is None else w.ctypes.data)


def hex_mass(sizes, density):
    """hex::mass (hex.rs:337-353) of each box cell: ``sizes`` (K, 3), ``density`` (K,). Returns
    (K, 24, 24)."""
    s = L.arr(sizes, np.float64).reshape(-1, 3)
    d = L.arr(density, np.float64).ravel()
    out = np.empty((len(s), 24, 24))
    L.check(L.lib().femgpu_hex_mass(len(s), s.ctypes.data, d.ctypes.data, out.ctypes.data))
    return out


def hex_elements(keys):
    """Hex::new (hex.rs:218-297) on the device for each row of ``keys`` (K, 12): the 3 sides and
    the 9 orthotropic constants of a box cell. Returns (K, 24, 24)."""
    k = L.arr(keys, np.float64).reshape(-1, 12)
    out = np.empty((len(k), 24, 24))
    L.check(L.lib().femgpu_hex_elements(len(k), k.ctypes.data, out.ctypes.data))
    return out


def symbolic_counts(a: Csr, unknowns: Unknowns):
    """(entries, flops) of the sparse Cholesky factor of ``a`` in the nested dissection order of
    the unknowns' points (order.rs, symbolic.rs): what Crossover.Flops compares."""
    keep = []
    u = unknowns_c(unknowns, keep)
    e, f = C.c_uint64(), C.c_double()
    L.check(L.lib().femgpu_symbolic_counts(a.handle, C.byref(u), C.byref(e), C.byref(f)))
    return e.value, f.value


def coarse_matrix(a: Csr, unknowns: Unknowns, level: int, cells: Cells | None = None):
    """The matrix (ptr, idx, val) of multigrid level ``level`` as the solver forms it (the
    Galerkin products, or with ``cells`` the cell-condensed matrices), and the grid point (3
    plane indices) and component of each of its unknowns, which are numbered in grid order (z,
    y, x, component): (ptr, idx, val, points, comp)."""
    keep = []
    u = unknowns_c(unknowns, keep)
    cc = C.byref(cells._c(keep)) if cells is not None else None
    n, nnz = C.c_size_t(), C.c_size_t()
    L.check(L.lib().femgpu_coarse_matrix(a.handle, C.byref(u), cc, level, C.byref(n),
                                         C.byref(nnz), None, None, None, None, None))
    ptr = np.empty(n.value + 1, np.int64)
    idx = np.empty(nnz.value, np.uint32)
    val = np.empty(nnz.value, np.float64)
    pts = np.empty((n.value, 3), np.uint32)
    comp = np.empty(n.value, np.uint8)
    L.check(L.lib().femgpu_coarse_matrix(a.handle, C.byref(u), cc, level, C.byref(n),
                                         C.byref(nnz), ptr.ctypes.data, idx.ctypes.data,
                                         val.ctypes.data, pts.ctypes.data, comp.ctypes.data))
    return ptr, idx, val, pts, comp


class Solver:
    """solve.rs:58-250 on the device."""

    def __init__(self, a: Csr, unknowns: Unknowns, method: Method | None = None,
                 crossover: Crossover | None = None, cells: Cells | None = None, *,
                 precision=L.FP64, options: Options | None = None):
        crossover = crossover or Crossover.Unknowns(STEADY_DIRECT_LIMIT)
        opts = options or Options()
        opts.precision = precision if options is None else opts.precision
        keep = []  # arrays that must live through the call
        u = unknowns_c(unknowns, keep)
        n = a.n
        m = -1 if method is None else int(method)
        h = C.c_void_p()
        cr = crossover._c()
        oc = opts._c()
        cc = C.byref(cells._c(keep)) if cells is not None else None
        L.check(L.lib().femgpu_solver_new_cells(a.handle, C.byref(u), m, C.byref(cr),
                                                C.byref(oc), cc, C.byref(h)))
        self._h = h.value
        self.n = n

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and not getattr(self, "_owner", None):
            L.lib().femgpu_solver_free(h)
            self._h = None

    @classmethod
    def _borrowed(cls, handle, n, owner):
        """The solver of another handle (a transient loop's), freed with its owner."""
        s = cls.__new__(cls)
        s._h, s.n, s._owner = handle, n, owner
        return s

    @property
    def handle(self):
        return self._h

    def with_max_iter(self, max_iter):
        """solve.rs:187-189"""
        L.check(L.lib().femgpu_solver_set_max_iter(self._h, max_iter))
        return self

    def with_tol(self, tol):
        L.check(L.lib().femgpu_solver_set_tol(self._h, tol))
        return self

    def method(self) -> Method:
        """solve.rs:191-196"""
        return Method(L.lib().femgpu_solver_method(self._h))

    def levels(self):
        sizes = (C.c_size_t * 64)()
        k = L.lib().femgpu_solver_levels(self._h, sizes, 64)
        return [sizes[i] for i in range(k)]

    def device_bytes(self):
        return L.lib().femgpu_solver_bytes(self._h)

    def breakdown(self):
        """The device time of each kernel of 1 PCG iteration (overwrites the solver's vectors)."""
        buf = C.create_string_buffer(16384)
        L.lib().femgpu_solver_breakdown(self._h, buf, 16384)
        return buf.value.decode()

    def describe(self):
        """The levels, their storage formats and the kernels the autotuner chose."""
        buf = C.create_string_buffer(8192)
        L.lib().femgpu_solver_describe(self._h, buf, 8192)
        return buf.value.decode()

    def solve(self, b, x=None, cancelled=None) -> Stats:
        """solve.rs:199-250: solve A x = b; ``x`` (numpy, updated in place) holds the start
        value. ``cancelled`` is a callable or a ctypes int flag read before each iteration;
        a set flag raises FemError("cancelled")."""
        b = L.arr(b, np.float64)
        if x is None:
            x = np.zeros(self.n)
        if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
            raise TypeError("x must be a contiguous float64 numpy array (it gets the solution)")
        flag = None
        if isinstance(cancelled, C.c_int):
            flag = C.byref(cancelled)
        elif callable(cancelled) and cancelled():
            flag = C.byref(C.c_int(1))
        st = L.Stats_t()
        L.check(L.lib().femgpu_solver_solve(self._h, L.ptr(b), L.ptr(x), flag, C.byref(st)))
        return Stats(st.iterations, st.residual, st.true_residual, st.seconds, st.launches)

    def solve_zero(self, b, x=None, cancelled=None) -> Stats:
        """``solve`` from x = 0 (the start value of the reference's steady callers): ``x`` only
        gets the solution, so its start value is not copied to the device."""
        b = L.arr(b, np.float64)
        if x is None:
            x = np.empty(self.n)
        if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
            raise TypeError("x must be a contiguous float64 numpy array (it gets the solution)")
        flag = C.byref(cancelled) if isinstance(cancelled, C.c_int) else None
        st = L.Stats_t()
        L.check(L.lib().femgpu_solver_solve_zero(self._h, L.ptr(b), L.ptr(x), flag,
                                                 C.byref(st)))
        return Stats(st.iterations, st.residual, st.true_residual, st.seconds, st.launches)

    def solve_device(self, b_ptr: int, x_ptr: int, cancel=None) -> Stats:
        """The same on device vectors (raw CUDA pointers, e.g. torch ``data_ptr()``)."""
        st = L.Stats_t()
        flag = C.byref(cancel) if isinstance(cancel, C.c_int) else None
        L.check(L.lib().femgpu_solver_solve_device(self._h, C.c_void_p(b_ptr), C.c_void_p(x_ptr),
                                                   flag, C.byref(st)))
        return Stats(st.iterations, st.residual, st.true_residual, st.seconds, st.launches)


def prolongation(points, corners, edges, free):
    """pmultigrid.rs:104-151: (P, coarse points) from the free corner unknowns of a quadratic
    mesh to its free unknowns."""
    pts = L.arr(points, np.float64)
    e = L.arr(edges, np.uint32)
    f = L.arr(free, np.int64)
    nnz, nc = C.c_size_t(), C.c_size_t()
    lib = L.lib()
    L.check(lib.femgpu_prolongation(len(pts), L.ptr(pts), corners, len(e), L.ptr(e), len(f),
                                    L.ptr(f), C.byref(nnz), C.byref(nc), None, None, None, None))
    ptr = np.empty(len(f) + 1, np.int64)
    idx = np.empty(nnz.value, np.uint32)
    val = np.empty(nnz.value, np.float64)
    cx = np.empty((nc.value, 3))
    L.check(lib.femgpu_prolongation(len(pts), L.ptr(pts), corners, len(e), L.ptr(e), len(f),
                                    L.ptr(f), C.byref(nnz), C.byref(nc), L.ptr(ptr), L.ptr(idx),
                                    L.ptr(val), L.ptr(cx)))
    return Rect(len(f), nc.value, ptr, idx, val), cx


def reduced_rhs(a: Csr, load, t, free):
    """heat.rs:1219-1244 (steady): the right side of the free unknowns."""
    load = L.arr(load, np.float64)
    t = L.arr(t, np.float64)
    f = L.arr(free, np.int64)
    out = np.empty(len(f))
    L.check(L.lib().femgpu_reduced_rhs(a.handle, L.ptr(load), L.ptr(t), L.ptr(f), len(f),
                                       L.ptr(out)))
    return out


class Quadratic:
    """tet10.rs:232-272: the quadratic mesh of a mesh of 4-node tetrahedra, numbered on the
    device in the reference's order."""

    def __init__(self, points, corners, edges, tets):
        self.points, self.corners, self.edges, self.tets = points, corners, edges, tets

    @classmethod
    def new(cls, points, tets):
        pts = np.asarray(points, dtype=np.float64)
        t = L.arr(tets, np.uint32)
        t10 = np.empty((len(t), 10), np.uint32)
        edges = np.empty((6 * len(t), 2), np.uint32)
        ne = C.c_size_t()
        L.check(L.lib().femgpu_quadratic(len(pts), len(t), L.ptr(t), L.ptr(t10), L.ptr(edges),
                                         C.byref(ne)))
        edges = edges[:ne.value].copy()
        mid = 0.5 * (pts[edges[:, 0]] + pts[edges[:, 1]])
        return cls(np.concatenate([pts, mid]), len(pts), edges, t10)


@dataclass
class Convergence:
    """multigrid.rs:680-686: the iterations and |b - A x| / |b| at the end."""
    iterations: int
    residual: float


def pcg(a: Csr, b, x, precondition=None, tol=PCG_TOL, max_iter=PCG_MAX_ITER,
        cancelled=None) -> Convergence:
    """multigrid::pcg (multigrid.rs:692-753): conjugate gradients from the start value in ``x``
    (numpy, updated in place, the last iterate also on failure) with the preconditioner
    ``precondition(r, z)`` (numpy arrays; it writes z = M^-1 r), None for z = r. ``cancelled``
    is a ctypes int flag read before each step (or a callable read once). Raises FemError with
    the reference's texts."""
    b = L.arr(b, np.float64)
    if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
        raise TypeError("x must be a contiguous float64 numpy array (it gets the solution)")
    failure = []

    def call(r, z, n, _ctx):
        try:
            zr = np.ctypeslib.as_array(z, shape=(n,))
            precondition(np.ctypeslib.as_array(r, shape=(n,)).copy(), zr)
        except BaseException as e:  # noqa: BLE001 - reported after the call
            failure.append(e)

    cb = L.PRECONDITION_FN(call) if precondition is not None else L.PRECONDITION_FN()
    flag = None
    if isinstance(cancelled, C.c_int):
        flag = C.byref(cancelled)
    elif callable(cancelled) and cancelled():
        flag = C.byref(C.c_int(1))
    out = L.Convergence_t()
    status = L.lib().femgpu_pcg(a.handle, L.ptr(b), L.ptr(x), cb, None, float(tol),
                                int(max_iter), flag, C.byref(out))
    if failure:
        raise failure[0]
    L.check(status)
    return Convergence(out.iterations, out.residual)
