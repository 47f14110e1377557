"""The reference's prism meshes (crates/fem/src/prism.rs, mesh2d.rs, grid.rs axis_planes) on the
C ABI: footprints (polygons and circles with holes) across an extrusion axis, meshed together in
1 quality triangle mesh on the host, extruded through the graded planes of the axis and cut into
tetrahedra on the device, where they stay for the assembly (``TetMesh.device``).

Names follow the crate: ``Outline.polygon`` / ``Outline.circle`` (prism.rs:29-37), ``Footprint``
(:40-44), ``Part`` and ``Spacing`` (grid.rs:22-46), ``mesh`` / ``mesh_hollow`` (prism.rs:170-380),
``split_prism`` (:144-154), ``axis_planes`` (grid.rs:418), ``Size``, ``Mesh2`` and ``mesh2d`` /
``periodic_mesh2d`` (mesh2d.rs:64-110). Errors are ``FemError`` with the reference's texts.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from ._lib import (CLASSIFY_FN, FemError, INVALID, Outline_t, Part_t, Spacing_t, TetmeshCounts_t,
                   check, lib, ptr)

OUTSIDE = 0xFFFFFFFF          # mesh2d.rs:48
RATIO = 2.0 ** 0.5            # mesh2d.rs:53
MIN_ANGLE = 20.7              # mesh2d.rs:56
NO_PART = 0xFFFFFFFF          # BoundaryFace.beyond when no hollow part is beyond


@dataclass
class Outline:
    """A closed outline across the extrusion axis: a polygon (corners, either direction) or a
    circle (prism.rs:29-37)."""
    corners: np.ndarray | None = None
    centre: tuple = (0.0, 0.0)
    radius: float = 0.0

    @staticmethod
    def polygon(corners) -> "Outline":
        return Outline(corners=np.asarray(corners, dtype=np.float64).reshape(-1, 2))

    @staticmethod
    def circle(centre, radius) -> "Outline":
        return Outline(centre=(float(centre[0]), float(centre[1])), radius=float(radius))

    @property
    def is_circle(self) -> bool:
        return self.corners is None


@dataclass
class Footprint:
    outline: Outline
    holes: list = field(default_factory=list)


@dataclass
class Part:
    """A box of 1 material, or the prism of ``footprint`` between lo and hi on the extrusion
    axis (grid.rs:22-35)."""
    name: str
    material: int
    priority: int
    lo: tuple
    hi: tuple
    footprint: Footprint | None = None


@dataclass
class Spacing:
    max_cell: float
    max_growth: float
    min_cells: int


@dataclass
class Size:
    max_size: float
    max_growth: float


@dataclass
class BoundaryFace:
    nodes: tuple
    tet: int
    beyond: int
    circles: list


class _Structs:
    """The C structures of a part list, kept alive while the call runs."""

    def __init__(self, parts: Sequence[Part]):
        self.keep = []
        self.parts = (Part_t * max(len(parts), 1))()
        for k, p in enumerate(parts):
            q = self.parts[k]
            name = p.name.encode()
            self.keep.append(name)
            q.name = name
            q.material = int(p.material)
            q.priority = int(p.priority)
            for d in range(3):
                q.lo[d] = float(p.lo[d])
                q.hi[d] = float(p.hi[d])
            q.has_footprint = p.footprint is not None
            if p.footprint is not None:
                self._outline(q.outline, p.footprint.outline)
                holes = (Outline_t * max(len(p.footprint.holes), 1))()
                for h, o in enumerate(p.footprint.holes):
                    self._outline(holes[h], o)
                self.keep.append(holes)
                q.nholes = len(p.footprint.holes)
                q.holes = C.cast(holes, C.c_void_p)

    def _outline(self, t, o: Outline):
        t.circle = o.is_circle
        if o.is_circle:
            t.centre[0], t.centre[1] = o.centre
            t.radius = o.radius
        else:
            c = np.ascontiguousarray(o.corners, dtype=np.float64)
            self.keep.append(c)
            t.ncorners = len(c)
            t.corners = c.ctypes.data_as(C.c_void_p)


def _spacing(s: Spacing) -> Spacing_t:
    return Spacing_t(float(s.max_cell), float(s.max_growth), int(s.min_cells))


class TetMesh:
    """prism.rs:117-132 TetMesh: ``points`` (n, 3), ``tets`` (t, 4) with positive volumes,
    ``part`` per tetrahedron, the boundary ``faces`` sorted by (tet, nodes), the ``circles``
    (centre, radius) of the parts' circle outlines, and the counts of ``triangles`` of the 2D
    mesh and of ``planes`` of the axis. The points and tetrahedra also stay on the device."""

    def __init__(self, handle):
        self._h = handle
        L = lib()
        n = TetmeshCounts_t()
        check(L.femgpu_tetmesh_sizes(handle, C.byref(n)))
        self.points = np.empty((n.points, 3))
        self.tets = np.empty((n.tets, 4), dtype=np.uint32)
        self.part = np.empty(n.tets, dtype=np.uint32)
        self.face_nodes = np.empty((n.faces, 3), dtype=np.uint32)
        self.face_tet = np.empty(n.faces, dtype=np.uint32)
        self.face_beyond = np.empty(n.faces, dtype=np.uint32)
        self.face_circle_start = np.empty(n.faces + 1, dtype=np.uint64)
        self.face_circles = np.empty(max(n.face_circles, 1), dtype=np.uint32)
        circles = np.empty((max(n.circles, 1), 3))
        check(L.femgpu_tetmesh_copy(handle, ptr(self.points), ptr(self.tets), ptr(self.part),
                                    ptr(self.face_nodes), ptr(self.face_tet),
                                    ptr(self.face_beyond), ptr(self.face_circle_start),
                                    ptr(self.face_circles), ptr(circles)))
        self.face_circles = self.face_circles[:n.face_circles]
        self.circles = [((c[0], c[1]), c[2]) for c in circles[:n.circles]]
        self.triangles = n.triangles
        self.planes = n.planes

    @property
    def faces(self) -> list:
        s = self.face_circle_start
        return [BoundaryFace(tuple(int(v) for v in self.face_nodes[f]), int(self.face_tet[f]),
                             int(self.face_beyond[f]),
                             [int(c) for c in self.face_circles[s[f]:s[f + 1]]])
                for f in range(len(self.face_tet))]

    def device(self):
        """The device pointers (points, tets, part), owned by this mesh (femgpu_assemble_device
        takes the first 2)."""
        p, t, q = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib().femgpu_tetmesh_device(self._h, C.byref(p), C.byref(t), C.byref(q)))
        return p.value, t.value, q.value

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            lib().femgpu_tetmesh_free(h)


def mesh_hollow(parts: Sequence[Part], axis: int, spacing: Spacing, max_points: int,
                refusal: str, periodic: bool = False, hollow: Sequence[bool] = ()) -> TetMesh:
    """prism::mesh_hollow (prism.rs:185-380): no tetrahedra in the parts k with hollow[k]."""
    st = _Structs(parts)
    hol = np.asarray([1 if h else 0 for h in hollow], dtype=np.uint8)
    out = C.c_void_p()
    sp = _spacing(spacing)
    check(lib().femgpu_prism_mesh(C.cast(st.parts, C.c_void_p), len(parts), int(axis),
                                  C.byref(sp), int(max_points), refusal.encode(),
                                  1 if periodic else 0, ptr(hol) if len(hol) else None, len(hol),
                                  C.byref(out)))
    return TetMesh(out.value)


def mesh(parts: Sequence[Part], axis: int, spacing: Spacing, max_points: int, refusal: str,
         periodic: bool = False) -> TetMesh:
    """prism::mesh (prism.rs:170-181)."""
    return mesh_hollow(parts, axis, spacing, max_points, refusal, periodic, ())


def axis_planes(parts: Sequence[Part], d: int, spacing: Spacing, extra=()) -> np.ndarray:
    """grid::axis_planes (grid.rs:418-484): the graded planes of axis d. Host only."""
    st = _Structs(parts)
    ex = np.ascontiguousarray(extra, dtype=np.float64)
    sp = _spacing(spacing)
    count = C.c_size_t()
    L = lib()
    args = (C.cast(st.parts, C.c_void_p), len(parts), int(d), C.byref(sp),
            ptr(ex) if len(ex) else None, len(ex))
    check(L.femgpu_axis_planes(*args, None, 0, C.byref(count)))
    out = np.empty(count.value)
    check(L.femgpu_axis_planes(*args, ptr(out), len(out), C.byref(count)))
    return out


def split_prism(g) -> list:
    """prism::split_prism (prism.rs:144-154): 3 tetrahedra of local corners."""
    gg = np.ascontiguousarray(g, dtype=np.uint64)
    if gg.shape != (6,):
        raise FemError(INVALID, "a prism has 6 corners")
    out = np.empty(12, dtype=np.int32)
    check(lib().femgpu_split_prism(ptr(gg), ptr(out)))
    return [[int(v) for v in out[4 * i:4 * i + 4]] for i in range(3)]


@dataclass
class Mesh2:
    """mesh2d.rs:72-82 Mesh2: points (n, 2), counterclockwise triangles (t, 3), a label per
    triangle, the triangle across each edge (t, 3; OUTSIDE where none) and the input segments
    of each edge on a segment, keyed by its 2 points (smaller first)."""
    points: np.ndarray
    triangles: np.ndarray
    label: np.ndarray
    across: np.ndarray
    segments: dict


def _mesh2d(points, segments, size: Size, classify: Callable, periodic: bool) -> Mesh2:
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
    segs = np.ascontiguousarray(segments, dtype=np.uint32).reshape(-1, 2)
    failure = []

    def call(p, _ctx):
        try:
            return int(classify((p[0], p[1])))
        except BaseException as e:  # noqa: BLE001 - reported after the call
            failure.append(e)
            return OUTSIDE

    cb = CLASSIFY_FN(call)
    out = C.c_void_p()
    status = lib().femgpu_mesh2d(ptr(pts), len(pts), ptr(segs), len(segs), float(size.max_size),
                                 float(size.max_growth), 1 if periodic else 0, cb, None,
                                 C.byref(out))
    if failure:
        if status == 0:
            lib().femgpu_mesh2_free(out)
        raise failure[0]
    check(status)
    try:
        n, t, e, o = (C.c_size_t() for _ in range(4))
        check(lib().femgpu_mesh2_sizes(out, C.byref(n), C.byref(t), C.byref(e), C.byref(o)))
        P = np.empty((n.value, 2))
        T = np.empty((t.value, 3), dtype=np.uint32)
        lab = np.empty(t.value, dtype=np.uint32)
        acr = np.empty((t.value, 3), dtype=np.uint32)
        E = np.empty((max(e.value, 1), 2), dtype=np.uint32)
        start = np.empty(e.value + 1, dtype=np.uint64)
        O = np.empty(max(o.value, 1), dtype=np.uint32)
        check(lib().femgpu_mesh2_copy(out, ptr(P), ptr(T), ptr(lab), ptr(acr), ptr(E),
                                      ptr(start), ptr(O)))
    finally:
        lib().femgpu_mesh2_free(out)
    seg = {(int(E[k, 0]), int(E[k, 1])): [int(v) for v in O[start[k]:start[k + 1]]]
           for k in range(e.value)}
    return Mesh2(P, T, lab, acr, seg)


def mesh2d(points, segments, size: Size, classify: Callable) -> Mesh2:
    """mesh2d::mesh (mesh2d.rs:87-96). Host only."""
    return _mesh2d(points, segments, size, classify, False)


def periodic_mesh2d(points, segments, size: Size, classify: Callable) -> Mesh2:
    """mesh2d::periodic_mesh (mesh2d.rs:100-110). Host only."""
    return _mesh2d(points, segments, size, classify, True)
