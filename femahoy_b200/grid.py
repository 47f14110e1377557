"""The reference's graded box grid (crates/fem/src/grid.rs Grid::build) and the hex mesh of its
cells (heat.rs:1165-1210 number), built on the device behind ``femgpu_box_grid``: the planes of
each axis, the part of each cell, the mesh points numbered in first use over the cells of the
parts with their grid points (the ``Level`` of the multigrid), the cells in VTK corner order and
the model's faces. The mesh stays on the device for the assembly (``BoxGrid.device``)."""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from ._lib import BoxgridCounts_t, check, lib, ptr
from .prism import Part, Spacing, _spacing, _Structs

VOID = 0xFFFFFFFF  # grid.rs:105
SIDES = ("x-", "x+", "y-", "y+", "z-", "z+")  # grid.rs:54-81 Side::ALL


class BoxGrid:
    """grid.rs:108-114 Grid (``planes``, ``part`` per cell, cell (i, j, k) at i + nx (j + ny k))
    with heat.rs:1153-1162 Numbering (``points``, ``ijk``, ``cells`` (E, 8), ``cell_of``,
    ``mesh_part``) and the faces (``face_cell``, ``face_side`` into SIDES)."""

    def __init__(self, handle):
        self._h = handle
        n = BoxgridCounts_t()
        check(lib().femgpu_boxgrid_sizes(handle, C.byref(n)))
        self.planes = [np.empty(n.planes[d]) for d in range(3)]
        self.part = np.empty(n.grid_cells, dtype=np.uint32)
        self.points = np.empty((n.points, 3))
        self.ijk = np.empty((n.points, 3), dtype=np.uint32)
        self.cells = np.empty((n.cells, 8), dtype=np.uint32)
        self.cell_of = np.empty(n.cells, dtype=np.uint64)
        self.mesh_part = np.empty(n.cells, dtype=np.uint32)
        self.face_cell = np.empty(n.faces, dtype=np.uint64)
        self.face_side = np.empty(n.faces, dtype=np.uint8)
        planes = (C.c_void_p * 3)(*[p.ctypes.data for p in self.planes])
        check(lib().femgpu_boxgrid_copy(handle, C.cast(planes, C.c_void_p), ptr(self.part),
                                        ptr(self.points), ptr(self.ijk), ptr(self.cells),
                                        ptr(self.cell_of), ptr(self.mesh_part),
                                        ptr(self.face_cell), ptr(self.face_side)))

    def dims(self):
        return tuple(len(p) - 1 for p in self.planes)

    def size(self, cell):
        """The side lengths of grid cell ``cell`` (grid.rs:195-199)."""
        nx, ny, _ = self.dims()
        c = (cell % nx, (cell // nx) % ny, cell // (nx * ny))
        return np.array([self.planes[d][c[d] + 1] - self.planes[d][c[d]] for d in range(3)])

    def device(self):
        """The device pointers of the mesh points and cells, owned by this grid."""
        p, c = C.c_void_p(), C.c_void_p()
        check(lib().femgpu_boxgrid_device(self._h, C.byref(p), C.byref(c)))
        return p.value, c.value

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            lib().femgpu_boxgrid_free(h)


def build(parts: Sequence[Part], spacing: Spacing, extra=((), (), ()), max_points=2**32 - 1,
          refusal: str = "the grid has too many points") -> BoxGrid:
    """Grid::build (grid.rs:119-154) and number (heat.rs:1165-1210)."""
    st = _Structs(parts)
    ex = [np.ascontiguousarray(e, dtype=np.float64) for e in extra]
    eptr = (C.c_void_p * 3)(*[e.ctypes.data if len(e) else None for e in ex])
    en = (C.c_size_t * 3)(*[len(e) for e in ex])
    sp = _spacing(spacing)
    out = C.c_void_p()
    check(lib().femgpu_box_grid(C.cast(st.parts, C.c_void_p), len(parts), C.byref(sp),
                                C.cast(eptr, C.c_void_p), C.cast(en, C.c_void_p), int(max_points),
                                refusal.encode(), C.byref(out)))
    return BoxGrid(out.value)
