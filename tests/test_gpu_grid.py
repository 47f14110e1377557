"""The box grid on the device (grid.rs Grid::build, heat.rs:1165-1210 number): bit-identical
with the oracle's sequential restatement (planes, each cell's part, the mesh points, their grid
points, the cells, the faces), the reference's own tests (grid.rs:548-642), the errors with the
reference's texts, and a box-cell heat solve on the grid's own mesh against the oracle."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import femahoy_b200 as fg
import oracle
from femahoy_b200 import _lib as L
from femahoy_b200 import grid as G
from femahoy_b200 import prism as P
from femahoy_b200._lib import FemError
from oracle import grid as OG

pytestmark = pytest.mark.gpu

SPACING = P.Spacing(1.0, 1.3, 2)


def _part(name, material, priority, lo, hi):
    return P.Part(name, material, priority, tuple(lo), tuple(hi))


def _same(g, parts, spacing, extra=((), (), ())):
    tuples = [(p.name, p.material, p.priority, p.lo, p.hi) for p in parts]
    planes, part = OG.build(tuples, (spacing.max_cell, spacing.max_growth, spacing.min_cells),
                            extra)
    for d in range(3):
        assert g.planes[d].tolist() == planes[d]
    assert g.part.tolist() == part
    points, ijk, cells, cell_of, mpart = OG.number(planes, part)
    assert g.points.tolist() == points
    assert g.ijk.tolist() == [list(v) for v in ijk]
    assert g.cells.tolist() == cells
    assert g.cell_of.tolist() == cell_of
    assert g.mesh_part.tolist() == mpart
    assert list(zip(g.face_cell.tolist(), g.face_side.tolist())) == OG.faces(planes, part)


def test_each_part_face_is_a_plane_and_the_grid_equals_the_oracle():
    parts = [_part("block", 0, 0, (0.0, 0.0, 0.0), (10.0, 10.0, 5.0)),
             _part("layer", 1, 0, (2.0, 3.0, 5.0), (7.0, 6.0, 5.01))]
    g = G.build(parts, SPACING)
    _same(g, parts, SPACING)
    for p in parts:
        for d in range(3):
            for x in (p.lo[d], p.hi[d]):
                assert np.abs(g.planes[d] - x).min() < 1e-12


def test_the_part_with_the_higher_priority_holds_the_overlap():
    parts = [_part("a", 0, 0, (0.0,) * 3, (2.0,) * 3), _part("b", 1, 1, (1.0,) * 3, (3.0,) * 3)]
    g = G.build(parts, SPACING)
    _same(g, parts, SPACING)
    nx, ny, _ = g.dims()

    def cell_at(x):
        i = [int(np.searchsorted(g.planes[d], x[d]) - 1) for d in range(3)]
        return i[0] + nx * (i[1] + ny * i[2])

    assert g.part[cell_at((1.5, 1.5, 1.5))] == 1
    assert g.part[cell_at((0.5, 0.5, 0.5))] == 0
    assert g.part[cell_at((2.5, 0.5, 0.5))] == G.VOID
    same = [_part("a", 0, 0, (0.0,) * 3, (2.0,) * 3), _part("b", 1, 0, (1.0,) * 3, (3.0,) * 3)]
    with pytest.raises(FemError, match=r"parts a and b overlap at \(1\.\d+, 1\.\d+, 1\.\d+\) "
                                       "with the same priority and other materials"):
        G.build(same, SPACING)


def test_the_faces_of_a_box_cover_its_surface():
    g = G.build([_part("a", 0, 0, (0.0,) * 3, (2.0, 3.0, 4.0))], SPACING)
    area = 0.0
    for cell, side in zip(g.face_cell, g.face_side):
        s = g.size(int(cell))
        area += np.prod([s[d] for d in range(3) if d != side // 2])
    assert abs(area - 2.0 * (6.0 + 8.0 + 12.0)) < 1e-9


def test_random_parts_with_priorities_and_a_symmetry_plane_equal_the_oracle():
    rng = np.random.default_rng(11)
    for trial in range(8):
        parts = []
        for i in range(5):
            lo = rng.uniform(0.0, 6.0, 3)
            hi = lo + 0.05 + 4.0 * rng.uniform(0.0, 1.0, 3) ** 3
            # Distinct priorities, or the same material at equal priority: no refusal.
            parts.append(_part(f"p{i}", i % 2 if trial % 2 else 0, i if trial % 2 else 0, lo, hi))
        extra = ((), (3.0,), ()) if trial % 3 == 0 else ((), (), ())
        g = G.build(parts, P.Spacing(0.7, 1.3, 2), extra=extra)
        _same(g, parts, P.Spacing(0.7, 1.3, 2), extra)


def test_box_grid_errors_carry_the_reference_texts():
    a = _part("a", 0, 0, (0.0,) * 3, (1.0,) * 3)
    for sp, text in ((P.Spacing(0.0, 1.3, 2), "max_cell must be a number above 0"),
                     (P.Spacing(0.5, 1.0, 2), "max_growth must be a number above 1"),
                     (P.Spacing(0.5, 1.3, 0), "min_cells must be 1 or more")):
        with pytest.raises(FemError, match=text):
            G.build([a], sp)
    with pytest.raises(FemError, match="the model has no part"):
        G.build([], SPACING)
    bad = _part("bad", 0, 0, (0.0, 1.0, 0.0), (1.0, 1.0, 1.0))
    with pytest.raises(FemError, match="part bad: its y range must be 2 finite numbers"):
        G.build([bad], SPACING)
    with pytest.raises(FemError, match="the grid has more than 10 points") as e:
        G.build([a], SPACING, max_points=10, refusal="the grid has more than 10 points")
    assert e.value.code == L.TOO_LARGE


def test_a_box_cell_heat_solve_on_the_grid_mesh_equals_the_oracle():
    """heat.rs:755-830's path on the grid's own mesh: 2 materials with priorities and a void
    corner, the box-cell conduction assembled from the grid's device arrays (bit-identical with
    the host assembly), 0 at z = 0 and 100 at the top; the grid's V-cycle on the mesh points'
    grid points reaches the oracle's direct solution."""
    torch = pytest.importorskip("torch")
    parts = [_part("slab", 0, 0, (0.0, 0.0, 0.0), (2.0, 1.5, 1.0)),
             _part("insert", 1, 1, (0.5, 0.25, 0.3), (1.2, 1.0, 0.7)),
             _part("post", 0, 0, (0.0, 0.0, 1.0), (0.6, 0.6, 1.8))]
    g = G.build(parts, P.Spacing(0.08, 1.3, 2))
    k = np.array([[1.0, 1.0, 1.0], [20.0, 20.0, 5.0]])
    coef = np.array([k[[0, 1, 0][p]] for p in g.mesh_part.tolist()])
    xyz, cells = g.device()
    dc = torch.tensor(coef, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    h = C.c_void_p()
    L.check(L.lib().femgpu_assemble_device(fg.HEX8_HEAT, fg.GATHER, len(g.points), xyz,
                                           len(g.cells), cells, C.c_void_p(dc.data_ptr()),
                                           C.byref(h)))
    K = fg.Csr(h.value)
    Kh = fg.Csr.assemble(fg.HEX8_HEAT, g.points, g.cells, coef)
    for a, b in zip(K.arrays(), Kh.arrays()):
        assert np.array_equal(a, b)
    z = g.points[:, 2]
    fixed = (z == 0.0) | (z == z.max())
    values = np.where(z == z.max(), 100.0, 0.0)
    free = np.nonzero(~fixed)[0].astype(np.int64)
    A = K.submatrix(free)
    rhs = fg.reduced_rhs(K, np.zeros(len(g.points)), values, free)
    lv = fg.Level(g.planes, g.ijk[free].astype(np.uint32), np.zeros(len(free), np.uint8))
    s = fg.Solver(A, fg.Unknowns.Grid(lv), fg.Method.Multigrid,
                  options=fg.Options(coarsest=500)).with_tol(1e-10)
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.true_residual <= 1.2e-10
    Ko = oracle.pattern(len(g.points), g.cells)
    Ko.assemble(5, g.points, g.cells, coef)
    xd, _ = oracle.direct_solve(Ko.submatrix(free), g.points[free],
                                Ko.reduced_rhs(np.zeros(len(g.points)), values, free))
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
