"""The prism mesh on the device (prism.rs:185-380): the extrusion equals the oracle's sequential
restatement bit for bit (points, tetrahedra, parts, boundary faces with their hollow parts and
circles) on the same 2D mesh, the reference's own checks of tests/tet.rs:142-214 hold, the
errors carry the reference's texts, the device copy feeds the assembly directly, and a P2
elasticity solve on a prism mesh equals the oracle's direct solution."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

import femahoy_b200 as fg
import oracle
from femahoy_b200 import prism as P
from femahoy_b200 import _lib as L
from femahoy_b200._lib import FemError
from oracle import prism as O

pytestmark = pytest.mark.gpu

HOLE = ("circle", (1.0, 1.0), 0.4)
PLATE = ("plate", 0, 0, (0.0, 0.0, 0.0), (0.0, 0.0, 0.2),
         (("polygon", [(0.0, 0.0), (3.0, 0.0), (3.0, 2.0), (0.0, 2.0)]), [HOLE]))
LID = ("lid", 1, 0, (0.0, 0.0, 0.2), (0.0, 0.0, 0.5),
       (("polygon", [(2.0, 0.5), (2.8, 0.5), (2.4, 1.5)]), []))


def _outline(o):
    return P.Outline.circle(o[1], o[2]) if o[0] == "circle" else P.Outline.polygon(o[1])


def _part(p):
    name, material, priority, lo, hi, fp = p
    f = None if fp is None else P.Footprint(_outline(fp[0]), [_outline(h) for h in fp[1]])
    return P.Part(name, material, priority, lo, hi, f)


def _reference(parts, axis, spacing, max_points=10**9, hollow=()):
    """The oracle's mesh of the same parts on the same 2D mesh (the product's mesh2d fed the
    oracle's footprints and labels)."""
    pts, segs, segcirc, circles, classify, covers = O.footprint_inputs(parts, axis,
                                                                       spacing.max_cell)
    m2 = P.mesh2d(np.array(pts), np.array(segs, dtype=np.uint32),
                  P.Size(spacing.max_cell, spacing.max_growth), classify)
    planes = O.axis_planes([(p[3], p[4]) for p in parts], axis,
                           (spacing.max_cell, spacing.max_growth, spacing.min_cells))
    out = O.extrude(parts, axis, planes, [tuple(p) for p in m2.points], m2.triangles.tolist(),
                    m2.label.tolist(), covers, m2.segments, segcirc, max_points, hollow)
    return out, circles, len(m2.triangles), len(planes)


def _same(tm, ref):
    (pts, tets, part, faces), circles, ntri, nplanes = ref
    assert tm.points.tolist() == [list(p) for p in pts]
    assert tm.tets.tolist() == tets
    assert tm.part.tolist() == part
    got = [(f.nodes, f.tet, f.beyond, f.circles) for f in tm.faces]
    assert got == [(tuple(f[0]), f[1], f[2], list(f[3])) for f in faces]
    assert tm.circles == [((c[0][0], c[0][1]), c[1]) for c in circles]
    assert tm.triangles == ntri and tm.planes == nplanes


def test_the_plate_with_a_hole_and_a_lid_equals_the_oracle_and_is_conforming():
    """tests/tet.rs:142-214: each inner face has 2 tetrahedra, the volumes are the parts', the
    boundary faces close the surface and the faces on the hole have its area."""
    parts = [PLATE, LID]
    sp = P.Spacing(0.2, 1.3, 2)
    tm = P.mesh([_part(p) for p in parts], 2, sp, 10**9, "")
    _same(tm, _reference(parts, 2, sp))
    vol = np.zeros(2)
    for t, tet in enumerate(tm.tets):
        v = O.volume(tm.points[tet].tolist())
        assert v > 0.0
        vol[tm.part[t]] += v
    n = len(O.circle_corners((1.0, 1.0), 0.4, 0.2))
    polygon_hole = 0.5 * n * 0.4 ** 2 * math.sin(2 * math.pi / n)
    assert abs(vol[0] - (6.0 - polygon_hole) * 0.2) < 1e-9
    assert abs(vol[1] - 0.4 * 0.3) < 1e-9
    count = {}
    for tet in tm.tets.tolist():
        for f in ((1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1)):
            key = tuple(sorted(tet[k] for k in f))
            count[key] = count.get(key, 0) + 1
    assert max(count.values()) <= 2
    total = np.zeros(3)
    on_hole = 0.0
    for f in tm.faces:
        p = tm.points[list(f.nodes)]
        nrm = np.cross(p[1] - p[0], p[2] - p[0])
        total += 0.5 * nrm
        if f.circles:
            on_hole += 0.5 * np.linalg.norm(nrm)
    assert np.abs(total).max() < 1e-12
    assert sum(1 for c in count.values() if c == 1) == len(tm.faces)
    perimeter = n * 2.0 * 0.4 * math.sin(math.pi / n)
    assert abs(on_hole - perimeter * 0.2) < 1e-9


def test_a_hollow_part_keeps_its_space_and_its_faces_name_it():
    """prism.rs:183-184: the lid hollow: no tetrahedra in it, the plate's faces under it are
    boundary faces with the lid beyond; equal to the oracle."""
    parts = [PLATE, LID]
    sp = P.Spacing(0.25, 1.4, 2)
    tm = P.mesh_hollow([_part(p) for p in parts], 2, sp, 10**9, "", hollow=[False, True])
    _same(tm, _reference(parts, 2, sp, hollow=[False, True]))
    assert set(tm.part.tolist()) == {0}
    assert any(f.beyond == 1 for f in tm.faces)


def test_boxes_and_priorities_along_x_equal_the_oracle():
    """Box parts (no footprint) extruded along x, overlapping with priorities, and a circle part:
    the part of each prism by priority, the later part first at equal priority."""
    parts = [("base", 0, 0, (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), None),
             ("insert", 1, 2, (0.3, 0.5, 0.2), (0.8, 1.2, 0.9), None),
             ("rod", 2, 1, (0.0, 0.0, 0.0), (1.0, 0.0, 0.0),
              (("circle", (1.5, 0.5), 0.3), []))]
    sp = P.Spacing(0.15, 1.3, 2)
    tm = P.mesh([_part(p) for p in parts], 0, sp, 10**9, "")
    _same(tm, _reference(parts, 0, sp))
    assert set(tm.part.tolist()) == {0, 1, 2}


def test_a_periodic_unit_cell_equals_the_oracle_and_its_sides_match():
    """prism.rs:170's `periodic` (mesh2d.rs:1136-1197): a unit cell with an off-centre round
    inclusion, extruded along z; the points on x = 0 and x = 1 (and on y = 0, y = 1) pair up."""
    cell = ("matrix", 0, 0, (0.0, 0.0, 0.0), (1.0, 1.0, 0.5),
            (("polygon", [(0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0)]), []))
    fibre = ("fibre", 1, 1, (0.0, 0.0, 0.0), (0.0, 0.0, 0.5),
             (("circle", (0.4, 0.55), 0.2), []))
    parts = [cell, fibre]
    sp = P.Spacing(0.2, 1.3, 2)
    tm = P.mesh([_part(p) for p in parts], 2, sp, 10**9, "", periodic=True)
    pts, segs, segcirc, circles, classify, covers = O.footprint_inputs(parts, 2, sp.max_cell)
    m2 = P.periodic_mesh2d(np.array(pts), np.array(segs, dtype=np.uint32),
                           P.Size(sp.max_cell, sp.max_growth), classify)
    planes = O.axis_planes([(p[3], p[4]) for p in parts], 2, (0.2, 1.3, 2))
    ref = O.extrude(parts, 2, planes, [tuple(p) for p in m2.points], m2.triangles.tolist(),
                    m2.label.tolist(), covers, m2.segments, segcirc, 10**9)
    _same(tm, (ref, circles, len(m2.triangles), len(planes)))
    for d in range(2):
        o = 1 - d
        lo = sorted((round(q[o], 12), round(q[2], 12)) for q in tm.points if abs(q[d]) < 1e-12)
        hi = sorted((round(q[o], 12), round(q[2], 12)) for q in tm.points
                    if abs(q[d] - 1.0) < 1e-12)
        assert lo == hi and lo


def test_prism_mesh_errors_carry_the_reference_texts():
    sp = P.Spacing(0.2, 1.3, 2)
    with pytest.raises(FemError, match="too many tetrahedra for this case") as e:
        P.mesh([_part(PLATE)], 2, sp, 100, "too many tetrahedra for this case")
    assert e.value.code == L.TOO_LARGE
    with pytest.raises(FemError, match="the parts hold no volume"):
        P.mesh_hollow([_part(PLATE)], 2, sp, 10**9, "", hollow=[True])
    with pytest.raises(FemError, match="the model has no part"):
        P.mesh([], 2, sp, 10**9, "")
    with pytest.raises(FemError, match="max_cell must be a number above 0"):
        P.mesh([_part(PLATE)], 2, P.Spacing(0.0, 1.3, 2), 10**9, "")
    a = ("a", 0, 0, (0.0, 0.0, 0.0), (2.0, 2.0, 2.0), None)
    b = ("b", 1, 0, (1.0, 1.0, 1.0), (3.0, 3.0, 3.0), None)
    with pytest.raises(FemError, match="overlap with the same priority"):
        P.mesh([_part(a), _part(b)], 2, P.Spacing(0.5, 1.3, 2), 10**9, "")
    c = ("c", 0, 0, (0.0, 0.0, 1.0), (1.0, 1.0, 1.0), None)
    with pytest.raises(FemError, match="part c: its z range must be 2 finite numbers"):
        P.mesh([_part(c)], 2, sp, 10**9, "")


def test_the_device_mesh_feeds_the_assembly_bit_for_bit():
    """femgpu_assemble_device on the mesh's own device arrays equals the host-pointer assembly of
    its copies (P1 heat)."""
    torch = pytest.importorskip("torch")
    tm = P.mesh([_part(PLATE)], 2, P.Spacing(0.2, 1.3, 2), 10**9, "")
    coef = np.tile([1.0, 2.0, 3.0], (len(tm.tets), 1))
    host = fg.Csr.assemble(fg.P1_HEAT, tm.points, tm.tets, coef)
    xyz, tets, _ = tm.device()
    dc = torch.tensor(coef, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    h = C.c_void_p()
    L.check(L.lib().femgpu_assemble_device(fg.P1_HEAT, fg.GATHER, len(tm.points), xyz,
                                           len(tm.tets), tets, C.c_void_p(dc.data_ptr()),
                                           C.byref(h)))
    dev = fg.Csr(h.value)
    for a, b in zip(host.arrays(), dev.arrays()):
        assert np.array_equal(a, b)


def test_a_p2_solve_on_a_prism_mesh_equals_the_oracle_direct_solution():
    """elastic_tet.rs:98-330's path on the reference's own mesh: a block with a round hole
    through it (the plate's footprint, 1 thick), P2 elasticity clamped at x = 0 with a load at
    x = 3, p-multigrid to the corners and z-only geometric levels; the PCG solution equals the
    oracle's direct one."""
    block = PLATE[:4] + ((0.0, 0.0, 1.0), PLATE[5])
    tm = P.mesh([_part(block)], 2, P.Spacing(0.5, 1.3, 2), 250_000, "")
    q = fg.Quadratic.new(tm.points, tm.tets)
    n = len(q.points)
    coef = np.tile([1000.0, 0.3], (len(q.tets), 1))
    fixed = np.repeat(q.points[:, 0] == 0.0, 3)
    free = np.nonzero(~fixed)[0].astype(np.int64)
    load = np.zeros(3 * n)
    load[3 * np.nonzero(q.points[:, 0] == 3.0)[0] + 2] = -1e-3
    K = fg.Csr.assemble(fg.P2_ELASTIC, q.points, q.tets, coef)
    A = K.submatrix(free)
    rhs = fg.reduced_rhs(K, load, np.zeros(3 * n), free)
    Pm, coarse = fg.prolongation(q.points, len(tm.points), q.edges, free)
    u = fg.Unknowns.Quadratic(q.points[free // 3], Pm, coarse)
    s = fg.Solver(A, u, fg.Method.Multigrid,
                  options=fg.Options(axes=4, coarsest=4000)).with_tol(1e-10)
    assert len(s.levels()) >= 2
    x = np.zeros(A.n)
    st = s.solve(rhs, x)
    assert st.true_residual <= 1.2e-10
    Ko = oracle.pattern(3 * n, oracle.dof_elements(q.tets))
    Ko.assemble(2, q.points, q.tets, coef)
    xd, _ = oracle.direct_solve(Ko.submatrix(free), q.points[free // 3],
                                Ko.reduced_rhs(load, np.zeros(3 * n), free))
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
