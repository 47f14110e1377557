"""The device assembly against the oracle: the pattern, the Quadratic numbering, the colouring
and the submatrix are bit-exact; the gathered values are bit-identical with the reference's
element-ordered sums; the colour-scattered values agree to a few ulp."""
import numpy as np
import pytest

import femahoy_b200 as fg
import oracle
from femahoy_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _same_pattern(a, b):
    pa, ia, _ = a.arrays()
    pb, ib, _ = b.arrays()
    assert np.array_equal(pa, pb)
    assert np.array_equal(ia, ib)


def test_pattern_known_answer():
    """sparse.rs:299-305 on the device."""
    a = fg.Csr.pattern(3, np.array([[0, 1], [1, 2]]))
    ptr, idx, val = a.arrays()
    assert ptr.tolist() == [0, 2, 5, 7]
    assert idx.tolist() == [0, 1, 0, 1, 2, 1, 2]
    assert not val.any()


@pytest.mark.parametrize("dims", [(40, 4, 4), (16, 16, 16), (7, 3, 5)])
def test_pattern_matches_oracle(dims):
    m = mg.box(*dims)
    _same_pattern(fg.Csr.pattern(m.n, m.tets), oracle.pattern(m.n, m.tets))


def test_pattern_of_p2_unknowns_matches_oracle():
    m = mg.box(5, 3, 2)
    edges, t10 = oracle.quadratic(m.points, m.tets)
    n = m.n + len(edges)
    dof = oracle.dof_elements(t10)
    _same_pattern(fg.Csr.pattern(3 * n, dof), oracle.pattern(3 * n, dof))


def test_quadratic_numbering_matches_oracle():
    m = mg.box(9, 4, 3)
    q = fg.Quadratic.new(m.points, m.tets)
    edges, t10 = oracle.quadratic(m.points, m.tets)
    assert np.array_equal(q.edges, edges)
    assert np.array_equal(q.tets, t10)


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


@pytest.mark.parametrize("n", [8, 24])
def test_gather_p1_heat_is_bit_identical(n):
    h = mg.heat_cube(n)
    g = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    o = oracle.pattern(h.n_points, h.nodes)
    o.assemble(0, h.xyz, h.nodes, h.coef)
    _same_pattern(g, o)
    assert np.array_equal(_bits(g.arrays()[2]), _bits(o.arrays()[2]))


def test_gather_p1_elastic_is_bit_identical():
    p = mg.cantilever_p1()
    g = fg.Csr.assemble(fg.P1_ELASTIC, p.xyz, p.nodes, p.coef)
    o = oracle.pattern(3 * p.n_points, oracle.dof_elements(p.nodes))
    o.assemble(1, p.xyz, p.nodes, p.coef)
    _same_pattern(g, o)
    assert g.shape == (3075, 108873)
    assert np.array_equal(_bits(g.arrays()[2]), _bits(o.arrays()[2]))


def test_gather_p2_elastic_is_bit_identical():
    m = mg.box(10, 3, 3, (50.0, 15.0, 15.0))
    edges, t10 = oracle.quadratic(m.points, m.tets)
    prob = mg.beam_p2(edges, t10, mesh=m)
    g = fg.Csr.assemble(fg.P2_ELASTIC, prob.xyz, prob.nodes, prob.coef)
    o = oracle.pattern(3 * prob.n_points, oracle.dof_elements(prob.nodes))
    o.assemble(2, prob.xyz, prob.nodes, prob.coef)
    _same_pattern(g, o)
    assert np.array_equal(_bits(g.arrays()[2]), _bits(o.arrays()[2]))


def test_colouring_matches_oracle():
    m = mg.box(12, 7, 5)
    c, nc = fg.colour(m.n, m.tets)
    co, nco = oracle.colour(m.n, m.tets)
    assert nc == nco
    assert np.array_equal(c, co)


@pytest.mark.parametrize("kind", [fg.P1_HEAT, fg.P1_ELASTIC, fg.P2_ELASTIC])
def test_colour_scatter_agrees_to_rounding(kind):
    m = mg.box(8, 4, 4, (40.0, 20.0, 20.0))
    if kind == fg.P1_HEAT:
        xyz, nodes = m.points, m.tets
        coef = np.exp(np.random.default_rng(5).standard_normal((len(m.tets), 1))) * np.ones(3)
    elif kind == fg.P1_ELASTIC:
        xyz, nodes = m.points, m.tets
        coef = np.tile([70e3, 0.33], (len(m.tets), 1))
    else:
        edges, t10 = oracle.quadratic(m.points, m.tets)
        xyz = mg.beam_p2(edges, t10, mesh=m).xyz
        nodes = t10
        coef = np.tile([70e3, 0.33], (len(m.tets), 1))
    a = fg.Csr.assemble(kind, xyz, nodes, coef, mode=fg.GATHER)
    b = fg.Csr.assemble(kind, xyz, nodes, coef, mode=fg.COLOUR)
    pa, ia, va = a.arrays()
    pb, ib, vb = b.arrays()
    assert np.array_equal(pa, pb) and np.array_equal(ia, ib)
    # Sums of at most 24 terms in another order: a few ulp of the row's largest entry.
    rows = np.repeat(np.arange(len(pa) - 1), np.diff(pa))
    scale = np.maximum.reduceat(np.abs(va), pa[:-1])[rows]
    assert np.all(np.abs(va - vb) <= 1e-13 * scale)


def test_submatrix_and_reduced_rhs_are_bit_identical():
    h = mg.heat_cube(12)
    g = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    o = oracle.pattern(h.n_points, h.nodes)
    o.assemble(0, h.xyz, h.nodes, h.coef)
    gs, os_ = g.submatrix(h.free), o.submatrix(h.free)
    _same_pattern(gs, os_)
    assert np.array_equal(_bits(gs.arrays()[2]), _bits(os_.arrays()[2]))
    rg = fg.reduced_rhs(g, h.load, h.values, h.free)
    ro = o.reduced_rhs(h.load, h.values, h.free)
    assert np.array_equal(_bits(rg), _bits(ro))
    x = np.random.default_rng(1).standard_normal(gs.n)
    assert np.array_equal(_bits(gs.mul(x)), _bits(os_.mul(x)))


def test_unsorted_keep_sorts_rows_as_the_reference():
    """sparse.rs:137-148: a keep list out of order gives sorted rows with their values."""
    h = mg.heat_cube(4)
    g = fg.Csr.assemble(fg.P1_HEAT, h.xyz, h.nodes, h.coef)
    o = oracle.pattern(h.n_points, h.nodes)
    o.assemble(0, h.xyz, h.nodes, h.coef)
    keep = np.random.default_rng(2).permutation(h.n_points)[: h.n_points // 2]
    gs, os_ = g.submatrix(keep), o.submatrix(keep)
    _same_pattern(gs, os_)
    assert np.array_equal(gs.arrays()[2], os_.arrays()[2])


def test_element_out_of_range_is_an_error():
    with pytest.raises(fg.FemError) as e:
        fg.Csr.pattern(3, np.array([[0, 5]]))
    assert e.value.code == 5


def test_bad_material_is_the_reference_error():
    m = mg.box(2, 1, 1)
    coef = np.tile([70e3, 0.6], (len(m.tets), 1))
    with pytest.raises(fg.FemError, match="Poisson ratios give no stable material"):
        fg.Csr.assemble(fg.P1_ELASTIC, m.points, m.tets, coef)


def test_orthotropic_p2_assembly_is_bit_identical():
    """Orthotropic::stiffness (hex.rs:69-117) per element on the device: the same bits as the
    oracle for random stable constants; a modulus below 0 gives the reference's text."""
    m = mg.box(4, 2, 2, (40.0, 10.0, 10.0))
    q = fg.Quadratic.new(m.points, m.tets)
    rng = np.random.default_rng(8)
    ne = len(q.tets)
    e = rng.uniform(50e3, 200e3, (ne, 3))
    nu = rng.uniform(0.1, 0.3, (ne, 3))
    g = rng.uniform(20e3, 80e3, (ne, 3))
    coef = np.hstack([e, nu, g])
    K = fg.Csr.assemble(fg.P2_ELASTIC_ORTHO, q.points, q.tets, coef)
    Ko = oracle.pattern(3 * len(q.points), oracle.dof_elements(q.tets))
    Ko.assemble(4, q.points, q.tets, coef)
    for a, b in zip(K.arrays(), Ko.arrays()):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    bad = coef.copy()
    bad[3, 1] = -1.0
    with pytest.raises(fg.FemError) as err:
        fg.Csr.assemble(fg.P2_ELASTIC_ORTHO, q.points, q.tets, bad)
    assert err.value.code == fg._lib.MATERIAL and "moduli must be above 0" in str(err.value)

