"""Probes of a P2 elasticity model (elastic_tet.rs:428-467, cells_at at elastic_tet.rs:538-553).

CPU: the oracle against analytic answers (a P2 mesh holds a linear displacement and a linear
temperature exactly, and the stress of a uniform strain is exact at any point, whichever cells
share it). GPU: the device probes against the oracle bit for bit, at points inside cells, on
faces, edges and corners (several cells each), and the reference's error text for a point in no
cell.
"""
import numpy as np
import pytest

import oracle
from test_recovery import iso_stress, linear_u, p2_box


def _probe_points(xyz, rng):
    """Interior points, corners (many cells), edge and face midpoints (2+ cells)."""
    lo, hi = xyz.min(axis=0), xyz.max(axis=0)
    inner = lo + (hi - lo) * rng.uniform(0.05, 0.95, size=(6, 3))
    corners = xyz[[0, 7, 13, 40]]
    return np.concatenate([inner, corners, [0.5 * (lo + hi)], [[lo[0], 0.5 * (lo[1] + hi[1]),
                                                                 0.5 * (lo[2] + hi[2])]]])


def test_oracle_probes_are_exact_for_linear_fields():
    xyz, t10 = p2_box((4, 3, 2))
    e, nu = 200.0, 0.3
    coef = np.tile([e, nu], (len(t10), 1))
    h = np.array([[1e-3, 2e-4, 0.0], [0.0, -5e-4, 1e-4], [3e-4, 0.0, 2e-4]])
    u = linear_u(xyz, h)
    temp = 20.0 + xyz @ np.array([1.0, -2.0, 0.5])
    pts = _probe_points(xyz, np.random.default_rng(1))
    disp, stress, mises, tv, hits = oracle.probes(xyz, t10, coef, u, pts, temperature=temp)
    assert hits.min() >= 1 and hits.max() >= 6  # corners are shared by several cells
    assert np.allclose(disp, pts @ h.T, rtol=0, atol=1e-14)
    eps = 0.5 * (h + h.T)
    want = iso_stress([eps[0, 0], eps[1, 1], eps[2, 2], eps[0, 1], eps[1, 2], eps[0, 2]], e, nu)
    assert np.allclose(stress, want, rtol=1e-12, atol=1e-12)
    assert np.allclose(tv, 20.0 + pts @ np.array([1.0, -2.0, 0.5]), rtol=0, atol=1e-12)
    with pytest.raises(oracle.OracleError):
        oracle.probes(xyz, t10, coef, u, [[100.0, 0.0, 0.0]])


@pytest.mark.gpu
def test_gpu_probes_are_bit_identical_with_the_oracle():
    from femahoy_b200.recover import Recovery
    xyz, t10 = p2_box((6, 4, 3))
    rng = np.random.default_rng(5)
    coef = np.column_stack([rng.uniform(100, 300, len(t10)), rng.uniform(0.2, 0.35, len(t10))])
    exp = rng.uniform(0, 1e-5, size=(len(t10), 3))
    u = rng.standard_normal(3 * len(xyz)) * 1e-3
    temp = 20.0 + rng.standard_normal(len(xyz))
    dtemp = temp - 20.0
    pts = _probe_points(xyz, rng)
    rec = Recovery(xyz, t10, coef, expansion=exp)
    got = rec.probes(u, pts, dtemp=dtemp, temperature=temp)
    want = oracle.probes(xyz, t10, coef, u, pts, expansion=exp, dtemp=dtemp, temperature=temp)
    for key, w in zip(("displacement", "stress", "mises", "temperature", "hits"), want):
        g = got[key]
        assert g.shape == w.shape, key
        if g.dtype == np.float64:
            assert np.array_equal(g.view(np.uint64), w.view(np.uint64)), key
        else:
            assert np.array_equal(g, w), key
    # Without a temperature field the temperature is 0 and the stress has no thermal part.
    got = rec.probes(u, pts)
    want = oracle.probes(xyz, t10, coef, u, pts, expansion=exp)
    assert np.array_equal(got["stress"].view(np.uint64), want[1].view(np.uint64))
    assert not got["temperature"].any()


@pytest.mark.gpu
def test_gpu_probe_in_no_cell_has_the_reference_text():
    import femahoy_b200 as fg
    from femahoy_b200.recover import Recovery
    xyz, t10 = p2_box((3, 2, 2))
    rec = Recovery(xyz, t10, np.tile([200.0, 0.3], (len(t10), 1)))
    u = np.zeros(3 * len(xyz))
    with pytest.raises(fg.FemError) as e:
        rec.probes(u, [[1.0, 1.0, 0.5], [1000.5, 0.0, -0.25]], names=["mid", "tip"])
    assert str(e.value) == "probe tip at (1000.5, 0, -0.25) is in no part"
    assert e.value.code == 5
