"""Post-solve recovery of P2 elasticity (elastic_tet.rs:367-427, 482-483).

CPU: the oracle against the analytic answers of the reference's integration tests (a uniform
stress is exact, tests/elastic_tet.rs:134-197; a free body under a uniform temperature change
has no stress, tests/elastic_tet.rs:209-225) and against an independent numpy restatement of
the loop. GPU: the CUDA recovery against the oracle, bit for bit (the principal stresses to a few
ulp: they call acos and cos)."""
import numpy as np
import pytest

import oracle
from femahoy_b200 import meshgen as mg

SHEAR = [(1, 2), (0, 2), (0, 1)]


def p2_box(dims, lengths=(3.0, 2.0, 1.5)):
    mesh = mg.box(*dims, lengths)
    edges, t10 = oracle.quadratic(mesh.points, mesh.tets)
    mid = 0.5 * (mesh.points[edges[:, 0]] + mesh.points[edges[:, 1]])
    return np.concatenate([mesh.points, mid]), t10


def linear_u(xyz, h):
    """u = H x: the displacement of the uniform strain sym(H) (plus a rotation)."""
    return (xyz @ np.asarray(h).T).reshape(-1)


def iso_stress(eps, e, nu):
    """The stress of the tensor strain eps (xx, yy, zz, xy, yz, xz) in an isotropic material."""
    lam = e * nu / ((1 + nu) * (1 - 2 * nu))
    mu = e / (2 * (1 + nu))
    tr = eps[0] + eps[1] + eps[2]
    return np.array([lam * tr + 2 * mu * eps[0], lam * tr + 2 * mu * eps[1],
                     lam * tr + 2 * mu * eps[2], 2 * mu * eps[3], 2 * mu * eps[4],
                     2 * mu * eps[5]])


def pair_values(xyz, t10, coef, u, expansion=None, dtemp=None):
    """numpy restatement of the (cell, point) values of the loop: stress and strain (E, 10, 6)
    in the output order, from tet10.rs:77-87 and 142-169 and elastic.rs:967-975."""
    ne = len(t10)
    g = np.stack([oracle.tet_gradients(xyz[t10[e, :4]])[0] for e in range(ne)])
    ue = u.reshape(-1, 3)[t10]
    sig = np.empty((ne, 10, 6))
    eps = np.empty((ne, 10, 6))
    for e in range(ne):
        normal, shear = oracle.isotropic(*coef[e])
        alpha = np.zeros(3) if expansion is None else expansion[e]
        thermal = normal @ alpha
        te = np.zeros(4) if dtemp is None else dtemp[t10[e, :4]]
        for c in range(10):
            lc = np.zeros(4)
            if c < 4:
                lc[c] = 1.0
            else:
                lc[mg.EDGES[c - 4]] = 0.5
            gr = np.empty((10, 3))
            for i in range(4):
                gr[i] = (4 * lc[i] - 1) * g[e, i]
            for k, (i, j) in enumerate(mg.EDGES):
                gr[4 + k] = 4 * (lc[i] * g[e, j] + lc[j] * g[e, i])
            en = np.zeros(6)
            for i in range(10):
                en[:3] += gr[i] * ue[e, i]
                for s, (a, b) in enumerate(SHEAR):
                    en[3 + s] += gr[i, a] * ue[e, i, b] + gr[i, b] * ue[e, i, a]
            s = np.concatenate([normal @ en[:3], shear * en[3:]])
            s[:3] -= thermal * (lc @ te)
            sig[e, c] = s[[0, 1, 2, 5, 3, 4]]
            eps[e, c] = [en[0], en[1], en[2], 0.5 * en[5], 0.5 * en[3], 0.5 * en[4]]
    return sig, eps


def mises(s):
    xx, yy, zz, xy, yz, xz = np.moveaxis(s, -1, 0)
    return np.sqrt(0.5 * ((xx - yy) ** 2 + (yy - zz) ** 2 + (zz - xx) ** 2)
                   + 3 * (xy * xy + yz * yz + xz * xz))


def random_case(dims=(3, 2, 2), seed=5, nparts=3, extra_point=True):
    rng = np.random.default_rng(seed)
    xyz, t10 = p2_box(dims)
    if extra_point:  # a point of no cell: its mean is 0 / max(count, 1)
        xyz = np.concatenate([xyz, [[9.0, 9.0, 9.0]]])
    n, ne = len(xyz), len(t10)
    coef = np.column_stack([rng.uniform(50e3, 210e3, ne), rng.uniform(0.1, 0.45, ne)])
    u = rng.standard_normal(3 * n) * 1e-3
    expansion = rng.uniform(1e-6, 2e-5, (ne, 3))
    dtemp = rng.uniform(-50, 50, n)
    part = rng.integers(0, nparts, ne).astype(np.uint32)
    singular = (rng.random(n) < 0.05).astype(np.uint8)
    return dict(xyz=xyz, t10=t10, coef=coef, u=u, expansion=expansion, dtemp=dtemp, part=part,
                nparts=nparts, singular=singular)


def oracle_of(c):
    return oracle.recover(c["xyz"], c["t10"], c["coef"], c["u"], expansion=c["expansion"],
                          dtemp=c["dtemp"], part=c["part"], nparts=c["nparts"],
                          singular=c["singular"])


# ------------------------------------------------------------------ oracle, CPU


def test_uniform_stress_is_exact():
    """tests/elastic_tet.rs:134-197: the displacement of szz = 10 gives szz = 10 and no other
    stress at every point, to 1e-8 as the reference asserts."""
    xyz, t10 = p2_box((3, 2, 2))
    e, nu = 70e3, 0.33
    coef = np.tile([e, nu], (len(t10), 1))
    h = np.diag([-nu * 10 / e, -nu * 10 / e, 10 / e])
    r = oracle.recover(xyz, t10, coef, linear_u(xyz, h))
    assert np.abs(r["stress"] - [0, 0, 10, 0, 0, 0]).max() < 1e-8
    assert np.abs(r["strain"] - [h[0, 0], h[1, 1], h[2, 2], 0, 0, 0]).max() < 1e-16
    assert np.abs(r["mises"] - 10).max() < 1e-8
    # Smith's closed form loses about half the digits at a double eigenvalue (acos near 1).
    assert np.abs(r["principal"] - [10, 0, 0]).max() < 1e-6


def test_general_uniform_strain_is_exact():
    """Any linear displacement: the tensor strain is sym(H) at every point, and the stress
    D eps (P2 holds linear fields exactly, tet10.rs:10-12)."""
    rng = np.random.default_rng(3)
    xyz, t10 = p2_box((2, 3, 2))
    e, nu = 210e3, 0.3
    h = rng.standard_normal((3, 3)) * 1e-3
    sym = 0.5 * (h + h.T)
    eps = np.array([sym[0, 0], sym[1, 1], sym[2, 2], sym[0, 1], sym[1, 2], sym[0, 2]])
    r = oracle.recover(xyz, t10, np.tile([e, nu], (len(t10), 1)), linear_u(xyz, h))
    assert np.abs(r["strain"] - eps).max() < 1e-15
    sig = iso_stress(eps, e, nu)
    assert np.abs(r["stress"] - sig).max() < 1e-9 * np.abs(sig).max()
    full = np.array([[sig[0], sig[3], sig[5]], [sig[3], sig[1], sig[4]],
                     [sig[5], sig[4], sig[2]]])
    ev = np.sort(np.linalg.eigvalsh(full))[::-1]
    assert np.abs(r["principal"] - ev).max() < 1e-9 * np.abs(sig).max()


def test_free_expansion_has_no_stress():
    """tests/elastic_tet.rs:209-225: a uniform temperature change on a free body expands it by
    alpha dT x with no stress (E alpha dT = 200 there; the same scale here)."""
    xyz, t10 = p2_box((3, 2, 2))
    e, nu, alpha, dtemp = 200e3, 0.3, 1e-5, 100.0
    u = (alpha * dtemp * xyz).reshape(-1)
    r = oracle.recover(xyz, t10, np.tile([e, nu], (len(t10), 1)), u,
                       expansion=np.full((len(t10), 3), alpha), dtemp=np.full(len(xyz), dtemp))
    assert np.abs(r["stress"]).max() < 1e-9 * e * alpha * dtemp
    assert np.abs(r["strain"] - np.array([alpha * dtemp] * 3 + [0.0] * 3)).max() < 1e-16


def test_oracle_matches_numpy_restatement():
    c = random_case()
    r = oracle_of(c)
    sig, eps = pair_values(c["xyz"], c["t10"], c["coef"], c["u"], c["expansion"], c["dtemp"])
    n = len(c["xyz"])
    ssum, esum, cnt = np.zeros((n, 6)), np.zeros((n, 6)), np.zeros(n)
    for e in range(len(c["t10"])):
        for k in range(10):
            v = c["t10"][e, k]
            ssum[v] += sig[e, k]
            esum[v] += eps[e, k]
            cnt[v] += 1
    cnt = np.maximum(cnt, 1)[:, None]
    scale = np.abs(ssum).max()
    assert np.abs(r["stress"] - ssum / cnt).max() <= 1e-13 * scale
    assert np.abs(r["strain"] - esum / cnt).max() <= 1e-13 * np.abs(esum).max()
    assert np.all(r["stress"][-1] == 0) and np.all(r["strain"][-1] == 0)
    assert np.abs(r["mises"] - mises(r["stress"])).max() <= 1e-13 * scale
    # The peaks: the largest value of each part, first on ties; the regular one over the pairs
    # whose point and corners are not singular.
    vm = mises(sig)
    sing = c["singular"].astype(bool)
    t10 = c["t10"]
    regular = ~(sing[t10] | sing[t10[:, :4]].any(axis=1)[:, None])
    for p, pk in enumerate(r["peaks"]):
        mask = np.broadcast_to((c["part"] == p)[:, None], vm.shape)
        assert abs(pk.mises - vm[mask].max()) <= 1e-13 * vm.max()
        assert abs(vm[pk.element, pk.local] - pk.mises) <= 1e-13 * vm.max()
        assert pk.point == t10[pk.element, pk.local]
        assert bool(pk.singular) == (not regular[pk.element, pk.local])
        rm = mask & regular
        assert abs(pk.regular_mises - vm[rm].max()) <= 1e-13 * vm.max()
        assert regular[pk.regular_element, pk.regular_local]


def test_zero_displacement_peaks_are_the_first_pairs():
    """All values 0: the peak stays at the first pair of each part (strict >), and the regular
    peak at the first regular pair."""
    c = random_case(seed=9)
    c["u"] = np.zeros_like(c["u"])
    c["expansion"] = None
    r = oracle_of(c)
    assert np.all(r["stress"] == 0)
    t10 = c["t10"]
    sing = c["singular"].astype(bool)
    for p, pk in enumerate(r["peaks"]):
        first = int(np.flatnonzero(c["part"] == p)[0])
        assert (pk.element, pk.local, pk.mises) == (first, 0, 0.0)
        pairs = [(e, k) for e in np.flatnonzero(c["part"] == p) for k in range(10)
                 if not (sing[t10[e, k]] or sing[t10[e, :4]].any())]
        assert (pk.regular_element, pk.regular_local) == pairs[0]


# ------------------------------------------------------------------ CUDA against the oracle


def peak_tuple(p):
    return (p.mises, p.element, p.local, p.point, int(p.singular), p.regular_mises,
            p.regular_element, p.regular_local, p.regular_point)


def same_bits(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def gpu_recover(c, **kw):
    from femahoy_b200.recover import Recovery
    rec = Recovery(c["xyz"], c["t10"], c["coef"], expansion=c["expansion"], part=c["part"],
                   nparts=c["nparts"], singular=c["singular"])
    return rec, rec.run(c["u"], c["dtemp"], **kw)


def check_parity(c):
    ref = oracle_of(c)
    _, got = gpu_recover(c)
    assert same_bits(got["stress"], ref["stress"])
    assert same_bits(got["strain"], ref["strain"])
    assert same_bits(got["mises"], ref["mises"])
    scale = max(np.nanmax(np.abs(ref["stress"])), 1e-300)
    assert np.allclose(got["principal"], ref["principal"], rtol=0, atol=1e-12 * scale,
                       equal_nan=True)
    for g, o in zip(got["peaks"], ref["peaks"]):
        gt, ot = peak_tuple(g), peak_tuple(o)
        assert gt[1:5] == ot[1:5] and gt[6:] == ot[6:], (gt, ot)
        assert same_bits([gt[0], gt[5]], [ot[0], ot[5]])
    return ref, got


@pytest.mark.gpu
def test_gpu_recovery_is_bit_identical_to_the_oracle():
    check_parity(random_case(dims=(4, 3, 3), seed=11, nparts=3))


@pytest.mark.gpu
def test_gpu_recovery_many_parts():
    """More parts than a block keeps in shared memory (64): the maxima go to global memory."""
    check_parity(random_case(dims=(4, 4, 3), seed=15, nparts=100))


@pytest.mark.gpu
def test_gpu_recovery_without_options():
    """No expansion, no temperature change, 1 part, no singular points."""
    c = random_case(dims=(3, 3, 2), seed=12, nparts=1)
    c.update(expansion=None, dtemp=None, part=None, singular=None)
    check_parity(c)


@pytest.mark.gpu
def test_gpu_recovery_ties_and_nan():
    """All values 0 (ties everywhere: the first pair wins), then a NaN displacement at a
    point: the peaks skip NaN, and a NaN first regular pair stays the regular peak."""
    c = random_case(dims=(3, 2, 2), seed=13, nparts=2)
    c["u"] = np.zeros_like(c["u"])
    c["expansion"] = None
    check_parity(c)
    c["u"][3 * int(c["t10"][0, 0])] = np.nan
    ref, _ = check_parity(c)
    assert np.isnan(ref["stress"][c["t10"][0, 0]]).any()


@pytest.mark.gpu
def test_gpu_recovery_uniform_strain_at_scale():
    """A 40 x 16 x 16 box (61,440 cells): the strain of a linear field is exact at every point,
    and the device form gives the bits of the host form."""
    import torch
    from femahoy_b200.recover import Recovery
    xyz, t10 = p2_box((40, 16, 16), (4.0, 1.6, 1.6))
    rng = np.random.default_rng(4)
    h = rng.standard_normal((3, 3)) * 1e-3
    e, nu = 70e3, 0.33
    rec = Recovery(xyz, t10, np.tile([e, nu], (len(t10), 1)))
    u = linear_u(xyz, h)
    r = rec.run(u)
    sym = 0.5 * (h + h.T)
    eps = np.array([sym[0, 0], sym[1, 1], sym[2, 2], sym[0, 1], sym[1, 2], sym[0, 2]])
    assert np.abs(r["strain"] - eps).max() < 1e-14
    sig = iso_stress(eps, e, nu)
    assert np.abs(r["stress"] - sig).max() < 1e-9 * np.abs(sig).max()
    dev = torch.device("cuda:0")
    n = len(xyz)
    ud = torch.from_numpy(u).to(dev)
    st, sn = torch.empty((n, 6), dtype=torch.float64, device=dev), torch.empty(
        (n, 6), dtype=torch.float64, device=dev)
    mi = torch.empty(n, dtype=torch.float64, device=dev)
    peaks = rec.run_device(ud, st, sn, mises=mi)
    assert same_bits(st.cpu().numpy(), r["stress"])
    assert same_bits(sn.cpu().numpy(), r["strain"])
    assert same_bits(mi.cpu().numpy(), r["mises"])
    assert peak_tuple(peaks[0]) == peak_tuple(r["peaks"][0])
    ms, nbytes = rec.last_time()
    assert ms > 0 and nbytes > 0


@pytest.mark.gpu
def test_gpu_recovery_errors():
    from femahoy_b200 import _lib as L
    from femahoy_b200.recover import Recovery
    c = random_case(dims=(2, 2, 1), seed=14, nparts=2)
    bad = c["coef"].copy()
    bad[1, 1] = 0.7
    with pytest.raises(L.FemError) as e:
        Recovery(c["xyz"], c["t10"], bad)
    assert e.value.code == L.MATERIAL
    with pytest.raises(L.FemError) as e:
        Recovery(c["xyz"], c["t10"], c["coef"], part=np.full(len(c["t10"]), 2), nparts=2)
    assert e.value.code == L.INVALID and "part past the last" in str(e.value)
    t = c["t10"].copy()
    t[0, 5] = len(c["xyz"])
    with pytest.raises(L.FemError) as e:
        Recovery(c["xyz"], t, c["coef"])
    assert e.value.code == L.INVALID
