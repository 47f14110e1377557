"""The C-ABI boundary on the CPU: libfemgpu.so loads and exports every entry point of
include/femgpu.h; the host-only entry points (the prolongation) match the oracle; the host mirror
keeps the reference's constants. No device is touched."""
import ctypes
import os
import re

import numpy as np

import femahoy_b200 as fg
import oracle
from femahoy_b200 import _lib
from femahoy_b200 import meshgen as mg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            text = open(os.path.join(ROOT, "include", f)).read()
            names |= set(re.findall(r"\b(femgpu_[a-z_0-9]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _declared()
    assert len(declared) >= 20
    for name in sorted(declared):
        assert hasattr(lib, name), name
    assert set(_lib.SIGNATURES) >= declared


def test_version_and_error_buffer():
    lib = fg.lib()
    assert b"sm_100a" in lib.femgpu_version()
    buf = ctypes.create_string_buffer(8)
    lib.femgpu_last_error(buf, 8)


def test_prolongation_matches_oracle():
    m = mg.box(6, 3, 2, (30.0, 15.0, 10.0))
    edges, t10 = oracle.quadratic(m.points, m.tets)
    prob = mg.beam_p2(edges, t10, mesh=m)
    free = prob.free
    p, cx = fg.prolongation(prob.xyz, m.n, edges, free)
    po, cxo = oracle.prolongation(prob.xyz, m.n, edges, free)
    ptr, idx, val = po.arrays()
    assert np.array_equal(p.ptr, ptr) and np.array_equal(p.idx, idx)
    assert np.array_equal(p.val, val)
    assert np.array_equal(cx, cxo)


def test_reference_constants():
    assert fg.STEADY_DIRECT_LIMIT == 3000 and fg.PCG_TOL == 1e-10 and fg.PCG_MAX_ITER == 500
    assert fg.TRANSIENT_DIRECT_LIMIT == 40_000
    assert int(fg.Method.Direct) == 0 and int(fg.Method.Multigrid) == 1


def test_invalid_arguments_fail_before_the_device():
    with np.testing.assert_raises(fg.FemError):
        fg.prolongation(np.zeros((4, 3)), 4, np.zeros((0, 2), np.uint32), np.array([50]))


def test_recovery_arguments_fail_before_the_device():
    """femgpu_recovery_new checks its sizes on the host: no part, more than 2048 parts, an
    empty mesh, a null array."""
    from femahoy_b200.recover import Recovery
    xyz = np.zeros((10, 3))
    t10 = np.arange(10, dtype=np.uint32)[None, :]
    coef = np.array([[1.0, 0.3]])
    for kw, what in [(dict(nparts=0), "no part"), (dict(nparts=4096), "2048 parts")]:
        with np.testing.assert_raises(fg.FemError) as e:
            Recovery(xyz, t10, coef, **kw)
        assert what in str(e.exception)
    with np.testing.assert_raises(fg.FemError) as e:
        Recovery(np.zeros((0, 3)), t10[:0], coef[:0])
    assert "empty mesh" in str(e.exception)
    h = ctypes.c_void_p()
    st = fg.lib().femgpu_recovery_new(10, None, 1, None, None, None, None, 1, None,
                                      ctypes.byref(h))
    assert st == _lib.INVALID
