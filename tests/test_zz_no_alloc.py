"""femgpu_reduced_rhs_noalloc against femgpu_reduced_rhs and the oracle, through the C ABI.

The no-allocation entry point exists for callers that must not call cudaMalloc or cudaFree:
code that shares the GPU with other work in flight (cudaFree waits for the whole device and
would stall it) and code whose device memory is held by its own pool allocator. Such a caller
owns every buffer; here torch plays that caller and allocates the inputs and outputs, while the
entry point itself allocates nothing and keeps its scratch in a fixed array in the library.

The two calls in a row use matrices of different sizes, so the second call must clear what the
first left in the shared scratch. This file sorts last so that a run stopping at the first
failure has run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import femahoy_b200 as fg
from femahoy_b200 import _lib
from femahoy_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _problems(with_oracle=False):
    heat = mg.heat_cube(12)
    K1 = fg.Csr.assemble(fg.P1_HEAT, heat.xyz, heat.nodes, heat.coef)
    beam = mg.cantilever_p1(dims=(10, 2, 2), lengths=(25.0, 5.0, 5.0))
    K2 = fg.Csr.assemble(fg.P1_ELASTIC, beam.xyz, beam.nodes, beam.coef)
    rng = np.random.default_rng(7)
    t2 = np.where(beam.fixed, rng.uniform(-0.1, 0.1, beam.n_unknowns), 0.0)
    out = [(K1, heat.load, heat.values, heat.free), (K2, beam.load, t2, beam.free)]
    if not with_oracle:
        return out
    import oracle
    K1o = oracle.pattern(heat.n_points, heat.nodes)
    K1o.assemble(0, heat.xyz, heat.nodes, heat.coef)
    K2o = oracle.pattern(3 * beam.n_points, oracle.dof_elements(beam.nodes))
    K2o.assemble(1, beam.xyz, beam.nodes, beam.coef)
    return [p + (o,) for p, o in zip(out, (K1o, K2o))]


def _noalloc(torch, K, load, t, free, arrays=None, nfree=None, check=True):
    """The caller's device buffers, 1 call of the entry point, and the result (with
    check=False: the status code and the message)."""
    ptr, idx, val = K.arrays() if arrays is None else arrays
    dev = "cuda"
    d_ptr = torch.from_numpy(ptr).to(dev)
    d_idx = torch.from_numpy(idx.view(np.int32)).to(dev)
    d_val = torch.from_numpy(val).to(dev)
    d_load = torch.from_numpy(np.ascontiguousarray(load, dtype=np.float64)).to(dev)
    d_t = torch.from_numpy(np.ascontiguousarray(t, dtype=np.float64)).to(dev)
    d_free = torch.from_numpy(np.ascontiguousarray(free, dtype=np.int64)).to(dev)
    d_out = torch.full((len(free),), np.nan, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    stream.synchronize()
    rc = fg.lib().femgpu_reduced_rhs_noalloc(
        K.n, ctypes.c_void_p(d_ptr.data_ptr()), ctypes.c_void_p(d_idx.data_ptr()),
        ctypes.c_void_p(d_val.data_ptr()), ctypes.c_void_p(d_load.data_ptr()),
        ctypes.c_void_p(d_t.data_ptr()), ctypes.c_void_p(d_free.data_ptr()),
        len(free) if nfree is None else nfree,
        ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    if not check:
        buf = ctypes.create_string_buffer(256)
        fg.lib().femgpu_last_error(buf, 256)
        return rc, buf.value.decode()
    _lib.check(rc)
    stream.synchronize()
    return d_out.cpu().numpy()


def test_noalloc_right_side_equals_the_allocating_one_twice_in_a_row():
    """... and the oracle's reduced_rhs (heat.rs:1219-1244), bit for bit."""
    torch = pytest.importorskip("torch")
    for K, load, t, free, Ko in _problems(with_oracle=True):
        expected = fg.reduced_rhs(K, load, t, free)
        got = _noalloc(torch, K, load, t, free)
        # The same sums in the same order: equal bit for bit (the other right-side tests are
        # bit-exact too).
        assert np.array_equal(got.view(np.uint64), expected.view(np.uint64))
        want = Ko.reduced_rhs(load, t, free)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def test_noalloc_refuses_a_matrix_past_its_scratch():
    max_rows = 4194304
    rc = fg.lib().femgpu_reduced_rhs_noalloc(max_rows + 1, ctypes.c_void_p(8),
                                             ctypes.c_void_p(8), ctypes.c_void_p(8),
                                             ctypes.c_void_p(8), ctypes.c_void_p(8),
                                             ctypes.c_void_p(8), 1, ctypes.c_void_p(8), None)
    assert rc == 7  # FEMGPU_ERR_TOO_LARGE, before any device work
    buf = ctypes.create_string_buffer(256)
    fg.lib().femgpu_last_error(buf, 256)
    assert b"4194304" in buf.value


def test_noalloc_rejects_bad_free_rows_and_columns_then_still_works():
    """The argument checks run on the device before the result is trusted; every bad case is
    FEMGPU_ERR_INVALID with its own text, and a valid call afterwards is still bit-exact (the
    scratch is cleared per call)."""
    torch = pytest.importorskip("torch")
    K, load, t, free = _problems()[0]
    n = K.n
    cases = [
        (np.concatenate([free[:-1], [n + 5]]), None, "a free row is out of range"),
        (np.concatenate([free[:3], free[2:]]), None, "the free rows hold a row twice"),
        (free[::-1].copy(), None, "the free rows are not increasing"),
    ]
    for bad_free, arrays, text in cases:
        rc, msg = _noalloc(torch, K, load, t, bad_free, arrays=arrays, check=False)
        assert rc == 5 and msg == text, (rc, msg)
    # A column index past n in a free row.
    ptr, idx, val = K.arrays()
    idx = idx.copy()
    idx[ptr[free[0]]] = n + 7
    rc, msg = _noalloc(torch, K, load, t, free, arrays=(ptr, idx, val), check=False)
    assert rc == 5 and msg == "a column index of a free row is out of range", (rc, msg)
    # More free rows than rows, and a count whose size_t wraps to a negative int64.
    for nfree in (n + 1, 2**64 - 1):
        rc, msg = _noalloc(torch, K, load, t, free, nfree=nfree, check=False)
        assert rc == 5 and msg == "more free rows than rows", (rc, msg)
    expected = fg.reduced_rhs(K, load, t, free)
    got = _noalloc(torch, K, load, t, free)
    assert np.array_equal(got.view(np.uint64), expected.view(np.uint64))
