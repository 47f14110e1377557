"""Batches: many small systems with several right sides each, solved together on 1 GPU
(include/femgpu.h ``femgpu_batch_*``).

``Batch(matrices, unknowns, nrhs)`` builds each system's multigrid hierarchy and combines the
systems level by level into block-diagonal operators; ``solve(b)`` runs every (system, right
side) pair as its own PCG solve in 1 device-side loop. ``b`` and the result are lists of
``(rows, nrhs)`` arrays, one per system.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .solve import Options, Unknowns, unknowns_c
from .sparse import Csr


@dataclass
class BatchStats:
    max_iterations: int
    mean_iterations: float
    max_residual: float
    max_true_residual: float
    seconds: float
    launches: int
    not_converged: int
    restarts: int


class Batch:
    def __init__(self, matrices: list[Csr], unknowns: list[Unknowns], nrhs=16, *,
                 precision=L.MIXED, options: Options | None = None):
        if len(matrices) != len(unknowns):
            raise L.FemError(L.INVALID, "1 unknowns description per matrix")
        opts = options or Options(precision=precision)
        keep = []
        us = (L.Unknowns_t * len(matrices))()
        for k, u in enumerate(unknowns):
            us[k] = unknowns_c(u, keep)
        hs = (C.c_void_p * len(matrices))(*[m.handle for m in matrices])
        oc = opts._c()
        h = C.c_void_p()
        L.check(L.lib().femgpu_batch_new(len(matrices), hs, us, nrhs, C.byref(oc), C.byref(h)))
        self._h = h.value
        self.nrhs = nrhs
        count = L.lib().femgpu_batch_systems(self._h, None)
        off = np.zeros(count + 1, dtype=np.uint64)
        L.lib().femgpu_batch_systems(self._h, L.ptr(off))
        self.offsets = off.astype(np.int64)
        self.rows = int(self.offsets[-1])

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            L.lib().femgpu_batch_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @property
    def count(self):
        return len(self.offsets) - 1

    def with_tol(self, tol):
        L.check(L.lib().femgpu_batch_set_tol(self._h, tol))
        return self

    def with_max_iter(self, m):
        L.check(L.lib().femgpu_batch_set_max_iter(self._h, m))
        return self

    def describe(self):
        """The setup seconds by phase."""
        buf = C.create_string_buffer(4096)
        L.check(L.lib().femgpu_batch_describe(self._h, buf, 4096))
        return buf.value.decode()

    def levels(self):
        k = L.lib().femgpu_batch_levels(self._h, None)
        out = np.zeros(k, dtype=np.uint64)
        L.lib().femgpu_batch_levels(self._h, L.ptr(out))
        return [int(v) for v in out]

    def device_bytes(self):
        return L.lib().femgpu_batch_bytes(self._h)

    def kernel_time(self, reps=50):
        """(ms, bytes) of 1 launch of the finest Chebyshev step over all right sides."""
        ms, nb = C.c_double(), C.c_double()
        L.check(L.lib().femgpu_batch_kernel_time(self._h, reps, C.byref(ms), C.byref(nb)))
        return ms.value, nb.value

    def stream(self):
        return L.lib().femgpu_batch_stream(self._h)

    def pack(self, parts):
        """The interleaved vector of per-system (rows, nrhs) arrays."""
        out = np.empty((self.rows, self.nrhs))
        for k, p in enumerate(parts):
            out[self.offsets[k]:self.offsets[k + 1]] = np.asarray(p).reshape(-1, self.nrhs)
        return out

    def unpack(self, v):
        v = np.asarray(v).reshape(self.rows, self.nrhs)
        return [v[self.offsets[k]:self.offsets[k + 1]].copy() for k in range(self.count)]

    def solve_packed(self, b, x=None, cancel=None):
        """Solves with interleaved host vectors (rows x nrhs); x (the start value, zeros when
        None) gets the solution. Returns (x, BatchStats)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x is None else x
        st = L.BatchStats_t()
        flag = None if cancel is None else C.byref(cancel)
        L.check(L.lib().femgpu_batch_solve(self._h, L.ptr(b), L.ptr(x), flag, C.byref(st)))
        return x, _stats(st)

    def solve(self, parts, cancel=None):
        x, st = self.solve_packed(self.pack(parts), cancel=cancel)
        return self.unpack(x), st

    def solve_device(self, b, x, cancel=None):
        """Device tensors (torch, float64, rows * nrhs values, contiguous) on the batch's stream."""
        st = L.BatchStats_t()
        flag = None if cancel is None else C.byref(cancel)
        L.check(L.lib().femgpu_batch_solve_device(self._h, C.c_void_p(b.data_ptr()),
                                                  C.c_void_p(x.data_ptr()), flag, C.byref(st)))
        return _stats(st)

    def segments(self):
        """Per (system, right side) of the last solve: iterations, true residual, recurrence
        residual, status (0 converged, 1 iteration limit, 2 broke down), each (count, nrhs)."""
        n = self.count * self.nrhs
        it = np.zeros(n, dtype=np.uint64)
        tr = np.zeros(n)
        rr = np.zeros(n)
        stt = np.zeros(n, dtype=np.int32)
        L.check(L.lib().femgpu_batch_segments(self._h, L.ptr(it), L.ptr(tr), L.ptr(rr),
                                              L.ptr(stt)))
        shape = (self.count, self.nrhs)
        return (it.astype(np.int64).reshape(shape), tr.reshape(shape), rr.reshape(shape),
                stt.reshape(shape))


def _stats(st):
    return BatchStats(st.max_iterations, st.mean_iterations, st.max_residual,
                      st.max_true_residual, st.seconds, st.launches, st.not_converged,
                      st.restarts)


class StreamResult(C.Structure):
    _fields_ = [("iterations", C.c_size_t), ("residual", C.c_double),
                ("true_residual", C.c_double), ("status", C.c_int), ("latency_s", C.c_double)]


class Stream:
    """Continuous batching over a Batch (include/femgpu.h ``femgpu_stream_*``): ``submit(system,
    b)`` queues 1 right side of 1 system and returns a ticket; the device loop admits it into a
    free slot of its system while the other slots keep iterating; ``wait(ticket)`` returns
    (x, StreamResult). The batch then serves only this stream."""

    def __init__(self, batch: Batch):
        h = C.c_void_p()
        L.check(L.lib().femgpu_stream_new(batch._h, C.byref(h)))
        self._h = h.value
        self._batch = batch  # the stream uses the batch's operators

    def rows(self, system):
        return int(self._batch.offsets[system + 1] - self._batch.offsets[system])

    def submit(self, system, b):
        b = L.arr(b, np.float64).reshape(-1)
        if 0 <= system < len(self._batch.offsets) - 1 and len(b) != self.rows(system):
            raise L.FemError(L.INVALID, "the right side has the system's rows")
        t = C.c_uint64()
        L.check(L.lib().femgpu_stream_submit(self._h, system, L.ptr(b), C.byref(t)))
        return (t.value, system)

    def wait(self, ticket):
        t, system = ticket
        x = np.empty(self.rows(system))
        res = StreamResult()
        L.check(L.lib().femgpu_stream_wait(self._h, t, L.ptr(x), C.byref(res)))
        return x, res

    def counts(self):
        loops, served = C.c_size_t(), C.c_size_t()
        L.check(L.lib().femgpu_stream_counts(self._h, C.byref(loops), C.byref(served)))
        return loops.value, served.value

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            L.lib().femgpu_stream_free(h)
            self._h = None

    def __del__(self):
        self.close()
