"""Serving: many solve requests on 1 GPU (include/femgpu.h `femgpu_server_*`).

``Server(slots, budget_bytes)`` keeps solvers resident under keys (a mesh id), admits new ones
against a device-memory budget (least recently used idle solvers are freed first), and runs up
to ``slots`` solves at once, each on its solver's own stream, so requests overlap on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .solve import Solver, Stats


class Server:
    def __init__(self, slots=4, budget_bytes=150 << 30):
        h = C.c_void_p()
        L.check(L.lib().femgpu_server_new(slots, budget_bytes, C.byref(h)))
        self._h = h.value
        self._pending = {}  # ticket -> (b, x) kept alive until waited for

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            L.lib().femgpu_server_free(h)
            self._h = None

    def reserve(self, nbytes):
        """Frees idle resident solvers until ``nbytes`` more fit in the budget."""
        L.check(L.lib().femgpu_server_reserve(self._h, int(nbytes)))

    def put(self, key, solver: Solver):
        """The server takes ``solver`` (its handle is no longer the caller's)."""
        L.check(L.lib().femgpu_server_put(self._h, key, solver.handle))
        solver._h = None

    def has(self, key):
        return bool(L.lib().femgpu_server_has(self._h, key))

    def submit(self, key, b, x=None):
        """Queues a solve of the solver under ``key``; returns its ticket."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(len(b)) if x is None else x
        t = C.c_uint64()
        L.check(L.lib().femgpu_server_submit(self._h, key, L.ptr(b), L.ptr(x), C.byref(t)))
        self._pending[t.value] = (b, x)
        return t.value

    def wait(self, ticket):
        """(x, Stats, latency seconds); raises FemError with the solve's error."""
        st = L.Stats_t()
        lat = C.c_double()
        rc = L.lib().femgpu_server_wait(self._h, ticket, C.byref(st), C.byref(lat))
        b, x = self._pending.pop(ticket)
        L.check(rc)
        return x, Stats(st.iterations, st.residual, st.true_residual, st.seconds,
                        st.launches), lat.value

    @property
    def resident_bytes(self):
        return L.lib().femgpu_server_resident_bytes(self._h)

    @property
    def resident_count(self):
        return L.lib().femgpu_server_resident_count(self._h)
