"""Transient heat (include/femgpu.h ``femgpu_transient_*``): the backward-Euler loop of
crates/fem/src/heat.rs:686-733 with a lumped capacity, on the device.

``Transient(k, capacity, dt, free, unknowns)`` forms K + C/dt, its free-point submatrix and the
solver of that matrix once; ``run(steps, load, t0)`` steps from the temperatures ``t0``, each step
1 solve warm-started from the last temperatures, and returns the temperatures and energies of the
output steps.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .solve import Crossover, Options, Solver, Stats, Unknowns, unknowns_c
from .sparse import Csr

# solve.rs:24
TRANSIENT_DIRECT_LIMIT = 40_000


@dataclass
class Energy:
    """heat.rs:535-547 for a step with no radiation (see femgpu_energy)."""
    stored: float
    fixed: float
    gross: float


class Transient:
    def __init__(self, k: Csr, capacity, dt, free, unknowns: Unknowns, method=None,
                 crossover: Crossover | None = None, *, precision=L.FP64,
                 options: Options | None = None):
        capacity = L.arr(capacity, np.float64)
        free = L.arr(free, np.int64)
        crossover = crossover or Crossover.Unknowns(TRANSIENT_DIRECT_LIMIT)
        opts = options or Options(precision=precision)
        keep = []
        u = unknowns_c(unknowns, keep)
        cr, oc = crossover._c(), opts._c()
        h = C.c_void_p()
        m = -1 if method is None else int(method)
        L.check(L.lib().femgpu_transient_new(k.handle, L.ptr(capacity), float(dt), L.ptr(free),
                                             len(free), C.byref(u), m, C.byref(cr), C.byref(oc),
                                             C.byref(h)))
        self._h = h.value
        self._free = L.lib().femgpu_transient_free
        self.n = k.n
        self.nfree = len(free)
        self.solver = Solver._borrowed(L.lib().femgpu_transient_solver(self._h), len(free), self)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._free(h)
            self._h = None

    def run(self, steps, load, t0, output_every=1, cancelled=None):
        """heat.rs:709-733: returns (frames (F, n), energies (F Energy), temperatures after the
        last step, Stats summed over the steps). Frames are the steps s with
        s % output_every == 0 or s == steps."""
        n = self.n
        load = L.arr(load, np.float64)
        t = np.array(t0, dtype=np.float64, copy=True)
        every = max(int(output_every), 1)
        nframes = len([s for s in range(1, steps + 1) if s % every == 0 or s == steps])
        frames = np.empty((nframes, n))
        energies = (L.Energy_t * max(nframes, 1))()
        st = L.Stats_t()
        flag = cancelled if isinstance(cancelled, C.c_int) else None
        L.check(L.lib().femgpu_transient_run(self._h, steps, L.ptr(load), L.ptr(t), every,
                                             L.ptr(frames), C.cast(energies, C.c_void_p),
                                             C.byref(flag) if flag is not None else None,
                                             C.byref(st)))
        es = [Energy(e.stored, e.fixed, e.gross) for e in list(energies)[:nframes]]
        return frames, es, t, Stats(st.iterations, st.residual, st.true_residual, st.seconds,
                                    st.launches)
