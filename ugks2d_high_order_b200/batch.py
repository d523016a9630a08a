"""Batched S2CN2: many Couette instances of uneven grid and velocity-set sizes on one B200.

`Batch` mirrors `Solver`'s S2CN2 operators for a list of instances (case, velocity table): one
`run(n)` advances every instance by n steps with one CUDA graph launch per pair of steps
(libugks_b200.so, ugks_batch_*).  There is no counterpart in the reference, whose runs are one case
per MPI job; each instance follows exactly the single-instance S2CN2 step.
"""
import ctypes

import numpy as np

from . import capi
from .solver import Solver

_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return a.ctypes.data_as(_dp)


class Batch:
    def __init__(self, instances, device=0, max_streams=16):
        """instances: [(CouetteCase with method "S2CN2", (u, v, w))]."""
        self.L = capi.load()
        self.cases = [c for c, _ in instances]
        descs = (capi.UgksInstanceDesc * len(instances))()
        self._tables = []
        for d, (case, (u, v, w)) in zip(descs, instances):
            u, v, w = (np.ascontiguousarray(x, dtype=np.float64) for x in (u, v, w))
            self._tables.append((u, v, w))
            d.params = Solver.params_for(case, len(u))
            d.u, d.v, d.w = u.ctypes.data, v.ctypes.data, w.ctypes.data
        self.nvel = [len(t[0]) for t in self._tables]
        ptr = ctypes.c_void_p()
        capi.check(self.L, None, self.L.ugks_batch_create(len(instances), descs, device, max_streams, ctypes.byref(ptr)),
                   "ugks_batch_create")
        self.ptr = ptr
        self.n = len(instances)

    def close(self):
        if getattr(self, "ptr", None):
            self.L.ugks_batch_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def cell_velocities(self):
        return sum(c.nx * c.ny * nv for c, nv in zip(self.cases, self.nvel))

    def init_freestream(self, rho=1.0, U=0.0, V=0.0, tnative=2.0):
        capi.check(self.L, None, self.L.ugks_batch_init_freestream(self.ptr, rho, U, V, tnative), "batch init")

    def run(self, nsteps):
        """nsteps steps of every instance; returns (steps_done[n], status[n]).  Raises if any
        instance stopped (the others have still advanced)."""
        done = (ctypes.c_int * self.n)()
        st = (ctypes.c_uint * self.n)()
        code = self.L.ugks_batch_run(self.ptr, int(nsteps), done, st)
        self.last_done = np.array(done[:])
        self.last_status = np.array(st[:])
        if code != capi.UGKS_OK:
            bad = [(i, int(s), self.L.ugks_status_reference_code(s)) for i, s in enumerate(self.last_status) if s]
            raise capi.UgksError(code, f"batch run: instances stopped {bad[:8]}", int(bad[0][1]) if bad else 0,
                                 int(bad[0][2]) if bad else 0)
        return self.last_done, self.last_status

    def tune(self, steps=4):
        """Time 1, 2, 4, ... streams on the live batch (the instances advance) and keep the fastest."""
        k = ctypes.c_int()
        ms = ctypes.c_double()
        capi.check(self.L, None, self.L.ugks_batch_tune(self.ptr, int(steps), ctypes.byref(k), ctypes.byref(ms)), "tune")
        return k.value, ms.value

    def set_streams(self, k):
        capi.check(self.L, None, self.L.ugks_batch_set_streams(self.ptr, int(k)), "set_streams")

    def download(self, i):
        c, nv = self.cases[i], self.nvel[i]
        h = np.empty((c.ny, c.nx, nv))
        b = np.empty_like(h)
        W = np.empty((c.ny, c.nx, 4))
        capi.check(self.L, None, self.L.ugks_batch_download(self.ptr, i, _p(h), _p(b), _p(W)), "batch download")
        return h, b, W

    def upload(self, i, h, b, W):
        h, b, W = (np.ascontiguousarray(x, dtype=np.float64) for x in (h, b, W))
        capi.check(self.L, None, self.L.ugks_batch_upload(self.ptr, i, _p(h), _p(b), _p(W)), "batch upload")

    def report(self, i):
        r = np.zeros(capi.CN_REPORT_LEN)
        capi.check(self.L, None, self.L.ugks_batch_report(self.ptr, i, _p(r)), "batch report")
        return r

    def wall_aero(self, i):
        out = np.empty((2, self.cases[i].nx, 3))
        capi.check(self.L, None, self.L.ugks_batch_wall_aero(self.ptr, i, _p(out)), "batch wall_aero")
        return out

    @property
    def stream(self):
        return self.L.ugks_batch_stream(self.ptr)

    @property
    def launch_count(self):
        return self.L.ugks_batch_launch_count(self.ptr)
