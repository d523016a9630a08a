"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, and only
as the checker / reported CPU baseline.  The product library (ugks2d_high_order_b200) never
imports it and has no CPU fallback.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libugks_oracle.so")


class UOParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nvel", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("ck", ctypes.c_int),
        ("pr", ctypes.c_double), ("omega", ctypes.c_double), ("mu_ref", ctypes.c_double),
        ("gamma", ctypes.c_double), ("cfl", ctypes.c_double),
        ("wall_ux", ctypes.c_double * 2), ("wall_tnative", ctypes.c_double * 2),
        ("ncfl", ctypes.c_double), ("nslab", ctypes.c_int), ("mass_rescale", ctypes.c_int),
        ("macro_sweeps", ctypes.c_int),
        ("residual_tol", ctypes.c_double), ("moment_tol", ctypes.c_double), ("min_alpha", ctypes.c_double),
        ("high_order", ctypes.c_int),
        ("s2_kinetic_wall", ctypes.c_int), ("s2_time_centered", ctypes.c_int), ("s2_face_time", ctypes.c_int),
        ("s2_shared_predictor", ctypes.c_int),
    ]


def build():
    """The oracle and its tangent build (oracle/tangent.py)."""
    subprocess.run(["make", "-s", "-C", HERE, "all", "tangent"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.uo_create.restype = ctypes.c_void_p
        L.uo_create.argtypes = [ctypes.POINTER(UOParams), dp, dp, dp]
        L.uo_destroy.argtypes = [ctypes.c_void_p]
        L.uo_set_state.argtypes = [ctypes.c_void_p, dp, dp, dp]
        L.uo_get_state.argtypes = [ctypes.c_void_p, dp, dp, dp]
        L.uo_init_freestream.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 4
        L.uo_timestep.restype = ctypes.c_double
        L.uo_timestep.argtypes = [ctypes.c_void_p]
        L.uo_explicit_step.argtypes = [ctypes.c_void_p, dp, dp]
        L.uo_interpolation.argtypes = [ctypes.c_void_p]
        L.uo_evolution.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.uo_compute_residual.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.uo_apply_explicit_update.argtypes = [ctypes.c_void_p, ctypes.c_double, dp]
        L.uo_implicit_step.argtypes = [ctypes.c_void_p, dp, ctypes.c_int]
        L.uo_implicit_init.argtypes = [ctypes.c_void_p]
        L.uo_s2_evolution.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.uo_s2_compute_residual.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.uo_s2_init_state.argtypes = [ctypes.c_void_p]
        L.uo_s2cn2_init.argtypes = [ctypes.c_void_p]
        L.uo_s2cn2_step.argtypes = [ctypes.c_void_p, dp, ctypes.c_int]
        for name in ("uo_res_macro", "uo_res_h", "uo_res_b", "uo_wall_aero", "uo_face_x_h", "uo_face_y_h",
                     "uo_face_x_w", "uo_face_y_w", "uo_phys_eq_h", "uo_phys_col_h", "uo_phys_col_b"):
            f = getattr(L, name)
            f.restype = dp
            f.argtypes = [ctypes.c_void_p]
        L.uo_project_moments.argtypes = [ctypes.c_int, dp, dp, dp, dp, dp, dp, dp, dp]
        L.uo_solve_dense4.argtypes = [dp, dp, dp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """CPU restatement of the reference solver for one Couette domain."""

    def __init__(self, case, u, v, w):
        self.case = case
        self.nx, self.ny, self.nvel = case.nx, case.ny, len(u)
        self.u = np.ascontiguousarray(u, dtype=np.float64)
        self.v = np.ascontiguousarray(v, dtype=np.float64)
        self.w = np.ascontiguousarray(w, dtype=np.float64)
        p = UOParams()
        p.nx, p.ny, p.nvel = case.nx, case.ny, self.nvel
        p.dx, p.dy = case.dx, case.dy
        p.ck = case.ck
        p.pr, p.omega, p.mu_ref, p.gamma, p.cfl = case.pr, case.omega, case.mu_ref, case.gamma, case.cfl
        p.wall_ux[0], p.wall_ux[1] = case.wall_ux
        p.wall_tnative[0], p.wall_tnative[1] = case.wall_tnative
        p.ncfl = case.ncfl
        p.nslab = case.nslab
        p.mass_rescale = int(case.mass_rescale)
        p.macro_sweeps = case.macro_sweeps
        p.residual_tol, p.moment_tol, p.min_alpha = case.residual_tol, case.moment_tol, case.min_alpha
        p.high_order = int(case.method == "HighOrderImplicit")
        p.s2_kinetic_wall = int(case.flux_wall == 0)
        p.s2_time_centered, p.s2_face_time = int(case.s2w1_time_centered), int(case.s2w1d_face_time)
        p.s2_shared_predictor = int(case.s2w2r_shared_predictor)
        self._params = p
        self.ptr = lib().uo_create(ctypes.byref(p), _p(self.u), _p(self.v), _p(self.w))

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().uo_destroy(self.ptr)
            self.ptr = None

    @property
    def ncell(self):
        return self.nx * self.ny

    def init_freestream(self, rho=1.0, U=0.0, V=0.0, tnative=None):
        t = self.case.tinf if tnative is None else tnative
        e = lib().uo_init_freestream(self.ptr, rho, U, V, t)
        if not e and self.case.method in ("HighOrderImplicit", "S2CN2"):
            e = lib().uo_s2_init_state(self.ptr)   # S2NativeInitializeState cold start
        if not e and self.case.method == "S2CN2":
            e = lib().uo_s2cn2_init(self.ptr)      # the conservation ledger of the cold start
        if e:
            raise RuntimeError(f"oracle init failed: {e}")

    def set_state(self, h, b, W):
        h = np.ascontiguousarray(h, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        W = np.ascontiguousarray(W, dtype=np.float64)
        lib().uo_set_state(self.ptr, _p(h), _p(b), _p(W))

    def get_state(self):
        h = np.empty((self.ny, self.nx, self.nvel))
        b = np.empty_like(h)
        W = np.empty((self.ny, self.nx, 4))
        lib().uo_get_state(self.ptr, _p(h), _p(b), _p(W))
        return h, b, W

    def timestep(self):
        return lib().uo_timestep(self.ptr)

    def explicit_step(self):
        dt = np.zeros(1)
        res = np.zeros(4)
        e = lib().uo_explicit_step(self.ptr, _p(dt), _p(res))
        if e:
            raise RuntimeError(f"oracle explicit step aborted with reference code {e}")
        return float(dt[0]), res

    def implicit_init(self):
        e = lib().uo_implicit_init(self.ptr)
        if e:
            raise RuntimeError(f"oracle implicit init failed: {e}")

    def implicit_step(self, nout=80):
        out = np.zeros(nout)
        e = lib().uo_implicit_step(self.ptr, _p(out), nout)
        if e:
            raise RuntimeError(f"oracle implicit step aborted with reference code {e}")
        return out

    CN_OUT = 22

    def s2cn2_init(self):
        """Conservation ledger of the current state (total0, empty wall balance); targets not built."""
        e = lib().uo_s2cn2_init(self.ptr)
        if e:
            raise RuntimeError(f"oracle S2CN2 init failed: {e}")

    def s2cn2_step(self):
        """One S2CN2 step; returns the diagnostics vector (dt, cnres, mmerr, ..., drift, ledger)."""
        out = np.zeros(self.CN_OUT)
        e = lib().uo_s2cn2_step(self.ptr, _p(out), self.CN_OUT)
        if e:
            raise RuntimeError(f"oracle S2CN2 step rejected with reference code {e}")
        return out

    def view(self, name, shape):
        ptr = getattr(lib(), "uo_" + name)(self.ptr)
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(ptr, shape=(n,)).reshape(shape).copy()


def set_threads(n=None):
    """Number of pthreads the oracle uses over faces and cells (all host cores by default)."""
    L = lib()
    if not hasattr(L, "uo_set_threads"):
        return 1
    L.uo_set_threads.argtypes = [ctypes.c_int]
    L.uo_set_threads.restype = ctypes.c_int
    return L.uo_set_threads(0 if n is None else int(n))
