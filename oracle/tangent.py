"""ctypes binding of the oracle's tangent build -- TEST INFRASTRUCTURE ONLY.

The tangent build (oracle/tangent.hpp, Makefile target `tangent`) is the oracle itself compiled with
(value, derivative) numbers: every run carries the exact derivative of each value along one direction
of the inputs -- the state h, b, W and the parameters mu_ref (the tau / Kn scale), the wall speeds and
the wall temperatures.  Tests use it as the forward-mode (Jacobian-vector product) reference for the
device adjoint.  Only tests/ import this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libugks_oracle_tangent.so")


class D2(ctypes.Structure):
    """One (value, derivative) number; a Structure so that ctypes passes it by value."""
    _fields_ = [("v", ctypes.c_double), ("d", ctypes.c_double)]


class UOParamsT(ctypes.Structure):
    """uo_params of the tangent build: every double is a (value, derivative) pair."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nvel", ctypes.c_int),
        ("dx", D2), ("dy", D2),
        ("ck", ctypes.c_int),
        ("pr", D2), ("omega", D2), ("mu_ref", D2), ("gamma", D2), ("cfl", D2),
        ("wall_ux", D2 * 2), ("wall_tnative", D2 * 2),
        ("ncfl", D2), ("nslab", ctypes.c_int), ("mass_rescale", ctypes.c_int),
        ("macro_sweeps", ctypes.c_int),
        ("residual_tol", D2), ("moment_tol", D2), ("min_alpha", D2),
        ("high_order", ctypes.c_int),
        ("s2_kinetic_wall", ctypes.c_int), ("s2_time_centered", ctypes.c_int), ("s2_face_time", ctypes.c_int),
        ("s2_shared_predictor", ctypes.c_int),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "tangent"], check=True)


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.uo_create.restype = vp
        L.uo_create.argtypes = [ctypes.POINTER(UOParamsT), vp, vp, vp]
        L.uo_destroy.argtypes = [vp]
        L.uo_set_state.argtypes = [vp, vp, vp, vp]
        L.uo_get_state.argtypes = [vp, vp, vp, vp]
        L.uo_init_freestream.argtypes = [vp] + [D2] * 4
        L.uo_s2_init_state.argtypes = [vp]
        L.uo_s2cn2_init.argtypes = [vp]
        L.uo_s2cn2_step.argtypes = [vp, vp, ctypes.c_int]
        L.uo_timestep.argtypes = [vp]
        L.uo_timestep.restype = D2
        L.uo_face_y_w.argtypes = [vp]
        L.uo_face_y_w.restype = ctypes.POINTER(ctypes.c_double)
        L.uo_set_threads.argtypes = [ctypes.c_int]
        L.uo_set_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _pair(value, deriv=0.0):
    return D2(float(value), float(deriv))


def _dual(value, deriv=None):
    """An interleaved (value, derivative) float64 array of value's shape + (2,)."""
    value = np.asarray(value, dtype=np.float64)
    out = np.zeros(value.shape + (2,))
    out[..., 0] = value
    if deriv is not None:
        out[..., 1] = deriv
    return np.ascontiguousarray(out)


class TangentOracle:
    """The oracle of one Couette case with derivatives along one input direction.

    dparams: the parameter part of the direction -- "mu_ref": d mu_ref, "wall_ux": (d bottom, d top),
    "wall_tnative": (d bottom, d top).  The state part is given to set_state."""

    def __init__(self, case, u, v, w, dparams=None, threads=None):
        dparams = dparams or {}
        L = lib()
        L.uo_set_threads(0 if threads is None else int(threads))
        self.case = case
        self.nx, self.ny, self.nvel = case.nx, case.ny, len(u)
        p = UOParamsT()
        p.nx, p.ny, p.nvel = case.nx, case.ny, self.nvel
        p.dx, p.dy = _pair(case.dx), _pair(case.dy)
        p.ck = case.ck
        p.pr, p.omega, p.gamma, p.cfl = _pair(case.pr), _pair(case.omega), _pair(case.gamma), _pair(case.cfl)
        p.mu_ref = _pair(case.mu_ref, dparams.get("mu_ref", 0.0))
        dux = dparams.get("wall_ux", (0.0, 0.0))
        dtw = dparams.get("wall_tnative", (0.0, 0.0))
        for s in range(2):
            p.wall_ux[s] = _pair(case.wall_ux[s], dux[s])
            p.wall_tnative[s] = _pair(case.wall_tnative[s], dtw[s])
        p.ncfl = _pair(case.ncfl)
        p.nslab, p.mass_rescale, p.macro_sweeps = case.nslab, int(case.mass_rescale), case.macro_sweeps
        p.residual_tol, p.moment_tol, p.min_alpha = _pair(case.residual_tol), _pair(case.moment_tol), _pair(case.min_alpha)
        p.high_order = int(case.method == "HighOrderImplicit")
        p.s2_kinetic_wall = int(case.flux_wall == 0)
        p.s2_time_centered, p.s2_face_time = int(case.s2w1_time_centered), int(case.s2w1d_face_time)
        p.s2_shared_predictor = int(case.s2w2r_shared_predictor)
        self._params = p
        self.dux = np.array(dux, dtype=np.float64)
        self.wall_ux = np.array(case.wall_ux, dtype=np.float64)
        self._vel = [_dual(a) for a in (u, v, w)]
        self.ptr = L.uo_create(ctypes.byref(p), *(a.ctypes.data for a in self._vel))

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().uo_destroy(self.ptr)
            self.ptr = None

    def init_freestream(self, rho=1.0, U=0.0, V=0.0, tnative=None):
        """The S2 cold start and the S2CN2 ledger (no derivative: the initial state is fixed)."""
        t = self.case.tinf if tnative is None else tnative
        L = lib()
        e = L.uo_init_freestream(self.ptr, _pair(rho), _pair(U), _pair(V), _pair(t))
        e = e or L.uo_s2_init_state(self.ptr) or L.uo_s2cn2_init(self.ptr)
        if e:
            raise RuntimeError(f"tangent oracle init failed: {e}")

    def set_state(self, h, b, W, dh=None, db=None, dW=None):
        """State and its direction; the S2CN2 ledger and the volume targets are rebuilt from it."""
        hs, bs, Ws = _dual(h, dh), _dual(b, db), _dual(W, dW)
        L = lib()
        L.uo_set_state(self.ptr, hs.ctypes.data, bs.ctypes.data, Ws.ctypes.data)
        if L.uo_s2cn2_init(self.ptr):
            raise RuntimeError("tangent oracle S2CN2 init failed")

    def get_state(self):
        """(h, dh, b, db, W, dW) of the current state."""
        S = (self.ny, self.nx, self.nvel)
        h, b, W = np.zeros(S + (2,)), np.zeros(S + (2,)), np.zeros((self.ny, self.nx, 4, 2))
        lib().uo_get_state(self.ptr, h.ctypes.data, b.ctypes.data, W.ctypes.data)
        return h[..., 0], h[..., 1], b[..., 0], b[..., 1], W[..., 0], W[..., 1]

    def s2cn2_step(self):
        out = np.zeros((22, 2))
        e = lib().uo_s2cn2_step(self.ptr, out.ctypes.data, 22)
        if e:
            raise RuntimeError(f"tangent oracle S2CN2 step rejected with reference code {e}")
        return out[:, 0]

    def wall_outputs(self, dt):
        """[wall (bottom, top)][shear, heat] of the last evolution and their derivatives: the wall-face
        means of pnt = -rate_x and qn = rate_E - u_w rate_x, rate = wall macro flux / (dt dx), in the
        native frame of PublishWallDiagnostics (mod_S2NativeAdapter.f90:1075-1097)."""
        nx, ny = self.nx, self.ny
        n = (ny + 1) * nx * 4 * 2
        fy = np.ctypeslib.as_array(lib().uo_face_y_w(self.ptr), shape=(n,)).reshape(ny + 1, nx, 4, 2).copy()
        val = np.zeros((2, 2))
        der = np.zeros((2, 2))
        for wall, row in ((0, 0), (1, ny)):
            r = fy[row] / (dt * self.case.dx)   # [nx][4][value, derivative]
            ux, dux = self.wall_ux[wall], self.dux[wall]
            val[wall, 0] = (-r[:, 1, 0]).mean()
            der[wall, 0] = (-r[:, 1, 1]).mean()
            val[wall, 1] = (r[:, 3, 0] - ux * r[:, 1, 0]).mean()
            der[wall, 1] = (r[:, 3, 1] - ux * r[:, 1, 1] - dux * r[:, 1, 0]).mean()
        return val, der
