"""Host-side mirror of the reference's hot-path operator interface.

The reference calls argument-less Fortran subroutines from Solve_UGKS (src/mod_Solve.f90:84-186):
TimeStep, Interpolation, Evolution, ComputeResidual, ApplyExplicitUpdate,
ApplySteadyImplicitUpdate.  `Solver` exposes the same operators, in the same order and with the
same failure behaviour (a numerical gate failure raises `UgksError` carrying the reference's
MPI_Abort code), over one device-resident Couette domain.  All compute runs in libugks_b200.so.
"""
import ctypes

import numpy as np

from . import capi
from .case import CouetteCase

_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return a.ctypes.data_as(_dp)


class Solver:
    """One Couette domain resident on a B200."""

    def __init__(self, case: CouetteCase, u, v, w, device=0):
        self.L = capi.load()
        self.case = case
        self.u = np.ascontiguousarray(u, dtype=np.float64)
        self.v = np.ascontiguousarray(v, dtype=np.float64)
        self.w = np.ascontiguousarray(w, dtype=np.float64)
        self.nx, self.ny, self.nvel = case.nx, case.ny, len(self.u)
        p = self.params_for(case, self.nvel)
        self._params = p
        ctx = ctypes.c_void_p()
        self._check(self.L.ugks_ctx_create(ctypes.byref(p), _p(self.u), _p(self.v), _p(self.w), device,
                                           ctypes.byref(ctx)), "ugks_ctx_create", None)
        self.ctx = ctx

    @staticmethod
    def params_for(case, nvel):
        """ugks_params of a case (the C ABI's view of Config.ini)."""
        p = capi.UgksParams()
        p.nx, p.ny, p.nvel = case.nx, case.ny, nvel
        p.dx, p.dy = case.dx, case.dy
        p.ck = case.ck
        p.pr, p.omega, p.mu_ref, p.cfl = case.pr, case.omega, case.mu_ref, case.cfl
        p.wall_ux[0], p.wall_ux[1] = case.wall_ux
        p.wall_tnative[0], p.wall_tnative[1] = case.wall_tnative
        p.fixed_dt = 0.0
        p.method = {"ImplicitSteady": capi.UGKS_METHOD_IMPLICIT_STEADY,
                    "HighOrderImplicit": capi.UGKS_METHOD_HIGH_ORDER_IMPLICIT,
                    "S2CN2": capi.UGKS_METHOD_S2CN2}.get(case.method, capi.UGKS_METHOD_EXPLICIT)
        p.ncfl, p.nslab, p.mass_rescale, p.macro_sweeps = case.ncfl, case.nslab, int(case.mass_rescale), case.macro_sweeps
        p.residual_tol, p.moment_tol, p.min_alpha = case.residual_tol, case.moment_tol, case.min_alpha
        p.s2_kinetic_wall = int(case.flux_wall == 0)
        p.s2_time_centered, p.s2_face_time = int(case.s2w1_time_centered), int(case.s2w1d_face_time)
        p.s2_shared_predictor = int(case.s2w2r_shared_predictor)
        return p

    def _check(self, code, what, ctx="self"):
        capi.check(self.L, self.ctx if ctx == "self" else ctx, code, what)

    def close(self):
        if getattr(self, "ctx", None):
            self.L.ugks_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ncell(self):
        return self.nx * self.ny

    # ---- state
    def init_freestream(self, rho=1.0, U=0.0, V=0.0, tnative=None):
        t = self.case.tinf if tnative is None else tnative
        self._check(self.L.ugks_init_freestream(self.ctx, rho, U, V, t), "ugks_init_freestream")

    def upload(self, h, b, W):
        h = np.ascontiguousarray(h, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        W = np.ascontiguousarray(W, dtype=np.float64)
        assert h.size == self.ncell * self.nvel and W.size == self.ncell * 4
        self._check(self.L.ugks_upload_state(self.ctx, _p(h), _p(b), _p(W)), "ugks_upload_state")

    def download(self):
        h = np.empty((self.ny, self.nx, self.nvel))
        b = np.empty_like(h)
        W = np.empty((self.ny, self.nx, 4))
        self._check(self.L.ugks_download_state(self.ctx, _p(h), _p(b), _p(W)), "ugks_download_state")
        return h, b, W

    def upload_halo(self, h, b, W, lap=2):
        """Upload from the reference's backing stores with their LAP halo: h, b of shape
        [ny + 2 lap][nx + 2 lap][nvel] (cell_h_store(Nvel, 1-LAP:nx+LAP, 1-LAP:ny+LAP)); the halo is not read."""
        h = np.ascontiguousarray(h, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        W = np.ascontiguousarray(W, dtype=np.float64)
        assert h.shape == (self.ny + 2 * lap, self.nx + 2 * lap, self.nvel) and h.shape == b.shape
        assert W.size == self.ncell * 4
        self._check(self.L.ugks_upload_state_halo(self.ctx, _p(h), _p(b), _p(W), int(lap)), "ugks_upload_state_halo")

    def download_halo(self, h, b, W=None, lap=2):
        """Download into backing stores with a LAP halo (the arrays' halo is left as it is)."""
        assert h.flags.c_contiguous and b.flags.c_contiguous and h.dtype == np.float64 and b.dtype == np.float64
        assert h.shape == (self.ny + 2 * lap, self.nx + 2 * lap, self.nvel) and h.shape == b.shape
        if W is not None:
            assert W.flags.c_contiguous and W.dtype == np.float64 and W.size == self.ncell * 4
        self._check(self.L.ugks_download_state_halo(self.ctx, _p(h), _p(b), _p(W) if W is not None else None, int(lap)),
                    "ugks_download_state_halo")

    # ---- reference operators
    def time_step(self):
        """TimeStep (mod_Solve.f90:373-421): global CFL dt, computed on the device."""
        dt = np.zeros(1)
        self._check(self.L.ugks_timestep(self.ctx, _p(dt)), "TimeStep")
        return float(dt[0])

    def evolution(self):
        """Interpolation + Evolution (mod_Interpolation.f90:26-90, mod_Evolution.f90:35-41): the
        second-order evolution, or S2NativeEvolution on the S2 methods as the reference dispatches."""
        self._check(self.L.ugks_evolution(self.ctx), "Evolution")

    def evolution_s2(self, rebuild_targets=False):
        """S2NativeEvolution (mod_S2NativeAdapter.f90:469-599) with the volume targets rebuilt or kept."""
        self._check(self.L.ugks_evolution_s2(self.ctx, int(rebuild_targets)), "S2NativeEvolution")

    def compute_residual(self, with_collision=False):
        """ComputeResidual (mod_Residual.f90:17-132)."""
        self._check(self.L.ugks_compute_residual(self.ctx, int(with_collision)), "ComputeResidual")

    def apply_explicit_update(self):
        """ApplyExplicitUpdate (mod_TimeIntegrator.f90:16-134); returns the `res` vector."""
        res = np.zeros(4)
        self._check(self.L.ugks_apply_explicit_update(self.ctx, _p(res)), "ApplyExplicitUpdate")
        return res

    def step_explicit(self, nsteps=1):
        """nsteps Explicit steps (mod_Solve.f90:84-186) fused and graph-replayed; returns (dt, res)."""
        dt = np.zeros(1)
        res = np.zeros(4)
        self._check(self.L.ugks_step_explicit(self.ctx, int(nsteps), _p(dt), _p(res)), "Explicit step")
        return float(dt[0]), res

    # ---- ImplicitSteady (mod_SteadyImplicit.f90:379-462 + mod_ClosedCouetteMass.f90 + mod_R5Observe.f90)
    def implicit_init(self):
        """InitializeClosedMass: persistent M0 from the current state, new residual-reference epoch."""
        self._check(self.L.ugks_implicit_init(self.ctx), "InitializeClosedMass")

    def implicit_restore(self, m0, reference=None):
        """Resume a restarted run: the persistent M0 of closed_mass_rank*.bin and, when given, the
        (reference_h, reference_b) pair of residual_reference.in instead of a new epoch."""
        rh, rb = reference if reference is not None else (0.0, 0.0)
        self._check(self.L.ugks_implicit_restore(self.ctx, float(m0), float(rh), float(rb), int(reference is not None)),
                    "ReadMassRestart")

    def step_implicit(self, max_steps=1):
        """Up to max_steps accepted pseudo-steps; stops when the five-state gate has passed 5 times.
        Returns (steps_done, converged, report) where report is the last accepted state's
        sparse_residual.csv row (layout in include/ugks_b200.h)."""
        done = ctypes.c_int()
        conv = ctypes.c_int()
        rep = np.zeros(capi.REPORT_LEN)
        self._check(self.L.ugks_implicit_steps(self.ctx, int(max_steps), ctypes.byref(done), ctypes.byref(conv),
                                               _p(rep)), "ApplySteadyImplicitUpdate")
        return done.value, bool(conv.value), rep

    def implicit_state(self):
        st = np.zeros(16)
        rep = np.zeros(capi.REPORT_LEN)
        self._check(self.L.ugks_implicit_state(self.ctx, _p(st), _p(rep)), "implicit_state")
        return st, rep

    # ---- S2CN2, the explicit high-order method (S2NativeEvolution + S2NativeApplyUpdate)
    def s2cn2_init(self):
        """S2NativeInitializeState's ledger and the volume targets of the current state (done by
        init_freestream; needed after upload)."""
        self._check(self.L.ugks_s2cn2_init(self.ctx), "S2CN2 init")

    def step_s2cn2(self, nsteps=1):
        """nsteps S2CN2 steps.  Returns (steps_done, report) with report the last step's
        diagnostics (layout in include/ugks_b200.h).  A rejected step raises UgksError with
        reference code 203 after the accepted ones are kept."""
        done = ctypes.c_int()
        rep = np.zeros(capi.CN_REPORT_LEN)
        code = self.L.ugks_s2cn2_steps(self.ctx, int(nsteps), ctypes.byref(done), _p(rep))
        self.last_steps_done = done.value
        self._check(code, "S2NativeApplyUpdate")
        return done.value, rep

    def s2cn2_report(self):
        """The last S2CN2 step's report (layout in include/ugks_b200.h)."""
        rep = np.zeros(capi.CN_REPORT_LEN)
        self._check(self.L.ugks_s2cn2_report(self.ctx, _p(rep)), "S2CN2 report")
        return rep

    # ---- the S2CN2 adjoint: gradients of the wall outputs (bottom shear, bottom heat, top shear, top heat)
    # with respect to (mu_ref, wall_ux[0], wall_ux[1], wall_tnative[0], wall_tnative[1])
    def s2cn2_forward_checkpointed(self, nsteps, every=50):
        """nsteps S2CN2 steps storing a checkpoint every `every` steps; returns the wall outputs [4]."""
        out = np.zeros(4)
        self._check(self.L.ugks_s2cn2_forward_checkpointed(self.ctx, int(nsteps), int(every), _p(out)),
                    "S2CN2 checkpointed forward")
        return out

    def s2cn2_backward(self, seed, initial_state=False):
        """The reverse sweep of the last checkpointed forward: the gradient [5] of sum(seed * outputs),
        and, with initial_state, the cotangents (h, b, W) of the initial state."""
        seed = np.ascontiguousarray(seed, dtype=np.float64)
        assert seed.size == 4
        grad = np.zeros(5)
        if initial_state:
            gh = np.zeros((self.ny, self.nx, self.nvel))
            gb = np.zeros_like(gh)
            gW = np.zeros((self.ny, self.nx, 4))
            self._check(self.L.ugks_s2cn2_backward(self.ctx, _p(seed), _p(grad), _p(gh), _p(gb), _p(gW)),
                        "S2CN2 backward")
            return grad, (gh, gb, gW)
        self._check(self.L.ugks_s2cn2_backward(self.ctx, _p(seed), _p(grad), None, None, None), "S2CN2 backward")
        return grad

    def s2cn2_step_vjp(self, gh=None, gb=None, gW=None, seed=None):
        """The vector-Jacobian product of one S2CN2 step at the current state: output cotangents (gh, gb,
        gW; None = 0) and the wall outputs' seed [4] -> (gh_in, gb_in, gW_in, grad[5])."""
        def opt(a, shape):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            assert a.size == int(np.prod(shape))
            return a
        S = (self.ny, self.nx, self.nvel)
        gh, gb, gW = opt(gh, S), opt(gb, S), opt(gW, (self.ny, self.nx, 4))
        seed = opt(seed, (4,))
        oh, ob, oW, grad = np.zeros(S), np.zeros(S), np.zeros((self.ny, self.nx, 4)), np.zeros(5)
        P = lambda a: _p(a) if a is not None else None
        self._check(self.L.ugks_s2cn2_step_vjp(self.ctx, P(gh), P(gb), P(gW), P(seed), _p(oh), _p(ob), _p(oW), _p(grad)),
                    "S2CN2 step VJP")
        return oh, ob, oW, grad

    def s2cn2_test_reject(self, step):
        """Force step `step` (1-based) of the next step_s2cn2 call to fail its conservation gate
        (the reference's S2D3_TEST_GLOBAL_REJECT / S2E3_TEST_REJECT_STEP hooks)."""
        self._check(self.L.ugks_s2cn2_test_reject(self.ctx, int(step)), "S2CN2 test reject")

    def wall_aero(self):
        out = np.empty((2, self.nx, 3))
        self._check(self.L.ugks_wall_aero(self.ctx, _p(out)), "wall_aero")
        return out

    FIELDS = ("r", "u", "v", "T", "p", "sxx", "sxy", "syy", "qx", "qy")

    def macro_fields(self):
        """Output's steady fields per cell (mod_Output.f90:102-116), computed on the device:
        array [ny][nx][10] in the order of `FIELDS`."""
        out = np.empty((self.ny, self.nx, 10))
        self._check(self.L.ugks_macro_fields(self.ctx, _p(out)), "macro_fields")
        return out

    def profiles(self):
        """x-averaged 64-point profiles of `FIELDS` (the rows of profiles_three_methods.plt)."""
        return self.macro_fields().mean(axis=1)

    def array(self, name, shape):
        out = np.empty(int(np.prod(shape)))
        self._check(self.L.ugks_copy_array(self.ctx, name.encode(), _p(out), out.size), f"copy {name}")
        return out.reshape(shape)

    @property
    def stream(self):
        return self.L.ugks_stream(self.ctx)

    def synchronize(self):
        self._check(self.L.ugks_synchronize(self.ctx), "synchronize")

    def profile(self, enable=True, graph=False):
        """Per-kernel (explicit) and per-stage (implicit) event timing; graph=True times the implicit
        stages inside the batch graphs instead of in un-graphed steps."""
        self._check(self.L.ugks_profile_enable(self.ctx, 2 if (enable and graph) else int(bool(enable))), "profile")

    def profile_read(self, kernel):
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        self._check(self.L.ugks_profile_read(self.ctx, kernel.encode(), ctypes.byref(ms), ctypes.byref(n)),
                    "profile_read")
        return ms.value, n.value

    @property
    def launch_count(self):
        return self.L.ugks_launch_count(self.ctx)
