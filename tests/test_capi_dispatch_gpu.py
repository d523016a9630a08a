"""The per-operator C ABI on the S2 methods, and the backing-store (LAP halo) copies.

The reference's Evolution() dispatches on the method (mod_Evolution.f90:35-41): S2CN2 and
HighOrderImplicit run S2NativeEvolution, the second-order methods EvolutionNative.  A Fortran driver
that calls the operators one by one (TimeStep, Evolution, ComputeResidual, the update) must get the
same step as the fused entry point; on S2CN2 that is ugks_s2cn2_steps, kernel for kernel, so the
states are compared bit for bit.
"""
import numpy as np
import pytest

from ugks2d_high_order_b200.case import reference_case, velocity_table

pytestmark = pytest.mark.gpu

HO_TOL = 1e-11   # GPU S2 evaluation vs the oracle (per-lane + butterfly vs sequential moment sums)


def _s2cn2_case():
    return reference_case("S2CN2").with_(ny=16, dy=1.0 / 16.0)


def test_s2cn2_per_operator_sequence_equals_steps():
    from ugks2d_high_order_b200.solver import Solver
    case = _s2cn2_case()
    vel = velocity_table(24)
    a, b = Solver(case, *vel), Solver(case, *vel)
    try:
        a.init_freestream()
        b.init_freestream()
        done, rep_a = a.step_s2cn2(3)   # one graph-replayed pair, then a single step
        assert done == 3
        for _ in range(3):
            b.time_step()
            b.evolution()
            b.compute_residual()
            b.apply_explicit_update()
        rep_b = b.s2cn2_report()
        sa, sb = a.download(), b.download()
        for x, y in zip(sa, sb):
            assert np.array_equal(x, y)
        assert np.array_equal(a.wall_aero(), b.wall_aero())
        assert np.array_equal(rep_a[:22], rep_b[:22])
        assert rep_b[22] == 1.0
        # and the sequence goes on from there exactly as the fused steps do
        a.step_s2cn2(1)
        b.time_step()
        b.evolution_s2(rebuild_targets=False)
        b.compute_residual()
        b.apply_explicit_update()
        for x, y in zip(a.download(), b.download()):
            assert np.array_equal(x, y)
    finally:
        a.close()
        b.close()


def test_operators_out_of_order_are_refused():
    from ugks2d_high_order_b200 import capi
    from ugks2d_high_order_b200.solver import Solver
    s = Solver(_s2cn2_case(), *velocity_table(24))
    try:
        s.init_freestream()
        L = s.L
        assert L.ugks_compute_residual(s.ctx, 0) == capi.UGKS_EINVAL          # before the evolution
        assert L.ugks_apply_explicit_update(s.ctx, None) == capi.UGKS_EINVAL  # before the residual
        s.time_step()
        s.evolution()
        assert L.ugks_apply_explicit_update(s.ctx, None) == capi.UGKS_EINVAL  # residual skipped
    finally:
        s.close()
    e = Solver(reference_case("Explicit").with_(ny=8, dy=1.0 / 8.0), *velocity_table(24))
    try:
        assert e.L.ugks_evolution_s2(e.ctx, 1) == capi.UGKS_EUNSUPPORTED
    finally:
        e.close()


@pytest.mark.parametrize("method", ["S2CN2", "HighOrderImplicit"])
def test_evolution_dispatches_to_the_s2_evolution(method):
    """ugks_evolution on an S2 context gives the high-order face fluxes of the oracle's S2 evaluation."""
    from oracle.oracle import Oracle, set_threads
    from ugks2d_high_order_b200 import capi
    from ugks2d_high_order_b200.solver import Solver
    set_threads(None)
    vel = velocity_table(24)
    base = _s2cn2_case()
    src = Solver(base, *vel)   # a state with developed wall layers: a few S2CN2 steps of the cold start
    try:
        src.init_freestream()
        src.step_s2cn2(4)
        h, b, W = src.download()
    finally:
        src.close()
    case = base if method == "S2CN2" else reference_case("HighOrderImplicit").with_(ny=16, dy=1.0 / 16.0, nslab=2)
    s = Solver(case, *vel)
    o = Oracle(case, *vel)
    try:
        s.upload(h, b, W)
        if method == "S2CN2":
            s.s2cn2_init()
        dt = s.time_step()
        s.evolution()
        o.set_state(h, b, W)
        assert o.timestep() == dt
        from oracle.oracle import lib
        assert lib().uo_s2_evolution(o.ptr, dt) == 0
        nx, ny, nv = case.nx, case.ny, len(vel[0])
        for name, shape in (("fxh", (ny, nx, nv)), ("fxb", (ny, nx, nv)), ("fyh", (ny + 1, nx, nv)),
                            ("fyb", (ny + 1, nx, nv)), ("fxw", (ny, nx, 4)), ("fyw", (ny + 1, nx, 4))):
            g = s.array(name, shape)
            ov = {"fxh": "face_x_h", "fyh": "face_y_h", "fxw": "face_x_w", "fyw": "face_y_w"}.get(name)
            if ov is None:
                continue
            r = o.view(ov, shape)
            assert np.abs(g - r).max() <= HO_TOL * np.abs(r).max(), (method, name)
        if method == "HighOrderImplicit":
            assert s.L.ugks_compute_residual(s.ctx, 0) == capi.UGKS_EUNSUPPORTED
            assert s.L.ugks_apply_explicit_update(s.ctx, None) == capi.UGKS_EUNSUPPORTED
    finally:
        s.close()


def test_backing_store_halo_copies():
    """ugks_*_state_halo read and write only the interior of [ny + 2 lap][nx + 2 lap][nvel] stores."""
    from ugks2d_high_order_b200.solver import Solver
    case = reference_case("Explicit").with_(ny=8, dy=1.0 / 8.0)
    vel = velocity_table(24)
    s = Solver(case, *vel)
    try:
        s.init_freestream()
        s.step_explicit(3)
        h, b, W = s.download()
        lap, nx, ny, nv = 2, case.nx, case.ny, len(vel[0])
        rng = np.random.default_rng(7)
        hs = rng.standard_normal((ny + 2 * lap, nx + 2 * lap, nv))
        bs = rng.standard_normal((ny + 2 * lap, nx + 2 * lap, nv))
        hs[lap:-lap, lap:-lap] = h
        bs[lap:-lap, lap:-lap] = b
        halo_h, halo_b = hs.copy(), bs.copy()
        s.upload_halo(hs, bs, W, lap)
        h2, b2, W2 = s.download()
        assert np.array_equal(h2, h) and np.array_equal(b2, b) and np.array_equal(W2, W)
        s.step_explicit(2)
        h3, b3, W3 = s.download()
        out_h = halo_h.copy()
        out_b = halo_b.copy()
        out_W = np.empty_like(W)
        s.download_halo(out_h, out_b, out_W, lap)
        assert np.array_equal(out_h[lap:-lap, lap:-lap], h3) and np.array_equal(out_b[lap:-lap, lap:-lap], b3)
        assert np.array_equal(out_W, W3)
        mask = np.ones(out_h.shape[:2], dtype=bool)
        mask[lap:-lap, lap:-lap] = False
        assert np.array_equal(out_h[mask], halo_h[mask]) and np.array_equal(out_b[mask], halo_b[mask])
    finally:
        s.close()
