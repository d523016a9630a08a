"""The CPU oracle against the reference's own printed numbers (no GPU needed)."""
import numpy as np
import pytest

from oracle.oracle import Oracle, lib
from ugks2d_high_order_b200.case import reference_case


def _round_sig(x, digits):
    return float(f"{x:.{digits - 1}e}")


def test_explicit_two_steps_match_reference_log(velocity, golden):
    """docs/release_checks/low_explicit/stdout.log:41-43 prints dtPhysical and res after 2 steps."""
    g = golden["low_explicit_2step"]
    o = Oracle(reference_case("Explicit"), *velocity)
    o.init_freestream()
    for _ in range(2):
        dt, res = o.explicit_step()
    assert _round_sig(dt, 7) == pytest.approx(g["dtPhysical"], rel=0, abs=0)
    for m in range(4):
        assert _round_sig(res[m], 7) == g["res"][m], (m, res[m], g["res"][m])


def test_static_equilibrium_one_step(velocity, golden):
    """checks/static_equilibrium: stationary walls, uniform gas; one explicit step keeps the state
    (reference maxima in checks/VERIFICATION.json: residual ~3e-14, update ~1e-17)."""
    case = reference_case("Explicit").with_(wall_ux=(0.0, 0.0))
    o = Oracle(case, *velocity)
    o.init_freestream()
    h0, b0, W0 = o.get_state()
    o.explicit_step()
    h1, b1, W1 = o.get_state()
    ref = golden["static_equilibrium"]["final_static_le"]
    assert np.abs(W1 - W0).max() <= 100 * max(ref["update_max"]["W"], 1e-18)
    assert np.abs(h1 - h0).max() <= 1e-15
    assert np.abs(b1 - b0).max() <= 1e-15
    rw = np.abs(o.view("res_macro", (o.ncell, 4))).max()
    assert rw <= 1e-12


def test_projection_restores_moments(velocity):
    u, v, w = velocity
    rng = np.random.default_rng(7)
    n = len(u)
    h = np.exp(-0.5 * (u ** 2 + v ** 2)) * (1 + 0.01 * rng.standard_normal(n)) / (2 * np.pi)
    b = 0.5 * h
    target = np.array([1.0, 0.1, -0.2, 1.6])
    rh, rb = h.copy(), b.copy()
    import ctypes
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ok = lib().uo_project_moments(n, P(h), P(b), P(target), P(u), P(v), P(w), P(rh), P(rb))
    assert ok == 1
    m = np.array([np.sum(w * h), np.sum(w * u * h), np.sum(w * v * h), 0.5 * np.sum(w * ((u * u + v * v) * h + b))])
    assert np.abs(m - target).max() <= 1e-12


def test_solve_dense4_pivoting():
    import ctypes
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    rng = np.random.default_rng(1)
    A = rng.standard_normal((4, 4))
    A[0, 0] = 0.0   # forces a row swap
    x = rng.standard_normal(4)
    rhs = A @ x
    sol = np.zeros(4)
    assert lib().uo_solve_dense4(P(np.ascontiguousarray(A)), P(rhs), P(sol)) == 1
    assert np.allclose(sol, x, rtol=1e-12, atol=1e-12)
    singular = np.ones((4, 4))
    assert lib().uo_solve_dense4(P(singular), P(rhs), P(sol)) == 0


SPARSE_KEYS = (['original_gate', 'moment', 'M_W', 'M_h'] + [f'R{k}' for k in range(1, 9)] +
               [f'science_{k}' for k in range(1, 23)] + [f'flux_{k}' for k in range(1, 17)] +
               ['reference_h', 'reference_b', 'c_minus_1'])


def test_implicit_two_steps_match_sparse_residual(velocity, golden):
    """docs/release_checks/low_implicit/sparse_residual.csv: the accepted states 1 and 2 of the
    ImplicitSteady cold start (8 ranks in 1x8, PR(2) + one LU-SGS sweep pair, closed-mass
    rescale).  The oracle emulates the 8-rank block-Jacobi seams.  Bound: 1e-10 relative for
    every printed value above 1e-10, 1e-14 absolute below (cross-compiler libm noise)."""
    from oracle.oracle import set_threads
    set_threads(None)
    o = Oracle(reference_case("ImplicitSteady"), *velocity)
    o.init_freestream()
    o.implicit_init()
    for step, ref in enumerate(golden["low_implicit_sparse"]):
        row = o.implicit_step()
        for i, k in enumerate(SPARSE_KEYS):
            r = ref[k]
            if abs(r) > 1e-10:
                assert abs(row[i] - r) <= 1e-10 * abs(r), (step, k, row[i], r)
            else:
                assert abs(row[i] - r) <= 1e-14, (step, k, row[i], r)
        assert row[53] == 1.0 and row[54] == 1.0   # full micro and macro steps (CheckR5Policy)


def test_high_order_implicit_two_steps_match_sparse_residual(velocity, golden):
    """docs/release_checks/high_implicit/sparse_residual.csv: accepted states 1 and 2 of the
    HighOrderImplicit cold start (S2 tensor WENO-AO reconstruction, discrete-conservative Newton
    closure, Gauss-node UGKS faces, multiscale diffuse wall, S2 physical collision, PR(2) + LU-SGS
    with the high-order collision correction, closed-mass rescale).  Same bound as the
    second-order rows: 1e-10 relative above 1e-10, 1e-14 absolute below."""
    from oracle.oracle import set_threads
    set_threads(None)
    o = Oracle(reference_case("HighOrderImplicit"), *velocity)
    o.init_freestream()
    o.implicit_init()
    for step, ref in enumerate(golden["high_implicit_sparse"]):
        row = o.implicit_step()
        for i, k in enumerate(SPARSE_KEYS):
            r = ref[k]
            if abs(r) > 1e-10:
                assert abs(row[i] - r) <= 1e-10 * abs(r), (step, k, row[i], r)
            else:
                assert abs(row[i] - r) <= 1e-14, (step, k, row[i], r)
        assert row[53] == 1.0 and row[54] == 1.0
