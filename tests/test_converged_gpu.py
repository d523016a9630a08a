"""Converged-state parity against the reference's published end states.

docs/couette_results/profiles_three_methods.plt holds the x-averaged 64-row profiles of
r, u, v, T, p, sxx, sxy, syy, qx, qy of the reference's converged runs, and analysis.json the end
summaries (step count, c_final, per-wall native pnn/pnt/qn).  Both runs use the delivered case
(8x64 cells, 32x32 velocities, CFL 0.1): ImplicitSteady until the five-state gate (1096 steps),
Explicit for 200000 steps.  Fields are compared relative to each column's largest magnitude; the
reference's own two solvers agree to ~1e-12 on these profiles, and its x-spread is ~1e-13.
"""
import numpy as np
import pytest

from ugks2d_high_order_b200.case import reference_case

COLS = ["r", "u", "v", "T", "p", "sxx", "sxy", "syy", "qx", "qy"]
PROFILE_TOL = 1e-9   # relative to each column's max |value|


def _profile_errors(got, zone):
    ref = np.array(zone)[:, 2:]           # drop x, y
    scale = np.abs(ref).max(axis=0)
    return np.abs(got - ref).max(axis=0) / scale


@pytest.mark.gpu
def test_implicit_steady_reaches_reference_end_state(velocity, golden):
    from ugks2d_high_order_b200.solver import Solver
    fin = golden["low_implicit_final"]
    s = Solver(reference_case("ImplicitSteady"), *velocity)
    try:
        s.init_freestream()
        s.implicit_init()
        done, conv, rep = s.step_implicit(3000)
        assert conv, "five-state gate not reached within 3000 pseudo-steps"
        # the gate falls where science_3 (RrhoV) crosses 1e-8 on its round-off floor (~0.92-0.99e-8),
        # so the step count is set by rounding; the reference stopped at 1096, the C oracle at 1097
        assert abs(done - fin["steps"]) <= 10, done
        assert abs(rep[52]) <= 1e-14                     # c_minus_1 of the last accepted state
        assert rep[1] <= 1e-12                           # moment gate
        for key, col in (("1", 12), ("2", 13), ("4", 15), ("13", 24), ("14", 25)):
            assert rep[col] <= 1e-10, (key, rep[col])    # converged macro / micro residuals
        err = _profile_errors(s.profiles(), golden["profiles"]["VL implicit: converged"])
        bad = {c: e for c, e in zip(COLS, err) if not e <= PROFILE_TOL}
        assert not bad, bad
        # wall shear and heat flux: x-averages of the wall faces' local-frame (pnn, pnt, qn)
        aero = s.wall_aero().mean(axis=1)
        for w, row in (("1", 0), ("2", 1)):
            ref = fin["final_walls"][w]
            for q, col in (("native_pnn", 0), ("native_pnt", 1), ("native_qn", 2)):
                assert abs(abs(aero[row, col]) - abs(ref[q])) <= 1e-9 * abs(ref[q]), (w, q, aero[row], ref)
    finally:
        s.close()


@pytest.mark.gpu
def test_explicit_limit_matches_reference_profiles(velocity, golden):
    from ugks2d_high_order_b200.solver import Solver
    steps = golden["low_explicit_final"]["steps"]
    s = Solver(reference_case("Explicit"), *velocity)
    try:
        s.init_freestream()
        dt, res = s.step_explicit(steps)
        assert np.all(np.isfinite(res))
        err = _profile_errors(s.profiles(), golden["profiles"]["VL explicit: limit"])
        bad = {c: e for c, e in zip(COLS, err) if not e <= PROFILE_TOL}
        assert not bad, bad
    finally:
        s.close()


@pytest.mark.gpu
def test_high_order_implicit_reaches_reference_limit_state(velocity, golden):
    """HighOrderImplicit from the cold start to its 3000 pseudo-step cap (the reference run also stops
    at the iteration limit, not at the gate).  The state is still relaxing there, so the bound is the
    reference's own x-spread of each profile column (analysis.json high_implicit/x_spread): every
    x-averaged profile value lies within it of "S2 implicit: limit"."""
    from ugks2d_high_order_b200.solver import Solver
    fin = golden["high_implicit_final"]
    s = Solver(reference_case("HighOrderImplicit"), *velocity)
    try:
        s.init_freestream()
        s.implicit_init()
        done, conv, rep = s.step_implicit(fin["steps"])
        assert done == fin["steps"] and not conv
        ref = np.array(golden["profiles"]["S2 implicit: limit"])[:, 2:]
        dev = np.abs(s.profiles() - ref).max(axis=0)
        bad = {c: (d, fin["x_spread"][c]) for c, d in zip(COLS, dev) if not d <= fin["x_spread"][c]}
        assert not bad, bad
        assert abs(rep[52]) <= 1e-9, rep[52]              # c_minus_1 (reference: -2.2e-10)
        assert rep[1] <= 1e-12                            # moment gate of the last accepted state
        # wall shear and heat in the native frame (PublishWallDiagnostics), x-averaged
        aero = s.wall_aero().mean(axis=1)
        for w, row in (("1", 0), ("2", 1)):
            r = fin["final_walls"][w]
            for q, col in (("native_pnn", 0), ("native_pnt", 1), ("native_qn", 2)):
                assert abs(aero[row, col] - r[q]) <= 1e-7 * abs(r[q]), (w, q, aero[row, col], r[q])
    finally:
        s.close()


@pytest.mark.gpu
def test_repeated_solves_on_one_context_are_identical(velocity):
    """Two cold-start ImplicitSteady solves to the five-state gate on one context (as bench.py runs
    them): the second sees none of the first's stop state and reproduces it bitwise."""
    from ugks2d_high_order_b200.solver import Solver
    s = Solver(reference_case("ImplicitSteady"), *velocity)
    try:
        out = []
        for _ in range(2):
            s.init_freestream()
            s.implicit_init()
            done, conv, rep = s.step_implicit(3000)
            assert conv
            out.append((done, rep.copy(), s.download()))
        assert out[0][0] == out[1][0]
        assert np.array_equal(out[0][1], out[1][1])
        for x, y in zip(out[0][2], out[1][2]):
            assert np.array_equal(x, y)
    finally:
        s.close()


@pytest.mark.gpu
def test_implicit_steady_follows_the_oracle_past_the_gate(velocity):
    """3000 accepted pseudo-steps of the delivered case with the headline metric's 1e-10 gate, against the
    oracle's trajectory (tests/golden/oracle_implicit_3000.json, from make_oracle_trajectory.py).

    The residual columns are norms of the change of one pseudo-step.  While they are far above rounding
    the device and the oracle give the same numbers (within 1e-9 to step 100, 2e-6 at step 500, where the
    macro residuals are 1e-7).  From step 1000 on they are made of rounding: the device and the oracle
    each sit on their own round-off floor, and the columns agree in magnitude only.  science_3, the
    rho*V residual relative to a near-zero reference, crosses 1e-8 near step 1100 and then stays between
    1e-10 and 1e-8 on that floor in both:
    the 1e-10 gate is never reached (the reference's own explicit run stalls the same way, at a rho*V
    residual of 6.7e-9 after 200,000 steps).  The state itself is converged and the same: W at steps 1100
    and 3000 agrees with the oracle's to 1e-12 of its largest component."""
    import json
    import os
    from ugks2d_high_order_b200.solver import Solver
    with open(os.path.join(os.path.dirname(__file__), "golden", "oracle_implicit_3000.json")) as f:
        fx = json.load(f)
    rows = {int(k): np.array(v) for k, v in fx["rows"].items()}
    states = {int(k): np.array(v) for k, v in fx["W"].items()}
    cols = (12, 13, 14, 15, 24, 25)   # science_1..4, R_h, R_b
    s = Solver(reference_case("ImplicitSteady").with_(residual_tol=1e-10), *velocity)
    try:
        s.init_freestream()
        s.implicit_init()
        at = 0
        for n in sorted(rows):
            done, conv, rep = s.step_implicit(n - at)
            assert done == n - at and not conv
            at = n
            o = rows[n]
            if n <= 500:
                tol = 1e-9 if n <= 100 else 2e-6
                for col in cols:
                    assert abs(rep[col] - o[col]) <= tol * abs(o[col]), (n, col, rep[col], o[col])
            else:
                for col in (12, 13, 15, 24, 25):
                    assert rep[col] <= 1e-10 and o[col] <= 1e-10, (n, col, rep[col], o[col])
                assert 1e-10 < rep[14] < (1e-7 if n <= 1100 else 1e-8), (n, rep[14])
                assert 1e-10 < o[14], (n, o[14])
            assert abs(rep[52] - o[52]) <= 1e-13, (n, rep[52], o[52])   # c_minus_1
            if n in states:
                W = s.download()[2].reshape(-1)
                assert np.abs(W - states[n]).max() <= 1e-12 * np.abs(states[n]).max(), n
    finally:
        s.close()
