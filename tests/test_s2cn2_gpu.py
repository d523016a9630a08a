"""S2CN2, the explicit high-order step, on the GPU against the oracle.

The step is TimeStep, S2NativeEvolution with the volume targets kept between steps, ComputeResidual
and S2NativeApplyUpdate's advance_step on the stream state (mod_S2NativeAdapter.f90:469-490,867-940;
mod_S2D1.f90:1302-1435), through the C ABI.  The reference ships no S2CN2 output for this case
(consistency/high_explicit holds inputs only), so the oracle is the checker; its S2 evolution is the
code pinned to the reference's high_implicit rows.  GPU moment sums are per lane and in a butterfly, the
oracle's sequential; over a dozen steps the states differ by 3e-16 (W) and 1.4e-15 (h, b) relative and the
wall fluxes by 4e-13, so the bounds are 1e-12 for the states and 1e-11 for the report.
"""
import numpy as np
import pytest

from ugks2d_high_order_b200.case import reference_case

HO_TOL = 1e-12    # states against the oracle, relative to the largest component
REP_TOL = 1e-11   # report entries
GATE = 2e-12


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _pair(velocity):
    from oracle.oracle import Oracle, set_threads
    from ugks2d_high_order_b200.solver import Solver
    set_threads(None)
    case = reference_case("S2CN2")
    return Solver(case, *velocity), Oracle(case, *velocity)


@pytest.mark.gpu
def test_s2cn2_steps_match_oracle(velocity):
    s, o = _pair(velocity)
    try:
        s.init_freestream()
        o.init_freestream()
        hg, bg, Wg = s.download()
        ho, bo, Wo = o.get_state()
        assert _rel(hg, ho) <= 1e-12 and _rel(Wg, Wo) == 0.0
        for step in range(3):
            done, rep = s.step_s2cn2(1)
            out = o.s2cn2_step()
            assert done == 1 and rep[22] == 1.0
            assert rep[0] == out[0]                          # dt of the same state
            assert rep[1] <= GATE and rep[2] <= GATE and rep[9] <= GATE
            assert abs(rep[4] - out[4]) <= 1e-14             # transport CFL
            for q in (5, 6, 7, 8):                           # min/max of h and b
                assert abs(rep[q] - out[q]) <= REP_TOL * max(abs(out[q]), 1e-6), (step, q, rep[q], out[q])
            for q in range(10, 22):                          # wall fluxes and the ledger
                assert abs(rep[q] - out[q]) <= REP_TOL * max(abs(out[q]), 1e-3), (step, q, rep[q], out[q])
            hg, bg, Wg = s.download()
            ho, bo, Wo = o.get_state()
            assert _rel(Wg, Wo) <= HO_TOL and _rel(hg, ho) <= HO_TOL and _rel(bg, bo) <= HO_TOL, \
                (step, _rel(Wg, Wo), _rel(hg, ho), _rel(bg, bo))
    finally:
        s.close()


@pytest.mark.gpu
def test_s2cn2_graph_pairs_and_odd_tail_match_oracle(velocity):
    """Ten steps (five graph-replayed pairs), then seven (three pairs and one step that leaves the
    accepted state in the second buffer set, copied back), against the oracle."""
    s, o = _pair(velocity)
    try:
        s.init_freestream()
        o.init_freestream()
        for n in (10, 7):
            done, rep = s.step_s2cn2(n)
            for _ in range(n):
                out = o.s2cn2_step()
            assert done == n and rep[23] == n
            hg, bg, Wg = s.download()
            ho, bo, Wo = o.get_state()
            assert _rel(Wg, Wo) <= HO_TOL and _rel(hg, ho) <= HO_TOL and _rel(bg, bo) <= HO_TOL, \
                (n, _rel(Wg, Wo), _rel(hg, ho), _rel(bg, bo))
            for q in range(10, 22):
                assert abs(rep[q] - out[q]) <= REP_TOL * max(abs(out[q]), 1e-3), (n, q, rep[q], out[q])
    finally:
        s.close()


@pytest.mark.gpu
def test_s2cn2_collision_gate_stops_the_sequence(velocity):
    """W that disagrees with the moments of h by 1e-8 fails S2NativePhysicalCollision's moment gate
    (the reference aborts with 444; the oracle returns 444 too) in the residual of the first step;
    the rest of the graph-replayed sequence returns at entry, the state is untouched and the context
    stays usable."""
    from ugks2d_high_order_b200.capi import UgksError
    s, o = _pair(velocity)
    try:
        s.init_freestream()
        o.init_freestream()
        h, b, W = s.download()
        Wbad = W.copy()
        Wbad[..., 0] *= 1.0 + 1e-8
        o.set_state(h, b, Wbad)
        o.s2cn2_init()
        with pytest.raises(RuntimeError, match="444"):
            o.s2cn2_step()
        s.upload(h, b, Wbad)
        s.s2cn2_init()
        with pytest.raises(UgksError) as ei:
            s.step_s2cn2(4)
        assert ei.value.reference_code == 444
        assert s.last_steps_done == 0
        h2, b2, W2 = s.download()
        assert np.array_equal(h2, h) and np.array_equal(b2, b) and np.array_equal(W2, Wbad)
        s.upload(h, b, W)
        s.s2cn2_init()
        done, rep = s.step_s2cn2(2)
        assert done == 2 and rep[22] == 1.0
    finally:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("reject_at,nsteps", [(3, 4), (2, 5)])
def test_s2cn2_rejected_step_keeps_the_last_accepted_state(velocity, reject_at, nsteps):
    """The reference's rejection hook (S2D3_TEST_GLOBAL_REJECT / S2E3_TEST_REJECT_STEP) forces the
    conservation gate of one step to fail: the call returns the reference's abort code 203, the
    accepted steps before it are kept (bitwise equal to a run that stops there), nothing after it
    runs, and the next call continues from that state."""
    from ugks2d_high_order_b200.capi import UgksError
    from ugks2d_high_order_b200.solver import Solver
    case = reference_case("S2CN2")
    a = Solver(case, *velocity)
    r = Solver(case, *velocity)
    try:
        a.init_freestream()
        r.init_freestream()
        a.s2cn2_test_reject(reject_at)
        with pytest.raises(UgksError) as ei:
            a.step_s2cn2(nsteps)
        assert ei.value.reference_code == 203
        assert a.last_steps_done == reject_at - 1
        r.step_s2cn2(reject_at - 1)
        for x, y in zip(a.download(), r.download()):
            assert np.array_equal(x, y)
        da, ra = a.step_s2cn2(2)
        dr, rr = r.step_s2cn2(2)
        assert da == dr == 2
        for x, y in zip(a.download(), r.download()):
            assert np.array_equal(x, y)
        assert np.array_equal(ra[18:22], rr[18:22])   # the ledger advanced only on accepted steps
    finally:
        a.close()
        r.close()
