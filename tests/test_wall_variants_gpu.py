"""The research S2CN2 wall variants on the GPU against the oracle, through the C ABI.

FluxWall_type = 0 (the free-streaming wall s2w1_wall_node, mod_S2D1.f90:961-995), W1T (the midpoint
wall predictor, mod_S2NativeAdapter.f90:605-685), W1D (its face correction, :660-680) and W2R (the
shared predictor, mod_S2D1.f90:1152-1244).  The reference ships no output of any of them (they are off
in every case file), so the oracle's restatement is the checker.  The bounds are those of the delivered
S2CN2 step (states 1e-12 relative to their largest component, report entries 1e-11): the variants add
half-step evaluations, CN collisions and face corrections whose moment sums are summed in a different
order on the device, as the step's own are.
"""
import numpy as np
import pytest

from ugks2d_high_order_b200.case import reference_case, velocity_table

pytestmark = pytest.mark.gpu

HO_TOL = 1e-12
REP_TOL = 1e-11
GATE = 2e-12

VARIANTS = {
    "kinetic_wall": dict(flux_wall=0),
    "w1t_midpoint": dict(flux_wall=0, s2w1_time_centered=1),
    "w1d_face_time": dict(flux_wall=0, s2w1_time_centered=1, s2w1d_face_time=1),
    "w2r_shared": dict(pr=1.0, s2w2r_shared_predictor=1),
}


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _case(name, **kw):
    return reference_case("S2CN2").with_(**VARIANTS[name], **kw)


def _check(rep, out, step):
    assert rep[0] == out[0]
    assert rep[1] <= GATE and rep[2] <= GATE and rep[9] <= GATE
    for q in (5, 6, 7, 8):
        assert abs(rep[q] - out[q]) <= REP_TOL * max(abs(out[q]), 1e-6), (step, q, rep[q], out[q])
    for q in range(10, 22):                      # wall fluxes and the ledger
        assert abs(rep[q] - out[q]) <= REP_TOL * max(abs(out[q]), 1e-3), (step, q, rep[q], out[q])


@pytest.mark.parametrize("name", list(VARIANTS))
def test_variant_steps_match_the_oracle(name, velocity):
    """Three single steps, then four graph-replayed ones, of the delivered 8 x 64 x 32^2 S2CN2 case with
    the variant, against the oracle's steps."""
    from oracle.oracle import Oracle, set_threads
    from ugks2d_high_order_b200.solver import Solver
    set_threads(None)
    case = _case(name)
    s, o = Solver(case, *velocity), Oracle(case, *velocity)
    try:
        s.init_freestream()
        o.init_freestream()
        for step in range(3):
            done, rep = s.step_s2cn2(1)
            out = o.s2cn2_step()
            assert done == 1 and rep[22] == 1.0
            _check(rep, out, step)
            hg, bg, Wg = s.download()
            ho, bo, Wo = o.get_state()
            assert _rel(Wg, Wo) <= HO_TOL and _rel(hg, ho) <= HO_TOL and _rel(bg, bo) <= HO_TOL, \
                (step, _rel(Wg, Wo), _rel(hg, ho), _rel(bg, bo))
        done, rep = s.step_s2cn2(4)
        for _ in range(4):
            out = o.s2cn2_step()
        assert done == 4
        _check(rep, out, "graph")
        hg, bg, Wg = s.download()
        ho, bo, Wo = o.get_state()
        assert _rel(Wg, Wo) <= HO_TOL and _rel(hg, ho) <= HO_TOL and _rel(bg, bo) <= HO_TOL
    finally:
        s.close()


def test_variants_change_the_step(velocity):
    """Each variant moves the walls (and W1D / W2R the interior faces) away from the delivered step: a
    variant that silently ran the delivered walls would pass the parity test only if the oracle did the
    same, so the four GPU results must differ from the delivered one and from each other."""
    from ugks2d_high_order_b200.solver import Solver
    states = {}
    for name in ["delivered"] + list(VARIANTS):
        case = reference_case("S2CN2") if name == "delivered" else _case(name)
        s = Solver(case, *velocity)
        try:
            s.init_freestream()
            done, rep = s.step_s2cn2(2)
            assert done == 2
            states[name] = (s.download()[0], rep[10:18].copy())
        finally:
            s.close()
    names = list(states)
    for a in range(len(names)):
        for b in range(a + 1, len(names)):
            if {names[a], names[b]} == {"delivered", "w2r_shared"}:
                continue   # different Pr: compared through the oracle only
            assert not np.array_equal(states[names[a]][0], states[names[b]][0]), (names[a], names[b])


def test_w1d_per_operator_sequence_equals_steps():
    """TimeStep, Evolution, ComputeResidual and the update called one by one on a W1D context equal
    ugks_s2cn2_steps bit for bit (the variant runs inside the S2 evolution, as S2NativeEvolution runs it)."""
    from ugks2d_high_order_b200.solver import Solver
    case = _case("w1d_face_time", ny=16, dy=1.0 / 16.0)
    vel = velocity_table(24)
    a, b = Solver(case, *vel), Solver(case, *vel)
    try:
        a.init_freestream()
        b.init_freestream()
        done, rep_a = a.step_s2cn2(3)
        assert done == 3
        for _ in range(3):
            b.time_step()
            b.evolution()
            b.compute_residual()
            b.apply_explicit_update()
        rep_b = b.s2cn2_report()
        for x, y in zip(a.download(), b.download()):
            assert np.array_equal(x, y)
        assert np.array_equal(a.wall_aero(), b.wall_aero())
        assert np.array_equal(rep_a[:22], rep_b[:22])
    finally:
        a.close()
        b.close()


def test_w2r_small_case_matches_the_oracle():
    """W2R on 8 x 16 cells with the generated 24^2 table, ten steps (five graph pairs)."""
    from oracle.oracle import Oracle, set_threads
    from ugks2d_high_order_b200.solver import Solver
    set_threads(None)
    case = _case("w2r_shared", ny=16, dy=1.0 / 16.0)
    vel = velocity_table(24)
    s, o = Solver(case, *vel), Oracle(case, *vel)
    try:
        s.init_freestream()
        o.init_freestream()
        done, rep = s.step_s2cn2(10)
        for _ in range(10):
            out = o.s2cn2_step()
        assert done == 10
        _check(rep, out, "w2r")
        hg, bg, Wg = s.download()
        ho, bo, Wo = o.get_state()
        assert _rel(Wg, Wo) <= HO_TOL and _rel(hg, ho) <= HO_TOL and _rel(bg, bo) <= HO_TOL
    finally:
        s.close()


def test_variant_contexts_refuse_the_adjoint():
    """The adjoint transposes the delivered walls only: a variant context refuses its entry points."""
    import ctypes
    from ugks2d_high_order_b200 import capi
    from ugks2d_high_order_b200.solver import Solver
    s = Solver(_case("kinetic_wall", ny=16, dy=1.0 / 16.0), *velocity_table(24))
    try:
        s.init_freestream()
        out = (ctypes.c_double * 4)()
        assert s.L.ugks_s2cn2_forward_checkpointed(s.ctx, 4, 2, out) == capi.UGKS_EUNSUPPORTED
    finally:
        s.close()


@pytest.mark.parametrize("name", ["w1d_face_time", "w2r_shared"])
def test_variants_on_the_48_squared_table(name):
    """The variants with a table above 1024 velocities (48^2 = 2304: the 10-velocity-per-thread cell
    kernels, every velocity loop of the variant kernels past one pass), 8 x 16 cells, four steps."""
    from oracle.oracle import Oracle, set_threads
    from ugks2d_high_order_b200.solver import Solver
    set_threads(None)
    case = _case(name, ny=16, dy=1.0 / 16.0)
    vel = velocity_table(48)
    s, o = Solver(case, *vel), Oracle(case, *vel)
    try:
        s.init_freestream()
        o.init_freestream()
        done, rep = s.step_s2cn2(4)
        for _ in range(4):
            out = o.s2cn2_step()
        assert done == 4
        _check(rep, out, name)
        hg, bg, Wg = s.download()
        ho, bo, Wo = o.get_state()
        assert _rel(Wg, Wo) <= HO_TOL and _rel(hg, ho) <= HO_TOL and _rel(bg, bo) <= HO_TOL, \
            (_rel(Wg, Wo), _rel(hg, ho), _rel(bg, bo))
    finally:
        s.close()


def test_high_order_implicit_with_the_kinetic_wall(velocity):
    """HighOrderImplicit with FluxWall_type 0 (the reference admits the kinetic wall on both S2 methods;
    its implicit micro wall treatment does not depend on it): five pseudo-steps of the delivered 8 x 64 x 32^2
    case against the oracle, at the delivered method's bounds (states 1e-11, c_minus_1 5e-11)."""
    from oracle.oracle import Oracle, set_threads
    from ugks2d_high_order_b200.solver import Solver
    set_threads(None)
    case = reference_case("HighOrderImplicit").with_(flux_wall=0)
    s, o = Solver(case, *velocity), Oracle(case, *velocity)
    try:
        s.init_freestream(); s.implicit_init()
        o.init_freestream(); o.implicit_init()
        done, conv, rep = s.step_implicit(5)
        for _ in range(5):
            row = o.implicit_step()
        assert done == 5
        hg, bg, Wg = s.download()
        ho, bo, Wo = o.get_state()
        assert _rel(Wg, Wo) <= 1e-11 and _rel(hg, ho) <= 1e-11, (_rel(Wg, Wo), _rel(hg, ho))
        assert abs(rep[52] - row[52]) <= 5e-11 * max(abs(row[52]), 1e-3)
    finally:
        s.close()
