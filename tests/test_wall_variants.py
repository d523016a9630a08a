"""The research S2CN2 wall variants on the CPU: the option checks of the C ABI and of the case reader
(mod_ImportPara.f90:455-471, :527-528, whose failures are the reference's abort 200), and the oracle's
restatement of the variants (mod_S2D1.f90:961-995, :1052-1244; mod_S2NativeAdapter.f90:605-685;
mod_S2MultiscaleWall.f90:187-227) on their own invariants: every step passes the reference's gates,
conserves against the wall ledger, and its walls carry no mass.
"""
import ctypes

import numpy as np
import pytest

from ugks2d_high_order_b200.case import reference_case, velocity_table

GATE = 2e-12
VARIANTS = {
    "kinetic_wall": dict(flux_wall=0),
    "w1t_midpoint": dict(flux_wall=0, s2w1_time_centered=1),
    "w1d_face_time": dict(flux_wall=0, s2w1_time_centered=1, s2w1d_face_time=1),
    "w2r_shared": dict(pr=1.0, s2w2r_shared_predictor=1),
}
REFUSED = [   # (case fields, the C ABI's answer)
    (dict(s2w1_time_centered=1), "EINVAL"),                                   # W1T on the multiscale wall
    (dict(flux_wall=0, s2w1d_face_time=1), "EINVAL"),                          # W1D without W1T
    (dict(pr=1.0, flux_wall=0, s2w2r_shared_predictor=1), "EINVAL"),           # W2R on the kinetic wall
    (dict(s2w2r_shared_predictor=1), "EINVAL"),                                # W2R with Pr = 2/3
    (dict(pr=1.0, ck=2, s2w2r_shared_predictor=1), "EINVAL"),                  # W2R with ck = 2
    (dict(flux_wall=0, s2w1_time_centered=2), "EINVAL"),                       # switches are 0 or 1
]


def _small(method="S2CN2", **kw):
    return reference_case(method).with_(ny=16, dy=1.0 / 16.0, **kw)


@pytest.mark.parametrize("fields,code", REFUSED)
def test_c_abi_refuses_combinations_the_reference_rejects(fields, code):
    """ugks_ctx_create checks the switches before it touches a device, so this runs without a GPU."""
    from ugks2d_high_order_b200 import capi
    from ugks2d_high_order_b200.solver import Solver
    L = capi.load()
    u, v, w = (np.ascontiguousarray(a) for a in velocity_table(24))
    p = Solver.params_for(_small(**fields), len(u))
    ctx = ctypes.c_void_p()
    dp = ctypes.POINTER(ctypes.c_double)
    r = L.ugks_ctx_create(ctypes.byref(p), u.ctypes.data_as(dp), v.ctypes.data_as(dp), w.ctypes.data_as(dp), 0,
                          ctypes.byref(ctx))
    assert r == getattr(capi, "UGKS_" + code) and not ctx.value


def test_c_abi_keeps_the_variants_to_s2cn2():
    from ugks2d_high_order_b200 import capi
    from ugks2d_high_order_b200.solver import Solver
    L = capi.load()
    u, v, w = (np.ascontiguousarray(a) for a in velocity_table(24))
    dp = ctypes.POINTER(ctypes.c_double)
    refused = [("Explicit", dict(flux_wall=0)), ("ImplicitSteady", dict(flux_wall=0)),
               ("HighOrderImplicit", dict(flux_wall=0, s2w1_time_centered=1))]   # the kinetic wall alone is HO's
    for method, fields in refused:
        p = Solver.params_for(_small(method, **fields), len(u))
        ctx = ctypes.c_void_p()
        assert L.ugks_ctx_create(ctypes.byref(p), u.ctypes.data_as(dp), v.ctypes.data_as(dp), w.ctypes.data_as(dp), 0,
                                 ctypes.byref(ctx)) == capi.UGKS_EUNSUPPORTED


@pytest.mark.parametrize("name", list(VARIANTS))
def test_oracle_variant_steps_keep_the_gates_and_the_ledger(name):
    from oracle.oracle import Oracle, set_threads
    set_threads(None)
    case = _small(**VARIANTS[name])
    o = Oracle(case, *velocity_table(24))
    o.init_freestream()
    for _ in range(3):
        out = o.s2cn2_step()
        assert out[1] <= GATE and out[2] <= GATE      # cnres, mmerr
        assert out[9] <= GATE                         # conservation drift against the wall ledger
        assert abs(out[10]) <= 1e-12 and abs(out[14]) <= 1e-12   # the walls carry no mass
    h, b, W = o.get_state()
    assert np.all(np.isfinite(h)) and np.all(np.isfinite(b)) and np.all(W[..., 0] > 0.0)


def test_oracle_refuses_combinations_the_reference_rejects():
    from oracle.oracle import Oracle
    for fields, _ in REFUSED[:5]:
        o = Oracle(_small(**fields), *velocity_table(24))
        o.init_freestream()
        with pytest.raises(RuntimeError, match="code 200"):
            o.s2cn2_step()


def test_oracle_variants_differ_from_the_delivered_walls():
    """The kinetic wall, the midpoint wall and its face correction each change the step: a variant that
    fell back to the delivered walls would leave the state equal to the delivered step's."""
    from oracle.oracle import Oracle
    vel = velocity_table(24)
    states = {}
    for name, fields in [("delivered", {})] + [(n, f) for n, f in VARIANTS.items() if n != "w2r_shared"]:
        o = Oracle(_small(**fields), *vel)
        o.init_freestream()
        o.s2cn2_step()
        o.s2cn2_step()
        states[name] = o.get_state()[0]
    names = list(states)
    for a in range(len(names)):
        for b in range(a + 1, len(names)):
            assert not np.array_equal(states[names[a]], states[names[b]]), (names[a], names[b])


def test_case_reader_takes_the_variant_switches(tmp_path):
    """Config.ini's FluxWall_type and the S2W1/S2W2R switches load into the case, and the combinations
    the reference rejects raise its abort 200."""
    from ugks2d_high_order_b200 import refio
    for fields in VARIANTS.values():
        case = reference_case("S2CN2").with_(nslab=1, **fields)
        text = refio.config_text(case)
        got = refio.case_from_config(refio.parse_namelists(text), None)
        for k in ("flux_wall", "s2w1_time_centered", "s2w1d_face_time", "s2w2r_shared_predictor", "pr"):
            assert getattr(got, k) == getattr(case, k), k
    for fields, _ in REFUSED[:5]:
        case = reference_case("S2CN2").with_(nslab=1, **fields)
        with pytest.raises(refio.CaseError, match="reference abort 200"):
            refio.case_from_config(refio.parse_namelists(refio.config_text(case)), None)
    with pytest.raises(refio.CaseError):   # W1T / W1D / W2R are S2CN2's
        refio.case_from_config(refio.parse_namelists(refio.config_text(
            reference_case("HighOrderImplicit").with_(flux_wall=0, s2w1_time_centered=1))), None)
    got = refio.case_from_config(refio.parse_namelists(refio.config_text(   # the kinetic wall is HO's too
        reference_case("HighOrderImplicit").with_(flux_wall=0))), None)
    assert got.flux_wall == 0 and got.method == "HighOrderImplicit"


@pytest.mark.parametrize("fields", [{}, VARIANTS["w1d_face_time"], VARIANTS["w2r_shared"]])
def test_tangent_build_steps_as_the_oracle(fields):
    """The oracle's tangent build (every double a value / derivative pair) carries the same parameter block
    and arithmetic: its S2CN2 step values equal the plain oracle's bit for bit, delivered walls or variant."""
    from oracle.oracle import Oracle
    from oracle.tangent import TangentOracle
    case = _small(**fields).with_(ny=8, dy=0.125)
    vel = velocity_table(16)
    o, t = Oracle(case, *vel), TangentOracle(case, *vel)
    o.init_freestream()
    t.init_freestream()
    for _ in range(2):
        assert np.array_equal(o.s2cn2_step(), t.s2cn2_step())
    h, b, W = o.get_state()
    th, _, tb, _, tW, _ = t.get_state()
    assert np.array_equal(h, th) and np.array_equal(b, tb) and np.array_equal(W, tW)


def test_oracle_high_order_implicit_with_the_kinetic_wall():
    """The kinetic wall on the HighOrderImplicit pseudo-step: it runs, keeps the moment gate, and moves
    the state away from the multiscale wall's."""
    from oracle.oracle import Oracle
    vel = velocity_table(24)
    out = {}
    for fw in (1, 0):
        o = Oracle(_small("HighOrderImplicit", flux_wall=fw), *vel)
        o.init_freestream()
        o.implicit_init()
        for _ in range(2):
            row = o.implicit_step()
        out[fw] = o.get_state()[0]
        assert abs(row[1]) <= 1e-12   # the moment gate of the accepted state
    assert not np.array_equal(out[0], out[1])
