"""The reference's tangent routines of the high-order path (restated in oracle/ugks_oracle_reftan.c) against
central differences and against the oracle's tangent build.

analytic_maxwellian_direction_2d, dq_value_and_direction, projector_direction_2d
(mod_CorrectedWF2DEquilibrium.f90:67-101, mod_CorrectedWF2DClosure.f90:211-243,560-625) and the WENO-AO
first-direction kernels (mod_WENO5AOScalar.f90:98-201) give directional derivatives by hand-written
formulas.  Central differences of their own value outputs check the formulas; the tangent build of the
oracle (every double a (value, derivative) pair, oracle/tangent.hpp) differentiates the same value
arithmetic automatically, so its derivative of the value outputs must equal the routines' direction
outputs -- which is what ties the tangent build, the forward-mode reference of the device adjoint, to the
reference's own tangents.
"""
import ctypes

import numpy as np
import pytest

from ugks2d_high_order_b200.case import velocity_table

CK = 1
FD_TOL = 1e-6      # central difference (h = 1e-6 relative) against the routine's direction
AD_TOL = 1e-10     # the tangent build's derivative of the values against the routine's direction


def _plain():
    from oracle.oracle import lib
    L = lib()
    dp = ctypes.POINTER(ctypes.c_double)
    L.uo_ref_maxwellian_direction.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp, dp]
    L.uo_ref_dq_direction.argtypes = [dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp, dp, dp]
    L.uo_ref_projector_direction.argtypes = [dp, dp, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp,
                                             dp, dp]
    L.uo_ref_weno_direction.argtypes = [dp, dp, ctypes.c_double, dp, dp, ctypes.POINTER(ctypes.c_int)]
    return L


def _tangent():
    from oracle.tangent import D2, lib
    L = lib()
    vp = ctypes.c_void_p
    L.uo_ref_maxwellian_direction.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, vp]
    L.uo_ref_dq_direction.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp]
    L.uo_ref_projector_direction.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp,
                                             vp, vp]
    L.uo_ref_weno_direction.argtypes = [vp, vp, D2, vp, vp, ctypes.POINTER(ctypes.c_int)]
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _dual(v, d=None):
    out = np.zeros(np.shape(v) + (2,))
    out[..., 0] = v
    if d is not None:
        out[..., 1] = d
    return np.ascontiguousarray(out)


def _state(rho, u, v, temp):
    return np.array([rho, rho * u, rho * v, rho * (temp * (CK + 2) / 4.0 + 0.5 * (u * u + v * v))])


@pytest.fixture(scope="module")
def table():
    u, v, w = velocity_table(24)
    return np.ascontiguousarray(u), np.ascontiguousarray(v), np.ascontiguousarray(w)


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_maxwellian_direction(table):
    u, v, _ = table
    n = len(u)
    L, T = _plain(), _tangent()
    w = _state(1.1, 0.3, -0.2, 2.2)
    dw = np.array([0.05, -0.02, 0.03, 0.1])

    def run(wv):
        o = [np.zeros(n) for _ in range(4)]
        assert L.uo_ref_maxwellian_direction(_p(wv), _p(dw), CK, n, _p(u), _p(v), *map(_p, o)) == 1
        return o
    mh, mb, dmh, dmb = run(w)
    h = 1e-6
    p, m = run(w + h * dw), run(w - h * dw)
    assert _rel((p[0] - m[0]) / (2 * h), dmh) <= FD_TOL and _rel((p[1] - m[1]) / (2 * h), dmb) <= FD_TOL
    ud, vd = _dual(u), _dual(v)
    o = [np.zeros((n, 2)) for _ in range(4)]
    assert T.uo_ref_maxwellian_direction(_dual(w, dw).ctypes.data, _dual(dw).ctypes.data, CK, n, ud.ctypes.data,
                                         vd.ctypes.data, *(a.ctypes.data for a in o)) == 1
    assert np.array_equal(o[0][:, 0], mh) and np.array_equal(o[2][:, 0], dmh)
    assert _rel(o[0][:, 1], dmh) <= AD_TOL and _rel(o[1][:, 1], dmb) <= AD_TOL


def test_dq_and_projector_directions(table):
    u, v, wt = table
    n = len(u)
    L, T = _plain(), _tangent()
    rng = np.random.default_rng(11)
    w = _state(0.9, -0.4, 0.25, 1.8)
    dw = np.array([0.03, 0.01, -0.02, 0.05])
    m, dm = rng.standard_normal(4) * 0.1, rng.standard_normal(4) * 0.1

    def dq(wv, mv):
        o = [np.zeros(n) for _ in range(4)]
        assert L.uo_ref_dq_direction(_p(wv), _p(dw), _p(mv), _p(dm), CK, n, _p(u), _p(v), _p(wt), *map(_p, o)) == 1
        return o
    ch, cb, dch, dcb = dq(w, m)
    h = 1e-6
    p, q = dq(w + h * dw, m + h * dm), dq(w - h * dw, m - h * dm)
    assert _rel((p[0] - q[0]) / (2 * h), dch) <= FD_TOL and _rel((p[1] - q[1]) / (2 * h), dcb) <= FD_TOL
    dual = [_dual(a) for a in (u, v, wt)]
    o = [np.zeros((n, 2)) for _ in range(4)]
    assert T.uo_ref_dq_direction(_dual(w, dw).ctypes.data, _dual(dw).ctypes.data, _dual(m, dm).ctypes.data,
                                 _dual(dm).ctypes.data, CK, n, *(a.ctypes.data for a in dual),
                                 *(a.ctypes.data for a in o)) == 1
    assert _rel(o[0][:, 1], dch) <= AD_TOL and _rel(o[1][:, 1], dcb) <= AD_TOL
    # the projector: p = z - dq(w) J^-1 moments(z), along (w_direction, z_direction)
    mh = np.zeros(n)
    scratch = [np.zeros(n) for _ in range(3)]
    L.uo_ref_maxwellian_direction(_p(w), _p(dw), CK, n, _p(u), _p(v), _p(mh), *map(_p, scratch))
    zh = mh * (1.0 + 0.1 * rng.standard_normal(n))
    zb = 0.5 * CK * 1.8 * zh
    dzh, dzb = 0.01 * rng.standard_normal(n) * mh, 0.01 * rng.standard_normal(n) * mh

    def proj(wv, zhv, zbv):
        o = [np.zeros(n) for _ in range(4)]
        assert L.uo_ref_projector_direction(_p(wv), _p(dw), _p(zhv), _p(zbv), _p(dzh), _p(dzb), CK, n, _p(u), _p(v),
                                            _p(wt), *map(_p, o)) == 1
        return o
    ph, pb, dph, dpb = proj(w, zh, zb)
    p, q = proj(w + h * dw, zh + h * dzh, zb + h * dzb), proj(w - h * dw, zh - h * dzh, zb - h * dzb)
    assert _rel((p[0] - q[0]) / (2 * h), dph) <= FD_TOL and _rel((p[1] - q[1]) / (2 * h), dpb) <= FD_TOL
    o = [np.zeros((n, 2)) for _ in range(4)]
    assert T.uo_ref_projector_direction(_dual(w, dw).ctypes.data, _dual(dw).ctypes.data, _dual(zh, dzh).ctypes.data,
                                        _dual(zb, dzb).ctypes.data, _dual(dzh).ctypes.data, _dual(dzb).ctypes.data,
                                        CK, n, *(a.ctypes.data for a in dual), *(a.ctypes.data for a in o)) == 1
    assert _rel(o[0][:, 1], dph) <= AD_TOL and _rel(o[1][:, 1], dpb) <= AD_TOL
    # the projected state keeps the moments of w's closure: moments(p) = 0 along any direction
    mom = lambda fh, fb: np.array([np.sum(wt * fh), np.sum(wt * u * fh), np.sum(wt * v * fh),
                                   np.sum(0.5 * wt * ((u * u + v * v) * fh + fb))])
    assert np.abs(mom(ph, pb)).max() <= 1e-12 and np.abs(mom(dph, dpb)).max() <= 1e-12


@pytest.mark.parametrize("xi", [-0.5, 0.5, -0.5 * np.sqrt(0.6), 0.0])
def test_weno_first_direction(xi):
    from oracle.tangent import D2
    L, T = _plain(), _tangent()
    rng = np.random.default_rng(5)
    for trial in range(20):
        q = np.cumsum(rng.standard_normal(5)) * 0.3 + 1.0
        dq = rng.standard_normal(5)
        val, dval, diff = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()

        def at(qq):
            a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
            assert L.uo_ref_weno_direction(_p(np.ascontiguousarray(qq)), _p(dq), xi, ctypes.byref(a), ctypes.byref(b),
                                           ctypes.byref(c)) == 1
            return a.value
        assert L.uo_ref_weno_direction(_p(q), _p(dq), xi, ctypes.byref(val), ctypes.byref(dval), ctypes.byref(diff)) == 1
        assert diff.value == 1
        h = 1e-6
        fd = (at(q + h * dq) - at(q - h * dq)) / (2 * h)
        assert abs(fd - dval.value) <= FD_TOL * max(abs(dval.value), 1e-3), (trial, fd, dval.value)
        o = np.zeros(2)
        od = np.zeros(2)
        dflag = ctypes.c_int()
        assert T.uo_ref_weno_direction(_dual(q, dq).ctypes.data, _dual(dq).ctypes.data, D2(xi, 0.0), o.ctypes.data,
                                       od.ctypes.data, ctypes.byref(dflag)) == 1
        assert o[0] == val.value
        assert abs(o[1] - dval.value) <= AD_TOL * max(abs(dval.value), 1e-3), (trial, o[1], dval.value)
