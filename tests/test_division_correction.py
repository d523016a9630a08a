"""The division by a stored reciprocal used inside the PR(2) wavefront (div_by_recip,
ugks_implicit.cu): q0 = a r with r = 1/d, then q0 + fma(-d, q0, a) r in one fused multiply-add,
against IEEE a / d on the host, whose binary64 arithmetic and fma are the device's.

Random operands over 60 binades, and significands of all ones (the divisors whose reciprocal
rounds hardest), must give the quotient bit for bit."""
import ctypes
import ctypes.util

import numpy as np

_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_fma = _libm.fma
_fma.restype = ctypes.c_double
_fma.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]


def _div_by_recip(a, d, r):
    q0 = a * r
    return _fma(_fma(-d, q0, a), r, q0)


def _operands(rng, n):
    mant = rng.integers(0, 1 << 52, size=n, dtype=np.uint64)
    expo = rng.integers(1023 - 30, 1023 + 31, size=n, dtype=np.uint64)
    sign = rng.integers(0, 2, size=n, dtype=np.uint64) << np.uint64(63)
    return (sign | (expo << np.uint64(52)) | mant).view(np.float64)


def test_division_by_the_reciprocal_is_the_ieee_quotient():
    rng = np.random.default_rng(20261204)
    n = 100000
    a, d = _operands(rng, n), _operands(rng, n)
    ones = np.uint64((1 << 52) - 1)
    low = rng.integers(0, 256, size=n, dtype=np.uint64)
    d_hard = (d.view(np.uint64) | (ones ^ low)).view(np.float64)   # significands of (nearly) all ones
    a_hard = (a.view(np.uint64) | (ones ^ low)).view(np.float64)
    bad = 0
    for aa, dd in ((a, d), (a, d_hard), (a_hard, d), (a_hard, d_hard)):
        for x, y in zip(aa.tolist(), dd.tolist()):
            if _div_by_recip(x, y, 1.0 / y) != x / y:
                bad += 1
    assert bad == 0
