"""Half-range Gauss-Hermite velocity tables (mod_VelocityTables.f90) and their generator.

The reference ships half16 and half32 raw rules; the batched and refined cases need 24^2 and 48^2
tables it does not ship, so ugks2d_high_order_b200.velocity generates any half-range rule from its
moments at 100 digits.  Pinned here: the generator reproduces both shipped rules (nodes within a few
tens of ulp, weights within 1e-14 relative), and integrates the moments of exp(-x^2) on [0, inf)
at least as exactly as the shipped rules do; FillVelocity of the shipped half32 rule reproduces the
reference's velocity_half32_scale2.dat bitwise.
"""
import mpmath as mp
import numpy as np
import pytest

from ugks2d_high_order_b200.case import load_velocity_half32
from ugks2d_high_order_b200.velocity import fill_velocity, half_range_gauss_hermite, raw_rule, structured_table


def _moment_error(x, w):
    n = len(x)
    with mp.workdps(60):
        e = mp.mpf(0)
        for k in range(2 * n):
            mu = mp.gamma(mp.mpf(k + 1) / 2) / 2
            s = mp.fsum(mp.mpf(float(wi)) * mp.mpf(float(xi)) ** k for xi, wi in zip(x, w))
            e = max(e, abs(s - mu) / mu)
        return float(e)


@pytest.mark.parametrize("name,n", [("half16", 8), ("half32", 16)])
def test_generator_reproduces_reference_rules(golden, name, n):
    ref = golden["velocity_tables"][name]
    node, weight = raw_rule(n)
    rn, rw = np.array(ref["raw_node"]), np.array(ref["raw_weight"])
    assert np.all(np.abs(node - rn) <= 64 * np.spacing(np.abs(rn).max()))
    assert np.all(np.abs(weight - rw) <= 1e-14 * rw)
    # the generated rule is at least as exact on the moments as the shipped one
    assert _moment_error(node[n:], weight[n:]) <= max(2e-15, _moment_error(rn[n:], rw[n:]))


def test_fill_velocity_reproduces_the_reference_table_file(golden):
    ref = golden["velocity_tables"]["half32"]
    u, v, w = fill_velocity(ref["raw_node"], ref["raw_weight"], 2.0)
    uf, vf, wf = load_velocity_half32()
    assert np.array_equal(u, uf) and np.array_equal(v, vf) and np.array_equal(w, wf)


@pytest.mark.parametrize("n", [24, 48])
def test_generated_tables_are_symmetric_rules(n):
    u, v, w = structured_table(n)
    assert len(u) == n * n
    assert np.all(w > 0)
    assert np.array_equal(u.reshape(n, n)[0], -u.reshape(n, n)[0][::-1])
    x, wt = half_range_gauss_hermite(n // 2)
    assert _moment_error(x, wt) <= 2e-15
