"""Host logic of the central-difference wall sensitivities (no GPU): the instance layout and the
difference quotients, on outputs that are known functions of the parameters."""
import numpy as np

from ugks2d_high_order_b200.case import batched_cases
from ugks2d_high_order_b200.sensitivity import (PARAMS, central_differences, parameter_value, perturbed,
                                                sensitivity_instances)


def test_instances_are_the_base_case_then_plus_and_minus_steps():
    cases = [(c, n) for c, n in batched_cases(3)]
    inst = sensitivity_instances(cases, rel_step=1e-3)
    assert len(inst) == 7 * len(cases)
    for c, (case, _) in enumerate(cases):
        block = inst[7 * c:7 * (c + 1)]
        assert block[0][0] == case
        for j, p in enumerate(PARAMS):
            up, down = block[1 + 2 * j][0], block[2 + 2 * j][0]
            assert parameter_value(up, p) == parameter_value(case, p) * (1 + 1e-3)
            assert parameter_value(down, p) == parameter_value(case, p) * (1 - 1e-3)
            for q in PARAMS:                         # the other parameters are untouched
                if q != p:
                    assert parameter_value(up, q) == parameter_value(case, q)
    # both walls move together, in opposite directions
    up = perturbed(cases[0][0], "wall_speed", 2.0)
    assert up.wall_ux == (2 * cases[0][0].wall_ux[0], 2 * cases[0][0].wall_ux[1])


def test_central_differences_of_quadratic_outputs_are_exact():
    cases = [(c, n) for c, n in batched_cases(2)]
    h = 1e-4
    inst = sensitivity_instances(cases, rel_step=h)
    coef = np.array([[0.3, -1.1, 2.5], [0.7, 0.2, -0.4]])    # output k = sum_p coef[k,p] x_p^2

    def outputs(case):
        x = np.array([parameter_value(case, p) for p in PARAMS])
        f = coef @ (x * x)
        return np.stack([f, -f])                              # [wall][output]
    outs = np.stack([outputs(c) for c, _ in inst])
    values, grads = central_differences(cases, outs, h)
    for c, (case, _) in enumerate(cases):
        x = np.array([parameter_value(case, p) for p in PARAMS])
        exact = coef * (2 * x)                                # d/dx_p of sum coef x^2
        assert np.allclose(values[c], outputs(case))
        assert np.allclose(grads[c, 0], exact, rtol=1e-9, atol=0.0)
        assert np.allclose(grads[c, 1], -exact, rtol=1e-9, atol=0.0)
