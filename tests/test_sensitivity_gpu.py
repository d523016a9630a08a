"""Central-difference wall sensitivities on the batch (ugks2d_high_order_b200.sensitivity).

Two Couette cases of the batched distribution at 8 x 16 cells with the generated 24^2 velocity set,
10 S2CN2 steps from the cold start.  The base instance must reproduce a single-instance run bit for
bit, and the derivatives must be consistent: the relative steps 1e-6 and 1e-5 give the same
derivatives to 1e-4 (truncation O(h^2), rounding about 1e-16 / h).  The Couette problem's mirror
symmetry gives a physical check: equal wall shear and opposite wall heat flux on the two walls.
"""
import numpy as np
import pytest

from ugks2d_high_order_b200.case import batched_cases, velocity_table

STEPS = 10


def _cases():
    return [(c.with_(ny=16, dy=1.0 / 16), 24) for c, _ in batched_cases(2)]


@pytest.mark.gpu
def test_wall_sensitivities_are_consistent_central_differences():
    from ugks2d_high_order_b200.sensitivity import PARAMS, parameter_value, wall_outputs, wall_sensitivities
    from ugks2d_high_order_b200.solver import Solver
    cases = _cases()
    v6, g6 = wall_sensitivities(cases, STEPS, rel_step=1e-6)
    v5, g5 = wall_sensitivities(cases, STEPS, rel_step=1e-5)
    assert np.array_equal(v6, v5)
    for c, (case, nva) in enumerate(cases):
        s = Solver(case, *velocity_table(nva))
        try:
            s.init_freestream()
            s.step_s2cn2(STEPS)
            assert np.array_equal(wall_outputs(s.wall_aero()), v6[c])
        finally:
            s.close()
    assert g6.shape == (len(cases), 2, 2, len(PARAMS))
    assert np.all(np.isfinite(g6)) and np.all(np.abs(g6) > 0.0)
    # natural scale of d output / d parameter: max |output| / parameter, per case and parameter
    scale = np.array([[np.abs(v6[c]).max() / parameter_value(case, p) for p in PARAMS]
                      for c, (case, _) in enumerate(cases)])[:, None, None, :]
    assert np.all(np.abs(g6 - g5) <= 1e-4 * scale)
    # the problem is mirror-symmetric (y -> 1 - y, u -> -u): equal wall shear, opposite wall heat
    # flux, and the same for their derivatives (to the rounding of the differences, ~1e-10 of scale)
    assert np.allclose(v6[:, 0, 0], v6[:, 1, 0], rtol=1e-12, atol=0.0)
    assert np.allclose(v6[:, 0, 1], -v6[:, 1, 1], rtol=1e-12, atol=0.0)
    assert np.all(np.abs(g6[:, 0, 0] - g6[:, 1, 0]) <= 1e-8 * scale[:, 0, 0])
    assert np.all(np.abs(g6[:, 0, 1] + g6[:, 1, 1]) <= 1e-8 * scale[:, 0, 0])
