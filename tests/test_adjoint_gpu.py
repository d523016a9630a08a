"""The discrete adjoint of the S2CN2 step on the GPU, through the C ABI.

The adjoint is the transpose of the step's Jacobian.  It is checked three ways:
  * the dot-product identity <J v, u> = <v, J^T u> at one step, with J v from the oracle's tangent build
    (the oracle itself run with (value, derivative) numbers, oracle/tangent.py) and J^T u from the
    device's vector-Jacobian product, for directions in h, b, W and in each parameter;
  * gradients through several steps (checkpoint-and-recompute) against central differences of the GPU
    forward and against the tangent oracle's exact forward-mode derivatives;
  * the checkpoint interval does not change the gradient.
The GPU and the oracle evaluate the same step with differently ordered moment sums, so their Jacobians
agree to the tolerance of the high-order parity tests, not bit for bit.
"""
import numpy as np
import pytest

from ugks2d_high_order_b200.case import reference_case, velocity_table

pytestmark = pytest.mark.gpu

PARAMS = ("mu_ref", "wall_ux0", "wall_ux1", "wall_tnative0", "wall_tnative1")
DOT_TOL = 2e-11     # <J v, u> vs <v, J^T u>, GPU adjoint against the oracle's tangent, relative (worst seen 8e-12)
FD_TOL = 1e-6       # gradient vs central differences (h = 1e-6 relative), relative to the gradient's norm
EXACT_TOL = 1e-10   # gradient vs the tangent oracle's forward-mode derivative, relative to the gradient's norm


def _case():
    return reference_case("S2CN2").with_(ny=16, dy=1.0 / 16.0)


def _perturbed(case, p, d):
    if p == "mu_ref":
        return case.with_(mu_ref=case.mu_ref + d)
    if p.startswith("wall_ux"):
        w = int(p[-1])
        ux = list(case.wall_ux)
        ux[w] += d
        return case.with_(wall_ux=tuple(ux))
    w = int(p[-1])
    tw = list(case.wall_tnative)
    tw[w] += d
    return case.with_(wall_tnative=tuple(tw))


def _param_value(case, p):
    return {"mu_ref": case.mu_ref, "wall_ux0": case.wall_ux[0], "wall_ux1": case.wall_ux[1],
            "wall_tnative0": case.wall_tnative[0], "wall_tnative1": case.wall_tnative[1]}[p]


def _dparams(p):
    if p == "mu_ref":
        return {"mu_ref": 1.0}
    w = int(p[-1])
    d = [0.0, 0.0]
    d[w] = 1.0
    return {"wall_ux": tuple(d)} if p.startswith("wall_ux") else {"wall_tnative": tuple(d)}


def _moments(vel, h, b):
    u, v, w = vel
    return np.stack([np.sum(w * h, -1), np.sum(w * u * h, -1), np.sum(w * v * h, -1),
                     np.sum(0.5 * w * ((u * u + v * v) * h + b), -1)], -1)


@pytest.fixture(scope="module")
def developed_state():
    """A state with developed wall layers: 3 S2CN2 steps of the cold start, then h and b scaled per
    (cell, velocity) by factors in [0.9, 1.1] and W set to the moments of (h, b).

    The scaling makes the Jacobian well defined along every direction.  The Couette state is uniform in
    x, so wherever the positivity limiter acts (near the walls) the candidates of a cell's left and right
    face samples tie exactly (limit_cell_outputs, mod_S2D1.f90:315-345), and theta = min(candidates) has
    different one-sided derivatives along directions that break the uniformity.  The device and the
    oracle then pick different sides of the tie, each right for its own branch.  Directions that keep
    the uniformity (the parameters: wall speed, wall temperature, tau scale) see no kink.  On the
    scaled state no two candidates tie, and the device's vector-Jacobian product and the oracle's
    Jacobian-vector product describe the same derivative."""
    from ugks2d_high_order_b200.solver import Solver
    vel = velocity_table(24)
    s = Solver(_case(), *vel)
    try:
        s.init_freestream()
        s.step_s2cn2(3)
        h, b, _ = s.download()
    finally:
        s.close()
    g = np.random.default_rng(11)
    h = h * g.uniform(0.9, 1.1, size=h.shape)
    b = b * g.uniform(0.9, 1.1, size=b.shape)
    return vel, (h, b, _moments(vel, h, b))


def _tangent_step(case, vel, state, dstate=(None, None, None), dparams=None):
    """J v of one step by the tangent oracle: (dh', db', dW', d wall outputs[4])."""
    from oracle.tangent import TangentOracle
    t = TangentOracle(case, *vel, dparams=dparams)
    h, b, W = state
    t.set_state(h, b, W, *dstate)
    out = t.s2cn2_step()
    _, dh, _, db, _, dW = t.get_state()
    _, dwall = t.wall_outputs(out[0])
    return dh, db, dW, dwall.reshape(4)


def test_step_vjp_dot_product_with_the_tangent_oracle(developed_state):
    from ugks2d_high_order_b200.solver import Solver
    vel, state = developed_state
    case = _case()
    rng = np.random.default_rng(20261204)
    h, b, W = state
    u = [rng.standard_normal(h.shape), rng.standard_normal(b.shape), rng.standard_normal(W.shape)]
    seed = rng.standard_normal(4)
    s = Solver(case, *vel)
    try:
        s.upload(h, b, W)
        s.s2cn2_init()
        lh, lb, lW, grad = s.s2cn2_step_vjp(u[0], u[1], u[2], seed)
    finally:
        s.close()
    lam = (lh, lb, lW)

    def lhs(jv):
        return sum(float(np.sum(a * c)) for a, c in zip(u, jv[:3])) + float(np.dot(seed, jv[3]))

    # state directions, one field at a time (h, b, W)
    for which in range(3):
        v = [None, None, None]
        v[which] = rng.standard_normal(state[which].shape) * np.abs(state[which]).max()
        jv = _tangent_step(case, vel, state, tuple(v))
        a, c = lhs(jv), float(np.sum(v[which] * lam[which]))
        assert abs(a - c) <= DOT_TOL * max(abs(a), abs(c)), (which, a, c)
    # parameter directions: d(<u, x'> + seed . out) / dp = grad[p]
    for q, p in enumerate(PARAMS):
        jv = _tangent_step(case, vel, state, dparams=_dparams(p))
        a = lhs(jv)
        assert abs(a - grad[q]) <= DOT_TOL * max(abs(a), 1e-12), (p, a, grad[q])


def _gpu_outputs(case, vel, nsteps, state=False):
    from ugks2d_high_order_b200.sensitivity import wall_outputs
    from ugks2d_high_order_b200.solver import Solver
    s = Solver(case, *vel)
    try:
        s.init_freestream()
        done, _ = s.step_s2cn2(nsteps)
        assert done == nsteps
        out = wall_outputs(s.wall_aero()).reshape(4)
        return (out, s.download()) if state else out
    finally:
        s.close()


def _oracle_outputs(case, vel, nsteps):
    from oracle.oracle import Oracle, set_threads
    set_threads(None)
    o = Oracle(case, *vel)
    o.init_freestream()
    for _ in range(nsteps):
        out = o.s2cn2_step()
    # PublishWallDiagnostics (mod_S2NativeAdapter.f90:1075-1097): pnt = -rate_x, qn = rate_E - u_w rate_x,
    # rate = the wall face's macro flux / (dt dx), averaged over the wall
    fy = o.view("face_y_w", (case.ny + 1, case.nx, 4))
    res = []
    for wall, row in ((0, 0), (1, case.ny)):
        r = fy[row] / (out[0] * case.dx)
        res += [(-r[:, 1]).mean(), (r[:, 3] - case.wall_ux[wall] * r[:, 1]).mean()]
    return np.array(res)


def _gradient_checks(case, vel, nsteps, every, seed):
    """The adjoint's parameter gradient after nsteps from the cold start against central differences of
    the GPU forward and of the oracle forward (h = 1e-6 relative) and against the tangent oracle."""
    from oracle.tangent import TangentOracle
    from ugks2d_high_order_b200.solver import Solver
    s = Solver(case, *vel)
    try:
        s.init_freestream()
        out = s.s2cn2_forward_checkpointed(nsteps, every=every)
        end = s.download()
        grad = s.s2cn2_backward(seed)
    finally:
        s.close()
    # the checkpointed run is the plain run: the same state bit for bit; the outputs are wall means, summed
    # in another order on the host
    plain, plain_end = _gpu_outputs(case, vel, nsteps, state=True)
    assert all(np.array_equal(a, c) for a, c in zip(end, plain_end))
    assert np.abs(out - plain).max() <= 1e-14 * np.abs(plain).max()
    fd, fdo, exact = np.zeros(5), np.zeros(5), np.zeros(5)
    for q, p in enumerate(PARAMS):
        d = 1e-6 * abs(_param_value(case, p))
        cp, cm = _perturbed(case, p, d), _perturbed(case, p, -d)
        fd[q] = float(np.dot(seed, _gpu_outputs(cp, vel, nsteps) - _gpu_outputs(cm, vel, nsteps))) / (2.0 * d)
        fdo[q] = float(np.dot(seed, _oracle_outputs(cp, vel, nsteps) - _oracle_outputs(cm, vel, nsteps))) / (2.0 * d)
        t = TangentOracle(case, *vel, dparams=_dparams(p))
        t.init_freestream()
        for _ in range(nsteps):
            o = t.s2cn2_step()
        exact[q] = float(np.dot(seed, t.wall_outputs(o[0])[1].reshape(4)))
    scale = np.abs(grad).max()
    assert np.abs(grad - fd).max() <= FD_TOL * scale, (grad, fd)
    assert np.abs(grad - fdo).max() <= FD_TOL * scale, (grad, fdo)
    assert np.abs(grad - exact).max() <= EXACT_TOL * scale, (grad, exact)


def test_gradient_through_steps_matches_central_differences_and_the_tangent_oracle():
    _gradient_checks(_case(), velocity_table(24), 6, 4, np.array([0.7, -1.3, 0.4, 0.9]))


def test_gradient_of_an_adjoint_workload_instance():
    """One case of the adjoint workload's 64 (the batched distribution at 8 x 64 cells, 32^2
    velocities): six steps, checkpoints every four."""
    from ugks2d_high_order_b200.case import batched_cases
    case = batched_cases(64)[0][0].with_(ny=64, dy=1.0 / 64)
    _gradient_checks(case, velocity_table(32), 6, 4, np.array([1.0, 1.0, 1.0, 1.0]))


def test_checkpoint_interval_does_not_change_the_gradient():
    from ugks2d_high_order_b200.solver import Solver
    case, vel, nsteps = _case(), velocity_table(24), 7
    seed = np.array([1.0, 0.5, -0.25, 2.0])
    grads = []
    for every in (7, 3, 1):
        s = Solver(case, *vel)
        try:
            s.init_freestream()
            s.s2cn2_forward_checkpointed(nsteps, every=every)
            grads.append(s.s2cn2_backward(seed))
        finally:
            s.close()
    for g in grads[1:]:
        assert np.abs(g - grads[0]).max() <= 1e-12 * np.abs(grads[0]).max(), (g, grads[0])


def test_one_step_backward_equals_the_step_vjp():
    from ugks2d_high_order_b200.solver import Solver
    case, vel = _case(), velocity_table(24)
    seed = np.array([0.3, 1.1, -0.8, 0.6])
    s = Solver(case, *vel)
    try:
        s.init_freestream()
        h0, b0, W0 = s.download()
        s.s2cn2_forward_checkpointed(1, every=1)
        grad, (gh, gb, gW) = s.s2cn2_backward(seed, initial_state=True)
        s.upload(h0, b0, W0)
        s.s2cn2_init()
        vh, vb, vW, vgrad = s.s2cn2_step_vjp(seed=seed)
    finally:
        s.close()
    for a, c in ((grad, vgrad), (gh, vh), (gb, vb), (gW, vW)):
        assert np.abs(a - c).max() <= 1e-12 * max(np.abs(c).max(), 1e-300)


def test_autograd_function_gives_the_parameter_gradients():
    """WallOutputs (torch.autograd.Function over the C ABI): the gradient of a loss of the wall outputs in
    (wall speed, wall temperature, tau scale) of two cases against central differences of the loss."""
    import torch
    from ugks2d_high_order_b200.adjoint import case_at, wall_outputs
    vel = velocity_table(24)
    base = _case()
    cases = [(base, vel), (base.with_(mu_ref=base.mu_ref * 2.0), vel)]
    p0 = np.array([[abs(base.wall_ux[1]), base.wall_tnative[0], 1.0],
                   [0.7 * abs(base.wall_ux[1]), 1.1 * base.wall_tnative[0], 0.8]])
    wts = torch.tensor([[[1.0, -0.5], [0.25, 2.0]], [[-1.0, 0.3], [0.7, 1.5]]], dtype=torch.float64)
    nsteps = 5
    params = torch.tensor(p0, dtype=torch.float64, requires_grad=True)
    out = wall_outputs(params, cases, nsteps, every=2)
    loss = (wts * out).sum()
    loss.backward()

    def loss_at(p):
        return float((wts * wall_outputs(torch.tensor(p, dtype=torch.float64), cases, nsteps, every=nsteps)).sum())

    fd = np.zeros_like(p0)
    for n in range(2):
        for q in range(3):
            d = 1e-6 * abs(p0[n, q])
            pp, pm = p0.copy(), p0.copy()
            pp[n, q] += d
            pm[n, q] -= d
            fd[n, q] = (loss_at(pp) - loss_at(pm)) / (2.0 * d)
    g = params.grad.numpy()
    assert np.abs(g - fd).max() <= FD_TOL * np.abs(g).max(), (g, fd)
    assert case_at(base, 1.0, 2.0, 3.0).mu_ref == 3.0 * base.mu_ref
