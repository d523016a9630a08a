"""The host side of the differentiable wall outputs (ugks2d_high_order_b200/adjoint.py), without a GPU:
a stand-in for the solver records the cases it is given and returns fixed outputs and C-ABI gradients,
so the test checks the mapping between the autograd parameters (wall speed U, wall temperature T_w,
tau scale s per case) and the C ABI's (mu_ref, wall_ux[0], wall_ux[1], wall_tnative[0], wall_tnative[1])."""
import numpy as np
import pytest
import torch

from ugks2d_high_order_b200 import adjoint
from ugks2d_high_order_b200.case import reference_case


class FakeSolver:
    made = []

    def __init__(self, case, u, v, w, device=0):
        self.case = case
        self.closed = False
        FakeSolver.made.append(self)

    def init_freestream(self, tnative=None):
        pass

    def s2cn2_forward_checkpointed(self, steps, every):
        self.steps, self.every = steps, every
        c = self.case
        return np.array([c.wall_ux[1], c.wall_tnative[0], c.mu_ref, c.wall_ux[0]])

    def s2cn2_backward(self, seed):
        self.seed = np.array(seed)
        return np.array([10.0, 1.0, 2.0, 3.0, 4.0])   # d/d(mu_ref, ux0, ux1, tw0, tw1)

    def close(self):
        self.closed = True


@pytest.fixture
def fake(monkeypatch):
    FakeSolver.made = []
    monkeypatch.setattr(adjoint, "Solver", FakeSolver)
    return FakeSolver


def test_forward_builds_the_cases_and_backward_maps_the_gradients(fake):
    base = reference_case("S2CN2")
    vel = (np.zeros(4), np.zeros(4), np.ones(4))
    p = torch.tensor([[0.5, 1.2, 2.0], [0.25, 0.9, 0.5]], dtype=torch.float64, requires_grad=True)
    out = adjoint.wall_outputs(p, [(base, vel), (base, vel)], steps=7, every=3)
    assert out.shape == (2, 2, 2)
    for n, sv in enumerate(fake.made):
        U, Tw, s = p[n].tolist()
        assert sv.case.wall_ux == (-U, U) and sv.case.wall_tnative == (Tw, Tw)
        assert sv.case.mu_ref == pytest.approx(base.mu_ref * s)
        assert (sv.steps, sv.every) == (7, 3)
        assert out[n].reshape(4).tolist() == [U, Tw, pytest.approx(base.mu_ref * s), -U]
    g = torch.tensor([[[1.0, 2.0], [3.0, 4.0]], [[-1.0, 0.5], [0.25, 2.0]]], dtype=torch.float64)
    (out * g).sum().backward()
    for n, sv in enumerate(fake.made):
        assert np.array_equal(sv.seed, g[n].reshape(4).numpy()) and sv.closed
    # U: walls at (-U, +U) -> d ux1 - d ux0; T_w: both walls -> d tw0 + d tw1; s: mu_ref = s mu0 -> mu0 d mu
    expect = np.array([2.0 - 1.0, 3.0 + 4.0, base.mu_ref * 10.0])
    assert np.allclose(p.grad.numpy(), np.stack([expect, expect]))
