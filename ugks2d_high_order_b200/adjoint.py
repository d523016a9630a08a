"""Gradients of S2CN2 wall outputs through the discrete adjoint, as a torch.autograd.Function.

The outputs are the reference's wall aerodynamics of the last step's evaluation, averaged over each
wall (PublishWallDiagnostics, mod_S2NativeAdapter.f90:1075-1097): [wall (bottom, top)][shear pnt, heat
qn - u_w * mass flux].  The parameters of a case are its wall speed U_w (the walls move at -U_w and
+U_w), its wall temperature T_w (both walls, native units) and its tau scale s (mu_ref = s * mu_ref of
the case, so Kn scales with s).  The forward runs the S2CN2 steps on the GPU with a checkpoint every
`every` steps (ugks_s2cn2_forward_checkpointed); the backward is the device's reverse sweep with
recompute (ugks_s2cn2_backward), transposed onto (U_w, T_w, s).  torch holds no part of the solver: it
only carries the three parameters per case and the cotangents of the outputs.
"""
import numpy as np
import torch

from .solver import Solver

PARAMS = ("wall_speed", "wall_temperature", "tau_scale")


def case_at(case, U, Tw, s):
    """The case with wall speed U (walls at -U, +U), wall temperature Tw and tau scale s."""
    return case.with_(wall_ux=(-U, U), wall_tnative=(Tw, Tw), mu_ref=case.mu_ref * s)


class WallOutputs(torch.autograd.Function):
    """params [n, 3] float64 (U_w, T_w, s per case) -> outputs [n, 2, 2] float64 after `steps` S2CN2 steps
    from the cold start of each case (cases: [(CouetteCase of method S2CN2, (u, v, w))])."""

    @staticmethod
    def forward(ctx, params, cases, steps, every, tnative, device):
        p = params.detach().cpu().numpy().astype(np.float64)
        outs, solvers = [], []
        try:
            for (case, vel), (U, Tw, s) in zip(cases, p):
                sv = Solver(case_at(case, float(U), float(Tw), float(s)), *vel, device=device)
                solvers.append(sv)
                sv.init_freestream(tnative=tnative)
                outs.append(sv.s2cn2_forward_checkpointed(int(steps), int(every)).reshape(2, 2))
        except Exception:
            for sv in solvers:
                sv.close()
            raise
        ctx.solvers = solvers
        ctx.mu0 = np.array([case.mu_ref for case, _ in cases])
        return torch.from_numpy(np.stack(outs)).to(params.device)

    @staticmethod
    def backward(ctx, gout):
        g = gout.detach().cpu().numpy().astype(np.float64).reshape(len(ctx.solvers), 4)
        grads = np.zeros((len(ctx.solvers), 3))
        try:
            for n, sv in enumerate(ctx.solvers):
                d = sv.s2cn2_backward(g[n])   # d/d(mu_ref, wall_ux[0], wall_ux[1], wall_tnative[0], wall_tnative[1])
                sv.close()
                grads[n] = (d[2] - d[1], d[3] + d[4], ctx.mu0[n] * d[0])
        finally:
            for sv in ctx.solvers:
                sv.close()
            ctx.solvers = []
        return torch.from_numpy(grads).to(gout.device), None, None, None, None, None


def wall_outputs(params, cases, steps, every=50, tnative=None, device=0):
    """Differentiable wall outputs [n, 2, 2] of the cases at params [n, 3] (U_w, T_w, tau scale)."""
    return WallOutputs.apply(params, cases, steps, every, tnative, device)
