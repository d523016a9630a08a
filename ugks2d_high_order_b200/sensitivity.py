"""Wall shear and heat-flux sensitivities of S2CN2 Couette runs by central differences on the batch.

The quantities are the reference's wall aerodynamics per wall, averaged over the wall cells
(PublishWallDiagnostics, mod_S2NativeAdapter.f90:1075-1097; the wall_history.csv columns
shear_per_length and heat_per_length, mod_R5Observe.f90:379-404): the tangential stress pnt and the
heat flux qn - u_w * mass flux of each wall after `steps` S2CN2 steps from the cold start.

The parameters are the wall speed U_w (both walls, which move at -U_w and +U_w), the wall temperature
T_w (both walls, native units) and the tau scale (the viscosity mu_ref, so Kn = sqrt(pi) mu_ref).
Each case becomes 7 instances of one batch: the base case and, per parameter, the case with the
parameter scaled by (1 + h) and by (1 - h).  Every instance runs the single-instance kernels (the
batch is bitwise the single runs), so each derivative is the central difference
    dF/dp = (F(p (1 + h)) - F(p (1 - h))) / (2 h p),
with truncation error O(h^2) and rounding error of about eps |F| / h.

This is the finite-difference check that a hand-written adjoint of the step would be measured
against; the adjoint itself is not part of this package.
"""
import numpy as np

from .case import velocity_table

PARAMS = ("wall_speed", "wall_temperature", "tau_scale")
OUTPUTS = ("shear", "heat")


def perturbed(case, param, factor):
    """`case` with one parameter scaled by `factor`."""
    if param == "wall_speed":
        return case.with_(wall_ux=(case.wall_ux[0] * factor, case.wall_ux[1] * factor))
    if param == "wall_temperature":
        return case.with_(wall_tnative=(case.wall_tnative[0] * factor, case.wall_tnative[1] * factor))
    if param == "tau_scale":
        return case.with_(mu_ref=case.mu_ref * factor)
    raise ValueError(f"unknown parameter {param!r}")


def parameter_value(case, param):
    return {"wall_speed": case.wall_ux[1], "wall_temperature": case.wall_tnative[0], "tau_scale": case.mu_ref}[param]


def wall_outputs(aero):
    """[wall (bottom, top)][shear, heat]: the wall-cell means of pnt and qn - u_w * mass flux."""
    return np.stack([aero[:, :, 1].mean(axis=1), aero[:, :, 2].mean(axis=1)], axis=1)


def sensitivity_instances(cases, rel_step=1e-6):
    """The batch instances of `cases`: per case the base case, then per parameter the +h and -h cases."""
    tables = {}
    instances = []
    for case, nva in cases:
        if nva not in tables:
            tables[nva] = velocity_table(nva)
        instances.append((case, tables[nva]))
        for p in PARAMS:
            instances.append((perturbed(case, p, 1.0 + rel_step), tables[nva]))
            instances.append((perturbed(case, p, 1.0 - rel_step), tables[nva]))
    return instances


def central_differences(cases, outs, rel_step):
    """(values, grads) from the wall outputs of sensitivity_instances(cases), in their order."""
    k = 1 + 2 * len(PARAMS)
    values = np.empty((len(cases), 2, 2))
    grads = np.empty((len(cases), 2, 2, len(PARAMS)))
    for c, (case, _) in enumerate(cases):
        o = outs[c * k:(c + 1) * k]
        values[c] = o[0]
        for j, p in enumerate(PARAMS):
            grads[c, :, :, j] = (o[1 + 2 * j] - o[2 + 2 * j]) / (2.0 * rel_step * parameter_value(case, p))
    return values, grads


def wall_sensitivities(cases, steps, rel_step=1e-6, device=0, max_streams=16, tnative=2.0):
    """Central-difference sensitivities of the wall outputs of S2CN2 runs.

    cases: [(CouetteCase with method S2CN2, velocities per axis)].  Returns (values, grads):
    values[c][wall][output] after `steps` steps of case c, grads[c][wall][output][param] = d output /
    d param (PARAMS order, per unit of the parameter).  Raises UgksError if any instance's step is
    rejected."""
    from .batch import Batch
    from .capi import UgksError
    instances = sensitivity_instances(cases, rel_step)
    b = Batch(instances, device=device, max_streams=max_streams)
    try:
        b.init_freestream(tnative=tnative)
        done, status = b.run(steps)
        if not (np.all(done == steps) and not np.any(status)):
            raise UgksError(-1, "a sensitivity instance was rejected before the last step")
        outs = np.stack([wall_outputs(b.wall_aero(i)) for i in range(len(instances))])
    finally:
        b.close()
    return central_differences(cases, outs, rel_step)
