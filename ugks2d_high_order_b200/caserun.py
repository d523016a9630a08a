"""Run a reference case directory on the device (the role of run.sh + Solve_UGKS's outer loop).

`run_case_dir` reads Config.ini, Mesh2d.dat and the velocity file (refio.load_case_dir), starts
from the cold start (Iflag_InitFlow = 0) or from the restart files of the directory (2), advances
MAX_ITER steps (implicit methods stop earlier at the five-state gate), and writes what the
reference writes for this path:
  sparse_residual.csv          every Nstep_monitor-th accepted state (implicit methods),
  ResidualImplicit.plt         every Nstep_show-th step (implicit methods), with the reference's
                               'Implicit iter=' line on the log,
  flow2d.dat, vdf2d.dat,       every Nstep_restart steps and at the end when Iflag_WriteRestart = 1
  grid2d.grd                   (Output_restart_only, mod_Output.f90:30-56),
  closed_mass_rank<r>.bin,     with the mass rescale on (WriteMassRestart), and
  residual_reference.in        (WriteRestartReference).
The correction ledger of closed_mass_rank<r>.bin is written as zeros: the device keeps no ledger
(the reference uses it only for its light_steps.csv audit columns).
"""
import os
import time

import numpy as np

from . import refio
from .solver import Solver

IMPLICIT = ("ImplicitSteady", "HighOrderImplicit")


def write_restart_set(out, d, s, step):
    """The restart files of the current device state (and, for implicit methods, M0 and the
    residual references of the sequence)."""
    h, b, W = s.download()
    c = d.case
    refio.write_restart(out, W, h, b, c.nx, c.ny, d.gridx, d.gridy)
    if c.method in IMPLICIT:
        st, _ = s.implicit_state()
        if c.mass_rescale:
            refio.write_mass_restart(out, d.config, d.u, d.w, W, h, b, c.nx, c.ny, st[0], step=step)
        if st[3] != 0.0:
            refio.write_residual_reference(out, st[1], st[2], c.residual_tol, c.moment_tol)


def start(d, s):
    """Cold start or restart of the device state.  Returns the origin step of the run."""
    c = d.case
    if int(d.run["Iflag_InitFlow"]) != 2:
        s.init_freestream()
        if c.method in IMPLICIT:
            s.implicit_init()
        return 0
    W, h, b = refio.read_restart(d.path, c.nx, c.ny, len(d.u))
    s.upload(h, b, W)
    origin = 0
    if c.method in IMPLICIT:
        if not c.mass_rescale:
            raise refio.CaseError("implicit restart without ClosedCouetteMassRescale has no persistent M0")
        m0, _, origin = refio.read_mass_restart(d.path, d.config, d.u, d.w, c.nx, c.ny, len(d.u), W, h, b)
        ref = None
        if os.path.exists(os.path.join(d.path, "residual_reference.in")):
            epoch, rh, rb, rtol, mtol = refio.read_residual_reference(d.path)
            if rtol != c.residual_tol or mtol != c.moment_tol:
                raise refio.CaseError("reference inheritance convergence thresholds mismatch", 941)
            if epoch > origin:
                raise refio.CaseError("reference epoch after checkpoint", 941)
            ref = (rh, rb)
        else:
            raise refio.CaseError("Couette restart requires residual_reference.in; refusing reference reset", 941)
        s.implicit_restore(m0, ref)
    elif c.method == "S2CN2":
        s.s2cn2_init()
    return origin


def run_case_dir(path, out=None, steps=None, log=print):
    """Run the case in directory `path`, writing outputs into `out` (default: `path`).  Returns
    (steps done, converged or None, last report)."""
    d = refio.load_case_dir(path)
    out = out or path
    os.makedirs(out, exist_ok=True)
    c = d.case
    nsteps = int(steps if steps is not None else d.run["MAX_ITER"])
    show = max(1, int(d.run["Nstep_show"]))
    monitor = max(1, int(d.run["Nstep_monitor"]))
    every = int(d.run["Nstep_restart"])
    write_restart = int(d.run["Iflag_WriteRestart"]) == 1
    s = Solver(c, d.u, d.v, d.w)
    try:
        origin = start(d, s)
        sparse = refio.SparseResidualWriter(out, c.mass_rescale) if c.method in IMPLICIT else None
        plt = refio.ResidualImplicitWriter(out, c.ncfl, c.mass_rescale) if c.method in IMPLICIT else None
        t0 = time.perf_counter()
        done, conv, rep = 0, None, None
        while done < nsteps:
            if c.method in IMPLICIT:
                got, conv, rep = s.step_implicit(1)
                if got == 0:
                    break
                done += got
                if (origin + done) % monitor == 0:
                    sparse.append(done, origin + done, rep)
                if done % show == 0:
                    wall = time.perf_counter() - t0
                    plt.append(done, rep, wall)
                    log(refio.implicit_stdout_line(done, rep, c.ncfl, wall))
            else:
                n = min(show, nsteps - done)
                if every > 0 and write_restart:
                    n = min(n, every - (origin + done) % every)
                if c.method == "S2CN2":
                    got, rep = s.step_s2cn2(n)
                else:
                    dt, res = s.step_explicit(n)
                    got, rep = n, np.concatenate([[dt], res])
                done += got
                log(f"iter={origin + done:8d} dt={rep[0]:.7e}")
            if write_restart and every > 0 and (origin + done) % every == 0:
                write_restart_set(out, d, s, origin + done)
            if conv:
                break
        if write_restart:
            write_restart_set(out, d, s, origin + done)
        return done, conv, rep
    finally:
        s.close()
