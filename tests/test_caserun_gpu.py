"""Case directories and restarts on the device.

A run restarted from the files written at step N continues exactly as the uninterrupted run: the
restart set holds the full FP64 state (flow2d.dat, vdf2d.dat), M0 (closed_mass_rank*.bin) and the
residual references (residual_reference.in, 17 significant digits), and the kernels are
deterministic, so the comparison is bitwise.  The streak of the five-state gate restarts at 0 on
both sides of this comparison (no state passes the gate this early).
"""
import os
import shutil

import numpy as np
import pytest

from ugks2d_high_order_b200 import refio
from ugks2d_high_order_b200.case import load_velocity_half32, reference_case

N1, N2 = 25, 15
RESTART_FILES = ("flow2d.dat", "vdf2d.dat", "grid2d.grd", "residual_reference.in")


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["Explicit", "ImplicitSteady", "HighOrderImplicit", "S2CN2"])
def test_restart_continues_bitwise(tmp_path, method):
    from ugks2d_high_order_b200.caserun import run_case_dir
    from ugks2d_high_order_b200.solver import Solver
    case = reference_case(method)
    u, v, w = load_velocity_half32()
    a, b = str(tmp_path / "a"), str(tmp_path / "b")
    ctl = {"Nstep_restart": N1, "Iflag_WriteRestart": 1, "Nstep_show": 5}
    refio.write_case_dir(a, case, u, v, w, extra=ctl)
    done, conv, _ = run_case_dir(a, steps=N1, log=lambda m: None)
    assert done == N1 and not conv
    refio.write_case_dir(b, case, u, v, w, extra=dict(ctl, Iflag_InitFlow=2))
    for f in os.listdir(a):
        if f in RESTART_FILES or f.startswith("closed_mass_rank"):
            shutil.copy(os.path.join(a, f), os.path.join(b, f))
    done2, _, rep2 = run_case_dir(b, steps=N2, log=lambda m: None)
    assert done2 == N2

    s = Solver(case, u, v, w)
    try:
        s.init_freestream()
        if method in ("ImplicitSteady", "HighOrderImplicit"):
            s.implicit_init()
            s.step_implicit(N1)
            _, _, rep = s.step_implicit(N2)
            assert np.array_equal(rep2, rep)
        elif method == "S2CN2":
            s.step_s2cn2(N1)
            s.step_s2cn2(N2)
        else:
            s.step_explicit(N1)
            s.step_explicit(N2)
        h, bb, W = s.download()
    finally:
        s.close()
    W2, h2, b2 = refio.read_restart(b, case.nx, case.ny, len(u))
    assert np.array_equal(W2, W.reshape(-1, 4))
    assert np.array_equal(h2, h.reshape(h2.shape)) and np.array_equal(b2, bb.reshape(b2.shape))
    if method in ("ImplicitSteady", "HighOrderImplicit"):
        rows = open(os.path.join(b, "sparse_residual.csv")).read().splitlines()
        assert rows[0] == refio.SPARSE_HEADER and len(rows) == 1 + N2
        assert rows[1].startswith("1,%d,accepted_convergence_verification," % (N1 + 1))
        assert rows[-1] == refio.sparse_row(N2, N1 + N2, rep2, case.mass_rescale)
        m0, _, step = refio.read_mass_restart(b, refio.load_case_dir(b).config, u, w, case.nx, case.ny, len(u))
        assert step == N1 + N2 and m0 > 0.0
        plt = open(os.path.join(b, "ResidualImplicit.plt")).read().splitlines()
        assert plt[0] == refio.RESIDUAL_IMPLICIT_HEADER and len(plt) == 1 + N2 // 5
        assert plt[-1] == refio.residual_implicit_row(N2, rep2, case.ncfl, True, float(plt[-1][12 + 11 * 18 + 8:][:18]))


@pytest.mark.gpu
def test_delivered_implicit_case_runs_to_the_gate(tmp_path):
    """The delivered low_implicit case directory, run by the driver from the cold start: 1097 accepted
    states (the reference: 1096), the last five passing the gate, one sparse row per state and the
    restart set at the end."""
    from ugks2d_high_order_b200.caserun import run_case_dir
    case = reference_case("ImplicitSteady")
    u, v, w = load_velocity_half32()
    d = str(tmp_path / "low_implicit")
    refio.write_case_dir(d, case, u, v, w, extra={"Nstep_restart": 100, "Iflag_WriteRestart": 1, "Nstep_show": 100})
    done, conv, rep = run_case_dir(d, log=lambda m: None)
    assert conv and done == 1097
    rows = open(os.path.join(d, "sparse_residual.csv")).read().splitlines()[1:]
    assert len(rows) == done
    gate = [float(r.split(",")[3]) for r in rows]
    assert gate[-5:] == [1.0] * 5 and gate[-6] == 0.0
    assert rows[-1] == refio.sparse_row(done, done, rep, True)
    m0, _, step = refio.read_mass_restart(d, refio.load_case_dir(d).config, u, w, case.nx, case.ny, len(u))
    assert step == done and abs(m0 - 1.0) < 1e-14
