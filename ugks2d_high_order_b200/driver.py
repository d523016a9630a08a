"""Command-line driver for the Couette case (the role of the reference's run.sh + Solve_UGKS loop).

    python -m ugks2d_high_order_b200.driver --method Explicit --steps 200 [--cfl 0.5 --omega 0.81]
    python -m ugks2d_high_order_b200.driver --method S2CN2 --steps 20 [--nvel 48 --ny 128]
    python -m ugks2d_high_order_b200.driver --case-dir CASE [--out DIR] [--steps N]

The last form runs a reference case directory unchanged (Config.ini, Mesh2d.dat, velocity file;
restart files when Iflag_InitFlow = 2) and writes sparse_residual.csv and the restart set
(ugks2d_high_order_b200.caserun).

Runs the case on cuda:0 and prints the residual line every --show steps, as Write_residuals does
(src/mod_Solve.f90:427-461).  Also the small, self-contained command used for ncu captures.
"""
import argparse
import time

from .case import CouetteCase, reference_case, velocity_table
from .solver import Solver


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--method", default="Explicit",
                    choices=["Explicit", "ImplicitSteady", "HighOrderImplicit", "S2CN2"])
    ap.add_argument("--steps", type=int, default=None, help="steps to run (default 100; --case-dir: MAX_ITER)")
    ap.add_argument("--show", type=int, default=100)
    ap.add_argument("--cfl", type=float, default=None)
    ap.add_argument("--omega", type=float, default=None)
    ap.add_argument("--ny", type=int, default=None)
    ap.add_argument("--nx", type=int, default=None)
    ap.add_argument("--nvel", type=int, default=32, help="velocities per axis (32: the reference's table)")
    ap.add_argument("--case-dir", default=None, help="run this reference case directory instead")
    ap.add_argument("--out", default=None, help="output directory of --case-dir (default: the case directory)")
    a = ap.parse_args(argv)
    if a.case_dir:
        from .caserun import run_case_dir
        t0 = time.perf_counter()
        done, conv, _ = run_case_dir(a.case_dir, a.out, a.steps, log=lambda m: print(m, flush=True))
        print(f"{done} steps in {time.perf_counter() - t0:.3f} s" + ("" if conv is None else f", converged={conv}"))
        return
    if a.steps is None:
        a.steps = 100
    case = reference_case(a.method)
    kw = {}
    if a.cfl is not None:
        kw["cfl"] = a.cfl
    if a.omega is not None:
        kw["omega"] = a.omega
    if a.ny is not None:
        kw["ny"] = a.ny
        kw["dy"] = 1.0 / a.ny
    if a.nx is not None:
        kw["nx"] = a.nx
        kw["dx"] = 1.0 / a.nx
    case = case.with_(**kw) if kw else case
    s = Solver(case, *velocity_table(a.nvel))
    s.init_freestream()
    if a.method in ("ImplicitSteady", "HighOrderImplicit"):
        s.implicit_init()
    t0 = time.perf_counter()
    done = 0
    while done < a.steps:
        n = min(a.show, a.steps - done)
        if a.method == "Explicit":
            dt, res = s.step_explicit(n)
            done += n
            print(f"iter={done:8d} dt={dt:.7e} res={' '.join(f'{r:.7e}' for r in res)}", flush=True)
        elif a.method == "S2CN2":
            got, rep = s.step_s2cn2(n)
            done += n
            print(f"iter={done:8d} dt={rep[0]:.7e} cnres={rep[1]:.3e} mmerr={rep[2]:.3e} drift={rep[9]:.3e} "
                  f"wall_balance_rho={rep[18]:.6e}", flush=True)
        else:
            got, conv, rep = s.step_implicit(n)
            done += n
            print(f"iter={done:8d} Rrho={rep[12]:.4e} RrhoU={rep[13]:.4e} RrhoV={rep[14]:.4e} RE={rep[15]:.4e} "
                  f"Rh={rep[24]:.4e} Rb={rep[25]:.4e} moment={rep[1]:.4e} c_minus_1={rep[52]:.6e} "
                  f"streak={int(rep[56])}", flush=True)
            if conv or got < n:
                print(f"five-state gate reached after {int(s.implicit_state()[0][7])} accepted steps", flush=True)
                break
    el = time.perf_counter() - t0
    print(f"{a.steps} steps in {el:.3f} s ({case.nx * case.ny * s.nvel * a.steps / el:.3e} cell-vel updates/s)")
    s.close()


if __name__ == "__main__":
    main()
