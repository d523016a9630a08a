"""Record the oracle's long ImplicitSteady trajectory of the delivered Couette case as a fixture.

The case file's gate (1e-8) stops the reference at 1096 accepted pseudo-steps.  The headline metric's
gate is 1e-10, which the solve does not reach: science_3 (the rho*V residual, relative to a near-zero
reference) keeps decaying on its round-off floor.  This script runs the C oracle (the CPU restatement
of the reference) for 3000 accepted pseudo-steps of the cold start, never stopping, and writes the
sparse_residual.csv rows of selected steps, and the macro state W at some of them, so that the GPU test can show that the device follows the
same trajectory without the oracle's minutes of CPU time:

    python tests/golden/make_oracle_trajectory.py        # writes tests/golden/oracle_implicit_3000.json

The row layout is that of ugks_implicit_steps' report (include/ugks_b200.h).
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

STEPS = (1, 2, 100, 500, 1000, 1097, 1100, 1500, 2000, 2500, 3000)
STATE_STEPS = (1100, 3000)   # W recorded (the converged state, beside the round-off-floor residuals)
OUT = os.path.join(ROOT, "tests", "golden", "oracle_implicit_3000.json")


def main():
    from oracle.oracle import Oracle, set_threads
    from ugks2d_high_order_b200.case import reference_case, load_velocity_half32
    threads = set_threads(None)
    case = reference_case("ImplicitSteady")
    o = Oracle(case, *load_velocity_half32())
    o.init_freestream()
    o.implicit_init()
    rows, states = {}, {}
    t0 = time.perf_counter()
    for n in range(1, max(STEPS) + 1):
        r = o.implicit_step()
        if n in STEPS:
            rows[str(n)] = [float(x) for x in r[:57]]
            if n in STATE_STEPS:
                states[str(n)] = [float(x) for x in o.get_state()[2].reshape(-1)]
            print(f"step {n}: science_3 {r[14]:.6e}  ({time.perf_counter() - t0:.0f} s)", flush=True)
    with open(OUT, "w") as f:
        json.dump({"case": "cases/low_implicit (8x64 cells, 32x32 velocities), cold start, never stopped",
                   "threads": threads, "rows": rows, "W": states}, f, indent=0)


if __name__ == "__main__":
    main()
