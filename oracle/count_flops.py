"""Algorithmic FP64 operations per cell-velocity update, counted by the op-counting oracle build.

    python oracle/count_flops.py            (builds oracle/_build/libugks_oracle_flops.so first)

Measurement infrastructure: the oracle compiled as C++ with every FP64 value a counting type
(oracle/flopcount.hpp).  For each method on its bench case (8 x 64 cells, 32 x 32 velocities, the
reference's delivered case files) the script runs warm-up steps, then counts the steps that follow,
on one thread, and prints the operations per cell-velocity update as JSON.  It first checks that the
counting build reproduces the plain oracle bit for bit on the same steps.  The results are the
flop constants bench.py uses for the FP64 fractions.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NAMES = ("add", "mul", "div", "sqrt", "exp", "erfc", "pow", "acos")
PLAN = {"Explicit": (1, 2), "ImplicitSteady": (2, 2), "HighOrderImplicit": (2, 2), "S2CN2": (1, 2),
        "evaluation_lo": (2, 1), "evaluation_s2": (2, 1), "S2CN2_24": (1, 2), "S2CN2_48": (1, 2)}
# S2CN2 on the batched distribution's other velocity sets (the generated 24^2 and 48^2 tables), on the
# delivered 8 x 64 case otherwise
# the implicit pseudo-step evaluates twice (before the update and for the accepted state); the device
# reuses the accepted-state evaluation as the next pre-update one, so it runs one evaluation less
EVALUATION = {"ImplicitSteady": "evaluation_lo", "HighOrderImplicit": "evaluation_s2"}


def run_one(method, flops):
    """Child process: (state checksum, counts per update) of `method` with the plain or counting build."""
    # the oracle directory itself (this script's) would shadow the `oracle` package
    sys.path[:] = [ROOT] + [q for q in sys.path if os.path.abspath(q or ".") != HERE]
    import ctypes
    import numpy as np
    import oracle.oracle as oo
    if flops:
        oo.LIB_PATH = os.path.join(HERE, "_build", "libugks_oracle_flops.so")
    from ugks2d_high_order_b200.case import load_velocity_half32, reference_case
    oo.set_threads(1)
    base = {"evaluation_lo": "ImplicitSteady", "evaluation_s2": "HighOrderImplicit", "S2CN2_24": "S2CN2",
            "S2CN2_48": "S2CN2"}.get(method, method)
    case = reference_case(base)
    if method in ("S2CN2_24", "S2CN2_48"):
        from ugks2d_high_order_b200.case import velocity_table
        u, v, w = velocity_table(24 if method == "S2CN2_24" else 48)
    else:
        u, v, w = load_velocity_half32()
    o = oo.Oracle(case, u, v, w)
    o.init_freestream()
    if base in ("ImplicitSteady", "HighOrderImplicit"):
        o.implicit_init()
    L = oo.lib()

    def evaluation():   # one evaluation of the current state: fluxes and the residual with collision
        dt = L.uo_timestep(o.ptr)
        if method == "evaluation_lo":
            L.uo_interpolation(o.ptr)
            L.uo_evolution(o.ptr, dt)
            L.uo_compute_residual(o.ptr, dt, 1)
        else:
            L.uo_s2_evolution(o.ptr, dt)
            L.uo_s2_compute_residual(o.ptr, dt, 1)

    step = {"Explicit": o.explicit_step, "S2CN2": o.s2cn2_step, "S2CN2_24": o.s2cn2_step,
            "S2CN2_48": o.s2cn2_step}.get(method, o.implicit_step)
    warm, counted = PLAN[method]
    for _ in range(warm):
        o.implicit_step() if method.startswith("evaluation") else step()
    if flops:
        L.uo_flops_reset()
    for _ in range(counted):
        evaluation() if method.startswith("evaluation") else step()
    h, b, W = o.get_state()
    out = {"checksum": [float(np.sum(h)), float(np.sum(b)), float(np.sum(W))],
           "probe": [float(h.ravel()[777]).hex(), float(W.ravel()[5]).hex()]}
    if flops:
        c = (ctypes.c_ulonglong * 8)()
        L.uo_flops_read(c)
        n = case.nx * case.ny * len(u) * counted
        out["per_update"] = {k: c[i] / n for i, k in enumerate(NAMES)}
    return out


def main():
    subprocess.run(["make", "-C", HERE, "flops"], check=True, stdout=subprocess.DEVNULL)
    result = {}
    for method in PLAN:
        res = {}
        for flops in (False, True):
            p = subprocess.run([sys.executable, __file__, "--child", method, str(int(flops))],
                               check=True, capture_output=True, text=True)
            res[flops] = json.loads(p.stdout.strip().splitlines()[-1])
        same = res[False]["checksum"] == res[True]["checksum"] and res[False]["probe"] == res[True]["probe"]
        if not same:
            raise SystemExit(f"{method}: the counting build does not reproduce the oracle")
        pu = res[True]["per_update"]
        pu["flops"] = pu["add"] + pu["mul"] + pu["div"] + pu["sqrt"]
        result[method] = {k: round(x, 3) for k, x in pu.items()}
    for method, ev in EVALUATION.items():
        result[method]["flops_device"] = round(result[method]["flops"] - result[ev]["flops"], 3)
    print(json.dumps(result, indent=1))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--child":
        print(json.dumps(run_one(sys.argv[2], sys.argv[3] == "1")))
    else:
        main()
