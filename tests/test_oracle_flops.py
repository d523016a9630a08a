"""The op-counting build of the oracle (oracle/flopcount.hpp), which gives bench.py its FP64 operations
per update: it must compute exactly what the oracle computes, and count a plausible workload.

Each build runs in a child process (the oracle module binds one library per process) on a small
S2CN2 case: 8 x 16 cells, the generated 24 x 24 velocity set, one warm-up step and one counted step.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, json, os, sys
sys.path.insert(0, {root!r})
import numpy as np
import oracle.oracle as oo
flops = {flops}
if flops:
    oo.LIB_PATH = os.path.join({root!r}, "oracle", "_build", "libugks_oracle_flops.so")
from ugks2d_high_order_b200.case import reference_case, velocity_table
oo.set_threads(1)
case = reference_case("S2CN2").with_(ny=16, dy=1.0 / 16)
u, v, w = velocity_table(24)
o = oo.Oracle(case, u, v, w)
o.init_freestream()
o.s2cn2_step()
L = oo.lib()
if flops:
    L.uo_flops_reset()
o.s2cn2_step()
h, b, W = o.get_state()
out = {{"h": h.tobytes().hex()[:4096], "sum": [float(np.sum(h)), float(np.sum(b)), float(np.sum(W))]}}
if flops:
    c = (ctypes.c_ulonglong * 8)()
    L.uo_flops_read(c)
    out["counts"] = list(c)
    out["n"] = case.nx * case.ny * len(u)
print(json.dumps(out))
"""


def _run(flops):
    p = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, flops=flops)], check=True,
                       capture_output=True, text=True)
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_counting_build_reproduces_the_oracle_and_counts_the_step():
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "all", "flops"], check=True,
                   stdout=subprocess.DEVNULL)
    plain, counted = _run(False), _run(True)
    assert plain["sum"] == counted["sum"] and plain["h"] == counted["h"]
    add, mul, div = counted["counts"][:3]
    per_update = (add + mul + div) / counted["n"]
    # an S2CN2 step is ~2.8e4 FP64 operations per cell-velocity (WENO templates, closures, node fluxes)
    assert 1.5e4 < per_update < 5e4
    assert counted["counts"][4] > 0          # exp calls (closure Maxwellians)
