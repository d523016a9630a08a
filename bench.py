"""Benchmark: DVM cell-velocity updates per second of the UGKS2D hot path on B200.

Workload (one "step" of this script): 1000 second-order Explicit UGKS steps of the planar Couette
case, 8x64 cells, 32x32 velocities (velocity_half32_scale2), CFL 0.5, omega 0.81, Kn 0.1, FP64.
One update = one (cell, velocity) with both h and b advanced by one solver step; a bench step is
8*64*1024*1000 = 5.24e8 updates.

  value          device-resident throughput (state already in HBM), CUDA events on the solver's
                 stream, max over ranks.
  e2e            the same through the public C ABI with host buffers: every bench step uploads
                 h, b, W from pinned host memory, runs the 1000 steps and downloads the state.
  roofline       the dominant kernel (per-kernel CUDA events in a separate profiling pass).
  cpu_baseline   the CPU oracle (a restatement of the reference's Fortran; the Fortran itself
                 does not build here) on a bounded sample of the same workload.

Multi-GPU: single instances do not shard (one domain per GPU); N ranks run N independent replicas
("scaling": "weak").  --impl reference times the CPU restatement of the reference on host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DVM cell·vel updates/s + time-to-steady on 1 B200, batched vs plain, vs CPU ref"
UNIT = "cell·vel updates/s"
SOLVER_STEPS = 1000
BYTES_PER_UPDATE_EXPLICIT = 32   # read h,b + write h',b' (FP64), SURVEY 8(d) algorithmic bytes


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed region.

    NVML (the library nvidia-smi is built on) is polled from a host thread every `period` s;
    `nvidia-smi -lms` is the alternative (--sampler smi).  Reasons recorded: hw_slowdown,
    hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap.
    """

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, index, kind="nvml", period=0.2):
        self.index, self.kind, self.period = index, kind, period
        self.samples, self.reasons, self.smax = [], set(), None
        self._stop = threading.Event()
        self.proc = None
        self.lines = []

    def start(self):
        if self.kind == "none":
            return
        if self.kind == "smi":
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            try:
                self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                              "--format=csv,noheader,nounits", "-lms", str(int(self.period * 1000))],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.t = threading.Thread(target=self._read_smi, daemon=True)
                self.t.start()
            except Exception:
                self.proc = None
            return
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nv = None
            return
        self.t = threading.Thread(target=self._poll_nvml, daemon=True)
        self.t.start()

    def _poll_nvml(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, bit in self.REASONS.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(self.period)

    def _read_smi(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.strip().split(",")]
            if len(parts) < 9:
                continue
            try:
                self.samples.append(float(parts[1]))
                self.smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    self.reasons.add(n)

    def stop(self):
        if self.kind == "none":
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "sampler": "none"}
        self._stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        elif getattr(self, "t", None):
            self.t.join(timeout=2)
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(self.samples),
                "sampler": "nvml" if self.kind == "nvml" else "nvidia-smi"}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline(case, velocity, nsteps=20, threads=None):
    """The oracle (single-domain restatement of the reference Fortran) on `nsteps` solver steps."""
    from oracle.oracle import Oracle, set_threads
    nthreads = set_threads(threads)
    o = Oracle(case, *velocity)
    o.init_freestream()
    o.explicit_step()   # warm-up
    t0 = time.perf_counter()
    for _ in range(nsteps):
        o.explicit_step()
    el = time.perf_counter() - t0
    units = case.nx * case.ny * len(velocity[0]) * nsteps
    return {"value": units / el, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{nsteps} Explicit solver steps of the 8x64x1024 workload after 1 warm-up step "
                      f"({el:.2f} s, C oracle -O2, {nthreads} pthread(s) over faces/cells)"}


def run_reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from ugks2d_high_order_b200.case import baseline_explicit_case, load_velocity_half32
    case = baseline_explicit_case()
    vel = load_velocity_half32()
    from oracle.oracle import Oracle, set_threads
    nthreads = set_threads(None)
    o = Oracle(case, *vel)
    o.init_freestream()
    per_step = max(1, int(os.environ.get("UGKS_REF_SAMPLE_STEPS", "5")))
    for _ in range(args.warmup):
        o.explicit_step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for _ in range(per_step):
            o.explicit_step()
    el = time.perf_counter() - t0
    units = case.nx * case.ny * len(vel[0]) * per_step * args.steps
    v = units / el
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "explicit 2nd-order UGKS Couette 8x64 cells, 32x32 velocities, CFL 0.5, omega 0.81",
                       "solver_steps_per_bench_step": per_step, "parallelism": "host threads"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"{per_step} solver steps per bench step (the Fortran reference cannot "
                                       f"be built on this image; its C restatement is timed)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sampler", default="nvml", choices=["nvml", "smi", "none"],
                    help="clock sampler during the timed region")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
        return

    world, rank, local = dist_env()
    import torch
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist
    else:
        torch.cuda.set_device(local)

    from ugks2d_high_order_b200.case import baseline_explicit_case, load_velocity_half32
    from ugks2d_high_order_b200.solver import Solver
    case = baseline_explicit_case()
    vel = load_velocity_half32()
    s = Solver(case, *vel, device=local)
    nc, nv = case.nx * case.ny, len(vel[0])
    units_per_bench_step = nc * nv * SOLVER_STEPS
    stream = torch.cuda.ExternalStream(s.stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        if pg:
            t = torch.zeros(1, device=f"cuda:{local}")
            pg.all_reduce(t)
        torch.cuda.synchronize()

    # ---------------- device-resident timing
    s.init_freestream()
    for _ in range(args.warmup):
        s.step_explicit(SOLVER_STEPS)
    s.init_freestream()
    launches0 = s.launch_count
    sampler = ClockSampler(local, args.sampler)
    sampler.start()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for _ in range(args.steps):
            flush.zero_()          # L2 flush between bench steps (256 MB > 126 MB L2)
            s.step_explicit(SOLVER_STEPS)
        ev1.record(stream)
    ev1.synchronize()
    barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    launches = s.launch_count - launches0
    if pg:
        t = torch.tensor([ms], device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    value = world * units_per_bench_step * args.steps / (ms * 1e-3)

    # ---------------- end-to-end through the C ABI with pinned host buffers
    h, b, W = s.download()
    hp = torch.from_numpy(h).pin_memory()
    bp = torch.from_numpy(b).pin_memory()
    Wp = torch.from_numpy(W).pin_memory()
    ho = torch.empty_like(hp).pin_memory()
    bo = torch.empty_like(bp).pin_memory()
    Wo = torch.empty_like(Wp).pin_memory()
    import ctypes
    dp = ctypes.POINTER(ctypes.c_double)
    P = lambda t: ctypes.cast(t.data_ptr(), dp)
    L = s.L
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            flush.zero_()
            L.ugks_upload_state(s.ctx, P(hp), P(bp), P(Wp))
            L.ugks_step_explicit(s.ctx, SOLVER_STEPS, None, None)
            L.ugks_download_state(s.ctx, P(ho), P(bo), P(Wo))
        e1.record(stream)
    e1.synchronize()
    barrier()
    ems = e0.elapsed_time(e1)
    if pg:
        t = torch.tensor([ems], device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ems = float(t.item())
    e2e_value = world * units_per_bench_step * args.steps / (ems * 1e-3)
    state_bytes = (h.nbytes + b.nbytes + W.nbytes)

    # ---------------- per-kernel timing pass (events around each launch, no graph)
    s.init_freestream()
    s.step_explicit(20)
    s.profile(True)
    s.step_explicit(200)
    ktimes = {name: s.profile_read(short) for name, short in
              (("k_lo_slopes", "slopes"), ("k_lo_faces", "faces"), ("k_lo_walls", "walls"), ("k_lo_cells", "cells"))}
    s.profile(False)
    ktot = sum(t for t, _ in ktimes.values())
    top = max(ktimes, key=lambda k: ktimes[k][0])
    t_top, n_top = ktimes[top]
    avg_s = t_top / n_top * 1e-3
    peak, peak_kind = peaks()
    algo_bytes = BYTES_PER_UPDATE_EXPLICIT * nc * nv
    achieved = algo_bytes / avg_s / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": top, "peak_source": peak_kind,
                "kernel_avg_us": avg_s * 1e6,
                "kernel_share": {k: t / ktot for k, (t, _) in ktimes.items()},
                "kernel_avg_us_all": {k: 1e3 * t / max(n, 1) for k, (t, n) in ktimes.items()},
                "algorithmic_bytes_per_launch": algo_bytes}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(case, vel)
        except Exception as e:   # the checker is optional for the device number
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "port", "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "explicit 2nd-order UGKS Couette 8x64 cells, 32x32 velocities "
                                       "(velocity_half32_scale2), CFL 0.5, omega 0.81, Kn 0.1",
                           "solver_steps_per_bench_step": SOLVER_STEPS, "updates_per_bench_step": units_per_bench_step,
                           "parallelism": f"replicas x{world}" if world > 1 else "single instance",
                           "l2": "flushed (256 MB write) between bench steps; state is L2-resident within a step"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                        "d2h_bytes_per_step": state_bytes},
                "gpu_launches": int(launches),
                "roofline": roofline,
                "cpu_baseline": cpu,
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    s.close()
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
