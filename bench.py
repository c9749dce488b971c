#!/usr/bin/env python
"""Benchmark of the B200 FDTD engine on the 3D MMI workload (600 x 200 x 100 = 12 M cells of
20 nm, 10-cell CPML, a Gaussian-profile current at 1550 nm, flux planes on both arms at 51
wavelengths; photonoxide_b200.configs.mmi_3d).

A "step" is one FDTD time step of the whole grid: H and E with the CPML, the source, the probe
and the transforms' accumulation. ``value`` is Gcell-updates/s over all ranks with the fields
resident in HBM; ``e2e`` is the same through the C ABI with host buffers, the upload of the
coefficients and fields and the download of the fields and transforms inside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (under torchrun) every rank steps its own replica of the grid: the path has no
exchange between GPUs, so there is no collective beyond the barriers and the max over ranks of
the timed region. ``--impl reference`` times the CPU restatement of photonoxide's own kernel
(the oracle, f64 as the reference's default) on the host's cores instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FDTD Gcell-updates/s (3D MMI, 12M cells)"
UNIT = "Gcell-updates/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """DRAM bytes per launch of the step kernel from the committed ncu summary, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "step_kernel_mmi.json")) as f:
            return float(json.load(f)["dram_bytes_per_launch"])
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}",
                                          f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = max(mx, float(parts[2]))
                except ValueError:
                    continue
                for name, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(eps, target_seconds=15.0):
    """The oracle (f64, all host threads) on the same MMI problem, timed over a bounded number
    of steps (about 10-30 s of CPU work)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import OracleSimulation
    from photonoxide_b200 import configs

    def make(g, _geo, b, courant, precision=64):
        return OracleSimulation(g, eps, b, courant, precision=64)

    s, info = configs.mmi_3d(make)
    t0 = time.perf_counter()
    s.run(1)
    one = time.perf_counter() - t0
    n = max(1, min(200, int(target_seconds / max(one, 1e-3))))
    t0 = time.perf_counter()
    s.run(n)
    dt = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    value = n * info["cells"] / dt / 1e9
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} steps of the full 600x200x100 MMI grid, f64, OpenMP on {cores} threads "
                      f"({dt:.1f} s)"}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from photonoxide_b200 import configs
    from photonoxide_b200.fdtd import average
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import OracleSimulation, average_boxes
    from photonoxide_b200.types import Grid3d
    g = Grid3d(600, 200, 100, 0.02, 0.02, 0.02, -6.0, -2.0, -1.0)
    eps = average_boxes(g, configs.mmi_geometry())

    def make(grid, _geo, b, courant, precision=64):
        return OracleSimulation(grid, eps, b, courant, precision=64)

    s, info = configs.mmi_3d(make)
    t0 = time.perf_counter()
    s.run(max(1, min(args.warmup, 3)))
    one = (time.perf_counter() - t0) / max(1, min(args.warmup, 3))
    steps = max(1, min(args.steps, int(90.0 / max(one, 1e-3))))
    t0 = time.perf_counter()
    s.run(steps)
    dt = time.perf_counter() - t0
    value = steps * info["cells"] / dt / 1e9
    cores = os.cpu_count() or 1
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": min(args.warmup, 3), "ms_per_step": dt / steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "3D MMI 600x200x100 (20 nm), CPML 10, Gaussian-profile current, "
                               "2 flux planes x 51 wavelengths", "cells": info["cells"]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{steps} steps of the full grid (the oracle: photonoxide's CPU "
                                   f"kernel restated in C++, f64, OpenMP on {cores} threads)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    import torch.distributed as dist
    from photonoxide_b200 import configs
    from photonoxide_b200.engine import Engine
    from photonoxide_b200.fdtd import Simulation, average
    from photonoxide_b200.types import Boundaries

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    sim, info = configs.mmi_3d(Simulation)
    cells = info["cells"]
    sim.run(args.warmup)  # the first run uploads and configures; then warm
    eng = Engine(sim.engine())
    stream = torch.cuda.ExternalStream(eng.stream())
    # algorithmic bytes of one step (60 B/cell + 8 B per psi value, f32)
    psi = configs.psi_values(sim.grid, Boundaries.with_cpml(10))
    bytes_step = configs.mmi_bytes_per_step(cells, psi)

    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    eng.profile(True)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    eng.run_async(args.steps, sim.steps)
    stop.record(stream)
    eng.synchronize()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = start.elapsed_time(stop)
    kernel_ms, kernel_n = eng.profile_read()
    eng.profile(False)
    launches = eng.launches()
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * args.steps * cells / (ms / 1e3) / 1e9

    # end to end through the C ABI: host (pinned) buffers in, the run, the results back
    N = cells
    pin = lambda n: torch.zeros(n, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    cb = pin(3 * N)
    cb[:] = sim.tables(1)
    e_host, h_host = pin(3 * N), pin(3 * N)
    nsums = sim.transforms().size
    sums = pin(2 * nsums)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    wall0 = time.perf_counter()
    e0.record(stream)
    eng.upload_coeffs(None, cb)
    eng.upload_fields(e_host, h_host)
    eng.run_async(args.steps, 0)
    eng.download_fields(e_host, h_host)
    eng.read_dft(sums)
    e1.record(stream)
    eng.synchronize()
    wall = time.perf_counter() - wall0
    e2e_ms = max(e0.elapsed_time(e1), 0.0)
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * args.steps * cells / (e2e_ms / 1e3) / 1e9
    h2d = (3 * N + 6 * N) * 8 / args.steps
    d2h = (6 * N * 8 + 16 * nsums) / args.steps

    peak, peak_kind = peaks()
    per_launch_s = kernel_ms / max(kernel_n, 1) / 1e3
    achieved = bytes_step / per_launch_s / 1e9
    traffic = ncu_traffic()
    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            base = cpu_baseline(np.asarray(configs_eps(sim)), 15.0)
        except Exception as exc:  # the baseline is reported, not the target
            base = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                    "sample": f"failed: {exc}"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "3D MMI 600x200x100 (20 nm), CPML 10, Gaussian-profile current, "
                               "2 flux planes x 51 wavelengths, f32 fields, f64 transforms",
                   "cells": cells, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (fields+coefficients 432 MB)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "bytes_per_launch": bytes_step,
                     "kernel_ms_per_launch": per_launch_s * 1e3},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "wall_s": wall},
        "gpu_launches": launches,
        "clocks": clk,
        "cpu_baseline": base,
    }
    print(json.dumps(line), flush=True)
    return 0


def configs_eps(sim):
    """The per-value permittivity the engine's host averaged (eps = dt / cb away from walls and
    conductivity), for the CPU baseline's input: the same bits the oracle's averaging gives."""
    from photonoxide_b200 import configs
    from photonoxide_b200.fdtd import average
    return average(sim.grid, configs.mmi_geometry())


if __name__ == "__main__":
    sys.exit(main())
