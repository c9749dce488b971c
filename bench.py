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
import tempfile
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
    """SM clocks and clock-event reasons sampled while the timed region runs: NVML polled every
    2 ms from a thread (the timed regions here can be a few milliseconds, shorter than
    nvidia-smi's sampling), else nvidia-smi every 200 ms. Read-only queries."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        self.thread = None
        self.samples = []  # (sm MHz, max MHz, set of reasons)
        try:
            self._start_nvml(gpu_index)
        except Exception:
            self.thread = None
            self._start_smi(gpu_index)

    def _start_nvml(self, gpu_index):
        import threading
        import pynvml as nv
        import torch
        nv.nvmlInit()
        try:
            p = torch.cuda.get_device_properties(gpu_index)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            handle = nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            handle = nv.nvmlDeviceGetHandleByIndex(gpu_index)
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        mx = float(nv.nvmlDeviceGetMaxClockInfo(handle, nv.NVML_CLOCK_SM))
        self.stop_flag = threading.Event()

        def poll():
            while not self.stop_flag.is_set():
                try:
                    sm = float(nv.nvmlDeviceGetClockInfo(handle, nv.NVML_CLOCK_SM))
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(handle)
                    self.samples.append((sm, mx, {k for k, b in bits.items() if r & b}))
                except Exception:
                    pass
                self.stop_flag.wait(0.002)
        self.thread = threading.Thread(target=poll, daemon=True)
        self.thread.start()

    def _start_smi(self, gpu_index):
        # the samples' file: PHOTONOXIDE_CLOCKS_DIR, else the system's temporary directory
        where = os.environ.get("PHOTONOXIDE_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(where, f"clocks_{os.getpid()}.csv")
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}",
                                          f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def _read_smi(self):
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm, mx = float(parts[1]), float(parts[2])
                except ValueError:
                    continue
                self.samples.append((sm, mx, {n for n, v in zip(self.NAMES, parts[5:9])
                                              if v.lower().startswith("active")}))

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            source = "nvml, every 2 ms"
        elif self.proc is not None:
            self._read_smi()
            source = "nvidia-smi, every 200 ms"
        else:
            return None
        if not self.samples:
            return None
        reasons = set().union(*(r for _, _, r in self.samples))
        return {"sm_mhz": float(np.median([s for s, _, _ in self.samples])),
                "sm_max_mhz": max(m for _, m, _ in self.samples), "reasons": sorted(reasons),
                "samples": len(self.samples), "source": source}


def aggregate(ms, steps, cells, dist=None, device="cpu"):
    """The slowest rank's time of a timed region (every rank steps its own replica of the grid,
    so the job ends when the last one does) and the whole job's rate in Gcell-updates/s."""
    world = 1
    if dist is not None and dist.is_initialized():
        import torch
        world = dist.get_world_size()
        t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, world * steps * cells / (ms / 1e3) / 1e9


WORKLOAD = ("3D MMI 600x200x100 (20 nm), CPML 10, Gaussian-profile current, 2 flux planes x 51 "
            "wavelengths, f32 fields, f64 transforms")


def config_of(cells: int, world: int) -> dict:
    """The workload's description, the same on both arms."""
    return {"workload": WORKLOAD, "cells": cells, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (fields+coefficients 432 MB)"}


def _oracle_rate(eps, precision, target_seconds):
    """The oracle's Gcell-updates/s on the MMI at `precision`, over about target_seconds of
    steps (at most 200), and the steps and seconds it took."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import OracleSimulation
    from photonoxide_b200 import configs

    def make(g, _geo, b, courant, precision=precision):
        return OracleSimulation(g, eps, b, courant, precision=precision)

    s, info = configs.mmi_3d(make)
    t0 = time.perf_counter()
    s.run(1)
    one = time.perf_counter() - t0
    n = max(1, min(200, int(target_seconds / max(one, 1e-3))))
    t0 = time.perf_counter()
    s.run(n)
    dt = time.perf_counter() - t0
    return n * info["cells"] / dt / 1e9, n, dt


def cpu_baseline(eps, target_seconds=12.0):
    """The oracle (photonoxide's CPU kernel restated, all host threads) on the same MMI problem,
    timed over a bounded number of steps: f64 (the reference's default arithmetic, the value) and
    f32 (its Yee<f32> kernel, the like-for-like arithmetic), with the host's STREAM triad."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import triad
    v64, n64, s64 = _oracle_rate(eps, 64, target_seconds)
    v32, n32, s32 = _oracle_rate(eps, 32, target_seconds)
    bw = triad()
    cores = os.cpu_count() or 1
    return {"value": v64, "unit": UNIT, "cores": cores, "kind": "port",
            "f32": {"value": v32, "unit": UNIT, "steps": n32, "seconds": s32},
            "triad_gbs": bw,
            "sample": f"{n64} steps (f64, {s64:.1f} s) and {n32} steps (f32, {s32:.1f} s) of the "
                      f"full 600x200x100 MMI grid, OpenMP on {cores} threads; STREAM triad "
                      f"{bw:.0f} GB/s on the same threads"}


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
    s.run(args.warmup)
    one = (time.perf_counter() - t0) / args.warmup
    steps = max(1, min(args.steps, int(90.0 / max(one, 1e-3))))
    t0 = time.perf_counter()
    s.run(steps)
    dt = time.perf_counter() - t0
    value = steps * info["cells"] / dt / 1e9
    cores = os.cpu_count() or 1
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": dt / steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": config_of(info["cells"], int(os.environ.get("WORLD_SIZE", "1"))),
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
    ap.add_argument("--edges", default="cpml",
                    choices=["cpml", "walls", "periodic", "cpml-x", "cpml-y", "cpml-z"],
                    help="the MMI grid's edges: cpml (the configuration) or, to compare the "
                         "step's cost without CPMLs, walls or periodic sides, or the CPMLs of "
                         "one axis only (walls elsewhere)")
    ap.add_argument("--batch-steps", type=int, default=6000,
                    help="the batch workload's steps (6000: the configuration; fewer for a "
                         "profiler's small case)")
    ap.add_argument("--workload", default="mmi", choices=sorted(["mmi"] + list(WORKLOADS)),
                    help="mmi: the 3D MMI step (this benchmark's line); the others measure the "
                         "remaining configurations, one JSON line each")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload != "mmi":
        return WORKLOADS[args.workload](args)

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

    sim, info = configs.mmi_3d(Simulation, edges=args.edges)
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
    ms, value = aggregate(ms, args.steps, cells, dist if world > 1 else None, "cuda")

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
    # each call returns once its copies are done (the run once its steps are): the wall time
    # between returns is the phase's
    phases, marks = {}, [time.perf_counter()]
    e0.record(stream)
    for name, call in (("upload_coeffs", lambda: eng.upload_coeffs(None, cb)),
                       ("upload_fields", lambda: eng.upload_fields(e_host, h_host)),
                       ("steps", lambda: (eng.run_async(args.steps, 0), eng.synchronize())),
                       ("download_fields", lambda: eng.download_fields(e_host, h_host)),
                       ("read_dft", lambda: eng.read_dft(sums))):
        call()
        marks.append(time.perf_counter())
        phases[name] = marks[-1] - marks[-2]
    e1.record(stream)
    eng.synchronize()
    wall = time.perf_counter() - marks[0]
    e2e_ms = max(e0.elapsed_time(e1), 0.0)
    e2e_ms, e2e_value = aggregate(e2e_ms, args.steps, cells, dist if world > 1 else None, "cuda")
    h2d = (3 * N + 6 * N) * 8 / args.steps
    d2h = (6 * N * 8 + 16 * nsums) / args.steps

    peak, peak_kind = peaks()
    per_launch_s = kernel_ms / max(kernel_n, 1) / 1e3
    achieved = bytes_step / per_launch_s / 1e9
    traffic = ncu_traffic()
    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            base = cpu_baseline(np.asarray(configs_eps(sim)))
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
        "config": config_of(cells, world),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "bytes_per_launch": bytes_step,
                     "kernel_ms_per_launch": per_launch_s * 1e3},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "wall_s": wall,
                "phases_s": phases},
        "gpu_launches": launches,
        "clocks": clk,
        "cpu_baseline": base,
    }
    print(json.dumps(line), flush=True)
    return 0


# -- the other configurations -----------------------------------------------------------------
# Each prints one JSON line. Timings of whole runs through the Python API are wall-clock around
# a synchronized run (host work included); the kernel-level figures come from CUDA events.

def _rel_l2(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    n = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a))


def _timed(fn):
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = fn()
    torch.cuda.synchronize()
    return out, time.perf_counter() - t0


def workload_strip2d(args):
    """Configuration 1: the 2D TE strip, 4000 steps, f32 on the GPU against f64 (the engine's
    f64, which is the oracle's bits): relative L2 of the probe's time series and of |DFT| over the
    plane at 21 wavelengths."""
    from photonoxide_b200 import configs
    from photonoxide_b200.fdtd import Simulation
    s32, info = configs.strip_2d(Simulation, 32)
    s64, _ = configs.strip_2d(Simulation, 64)
    steps = info["steps"]
    s32.run(args.warmup)
    _, dt = _timed(lambda: s32.run(steps - args.warmup))
    s64.run(steps)
    cells = s32.grid.cells()
    line = {"metric": "FDTD Gcell-updates/s (2D TE strip 400x200, 21-wavelength plane DFT)",
            "value": (steps - args.warmup) * cells / dt / 1e9, "unit": UNIT, "n_gpus": 1,
            "steps": steps - args.warmup, "warmup": args.warmup, "dtype": "f32",
            "higher_is_better": True, "data": "synthetic",
            "config": {"workload": "2D TE Si strip 0.5 um in SiO2, 400x200 at 20 nm, CPML 12, "
                                   "H_z line source, 4000 steps, DFT of the whole plane at 21 "
                                   "wavelengths", "cells": cells, "l2": "L2-resident"},
            "parity_vs_f64": {"probe_rel_l2": _rel_l2(s32.probe(info["probe"]), s64.probe(info["probe"])),
                              "dft_abs_rel_l2": _rel_l2(np.abs(s32.transforms()),
                                                        np.abs(s64.transforms())),
                              "tolerance": 1e-4}}
    print(json.dumps(line), flush=True)
    return 0


def workload_mmi_parity(args):
    """Configuration 2 at full size: 20000 steps of the MMI in f32 and in f64 (the engine's f64,
    the oracle's bits): the arms' flux spectra (|dT| relative to the largest flux) and the probe's
    time series (relative L2)."""
    from photonoxide_b200 import configs
    from photonoxide_b200.fdtd import Simulation
    s32, info = configs.mmi_3d(Simulation, 32)
    s64, _ = configs.mmi_3d(Simulation, 64)
    steps = int(os.environ.get("PHOTONOXIDE_MMI_STEPS", info["steps"]))
    _, t32 = _timed(lambda: s32.run(steps))
    _, t64 = _timed(lambda: s64.run(steps))
    f32 = np.array([s32.flux(n) for n in info["fluxes"]])
    f64 = np.array([s64.flux(n) for n in info["fluxes"]])
    scale = float(np.max(np.abs(f64)))
    line = {"metric": "MMI f32 vs f64 over a full run", "steps": steps, "dtype": "f32",
            "value": float(np.max(np.abs(f32 - f64)) / scale), "unit": "max |dT| / max T",
            "higher_is_better": False, "data": "synthetic",
            "probe_rel_l2": _rel_l2(s32.probe(info["probe"]), s64.probe(info["probe"])),
            "seconds": {"f32": t32, "f64": t64}, "tolerance": 1e-4,
            "config": {"workload": "3D MMI 600x200x100, CPML 10, 2 arm flux planes x 51 "
                                   "wavelengths", "cells": info["cells"]}}
    print(json.dumps(line), flush=True)
    return 0


def workload_dispersive(args):
    """Configuration 3: 256x256x128 with Drude and two-pole Lorentz boxes, the ADE fused into the
    E update; kernel time by CUDA events, algorithmic bytes 60 B/cell + 8 B/psi value + 8 B per
    dispersive value + 16 B per pole of it."""
    import ctypes as C
    import torch
    from photonoxide_b200 import configs
    from photonoxide_b200.engine import Engine
    from photonoxide_b200.fdtd import Simulation, library
    from photonoxide_b200.types import Boundaries
    s, info = configs.dispersive_3d(Simulation, 7, 32)
    steps = args.steps
    s.run(args.warmup)
    eng = Engine(s.engine())
    stream = torch.cuda.ExternalStream(eng.stream())
    clocks = Clocks(0)
    torch.cuda.synchronize()
    eng.profile(True)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    eng.run_async(steps, s.steps)
    b.record(stream)
    eng.synchronize()
    clk = clocks.stop()
    ms = a.elapsed_time(b)
    kms, kn = eng.profile_read()
    eng.profile(False)
    counts = (C.c_int64 * 2)()
    library().pxs_media_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    library().pxs_media_counts(s._h, counts)
    psi = configs.psi_values(s.grid, Boundaries.with_cpml(10))
    bytes_step = 60 * info["cells"] + 8 * psi + 8 * counts[0] + 16 * counts[1]
    peak, kind = peaks()
    achieved = bytes_step / (kms / max(kn, 1) / 1e3) / 1e9
    line = {"metric": "FDTD Gcell-updates/s (3D dispersive 256x256x128)",
            "value": steps * info["cells"] / (ms / 1e3) / 1e9, "unit": UNIT, "n_gpus": 1,
            "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps, "dtype": "f32",
            "higher_is_better": True, "data": "synthetic",
            "config": {"workload": "256x256x128 at 10 nm, Drude (wp 1.37e16 rad/s, gamma 1e14/s) "
                                   "and 2-pole Lorentz boxes, 12% fill, CPML 10",
                       "cells": info["cells"], "dispersive_values": counts[0],
                       "poles": counts[1], "l2": "inputs larger than L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": kind,
                         "bytes_per_launch": bytes_step,
                         "kernel_ms_per_launch": kms / max(kn, 1)},
            "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def _te_instances(count, seed=0, precision=32):
    from photonoxide_b200 import configs
    rng = np.random.default_rng(seed + 1)
    sims = []
    for (nx, ny) in configs.te_design_sides(count, seed):
        p = configs.te_design(nx, ny, precision=precision)
        eps = configs.N_SIO2 ** 2 + rng.uniform(0, 1, (100, 100)) * (configs.N_SI ** 2 - configs.N_SIO2 ** 2)
        sims.append(p.simulation(eps))
    return sims


def workload_batch(args):
    """Configuration 4, forward: 64 uneven 2D TE instances (sides log-uniform 256-1024 cells) with
    100x100 design regions, 6000 steps, batched (one persistent launch per step for all, CUDA-
    graph chunks, tile shape by timing) against the same instances run one at a time: through the
    3D engine (``one_at_a_time``) and as batches of one on the same TE kernel and tile shape
    (``one_at_a_time_te_kernel``, which isolates the batching's own gain)."""
    from photonoxide_b200.batch import Batch
    steps = args.batch_steps
    sims = _te_instances(64)
    cells = sum(s.grid.cells() for s in sims)
    B = Batch(sims)
    B.run(480)  # the tile shape's trial chunks
    _, tb = _timed(lambda: B.run(steps))
    alone = _te_instances(64)
    for s in alone:
        s.run(3)
    _, ta = _timed(lambda: [s.run(steps) for s in alone])
    # one at a time on the same TE kernel: each instance a batch of one, the batch's tile shape
    ones = [Batch([s], tile=B.tile) for s in _te_instances(64)]
    for one in ones:
        one.run(3)
    _, t1 = _timed(lambda: [one.run(steps) for one in ones])
    line = {"metric": "batched 2D TE Gcell-updates/s vs one at a time (64 instances)",
            "value": steps * cells / tb / 1e9, "unit": UNIT, "n_gpus": 1, "steps": steps,
            "dtype": "f32", "higher_is_better": True, "data": "synthetic",
            "one_at_a_time": steps * cells / ta / 1e9,
            "speedup": ta / tb, "tile": list(B.tile),
            "one_at_a_time_te_kernel": steps * cells / t1 / 1e9,
            "speedup_vs_te_kernel_one_at_a_time": t1 / tb,
            "config": {"workload": "64 2D TE instances, sides log-uniform 256-1024 at 20 nm, "
                                   "100x100 random design, CPML 12, flux monitor at 1550 nm",
                       "cells": cells}}
    print(json.dumps(line), flush=True)
    return 0


def workload_adjoint(args):
    """Configuration 4, gradient: one instance's flux at 1550 nm through the arm, d/d(density) of
    its 100x100 design (Gaussian blur sigma 2 px, eps in [1.444^2, 3.48^2]) by the time-reversed
    adjoint (6000 steps, checkpoints every 500), against central differences on 16 seeded pixels
    (delta 1e-3) in f64; and the f32 gradient against the f64 one."""
    import torch
    from photonoxide_b200 import configs
    from photonoxide_b200.adjoint import central_differences, transmission
    nx, ny = configs.te_design_sides(64)[0]
    e0, e1 = configs.N_SIO2 ** 2, configs.N_SI ** 2
    rho = np.random.default_rng(11).uniform(0, 1, (100, 100))
    out = {}
    for prec in (32, 64):
        p = configs.te_design(nx, ny, precision=prec)
        r = torch.tensor(rho, requires_grad=True)
        t, tf = _timed(lambda: transmission(r, p, e0, e1))
        _, tbk = _timed(lambda: t[0].backward())
        out[prec] = (p, r.grad.numpy().copy(), tf, tbk, float(t[0].detach()))
    p64, g64 = out[64][0], out[64][1]

    def f(x):
        with torch.no_grad():
            return float(transmission(torch.tensor(x), p64, e0, e1)[0])
    pixels = np.random.default_rng(5).choice(rho.size, 16, replace=False)
    fd = central_differences(f, rho, pixels, 1e-3)
    ga = g64.reshape(-1)[pixels]
    line = {"metric": "adjoint gradient vs central differences (max relative error, 16 pixels)",
            "value": float(np.max(np.abs(ga - fd)) / np.max(np.abs(fd))), "unit": "relative",
            "higher_is_better": False, "dtype": "f64", "data": "synthetic", "steps": 6000,
            "rel_l2": _rel_l2(ga, fd), "tolerance": 1e-3,
            "f32_vs_f64_gradient_rel_l2": _rel_l2(out[32][1], g64),
            "seconds": {"f32_forward": out[32][2], "f32_backward": out[32][3],
                        "f64_forward": out[64][2], "f64_backward": out[64][3]},
            "flux": out[64][4],
            "config": {"workload": f"2D TE {nx}x{ny} at 20 nm, 100x100 design, 6000 steps, "
                                   "segments of 500", "cells": nx * ny}}
    print(json.dumps(line), flush=True)
    return 0


def workload_serving(args):
    """Configuration 5: a seeded Poisson stream of jobs (20/s; 70% 2D, 30% 3D; cells log-uniform
    1e5-5e7, or PHOTONOXIDE_SERVING_CELLS="lo,hi"; PHOTONOXIDE_SERVING_JOBS of them, 60 by default;
    steps 2000-20000; 1-4 Si boxes in SiO2; 1-51 DFT wavelengths) served
    by the resident loop (150 GB budget, continuous admission) against the same jobs run one at a
    time in arrival order, the 2D ones on the 3D engine (``one_at_a_time``) and as batches of one
    on the TE kernel the loop batches them on (``one_at_a_time_te_kernel``): p50/p99 latency and
    aggregate Gcell-updates/s. The offered load exceeds
    the GPU's capacity (a backlog builds), as at full scale. A job's results are its transforms
    (read back when it ends; its fields are not kept, in both arms). Each job's host set-up
    (permittivity averaging, tables) is made before the stream starts, for both arms: the
    comparison is of the device's work."""
    import torch
    from photonoxide_b200.serving import Server, job_stream, make_job
    count = int(os.environ.get("PHOTONOXIDE_SERVING_JOBS", "60"))
    lo, hi = (float(v) for v in os.environ.get("PHOTONOXIDE_SERVING_CELLS", "1e5,5e7").split(","))
    specs = job_stream(count, rate=20.0, seed=5, cells=(lo, hi), steps=(2000, 20000))
    work = sum(int(np.prod(sp.n)) * sp.steps for sp in specs)
    # one at a time, in arrival order: each job run and its results read back
    sims = [make_job(sp) for sp in specs]
    durations = []
    for sp, s in zip(specs, sims):
        def one():
            s.run(sp.steps)
            s.transforms()
        _, d = _timed(one)
        durations.append(d)
    t, lat1 = 0.0, []
    for sp, d in zip(specs, durations):
        t = max(t, sp.arrival) + d
        lat1.append(t - sp.arrival)
    span1 = t - specs[0].arrival
    # one at a time with each 2D job on the TE kernel the served loop batches them on (a batch
    # of one, on the loop's tiles): the baseline that leaves the loop's own gain
    from photonoxide_b200.batch import Batch
    sims = [make_job(sp) for sp in specs]
    durations = []
    for sp, s in zip(specs, sims):
        if sp.two_d:
            def one():
                Batch([s], tile=(124, 7) if s.grid.nx % 4 == 0 else (32, 16)).run(sp.steps)
                s.transforms()
        else:
            def one():
                s.run(sp.steps)
                s.transforms()
        _, d = _timed(one)
        durations.append(d)
    del sims
    t, lat2 = 0.0, []
    for sp, d in zip(specs, durations):
        t = max(t, sp.arrival) + d
        lat2.append(t - sp.arrival)
    span2 = t - specs[0].arrival
    # served: submitted at their arrival times
    sims = [make_job(sp) for sp in specs]
    torch.cuda.synchronize()
    with Server(hbm_budget=150e9, max_active=64, chunk=500) as server:
        start = time.perf_counter()
        jobs = []
        for sp, s in zip(specs, sims):
            delay = sp.arrival - (time.perf_counter() - start)
            if delay > 0:
                time.sleep(delay)
            jobs.append(server.submit(s, sp.steps, keep_fields=False))
        for j in jobs:
            j.wait()
        span = time.perf_counter() - start - specs[0].arrival
        loop = server.stats()
        lat = [j.latency() for j in jobs]
    line = {"metric": "served FDTD jobs: aggregate Gcell-updates/s and p99 latency",
            "value": work / span / 1e9, "unit": UNIT, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic", "jobs": count,
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "one_at_a_time": {"value": work / span1 / 1e9,
                              "latency_s": {"p50": float(np.percentile(lat1, 50)),
                                            "p99": float(np.percentile(lat1, 99))}},
            "speedup": span1 / span,
            "one_at_a_time_te_kernel": {"value": work / span2 / 1e9,
                                        "latency_s": {"p50": float(np.percentile(lat2, 50)),
                                                      "p99": float(np.percentile(lat2, 99))}},
            "speedup_vs_te_kernel_one_at_a_time": span2 / span,
            "loop_seconds": {k: loop[k] for k in ("launch_s", "host_s", "wait_s")},
            "config": {"workload": f"Poisson stream, 20 jobs/s, 70% 2D / 30% 3D, cells "
                                   f"log-uniform {lo:g}-{hi:g}, steps 2000-20000, 150 GB budget; "
                                   "host set-up before the stream", "cell_updates": work}}
    print(json.dumps(line), flush=True)
    return 0


WORKLOADS = {"strip2d": workload_strip2d, "mmi_parity": workload_mmi_parity,
             "dispersive": workload_dispersive, "batch": workload_batch,
             "adjoint": workload_adjoint, "serving": workload_serving}


def configs_eps(sim):
    """The per-value permittivity the engine's host averaged (eps = dt / cb away from walls and
    conductivity), for the CPU baseline's input: the same bits the oracle's averaging gives."""
    from photonoxide_b200 import configs
    from photonoxide_b200.fdtd import average
    return average(sim.grid, configs.mmi_geometry())


if __name__ == "__main__":
    sys.exit(main())
