"""Serving FDTD jobs: a resident loop on the GPU (include/photonoxide_sim.h, ``pxs_server_*``)
that admits simulations as memory and slots free up, steps the admitted ones together (2D TE
jobs in one batch, one launch per step for all of them; the others each on its own stream,
concurrently), and hands each back when its steps are done, its results read to the host and its
device memory freed. Jobs that arrive while others run join between chunks of steps: continuous
batching. Each job's results have the bits they have when it runs alone.

The reference runs one ``Simulation`` at a time; there is no counterpart.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from .fdtd import FDTD_E_INVALID, Simulation, library
from .types import (INF, Axis, Boundaries, Boxes, Field, FluxPlane, GpuError, Grid3d,
                    InvalidValue, Source, Waveform)

QUEUED, RUNNING, DONE, FAILED, CANCELLED = range(5)
_bound = False


def _lib():
    global _bound
    x = library()
    if not _bound:
        P, I32, I64 = C.c_void_p, C.c_int32, C.c_int64
        DP = C.POINTER(C.c_double)
        x.pxs_server_create.argtypes = [C.c_size_t, I32, I64, C.POINTER(P)]
        x.pxs_server_last_error.argtypes = [P]
        x.pxs_server_last_error.restype = C.c_char_p
        x.pxs_server_submit.argtypes = [P, P, I64, I32]
        x.pxs_server_submit.restype = I64
        x.pxs_server_poll.argtypes = [P, I64, DP]
        x.pxs_server_wait.argtypes = [P, I64]
        x.pxs_server_cancel.argtypes = [P, I64]
        x.pxs_server_stats.argtypes = [P, DP]
        x.pxs_server_destroy.argtypes = [P]
        _bound = True
    return x


class Job:
    """A submitted simulation. Its simulation belongs to the server until the job ends."""

    def __init__(self, server: "Server", id: int, sim: Simulation, steps: int):
        self.server, self.id, self.sim, self.steps = server, id, sim, steps

    def poll(self):
        """(state, (submitted, started, finished)) -- times on one steady clock, seconds."""
        t = (C.c_double * 3)()
        st = _lib().pxs_server_poll(self.server._h, self.id, t)
        return st, (t[0], t[1], t[2])

    def wait(self) -> int:
        st = _lib().pxs_server_wait(self.server._h, self.id)
        if st == FAILED:
            raise GpuError(_lib().pxs_server_last_error(self.server._h).decode())
        return st

    def cancel(self):
        _lib().pxs_server_cancel(self.server._h, self.id)

    def latency(self) -> float:
        """Seconds from submission to the results being on the host."""
        st, (a, _, c) = self.poll()
        return c - a if st >= DONE else math.nan


class Server:
    """The resident loop: ``hbm_budget`` bytes for the admitted jobs' device state (an upper
    estimate per job), at most ``max_active`` jobs on the device, ``chunk`` steps between
    admissions."""

    def __init__(self, hbm_budget: float = 150e9, max_active: int = 64, chunk: int = 500):
        h = C.c_void_p()
        code = _lib().pxs_server_create(int(hbm_budget), int(max_active), int(chunk), C.byref(h))
        self._h = h.value
        if code < 0:
            msg = _lib().pxs_server_last_error(self._h).decode()
            self.close()
            raise InvalidValue(msg)
        self.jobs: List[Job] = []

    def submit(self, sim: Simulation, steps: int, keep_fields: bool = True) -> Job:
        """Queues ``steps`` steps of ``sim``. With ``keep_fields`` off only its transforms,
        fluxes and probes come back when the job ends (its fields are dropped with the device
        memory, which saves reading them back)."""
        id = _lib().pxs_server_submit(self._h, sim._h, int(steps), 1 if keep_fields else 0)
        if id < 0:
            msg = _lib().pxs_server_last_error(self._h).decode()
            raise InvalidValue(msg) if id == FDTD_E_INVALID else GpuError(msg)
        job = Job(self, int(id), sim, int(steps))
        self.jobs.append(job)
        return job

    def stats(self) -> dict:
        out = (C.c_double * 6)()
        _lib().pxs_server_stats(self._h, out)
        return {"cell_updates": out[0], "chunks": int(out[1]), "bytes_admitted": out[2],
                "launch_s": out[3], "host_s": out[4], "wait_s": out[5]}

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            _lib().pxs_server_destroy(h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# -- the serving workload: a seeded Poisson stream of Si/SiO2 jobs -----------------------------

@dataclass(frozen=True)
class JobSpec:
    arrival: float      # seconds after the stream starts
    two_d: bool
    n: tuple            # cells along x, y, z
    steps: int
    boxes: tuple        # (x0, y0, x1, y1) in um, Si boxes in SiO2
    nfreq: int          # DFT wavelengths, 1.5..1.6 um


def job_stream(count: int, rate: float = 20.0, seed: int = 0, cells=(1e5, 5e7),
               steps=(2000, 20000), share_2d: float = 0.7) -> List[JobSpec]:
    """A seeded Poisson stream of ``count`` jobs at ``rate`` per second: 2D with probability
    share_2d (else 3D), cell counts log-uniform in ``cells``, steps uniform in ``steps``, 1-4 Si
    boxes in SiO2, 1-51 DFT wavelengths."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(count):
        t += rng.exponential(1.0 / rate)
        two_d = bool(rng.uniform() < share_2d)
        c = math.exp(rng.uniform(math.log(cells[0]), math.log(cells[1])))
        aspect = rng.uniform(0.5, 2.0)
        if two_d:
            nx = max(48, int(round(math.sqrt(c * aspect))))
            ny = max(48, int(round(c / nx)))
            n = (nx - nx % 4, ny, 1)
        else:
            nz = max(24, int(round((c / 8.0) ** (1 / 3))))
            nx = max(48, int(round(math.sqrt(c / nz * aspect))))
            ny = max(32, int(round(c / nz / nx)))
            n = (nx - nx % 4, ny, nz)
        k = int(rng.integers(1, 5))
        boxes = []
        for _ in range(k):
            x0, y0 = rng.uniform(-0.5, 0.3, 2)
            boxes.append((float(x0), float(y0), float(x0 + rng.uniform(0.1, 0.4)),
                          float(y0 + rng.uniform(0.1, 0.4))))
        out.append(JobSpec(t, two_d, n, int(rng.integers(steps[0], steps[1] + 1)), tuple(boxes),
                           int(rng.integers(1, 52))))
    return out


def make_job(spec: JobSpec, precision: int = 32) -> Simulation:
    """The simulation of one job: a grid of 20 nm cells centred on the origin, 10-cell CPMLs,
    the job's Si boxes (full height in z) in SiO2, a 1550 nm pulse from a point source (H_z in
    2D, E_y in 3D) near the low x side, a flux plane near the high x side at the job's
    wavelengths."""
    h = 0.02
    nx, ny, nz = spec.n
    g = Grid3d.centred((nx, ny, nz), h)
    eps = Boxes(1.444 ** 2)
    for (x0, y0, x1, y1) in spec.boxes:
        eps = eps.add((x0, y0, -INF), (x1, y1, INF), 3.48 ** 2)
    b = Boundaries.cpml_2d(10) if spec.two_d else Boundaries.with_cpml(10)
    s = Simulation(g, eps, b, 0.5, precision=precision)
    pulse = Waveform.pulse(1.0 / 1.55, 1.0 / 1.5 - 1.0 / 1.6)
    at = (16, ny // 2, nz // 2)
    s.add_source(Source(Field.H, Axis.Z, at, pulse) if spec.two_d
                 else Source(Field.E, Axis.Y, at, pulse))
    freqs = [1.0 / w for w in np.linspace(1.5, 1.6, spec.nfreq)]
    s.add_flux(FluxPlane(Axis.X, nx - 16), freqs)
    return s


def serve(specs: List[JobSpec], server: Server, precision: int = 32, realtime: bool = True):
    """Submits each job at its arrival time (``realtime``) or all at once, waits for all; returns
    the jobs. The simulations are made (on the host) as each job arrives."""
    start = time.perf_counter()
    jobs = []
    for sp in specs:
        if realtime:
            delay = sp.arrival - (time.perf_counter() - start)
            if delay > 0:
                time.sleep(delay)
        jobs.append(server.submit(make_job(sp, precision), sp.steps))
    for j in jobs:
        j.wait()
    return jobs
