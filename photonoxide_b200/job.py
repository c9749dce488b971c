"""FDTD job files: the subset of the reference's ``kind = "fdtd"`` task (src/job/fdtd.rs) that
runs on the engine, read from TOML or YAML and run with the job runner's own stop rule.

The subset is a 3D job on a ``[task.stack]`` table of fixed refractive indices, ``rect`` shapes,
``dipole`` sources and ``flux``, ``flux_box`` and ``field`` monitors. Each part is read as the
reference's ``Setup::new`` (src/job/fdtd.rs:414-712) reads it, with the same checks and the same
error messages where they apply:

- the window ``x_um``, ``y_um``, ``z_um`` (by default the task's layer with 1 um either side),
  ``step_nm``, ``courant`` (0.9), ``pml_cells`` (20) and ``boundaries`` (``cpml``, ``wall`` or
  ``periodic`` per axis): ``grid_of``, ``boundaries_of`` and ``time_step``
  (src/job/fdtd.rs:1726-1826);
- ``[task.stack]``: ``substrate``, ``cladding`` and ``[[task.stack.layer]]`` (``name``,
  ``thickness_um``, ``material``, ``background``), every medium a number, a fixed refractive index
  of at least 1 (``task_medium``, src/device/spec.rs:978-1027: "a benchmark's medium");
- ``[[task.rect]]`` (``layer``, ``center_um``, ``size_um``): a box of the layer's material, its
  edges included (``Bounds::contains``, src/geometry.rs:150-153);
- ``[task.spectrum]`` (``from_um``, ``to_um``, ``points``): the monitors' wavelengths, and the
  pulse that covers them, twice their reach from the carrier wide, at least 5 % of it;
- ``[[task.source]]`` of ``type = "dipole"`` (``position_um``, ``component``);
- ``[[task.monitor]]`` of ``type`` ``flux`` (``normal``, ``at_um``, windows along the plane's
  other axes), ``flux_box`` (``x_um``, ``y_um``, ``z_um``) and ``field`` (``wavelengths_um``, a
  DFT of the plane the view shows);
- ``[task.stop]``: ``until = "decay"`` (``fraction`` 1e-8, ``limit_um`` 2000) or ``"time"``
  (``time_um``), judged as the runner judges it (src/job/fdtd.rs:2700-2850): |E|^2 at each
  monitor's middle against its peak, every 10 carrier periods after the pulse, and a stop when
  the fields grow again (``Growth``, src/fdtd/monitors.rs:663-717).

The permittivity is the reference's 3D closure (src/job/fdtd.rs:1344-1425): the substrate below
z = 0, each layer's background or, inside one of its shapes, its material, the cladding above. It
becomes a box geometry whose boxes hold a point when lo < p < hi: a closed face at v is the open
face at the next double beyond v, which holds the same points, so the cell averages are the
reference's.

Refused with a message: 2D jobs (each slab's effective index is a mode solve:
src/job/fdtd.rs:1430-1480), named stacks and catalogue materials (their dispersion models),
circles, rings, paths, shapes, components and bodies, partial etches, mode, plane-wave and beam
sources, mode and resonance monitors (mode solves, harmonic inversion), Bloch wavenumbers. The
runner's record (frames, progress, events) is not written: :meth:`FdtdJob.run` returns the spectra.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field as dc_field
from typing import Dict, List, Optional, Tuple

import numpy as np

from .types import (INF, Axis, Boundaries, Boxes, Cpml, Dipole, Field, FluxPlane, Grid3d,
                    InvalidValue, Periodic, Pml, Waveform)

COMPONENTS = {"Ex": (Field.E, Axis.X), "Ey": (Field.E, Axis.Y), "Ez": (Field.E, Axis.Z),
              "Hx": (Field.H, Axis.X), "Hy": (Field.H, Axis.Y), "Hz": (Field.H, Axis.Z)}
AXIS_NAMES = ("x", "y", "z")
ALL3 = (Axis.X, Axis.Y, Axis.Z)
GROWTH = 1e3                 # src/fdtd/monitors.rs:665
MOST_CELLS = 2e7             # a job's grid, src/job/fdtd.rs:44
MOST_CELLS_PER_SIDE = 1e4    # src/job/check.rs:45
FEWEST_CELLS_PER_SIDE = 2.0  # src/job/check.rs:49

TASK_KEYS = {"kind", "stack", "core_nm", "bottom_oxide_um", "wavelength_um", "layer",
             "dimensions", "polarization", "x_um", "y_um", "z_um", "step_nm", "courant",
             "pml_cells", "boundaries", "spectrum", "rect", "circle", "ring", "path", "shape",
             "component", "body", "source", "monitor", "stop", "view", "export"}
ITEM_KEYS = {"type", "name", "normal", "at_um", "direction", "x_um", "y_um", "z_um",
             "position_um", "component", "polarization", "center_um", "waist_um", "focus_um",
             "angle_deg", "wavelengths_um"}
NOT_IN_SUBSET = {
    "circle": "circles", "ring": "rings", "path": "paths", "shape": "shapes",
    "component": "components", "body": "bodies in space", "export": "exports",
}


class JobError(InvalidValue):
    """A job the reference refuses (its ``task_error``), or one beyond the subset."""


def rust_round(x: float) -> float:
    """f64::round: half-way cases away from zero (Python's round() takes them to even)."""
    t = float(math.trunc(x))
    if abs(x - t) >= 0.5:
        t += math.copysign(1.0, x)
    return t


def _number(v, what: str) -> float:
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise JobError(f"{what} must be a number, got {v!r}")
    return float(v)


def _pair(v, what: str) -> Tuple[float, float]:
    if not isinstance(v, (list, tuple)) or len(v) != 2:
        raise JobError(f"{what} must be [low, high], got {v!r}")
    return _number(v[0], what), _number(v[1], what)


def check_window(name: str, w: Tuple[float, float]):
    """src/job/check.rs:21-30"""
    if not (math.isfinite(w[0]) and math.isfinite(w[1]) and w[1] > w[0]):
        raise JobError(f"{name} must go from a smaller to a larger number, got [{w[0]}, {w[1]}]")


def check_cells(name: str, w: Tuple[float, float], step_nm: float):
    """src/job/check.rs:51-90: at most 1e4 cells along a side, at least 2."""
    exact = (w[1] - w[0]) / (step_nm / 1000.0)
    if rust_round(exact) > MOST_CELLS_PER_SIDE:
        raise JobError(f"{name} at a step of {step_nm} nm is {rust_round(exact):.0f} cells, more "
                       f"than {MOST_CELLS_PER_SIDE:.0f}: take a larger step_nm or a smaller window")
    if exact < FEWEST_CELLS_PER_SIDE:
        raise JobError(f"{name} at a step of {step_nm} nm is fewer than "
                       f"{FEWEST_CELLS_PER_SIDE:.0f} cells: take a smaller step_nm")


def fixed_index(v, what: str) -> float:
    """A medium of ``[task.stack]`` as a number: a fixed refractive index of at least 1
    (src/device/spec.rs:985-1027). Its permittivity is n * n (``Model::Constant``)."""
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise JobError(f"{what}: this reader takes each medium as a fixed refractive index (a "
                       f"number); catalogue materials need their dispersion models, got {v!r}")
    n = float(v)
    if not (math.isfinite(n) and n >= 1.0):
        raise JobError(f"{what}: a fixed refractive index must be a number of at least 1, "
                       f"got {n}")
    return n


@dataclass
class Layer:
    name: str
    bottom: float
    top: float
    material: float  # refractive indices
    background: float


@dataclass
class Monitor:
    """A monitor as the run adds it: ``flux`` (one plane), ``flux_box`` (faces with their
    signs, outwards +) or ``field`` (a DFT of the plane of nodes ``k`` along z)."""

    kind: str
    name: Optional[str]
    faces: List[Tuple[FluxPlane, float]] = dc_field(default_factory=list)
    wavelengths_um: List[float] = dc_field(default_factory=list)
    k: int = 0


@dataclass
class FdtdJob:
    """A job read by :func:`load`: its grid, medium, sources, monitors and stop rule."""

    name: str
    grid: Grid3d
    boundaries: Boundaries
    geometry: Boxes
    courant: float
    wavelength_um: float
    wavelengths_um: List[float]
    carrier: float
    bandwidth: float
    dipoles: List[Dipole] = dc_field(default_factory=list)
    monitors: List[Monitor] = dc_field(default_factory=list)
    until: Tuple = ("decay", 1e-8, 2000.0)  # or ("time", time)

    def waveform(self) -> Waveform:
        """The run's pulse (src/job/fdtd.rs:1333-1341)."""
        return Waveform.pulse(self.carrier, self.bandwidth)

    def frequencies(self) -> List[float]:
        return [1.0 / w for w in self.wavelengths_um]

    def probe_points(self) -> List[Tuple[int, int, int]]:
        """Where the decay is judged: each flux plane's middle (each face's, for a box), or the
        window's middle without one (src/job/fdtd.rs:1527-1590)."""
        g = self.grid
        k_mid = g.nz // 2
        points = []
        for m in self.monitors:
            for face, _ in m.faces:
                p = [0, 0, 0]
                p[int(face.axis)] = face.plane
                for slot, t in enumerate(face.axis.others()):
                    w = face.window[slot]
                    p[int(t)] = ((w[0] + w[1]) // 2 if w is not None
                                 else (k_mid if t == Axis.Z else g.n(int(t)) // 2))
                points.append((p[0], p[1], min(p[2], g.nz - 1)))
        if not points:
            points.append((g.nx // 2, g.ny // 2, k_mid))
        return points

    def simulation(self, cls=None, precision: int = 32):
        """The job's simulation with its sources and monitors: (sim, each monitor's numbers),
        a flux box's one per face. ``cls``: the simulation class (the engine's
        :class:`~photonoxide_b200.fdtd.Simulation` by default; anything with its calls)."""
        if cls is None:
            from .fdtd import Simulation as cls
        s = cls(self.grid, self.geometry, self.boundaries, self.courant, precision=precision)
        for d in self.dipoles:
            s.add_dipole(d)
        freqs = self.frequencies()
        added = []
        g = self.grid
        for m in self.monitors:
            if m.kind == "field":
                added.append([s.add_dft((0, 0, m.k), (g.nx - 1, g.ny - 1, m.k),
                                        [1.0 / w for w in m.wavelengths_um])])
            else:
                added.append([s.add_flux(face, freqs) for face, _ in m.faces])
        return s, added

    def run(self, cls=None, precision: int = 32, spectrum=None) -> Dict:
        """Builds the job and steps it until its stop rule ends it, in runs of steps that end at
        each step the rule looks at. Returns ``steps``, ``time_um``, ``stopped`` ("decayed",
        "grew", "limit" or "time"), ``growth`` (the factor, when it grew), ``fluxes`` (each flux
        and flux-box monitor's raw flux by name), ``spectra`` (those per unit source spectrum,
        as the runner records them: src/job/fdtd.rs:2248-2420), ``incident`` (the pulse's
        |W|^2), ``transforms`` (every transform's sums) and ``simulation``.
        ``spectrum(waveform, field, dt, steps, freqs)``: the source spectrum (the engine's
        :func:`~photonoxide_b200.fdtd.waveform_spectrum` by default)."""
        s, added = self.simulation(cls, precision)
        points = self.probe_points()
        probes = [[s.add_probe(Field.E, c, p) for c in ALL3] for p in points]
        w = self.waveform()
        width, delay = w.params[1], w.params[2]
        pulse_end = delay + 6.0 * width
        check = 10.0 * (1.0 / self.carrier)
        limit = self.until[2] if self.until[0] == "decay" else self.until[1]
        dt = s.dt
        npts = len(points)
        peaks, block = [0.0] * npts, [0.0] * npts
        block_end = pulse_end + check
        growth = _Growth.after(pulse_end, check)
        stopped, grew = None, None
        seen = 0
        while stopped is None:
            # the steps to the next one the rule looks at: the next check's, or the limit's
            n = _first_step_at(min(block_end, limit), dt, s.steps)
            s.run(n - s.steps)
            series = [[np.asarray(s.probe(q), dtype=np.float64)[seen:] for q in pr]
                      for pr in probes]
            for m in range(n - seen):
                t = float(seen + m + 1) * dt
                for k in range(npts):
                    ex, ey, ez = (float(series[k][0][m]), float(series[k][1][m]),
                                  float(series[k][2][m]))
                    v = ex * ex + ey * ey + ez * ez
                    peaks[k] = max(peaks[k], v)
                    if t > pulse_end:
                        block[k] = max(block[k], v)
                if t >= block_end:
                    worst = 0.0
                    for p, b in zip(peaks, block):
                        worst = max(worst, b / p if p > 0.0 else 0.0)
                    decayed = (self.until[0] == "decay" and worst <= self.until[1]
                               and any(p > 0.0 for p in peaks))
                    level = 0.0
                    for b in block:
                        level = max(level, b)
                    factor = growth.check(level)
                    grew = grew if grew is not None else factor
                    block = [0.0] * npts
                    block_end += check
                    if decayed:
                        stopped = "decayed"
                    elif grew is not None:
                        stopped = "grew"
                if stopped is None and t >= limit:
                    stopped = "limit" if self.until[0] == "decay" else "time"
                if stopped is not None and m != n - seen - 1:
                    raise JobError("the stop rule's step fell inside a run of steps")
            seen = n
        if spectrum is None:
            from .fdtd import waveform_spectrum as spectrum
        freqs = self.frequencies()
        pulse = min(s.steps, int(math.ceil((delay + 6.0 * width) / dt)) + 1)
        W = np.asarray(spectrum(w, Field.H, dt, pulse, freqs))
        incident = W.real * W.real + W.imag * W.imag
        fluxes, spectra = {}, {}
        for m, ns in zip(self.monitors, added):
            if m.kind == "field":
                continue
            if m.kind == "flux":
                total = np.asarray(s.flux(ns[0]), dtype=np.float64)
            else:  # each face's flux with its sign, summed from zero in face order
                total = np.zeros(len(freqs))
                for (_, sign), q in zip(m.faces, ns):
                    total = total + sign * np.asarray(s.flux(q), dtype=np.float64)
            fluxes[m.name] = total
            safe = np.where(incident > 0.0, incident, 1.0)
            spectra[m.name] = np.where(incident > 0.0, total / safe, 0.0)
        return {"steps": s.steps, "time_um": float(s.steps) * dt, "stopped": stopped,
                "growth": grew, "fluxes": fluxes, "spectra": spectra, "incident": incident,
                "transforms": s.transforms(), "simulation": s}


def _first_step_at(target: float, dt: float, now: int) -> int:
    """The first step count n > now whose time n dt reaches target."""
    n = max(now + 1, int(math.ceil(target / dt)))
    while n - 1 > now and float(n - 1) * dt >= target:
        n -= 1
    while float(n) * dt < target:
        n += 1
    return n


class _Growth:
    """``Growth`` (src/fdtd/monitors.rs:663-717): the level rising at more checks in a row than
    the pulse lasts (4 at least), to GROWTH times where the rise began."""

    def __init__(self, needed: int):
        self.needed, self.start, self.last, self.rises = needed, 0.0, 0.0, 0

    @staticmethod
    def after(pulse_end: float, check: float) -> "_Growth":
        return _Growth(max(int(math.ceil(pulse_end / check)) + 1, 4))

    def check(self, level: float) -> Optional[float]:
        if self.last > 0.0 and level > self.last:
            if self.rises == 0:
                self.start = self.last
            self.rises += 1
        else:
            self.rises = 0
        self.last = level
        if self.rises >= self.needed and level >= GROWTH * self.start:
            return level / self.start
        return None


# -- reading -------------------------------------------------------------------------------------

def load(source, most_cells: float = MOST_CELLS) -> FdtdJob:
    """Reads a job: a path (``.toml``, ``.yaml``/``.yml`` or ``.json``), a job's text (TOML or
    YAML), or a dict (the whole job or its task). ``most_cells``: the largest grid taken, the
    reference's 2e7 by default (the engine takes far more on one GPU)."""
    if isinstance(source, dict):
        doc = source
    else:
        text, kind = str(source), None
        if "\n" not in text and os.path.exists(text):
            kind = os.path.splitext(text)[1].lower()
            with open(text, encoding="utf-8") as f:
                text = f.read()
        doc = _parse_text(text, kind)
    if not isinstance(doc, dict):
        raise JobError(f"a job is a table, got {type(doc).__name__}")
    if "task" in doc:
        for key in doc:
            if key not in ("name", "task", "timeout_minutes"):
                raise JobError(f"an fdtd job in this reader is its [task]: it doesn't take "
                               f"[{key}]" + (" (a device's structure)" if key == "device" else ""))
        task, name = doc["task"], str(doc.get("name", "fdtd"))
    else:
        task, name = doc, "fdtd"
    if not isinstance(task, dict) or task.get("kind") != "fdtd":
        kind = task.get("kind") if isinstance(task, dict) else task
        raise JobError(f"not an fdtd task: kind = {kind!r}")
    return _setup(task, name, most_cells)


def _parse_text(text: str, kind: Optional[str]):
    if kind == ".json":
        return json.loads(text)
    if kind in (".yaml", ".yml"):
        import yaml
        return yaml.safe_load(text)
    import tomllib
    try:
        return tomllib.loads(text)
    except tomllib.TOMLDecodeError:
        if kind == ".toml":
            raise
        import yaml
        return yaml.safe_load(text)


def _setup(task: dict, name: str, most_cells: float) -> FdtdJob:
    for key in task:
        if key not in TASK_KEYS:
            raise JobError(f"[task] doesn't take {key}")
        if key in NOT_IN_SUBSET and task[key]:
            raise JobError(f"{NOT_IN_SUBSET[key]} ([task] {key}) are beyond this reader's subset: "
                           "a 3D job of rects on a stack of fixed indices")
    x_um, y_um = _pair(task.get("x_um"), "x_um"), _pair(task.get("y_um"), "y_um")
    check_window("x_um", x_um)
    check_window("y_um", y_um)
    step_nm = _number(task.get("step_nm"), "step_nm")
    if not (math.isfinite(step_nm) and step_nm > 0.0):
        raise JobError(f"step_nm must be positive, got {step_nm}")
    check_cells("x_um", x_um, step_nm)
    check_cells("y_um", y_um, step_nm)
    dims = task.get("dimensions", 2)
    if dims not in (2, 3):
        raise JobError(f"dimensions must be 2 or 3, got {dims}")
    if dims == 2:
        raise JobError("a 2D job's plane takes each slab's effective index, a slab mode solve: "
                       "this reader takes 3D jobs (dimensions = 3)")
    if task.get("polarization") is not None:
        raise JobError("polarization is for a 2D job: a 3D job's sources and monitors each say "
                       "theirs")
    layers, substrate, cladding = _stack(task)
    by_name = {l.name: l for l in layers}
    own = task.get("layer")
    if own not in by_name:
        raise JobError(f"the stack has no layer {own}")
    bottom, top = by_name[own].bottom, by_name[own].top
    if "z_um" in task:
        z_um = _pair(task["z_um"], "z_um")
        check_window("z_um", z_um)
        check_cells("z_um", z_um, step_nm)
    else:
        z_um = (bottom - 1.0, top + 1.0)
    courant = _number(task.get("courant", 0.9), "courant")
    if not (courant > 0.0 and courant <= 1.0):
        raise JobError(f"courant must be in (0, 1], got {courant}")
    grid = grid_of(x_um, y_um, z_um, step_nm)
    if grid.cells() > most_cells:
        raise JobError(f"the grid is {grid.nx} x {grid.ny} x {grid.nz} = {grid.cells()} cells, "
                       f"more than {most_cells:e}: take a larger step_nm or a smaller window")
    pml = task.get("pml_cells", 20)
    if isinstance(pml, bool) or not isinstance(pml, int) or pml < 0:
        raise JobError(f"pml_cells must be a count of cells, got {pml!r}")
    boundaries = boundaries_of(task.get("boundaries") or {}, pml, grid)
    dt = time_step(grid, boundaries, courant)
    # the spectrum and the pulse that covers it (src/job/fdtd.rs:544-599)
    lam = _number(task.get("wavelength_um"), "wavelength_um")
    wavelengths = spectrum_of(task.get("spectrum"), lam)
    if not (math.isfinite(lam) and lam > 0.0):
        raise JobError(f"a wavelength must be positive and finite, got {lam} um")
    carrier = 1.0 / lam
    reach = 0.0
    for w in wavelengths:
        reach = max(reach, abs(1.0 / w - carrier))
    bandwidth = max(2.0 * reach, 0.05 * carrier)
    nyquist = 0.5 / dt
    for f in [1.0 / w for w in wavelengths] + [carrier + bandwidth]:
        if f >= 0.8 * nyquist:
            raise JobError(f"the pulse and the spectrum reach {f:.4f} c/um, too near the time "
                           f"step's Nyquist frequency {nyquist:.4f} c/um: take a smaller step_nm "
                           "or a narrower spectrum")
    until = stop_of(task.get("stop"))
    # the view's plane, which a field monitor transforms (src/job/fdtd.rs:618-636)
    view = task.get("view") or {}
    for key in view:
        if key not in ("field", "z_um", "every_um"):
            raise JobError(f"[task.view] doesn't take {key}")
    vz = _number(view.get("z_um", 0.5 * (bottom + top)), "the view's z_um")
    vk = math.floor((vz - grid.z0) / grid.dz) if math.isfinite(vz) else -1
    if not (math.isfinite(vz) and 0 <= vk < grid.nz):
        raise JobError(f"the view's z_um, {vz}, is outside the window's z, {z_um[0]} to "
                       f"{z_um[1]} um")
    geometry = permittivity(layers, substrate, cladding, task.get("rect") or [], by_name)
    job = FdtdJob(name, grid, boundaries, geometry, courant, lam, wavelengths, carrier,
                  bandwidth, until=until)
    sources = task.get("source") or []
    if not sources:
        raise JobError("an fdtd job needs at least one [[task.source]]")
    for k, spec in enumerate(sources):
        job.dipoles.append(_source(job, spec, k))
    for k, spec in enumerate(task.get("monitor") or []):
        job.monitors.append(_monitor(job, spec, k, vk))
    names = []
    for m in job.monitors:
        if m.name is not None:
            if m.name in names:
                raise JobError(f'two monitors are named "{m.name}": each needs its own name')
            names.append(m.name)
    return job


def _stack(task: dict):
    """``[task.stack]`` of fixed indices (src/device/spec.rs:928-976, LayerStack::new at
    src/stack.rs:78-102): its layers bottom up, each top the sum of the thicknesses below."""
    stack = task.get("stack")
    if stack is None:
        raise JobError('needs a stack, e.g. stack = "soi_220"')
    if isinstance(stack, str):
        raise JobError(f'stack "{stack}" is a named stack of catalogue materials (their '
                       "dispersion models): this reader takes a [task.stack] table of fixed "
                       "refractive indices")
    if not isinstance(stack, dict):
        raise JobError(f"[task.stack] must be a table, got {stack!r}")
    if task.get("core_nm") is not None or task.get("bottom_oxide_um") is not None:
        raise JobError("core_nm and bottom_oxide_um are a named stack's: a [task.stack] table "
                       "gives each layer's thickness")
    for key in stack:
        if key not in ("substrate", "cladding", "layer"):
            raise JobError(f"[task.stack] doesn't take {key}")
    for key in ("substrate", "cladding"):
        if key not in stack:
            raise JobError(f'[task.stack] needs a {key}, e.g. {key} = "sio2"')
    substrate = fixed_index(stack["substrate"], "[task.stack] substrate")
    cladding = fixed_index(stack["cladding"], "[task.stack] cladding")
    specs = stack.get("layer")
    if not isinstance(specs, list) or not specs:
        raise JobError("[task.stack] needs its layers, bottom to top: [[task.stack.layer]]")
    layers: List[Layer] = []
    z = 0.0
    for k, spec in enumerate(specs):
        at = f"[[task.stack.layer]] {k + 1}"
        if not isinstance(spec, dict):
            raise JobError(f"{at} must be a table")
        for key in spec:
            if key not in ("name", "thickness_um", "material", "background"):
                raise JobError(f"{at} doesn't take {key}")
        for key in ("name", "thickness_um", "material", "background"):
            if key not in spec:
                raise JobError(f"{at} needs a {key}")
        t = _number(spec["thickness_um"], f"{at} thickness_um")
        if not (math.isfinite(t) and t > 0.0):
            raise JobError(f"layer stack: layer {spec['name']} has thickness {t} um")
        if any(l.name == spec["name"] for l in layers):
            raise JobError(f"layer stack: two layers are named {spec['name']}")
        layers.append(Layer(str(spec["name"]), z, z + t,
                            fixed_index(spec["material"], f"{at} material"),
                            fixed_index(spec["background"], f"{at} background")))
        z = z + t
    if len(layers) > 16:
        raise JobError("an fdtd job's stack may have at most 16 layers")
    return layers, substrate, cladding


def grid_of(x_um, y_um, z_um, step_nm: float) -> Grid3d:
    """src/job/fdtd.rs:1726-1747 in 3D: cells of about step_nm filling the window."""
    h = step_nm / 1000.0
    cells = lambda w: int(max(rust_round((w[1] - w[0]) / h), 1.0))  # noqa: E731
    nx, ny, nz = cells(x_um), cells(y_um), cells(z_um)
    return Grid3d(nx, ny, nz, (x_um[1] - x_um[0]) / nx, (y_um[1] - y_um[0]) / ny,
                  (z_um[1] - z_um[0]) / nz, x_um[0], y_um[0], z_um[0])


def boundaries_of(spec: dict, pml: int, grid: Grid3d) -> Boundaries:
    """src/job/fdtd.rs:1749-1815 in 3D, without Bloch wavenumbers."""
    for key in spec:
        if key not in ("x", "y", "z", "bloch"):
            raise JobError(f"[task.boundaries] doesn't take {key}")
    bloch = spec.get("bloch", [0.0, 0.0, 0.0])
    if any(_number(k, "a Bloch wavenumber") != 0.0 for k in bloch):
        raise JobError("a Bloch wavenumber makes the fields complex: beyond this reader's subset")
    edges = []
    for a, name in enumerate(AXIS_NAMES):
        kind = spec.get(name, "cpml")
        if kind == "cpml":
            if 2 * pml + 4 > grid.n(a):
                raise JobError(f"CPMLs of {pml} cells at each end leave nothing of the "
                               f"{grid.n(a)} cells along {name}")
            edges.append(Pml(pml, pml))
        elif kind == "wall":
            edges.append(Pml(0, 0))
        elif kind == "periodic":
            edges.append(Periodic())
        else:
            raise JobError(f'unknown boundary "{kind}" along {name}: cpml, wall or periodic')
    return Boundaries(edges[0], edges[1], edges[2], Cpml())


def time_step(grid: Grid3d, b: Boundaries, courant: float) -> float:
    """src/job/fdtd.rs:1818-1826: C / sqrt(sum 1/d^2) over the axes the field varies along."""
    total = 0.0
    for a in range(3):
        if not (grid.n(a) == 1 and b.periodic(a)):
            total += 1.0 / (grid.step(a) * grid.step(a))
    return courant / math.sqrt(total)


def spectrum_of(sp, wavelength_um: float) -> List[float]:
    """src/job/fdtd.rs:544-572"""
    if sp is None:
        return [wavelength_um]
    for key in sp:
        if key not in ("from_um", "to_um", "points"):
            raise JobError(f"[task.spectrum] doesn't take {key}")
    lo, hi = _number(sp.get("from_um"), "from_um"), _number(sp.get("to_um"), "to_um")
    points = sp.get("points")
    if isinstance(points, bool) or not isinstance(points, int) or points < 0:
        raise JobError(f"the spectrum's points must be a count, got {points!r}")
    if points == 0 or not (math.isfinite(lo) and math.isfinite(hi)) or lo <= 0.0 or hi <= 0.0:
        raise JobError("the spectrum needs positive from_um and to_um and at least 1 point")
    if points > 1000:
        raise JobError(f"the spectrum's points must be at most 1000, got {points}")
    if points == 1:
        return [lo]
    return [lo + (hi - lo) * float(k) / float(points - 1) for k in range(points)]


def stop_of(stop) -> Tuple:
    """src/job/fdtd.rs:1679-1724"""
    stop = stop or {}
    for key in stop:
        if key not in ("until", "fraction", "time_um", "limit_um"):
            raise JobError(f"[task.stop] doesn't take {key}")

    def positive(what, v):
        v = _number(v, what)
        if not (math.isfinite(v) and v > 0.0):
            raise JobError(f"{what} must be positive, got {v}")
        return v

    until = stop.get("until", "decay")
    if until == "decay":
        if "time_um" in stop:
            raise JobError('time_um is for until = "time"; a run until the fields decay takes '
                           "fraction and limit_um")
        fraction = _number(stop.get("fraction", 1e-8), "fraction")
        if not (fraction > 0.0 and fraction < 1.0):
            raise JobError(f"fraction must be between 0 and 1, got {fraction}")
        return ("decay", fraction, positive("limit_um", stop.get("limit_um", 2000.0)))
    if until == "time":
        if "fraction" in stop or "limit_um" in stop:
            raise JobError('fraction and limit_um are for until = "decay"; a run for a time '
                           "takes time_um")
        if "time_um" not in stop:
            raise JobError('until = "time" needs time_um')
        return ("time", positive("time_um", stop["time_um"]))
    raise JobError(f'unknown until "{until}": decay or time')


def _below(v: float) -> float:
    return math.nextafter(v, -math.inf)


def _above(v: float) -> float:
    return math.nextafter(v, math.inf)


def permittivity(layers: List[Layer], substrate: float, cladding: float, rects,
                 by_name: Dict[str, Layer]) -> Boxes:
    """The reference's 3D permittivity (src/job/fdtd.rs:1396-1425) as open boxes: the cladding
    everywhere; the substrate where z < 0; layer i's background where bottom_i <= z < top_i;
    each rect of layer i, |x - cx| <= w/2 and |y - cy| <= h/2 edges included, over it. A face
    that holds its points (<=) is the open face at the next double out, which holds the same."""
    geo = Boxes(cladding * cladding)
    geo.add((-INF, -INF, -INF), (INF, INF, 0.0), substrate * substrate)
    for l in layers:
        geo.add((-INF, -INF, _below(l.bottom)), (INF, INF, l.top), l.background * l.background)
    for k, r in enumerate(rects):
        at = f"[[task.rect]] #{k + 1}"
        if not isinstance(r, dict):
            raise JobError(f"{at} must be a table")
        for key in r:
            if key not in ("layer", "center_um", "size_um", "etch"):
                raise JobError(f"{at} doesn't take {key}")
        if r.get("etch") is not None:
            raise JobError(f"{at}: an etched shape (a partial etch, sloped walls) is beyond this "
                           "reader's subset")
        if r.get("layer") not in by_name:
            raise JobError(f"{at}: the stack has no layer {r.get('layer')}")
        cx, cy = _pair(r.get("center_um"), f"{at} center_um")
        w, h = _pair(r.get("size_um"), f"{at} size_um")
        if not (math.isfinite(cx) and math.isfinite(cy)) or not all(
                math.isfinite(v) and v > 0.0 for v in (w, h)):
            raise JobError(f"rectangle: needs a finite centre and a positive size, got {w} x {h}")
        l = by_name[r["layer"]]
        geo.add((_below(cx - w / 2.0), _below(cy - h / 2.0), _below(l.bottom)),
                (_above(cx + w / 2.0), _above(cy + h / 2.0), l.top), l.material * l.material)
    return geo


def _only(spec: dict, what: str, allowed) -> None:
    """ItemSpec::only (src/job/fdtd.rs:141-152): refuses the fields a type doesn't read."""
    for key in spec:
        if key not in ITEM_KEYS:
            raise JobError(f"{what}: unknown field {key}")
    for key in sorted(k for k in spec if k != "type"):
        if key not in allowed:
            raise JobError(f"{what}: a {spec['type']} doesn't take {key} (it takes "
                           f"{', '.join(allowed)})")


def _source(job: FdtdJob, spec: dict, k: int) -> Dipole:
    """A dipole source (src/job/fdtd.rs:922-945): amplitude 1, the run's pulse."""
    kind = spec.get("type")
    what = f"source {k + 1} ({kind})"
    if kind in ("mode", "plane_wave", "beam"):
        raise JobError(f"{what}: a {kind} source is beyond this reader's subset (a mode solve or "
                       "a total-field box): it takes dipoles")
    if kind != "dipole":
        raise JobError(f'source {k + 1}: unknown type "{kind}": mode, dipole, plane_wave or beam')
    _only(spec, what, ["position_um", "component"])
    p = spec.get("position_um")
    if p is None:
        raise JobError(f"{what}: needs position_um")
    if not isinstance(p, (list, tuple)) or len(p) != 3:
        raise JobError(f"{what}: position_um must be [x, y], z")
    p = [_number(v, f"{what} position_um") for v in p]
    g = job.grid
    for a, v in enumerate(p):
        lo = g.origin(a)
        hi = lo + float(g.n(a)) * g.step(a)
        if not (math.isfinite(v) and lo <= v <= hi):
            raise JobError(f"{what}: its {AXIS_NAMES[a]} = {v} um is outside the window")
    name = spec.get("component")
    if name is None:
        raise JobError(f'{what}: needs a component, e.g. "Ez"')
    if name not in COMPONENTS:
        raise JobError(f'{what}: unknown component "{name}": Ex, Ey, Ez, Hx, Hy or Hz')
    field, comp = COMPONENTS[name]
    return Dipole(field, comp, tuple(p), 1.0 + 0.0j, job.waveform())


def _half_plane(job: FdtdJob, axis: int, v: float, what: str) -> int:
    """Setup::half_plane (src/job/fdtd.rs:1304-1322): the node before the half-plane nearest v,
    inside the grid and clear of the CPMLs."""
    g = job.grid
    e = job.boundaries.edges(axis)
    low, high = (e.low, e.high) if isinstance(e, Pml) else (0, 0)
    n = g.n(axis)
    ok = math.isfinite(v)
    m = rust_round((v - g.origin(axis)) / g.step(axis) - 0.5) if ok else 0.0
    if not (ok and m >= low and m + 1.0 + high <= n and m + 1.0 < n):
        raise JobError(f"{what}: {AXIS_NAMES[axis]} = {v} um is outside the window or inside "
                       f"its CPMLs ({low} and {high} cells)")
    return int(m)


def _window(job: FdtdJob, spec: dict, key: str, axis: int, what: str) -> Tuple[int, int]:
    w = _pair(spec[key], f"{what}'s {key}")
    check_window(f"{what}'s {key}", w)
    lo, hi = _half_plane(job, axis, w[0], what), _half_plane(job, axis, w[1], what)
    if hi <= lo:
        raise JobError(f"{what}: its {key} covers less than a cell")
    return lo, hi


def _monitor(job: FdtdJob, spec: dict, k: int, view_k: int) -> Monitor:
    """A flux, flux-box or field monitor (src/job/fdtd.rs:1113-1265)."""
    kind = spec.get("type")
    what = f"monitor {k + 1} ({kind})"
    name = spec.get("name", f"{str(kind).replace('_', ' ')} {k + 1}")
    if kind in ("mode", "resonance"):
        raise JobError(f"{what}: a {kind} monitor is beyond this reader's subset (a mode solve or "
                       "harmonic inversion): it takes flux, flux_box and field")
    if kind == "flux":
        _only(spec, what, ["name", "normal", "at_um", "x_um", "y_um", "z_um"])
        normal = spec.get("normal")
        if normal is None:
            raise JobError(f'{what}: needs a normal, "x" or "y"')
        if normal not in AXIS_NAMES:
            raise JobError(f'{what}: unknown normal "{normal}": x or y or z')
        axis = Axis(AXIS_NAMES.index(normal))
        if "at_um" not in spec:
            raise JobError(f"{what}: needs at_um, its plane")
        plane = _half_plane(job, int(axis), _number(spec["at_um"], f"{what} at_um"), what)
        if f"{normal}_um" in spec:
            raise JobError(f"{what}: give at_um, and windows along the plane's other axes")
        window = [None, None]
        for slot, t in enumerate(axis.others()):
            key = f"{AXIS_NAMES[int(t)]}_um"
            if key in spec:
                window[slot] = _window(job, spec, key, int(t), what)
        return Monitor("flux", name, [(FluxPlane(axis, plane, tuple(window)), 1.0)])
    if kind == "flux_box":
        _only(spec, what, ["name", "x_um", "y_um", "z_um"])
        planes = []
        for a, key in enumerate(("x_um", "y_um", "z_um")):
            if key not in spec:
                raise JobError(f"{what}: needs its box's {key}")
            planes.append(_window(job, spec, key, a, what))
        faces = []
        for axis in ALL3:
            lo, hi = planes[int(axis)]
            b, c = axis.others()
            for node, sign in ((lo, -1.0), (hi, 1.0)):
                faces.append((FluxPlane(axis, node, (planes[int(b)], planes[int(c)])), sign))
        return Monitor("flux_box", name, faces)
    if kind == "field":
        _only(spec, what, ["name", "wavelengths_um"])
        wl = spec.get("wavelengths_um")
        wl = [job.wavelength_um] if wl is None else [_number(v, f"{what} wavelengths_um")
                                                     for v in wl]
        if not wl or len(wl) > 20:
            raise JobError(f"{what}: wavelengths_um must hold 1 to 20 wavelengths")
        lowest = 1.0 / max(job.wavelengths_um)
        highest = 1.0 / min(job.wavelengths_um)
        lo = min(lowest, job.carrier - job.bandwidth)
        hi = max(highest, job.carrier + job.bandwidth)
        for w in wl:
            if not (math.isfinite(w) and w > 0.0):
                raise JobError(f"a wavelength must be positive and finite, got {w} um")
            if not (lo <= 1.0 / w <= hi):
                raise JobError(f"{what}: {w} um is outside the pulse's band, {1.0 / hi:.4f} to "
                               f"{1.0 / lo:.4f} um")
        return Monitor("field", None, [], wl, view_k)
    raise JobError(f'monitor {k + 1}: unknown type "{kind}": mode, flux, flux_box, field or '
                   "resonance")
