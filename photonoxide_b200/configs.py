"""The workloads the engine is measured on, built through the reference's API.

- :func:`strip_2d`: a 2D TE run of a straight Si strip (n = 3.48, 0.5 um wide) in SiO2
  (n = 1.444), 400 x 200 cells of 20 nm, a 12-cell CPML, a Gaussian-pulse line source at 1550 nm
  (100 nm bandwidth), Courant 0.5, a transform of the whole plane at 21 wavelengths 1.5-1.6 um.
- :func:`mmi_3d`: a 1x2 MMI on SOI: a 220 nm Si core, 0.5 um access guides, a 3 x 8 um body,
  SiO2 cladding, in a 12 x 4 x 2 um domain of 20 nm cells (600 x 200 x 100 = 12 M), a 10-cell
  CPML, a Gaussian-profile current at 1550 nm in the input guide and a flux plane across each
  arm at 51 wavelengths 1.5-1.6 um.
- :func:`dispersive_3d`: 256 x 256 x 128 cells of 10 nm holding seeded random Drude-metal boxes
  and two-pole Lorentz boxes, CPML on every face and a broadband pulse over 1.2-2.0 um.

Geometries are the reference's job surface restated (rectangular Si/SiO2 boxes, constant
indices at the carrier, src/job/fdtd.rs:76-230); the builders are the reference's bench problems'
shape (src/bench/fdtd.rs:27-61). Every call takes ``cls``, the simulation class, so the same
problem is built on the engine and on a CPU restatement alike.
"""
from __future__ import annotations

import math

import numpy as np

from .types import (INF, Axis, Boundaries, Boxes, Cpml, Current, Dispersive, Field, FluxPlane,
                    Grid3d, Periodic, Pml, Pole, Source, Waveform)

N_SI = 3.48
N_SIO2 = 1.444
C_UM_PER_S = 299_792_458e6  # light's speed in um/s


def wavelengths(lo: float, hi: float, count: int):
    """``count`` frequencies (c/um) of wavelengths evenly spaced from lo to hi um."""
    return [1.0 / w for w in np.linspace(lo, hi, count)]


def pulse_1550(lo: float = 1.5, hi: float = 1.6) -> Waveform:
    """A Gaussian pulse centred on 1550 nm whose half-power bandwidth covers lo..hi um
    (``Waveform::pulse``, src/fdtd.rs:300-312): bandwidth 1/lo - 1/hi in c/um."""
    return Waveform.pulse(1.0 / 1.55, 1.0 / lo - 1.0 / hi)


def strip_2d(cls, precision: int = 32, **kw):
    """Configuration 1: returns (simulation, monitor numbers)."""
    h = 0.02
    g = Grid3d(400, 200, 1, h, h, h, -4.0, -2.0, -h / 2)
    eps = Boxes(N_SIO2 ** 2).add((-INF, -0.25, -INF), (INF, 0.25, INF), N_SI ** 2)
    s = cls(g, eps, Boundaries.cpml_2d(12), 0.5, precision=precision, **kw)
    # a line source (one value in the plane) on H_z at the strip's centre, 1 um in from the CPML
    i = 12 + int(round(1.0 / h))
    s.add_source(Source(Field.H, Axis.Z, (i, g.ny // 2, 0), pulse_1550()))
    probe = s.add_probe(Field.H, Axis.Z, (g.nx - 12 - 50, g.ny // 2, 0))
    dft = s.add_dft((0, 0, 0), (g.nx - 1, g.ny - 1, 0), wavelengths(1.5, 1.6, 21))
    return s, {"probe": probe, "dft": dft, "steps": 4000}


def mmi_geometry() -> Boxes:
    core = (-0.11, 0.11)
    geo = Boxes(N_SIO2 ** 2)
    geo.add((-INF, -0.25, core[0]), (-4.0, 0.25, core[1]), N_SI ** 2)      # input guide
    geo.add((-4.0, -1.5, core[0]), (4.0, 1.5, core[1]), N_SI ** 2)          # 3 x 8 um body
    for yc in (-0.75, 0.75):                                                 # the two arms
        geo.add((4.0, yc - 0.25, core[0]), (INF, yc + 0.25, core[1]), N_SI ** 2)
    return geo


def mmi_3d(cls, precision: int = 32, steps: int = 20000, frequencies: int = 51,
           edges: str = "cpml", **kw):
    """Configuration 2: returns (simulation, info). ``edges`` "walls" or "periodic" replaces the
    CPMLs, and "cpml-x", "cpml-y" or "cpml-z" keeps those of one axis only, walls elsewhere (for
    comparing the step's cost without them; not the configuration)."""
    h = 0.02
    g = Grid3d(600, 200, 100, h, h, h, -6.0, -2.0, -1.0)
    one = {f"cpml-{a}": Boundaries(*[Pml(10, 10) if a == b else Pml(0, 0) for b in "xyz"], Cpml())
           for a in "xyz"}
    b = {"cpml": Boundaries.with_cpml(10), "walls": Boundaries.walls(),
         "periodic": Boundaries(Periodic(), Periodic(), Periodic(), Cpml()), **one}[edges]
    # Courant 0.9: the reference job's default (src/job/fdtd.rs:523)
    s = cls(g, mmi_geometry(), b, 0.9, precision=precision, **kw)
    # a Gaussian-profile E_y current across the input guide, 0.5 um in from the CPML
    i = 10 + 25
    values = []
    for k in range(g.nz):
        z = g.z0 + k * h
        for j in range(g.ny):
            y = g.y0 + (j + 0.5) * h
            a = math.exp(-(y / 0.25) ** 2 - (z / 0.15) ** 2)
            if a > 1e-3:
                values.append((Axis.Y, (i, j, k), complex(a, 0.0)))
    s.add_current(Current(Field.E, values, pulse_1550()))
    # a flux plane across each arm, 0.6 um before the CPML: |y - yc| < 0.5 um, |z| < 0.4 um
    plane = g.nx - 10 - 30
    freqs = wavelengths(1.5, 1.6, frequencies)
    fluxes = []
    for yc in (-0.75, 0.75):
        jlo = int(round((yc - 0.5 - g.y0) / h))
        jhi = int(round((yc + 0.5 - g.y0) / h))
        klo = int(round((-0.4 - g.z0) / h))
        khi = int(round((0.4 - g.z0) / h))
        fluxes.append(s.add_flux(FluxPlane(Axis.X, plane).within((jlo, jhi), (klo, khi)), freqs))
    probe = s.add_probe(Field.E, Axis.Y, (plane, int(round((0.75 - g.y0) / h)), g.nz // 2))
    return s, {"fluxes": fluxes, "probe": probe, "steps": steps, "cells": g.cells()}


def dispersive_3d(cls, seed: int = 7, precision: int = 32, fill: float = 0.12, **kw):
    """Configuration 3: seeded random Drude boxes (omega_p = 1.37e16 rad/s, gamma = 1e14 1/s) and
    two-pole Lorentz boxes (delta eps in [0.5, 2], resonances over 1-3 um, eps_inf 2.25) in
    vacuum, CPML of 10 cells on every face. Returns (simulation, info)."""
    rng = np.random.default_rng(seed)
    h = 0.01
    g = Grid3d(256, 256, 128, h, h, h, -1.28, -1.28, -0.64)
    lo = np.array([g.x0, g.y0, g.z0]) + 12 * h
    hi = np.array([g.x0 + g.nx * h, g.y0 + g.ny * h, g.z0 + g.nz * h]) - 12 * h
    drude_boxes, lorentz_boxes = Boxes(0.0), Boxes(0.0)
    volume = float(np.prod(hi - lo))
    filled = 0.0
    while filled < fill * volume:
        size = rng.uniform(0.05, 0.3, 3) * (hi - lo)
        start = rng.uniform(lo, hi - size)
        target = drude_boxes if rng.random() < 0.5 else lorentz_boxes
        target.add(tuple(start), tuple(start + size), 1.0)
        filled += float(np.prod(size))
    plasma = 1.37e16 / (2 * math.pi) / C_UM_PER_S       # c/um
    damping = 1e14 / (2 * math.pi) / C_UM_PER_S
    drude = Dispersive(1.0, [Pole.drude(plasma, damping)])
    lorentz = Dispersive(2.25, [Pole.lorentz(float(rng.uniform(0.5, 2.0)), 1.0 / float(rng.uniform(1.0, 3.0)), 0.01),
                                Pole.lorentz(float(rng.uniform(0.5, 2.0)), 1.0 / float(rng.uniform(1.0, 3.0)), 0.01)])
    s = cls(g, Boxes(1.0), Boundaries.with_cpml(10), 0.5, precision=precision, **kw)
    s.with_medium(drude, drude_boxes)
    s.with_medium(lorentz, lorentz_boxes)
    s.add_source(Source(Field.E, Axis.Z, (g.nx // 2, g.ny // 2, g.nz // 2),
                        Waveform.pulse(1.0 / 1.6, 1.0 / 1.2 - 1.0 / 2.0)))
    probe = s.add_probe(Field.E, Axis.Z, (g.nx // 2 + 40, g.ny // 2, g.nz // 2))
    return s, {"probe": probe, "steps": 10000, "cells": g.cells()}


def mmi_bytes_per_step(cells: int, psi_values: int, precision: int = 32) -> int:
    """The algorithmic bytes of one step (the reference's GPU roof, docs/methods/fdtd.md:
    1410-1412, 1481-1482): E and H read and written, cb read (60 B/cell in f32, lossless), and
    each CPML psi read and written (8 B)."""
    r = precision // 8
    return 15 * r * cells + 2 * r * psi_values


def psi_values(grid: Grid3d, boundaries: Boundaries) -> int:
    """The CPMLs' psi values: per slab cell along an axis, two components of E and two of H."""
    total = 0
    for a in range(3):
        e = boundaries.edges(a)
        if hasattr(e, "low"):
            total += 4 * (e.low + e.high) * (grid.cells() // grid.n(a))
    return total


def te_design(nx: int, ny: int, precision: int = 32, steps: int = 6000, segment: int = 500,
              design_cells: int = 100, h: float = 0.02, bandwidth: float = 0.3, cls=None):
    """Configuration 4, one instance: a 2D TE grid of nx x ny cells of 20 nm, 12-cell CPMLs, an
    input Si strip (0.5 um) from the left CPML into a design region of design_cells^2 cells at
    the centre and an output strip from it to the right CPML, all in SiO2. A Gaussian-profile
    current on E_y across the input strip carries a pulse centred on 1550 nm (``bandwidth`` c/um
    wide, so that it has passed within the run); flux monitor 0 sits across the output strip
    (the arm) at 1550 nm. Returns the adjoint's TeProblem (design permittivities
    eps in [1.444^2, 3.48^2] are the variables); ``cls`` the simulation class its builder makes
    (the engine's by default)."""
    from .adjoint import Design2d, TeProblem
    from .fdtd import Simulation, average

    g = Grid3d(nx, ny, 1, h, h, h, -0.5 * nx * h, -0.5 * ny * h, -h / 2)
    half = 0.5 * design_cells * h
    boxes = (Boxes(N_SIO2 ** 2)
             .add((-INF, -0.25, -INF), (-half, 0.25, INF), N_SI ** 2)
             .add((half, -0.25, -INF), (INF, 0.25, INF), N_SI ** 2))
    background = average(g, boxes)
    d0x, d0y = nx // 2 - design_cells // 2, ny // 2 - design_cells // 2
    design = Design2d(d0x, d0y, design_cells, design_cells)
    src_x = 12 + 25
    mon_x = nx - 12 - 25
    jc = ny // 2
    span = int(round(1.0 / h))  # the monitor's window: 1 um either side of the strip

    def build(eps, prec):
        s = (cls or Simulation)(g, eps, Boundaries.cpml_2d(12), 0.5, precision=prec)
        values = []
        for j in range(jc - 25, jc + 26):
            y = (j + 0.5 - ny / 2) * h
            values.append((Axis.Y, (src_x, j, 0), complex(math.exp(-(y / 0.25) ** 2))))
        s.add_current(Current(Field.E, values, Waveform.pulse(1.0 / 1.55, bandwidth)))
        window = ((max(jc - span, 13), min(jc + span, ny - 14)), None)  # all of z
        s.add_flux(FluxPlane(Axis.X, mon_x, window), [1.0 / 1.55])
        return s

    return TeProblem(g, background, design, build, steps, precision=precision, segment=segment)


def te_design_sides(count: int = 64, seed: int = 0, lo: int = 256, hi: int = 1024):
    """The instances' sides (nx, ny), log-uniform in [lo, hi] cells, seeded."""
    rng = np.random.default_rng(seed)
    return [tuple(int(v) for v in np.exp(rng.uniform(np.log(lo), np.log(hi), 2)))
            for _ in range(count)]
