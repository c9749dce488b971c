"""The plain types of photonoxide's FDTD API, as Python values.

Each mirrors the Rust type of the same name in the reference crate, so that a problem is
described here as it is there: the grid (``src/fdfd/three.rs:70-157``), the boundaries and the
CPML's parameters (``src/fdtd.rs:83-256``), waveforms and point sources (``src/fdtd.rs:259-456``),
currents and dipoles (``src/fdtd/sources.rs:46-70``), flux planes (``src/fdtd/monitors.rs:212-263``)
and dispersive media (``src/fdtd/media.rs:55-130``).

A closure ``eps(x, y, z)`` is how the reference takes a permittivity; a Python callable sampled
8^3 times per value of E would take hours on a 12 M-cell grid, so a geometry is given here as
:class:`Boxes` (a background and boxes over it, later ones on top), or as an array of the
per-value permittivity already averaged.
"""
from __future__ import annotations

import enum
import math
from dataclasses import dataclass, field as dc_field
from typing import List, Optional, Sequence, Tuple

import numpy as np

TAU = 2.0 * math.pi


class Axis(enum.IntEnum):
    """An axis of the grid and a field's component along it (``src/fdfd/three.rs:33-58``)."""

    X = 0
    Y = 1
    Z = 2

    def others(self) -> Tuple["Axis", "Axis"]:
        """The next two axes in cyclic order: (y, z) for x, (z, x) for y, (x, y) for z."""
        return Axis((self + 1) % 3), Axis((self + 2) % 3)


ALL_AXES = (Axis.X, Axis.Y, Axis.Z)


class Field(enum.IntEnum):
    """Which field a source drives or a probe records (``src/fdtd.rs:437-443``)."""

    E = 0
    H = 1


class InvalidValue(ValueError):
    """A value the API refuses: the reference's ``Error::InvalidValue`` (``src/error.rs:15-22``)."""


class GpuError(RuntimeError):
    """A device failure or a problem the device can't hold: ``Error::Gpu`` (``src/error.rs:49``)."""


class Growing(RuntimeError):
    """The fields grew again after the sources ended and the run stopped: ``Error::Growing``
    (``src/error.rs:59-69``)."""

    def __init__(self, message, time_um=float("nan"), checks=0, factor=float("nan")):
        super().__init__(message)
        self.time_um, self.checks, self.factor = time_um, checks, factor


@dataclass(frozen=True)
class Grid3d:
    """nx x ny x nz cells of dx x dy x dz um, the lowest corner at (x0, y0, z0)."""

    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    x0: float = 0.0
    y0: float = 0.0
    z0: float = 0.0

    @staticmethod
    def centred(n: Sequence[int], h: float) -> "Grid3d":
        """Cells of side h centred on the origin (the reference's test helper ``grid``,
        ``src/fdtd/checks.rs:8-20``)."""
        return Grid3d(n[0], n[1], n[2], h, h, h, -n[0] * h / 2.0, -n[1] * h / 2.0, -n[2] * h / 2.0)

    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def n(self, axis: int) -> int:
        return (self.nx, self.ny, self.nz)[axis]

    def step(self, axis: int) -> float:
        return (self.dx, self.dy, self.dz)[axis]

    def origin(self, axis: int) -> float:
        return (self.x0, self.y0, self.z0)[axis]

    def node(self, axis: int, m: int) -> float:
        return self.origin(axis) + float(m) * self.step(axis)

    def index(self, at: Tuple[int, int, int]) -> int:
        i, j, k = at
        return (k * self.ny + j) * self.nx + i

    def e_position(self, component: int, at: Tuple[int, int, int]) -> List[float]:
        p = [self.node(0, at[0]), self.node(1, at[1]), self.node(2, at[2])]
        p[component] += 0.5 * self.step(component)
        return p

    def h_position(self, component: int, at: Tuple[int, int, int]) -> List[float]:
        p = [self.node(0, at[0]) + 0.5 * self.dx, self.node(1, at[1]) + 0.5 * self.dy,
             self.node(2, at[2]) + 0.5 * self.dz]
        p[component] -= 0.5 * self.step(component)
        return p

    def as_arrays(self):
        return ((self.nx, self.ny, self.nz), (self.dx, self.dy, self.dz), (self.x0, self.y0, self.z0))


@dataclass(frozen=True)
class Pml:
    """A CPML of ``low`` and ``high`` cells inside the grid along an axis; 0 cells is a wall."""

    low: int
    high: int


@dataclass(frozen=True)
class Periodic:
    """A periodic axis (the reference's ``Edges::Bloch { k: 0 }``)."""


@dataclass(frozen=True)
class Bloch:
    """A Bloch-periodic axis (the reference's ``Edges::Bloch { k }``, ``src/fdtd.rs:206-256``):
    one period on, the field is e^(ikL) times itself; k (rad/um) not zero makes the fields
    complex (``src/fdtd/bloch.rs``)."""

    k: float


@dataclass(frozen=True)
class Cpml:
    """The convolutional PML's parameters (``src/fdtd.rs:83-118``)."""

    reflection: float = 1e-8
    sigma: Optional[float] = None
    order: float = 3.0
    kappa: float = 1.0
    alpha: float = 0.0

    def as_array(self) -> List[float]:
        return [self.reflection, math.nan if self.sigma is None else self.sigma, self.order,
                self.kappa, self.alpha]


@dataclass(frozen=True)
class Boundaries:
    """What is beyond each axis's ends (``src/fdtd.rs:206-256``)."""

    x: object
    y: object
    z: object
    cpml: Cpml = Cpml()

    @staticmethod
    def with_cpml(cells: int) -> "Boundaries":
        e = Pml(cells, cells)
        return Boundaries(e, e, e, Cpml())

    @staticmethod
    def walls() -> "Boundaries":
        return Boundaries.with_cpml(0)

    @staticmethod
    def cpml_2d(cells: int) -> "Boundaries":
        e = Pml(cells, cells)
        return Boundaries(e, e, Periodic(), Cpml())

    def edges(self, axis: int):
        return (self.x, self.y, self.z)[axis]

    def periodic(self, axis: int) -> bool:
        return isinstance(self.edges(axis), (Periodic, Bloch))

    def bloch(self) -> List[float]:
        """Each axis' Bloch wavenumber (0 for a plain periodic side or a CPML)."""
        return [float(self.edges(a).k) if isinstance(self.edges(a), Bloch) else 0.0
                for a in range(3)]

    def as_arrays(self):
        kind, low, high = [], [], []
        for a in range(3):
            e = self.edges(a)
            if isinstance(e, (Periodic, Bloch)):
                kind.append(1), low.append(0), high.append(0)
            else:
                kind.append(0), low.append(int(e.low)), high.append(int(e.high))
        return kind, low, high


class Waveform:
    """How a source varies in time (``src/fdtd.rs:259-434``)."""

    __slots__ = ("kind", "params")

    def __init__(self, kind: int, params: Sequence[float]):
        self.kind = kind
        self.params = tuple(float(p) for p in params)

    @staticmethod
    def gaussian(frequency: float, width: float, delay: float) -> "Waveform":
        """exp(-((t-delay)/width)^2) sin(omega (t-delay)), omega = 2 pi frequency (c/um)."""
        return Waveform(0, (frequency, width, delay))

    @staticmethod
    def differentiated_gaussian(width: float, delay: float) -> "Waveform":
        return Waveform(1, (width, delay))

    @staticmethod
    def continuous(frequency: float, amplitude: complex, ramp: float) -> "Waveform":
        return Waveform(2, (frequency, complex(amplitude).real, complex(amplitude).imag, ramp))

    @staticmethod
    def pulse(frequency: float, bandwidth: float) -> "Waveform":
        """A pulse whose power spectrum is ``bandwidth`` wide at half its peak (c/um):
        width sqrt(2 ln 2)/(pi bandwidth), its peak 6 widths in (``src/fdtd.rs:300-312``)."""
        if not (math.isfinite(bandwidth) and bandwidth > 0.0):
            raise InvalidValue(f"a pulse's bandwidth must be positive and finite, got {bandwidth}")
        width = math.sqrt(2.0 * math.log(2.0)) / (math.pi * bandwidth)
        return Waveform.gaussian(frequency, width, 6.0 * width)

    def as_array(self) -> List[float]:
        p = list(self.params) + [0.0] * (5 - len(self.params))
        return [float(self.kind)] + p

    def carrier(self) -> Optional[float]:
        return None if self.kind == 1 else self.params[0]

    def __repr__(self):
        names = {0: "Gaussian", 1: "DifferentiatedGaussian", 2: "Continuous"}
        return f"Waveform.{names[self.kind]}{self.params}"


@dataclass(frozen=True)
class Source:
    """A point source: a current on one value of E (J) or of H (M) (``src/fdtd.rs:446-456``)."""

    field: Field
    component: Axis
    at: Tuple[int, int, int]
    waveform: Waveform


@dataclass
class Current:
    """A current over many values, value r taking Re(a_r w(t)) (``src/fdtd/sources.rs:46-54``)."""

    field: Field
    values: List[Tuple[Axis, Tuple[int, int, int], complex]]
    waveform: Waveform


@dataclass(frozen=True)
class Dipole:
    """A point dipole anywhere, restricted to the grid with trilinear weights
    (``src/fdtd/sources.rs:56-70``)."""

    field: Field
    component: Axis
    position: Tuple[float, float, float]
    amplitude: complex
    waveform: Waveform


@dataclass(frozen=True)
class PlaneWave:
    """A plane wave on a total-field/scattered-field box (``src/fdtd/sources.rs:74-93``): the
    total field from nodes ``low`` to ``high`` (inclusive; whole along a periodic axis), going
    along ``direction`` = (p, q, s) cells (integers), E along ``polarization``'s part across it,
    in a background of ``eps`` uniform on the box's surface."""

    low: Tuple[int, int, int]
    high: Tuple[int, int, int]
    direction: Tuple[int, int, int]
    polarization: Tuple[float, float, float]
    eps: float
    waveform: "Waveform"


@dataclass(frozen=True)
class GaussianBeam:
    """A Gaussian beam launched from a plane of nodes, one way (``src/fdtd/sources.rs:104-133``):
    the plane ``plane`` normal to ``axis``, ``forward`` towards +axis; ``centre`` where its axis
    crosses the plane (along ``axis.others()``), ``waist`` w0 and the ``focus``'s distance ahead
    (um); tilted towards ``tilt`` by ``angle`` (radians); E across the tilt's plane
    (``parallel`` False, s) or in it (p); ``eps`` the medium's on the plane."""

    axis: Axis
    plane: int
    forward: bool
    centre: Tuple[float, float]
    waist: float
    focus: float
    tilt: Axis
    angle: float
    parallel: bool
    eps: float


@dataclass(frozen=True)
class FluxPlane:
    """Halfway between node planes ``plane`` and ``plane + 1`` along ``axis``, within a window
    along ``axis.others()`` (``src/fdtd/monitors.rs:212-263``)."""

    axis: Axis
    plane: int
    window: Tuple[Optional[Tuple[int, int]], Optional[Tuple[int, int]]] = (None, None)

    def within(self, b: Tuple[int, int], c: Tuple[int, int]) -> "FluxPlane":
        return FluxPlane(self.axis, self.plane, (tuple(b), tuple(c)))

    def window_array(self) -> List[int]:
        out = []
        for w in self.window:
            out += [-1, -1] if w is None else [int(w[0]), int(w[1])]
        return out


@dataclass(frozen=True)
class Pole:
    """One term of a dispersive medium (``src/fdtd/media.rs:55-109``): a Lorentz oscillator
    (strength, resonance f0, damping gamma/2pi) or a Drude term (plasma fp, damping)."""

    kind: int
    a: float
    b: float
    c: float = 0.0

    @staticmethod
    def lorentz(strength: float, resonance: float, damping: float) -> "Pole":
        return Pole(0, strength, resonance, damping)

    @staticmethod
    def drude(plasma: float, damping: float) -> "Pole":
        return Pole(1, plasma, damping, 0.0)

    def parts(self):
        if self.kind == 0:
            w0 = TAU * self.b
            return self.a * w0 * w0, w0 * w0, TAU * self.c
        wp = TAU * self.a
        return wp * wp, 0.0, TAU * self.b

    def coefficients(self, dt: float):
        """alpha, xi, gamma of the update at the step dt (``src/fdtd/media.rs:101-109``)."""
        a, w0sq, gamma = self.parts()
        d = 1.0 + gamma * dt / 2.0
        return ((2.0 - w0sq * dt * dt) / d, (gamma * dt / 2.0 - 1.0) / d, a * dt * dt / d)

    def as_array(self) -> List[float]:
        return [float(self.kind), self.a, self.b, self.c]


@dataclass
class Dispersive:
    """eps(omega) = eps_inf + sum of terms (``src/fdtd/media.rs:111-118``)."""

    eps_inf: float
    poles: List[Pole] = dc_field(default_factory=list)

    def check(self):
        if not (math.isfinite(self.eps_inf) and self.eps_inf > 0.0):
            raise InvalidValue(
                f"a dispersive medium's eps_inf must be positive and finite, got {self.eps_inf}")
        for p in self.poles:
            strength, damping = (p.a, p.c) if p.kind == 0 else (1.0, p.b)
            if not (math.isfinite(strength) and strength >= 0 and math.isfinite(damping)
                    and damping >= 0):
                raise InvalidValue(
                    f"a term of negative strength or damping is a gain, which FDTD can't step: {p}")


@dataclass
class Boxes:
    """A geometry: ``background`` everywhere, then each box (lo, hi, value) over it, a point
    inside when lo < p < hi on every axis; later boxes on top. It is the value of the
    reference's ``eps(x, y, z)`` closure, callable the same way."""

    background: float
    boxes: List[Tuple[Sequence[float], Sequence[float], float]] = dc_field(default_factory=list)

    def add(self, lo, hi, value) -> "Boxes":
        self.boxes.append((tuple(float(v) for v in lo), tuple(float(v) for v in hi), float(value)))
        return self

    def __call__(self, x, y, z):
        v = self.background
        for lo, hi, val in self.boxes:
            if lo[0] < x < hi[0] and lo[1] < y < hi[1] and lo[2] < z < hi[2]:
                v = val
        return v

    def as_array(self) -> np.ndarray:
        rows = [[lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], v] for lo, hi, v in self.boxes]
        return np.array(rows, dtype=np.float64).reshape(-1, 7)


INF = math.inf
