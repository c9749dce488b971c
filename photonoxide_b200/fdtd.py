"""photonoxide's FDTD ``Simulation`` (``src/fdtd.rs:469-1590``), stepped by the B200 engine.

The setup (cell-averaged permittivity, time step, walls, CPML tables, media, sources, monitors)
is the C++ host library's and the stepping the CUDA engine's, both in ``libphotonoxide_fdtd.so``
next to this file (``make -C photonoxide_b200/csrc`` builds it).
There is no CPU fallback: without the library, or without a CUDA device at the first run, the
calls raise.

The methods keep the reference's names and meanings: ``with_conductivity``, ``with_medium``,
``conductor``, ``add_source``, ``add_current``, ``add_dipole``, ``add_probe``, ``add_dft``,
``add_flux``, ``add_flux_box``, ``run``, ``step``, ``e``, ``h``, ``probe``, ``flux``. Errors are
:class:`~photonoxide_b200.types.InvalidValue` (``Error::InvalidValue``) and
:class:`~photonoxide_b200.types.GpuError` (``Error::Gpu``).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import Optional

import numpy as np

from .types import (Boxes, Current, Dipole, Dispersive, Field, FluxPlane, GaussianBeam,
                    GpuError, Grid3d, Growing, InvalidValue, PlaneWave, Source)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphotonoxide_fdtd.so")

FDTD_E_INVALID = -1
FDTD_E_GPU = -2
FDTD_E_BUDGET = -3
FDTD_E_GROWING = -6

_lib = None

D, I32, I64, P = C.c_double, C.c_int32, C.c_int64, C.c_void_p
DP, I32P, I64P = C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int64)


class Geometry(C.Structure):
    _fields_ = [("background", D), ("nboxes", I32), ("boxes", DP)]


def library():
    """The engine's shared library, loaded once. Raises if it isn't built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GpuError(
                f"{LIB_PATH} is not built: run make -C {HERE}/csrc")
        x = C.CDLL(LIB_PATH)
        x.pxs_create.restype = P
        x.pxs_create.argtypes = [I64P, DP, DP, I32P, I64P, I64P, DP, D, DP, C.POINTER(Geometry),
                                 I32, C.c_size_t, C.c_char_p, I32]
        x.pxs_destroy.argtypes = [P]
        x.pxs_last_error.argtypes = [P]
        x.pxs_last_error.restype = C.c_char_p
        x.pxs_average.argtypes = [I64P, DP, DP, C.POINTER(Geometry), DP]
        x.pxs_conductivity.argtypes = [P, DP, C.POINTER(Geometry)]
        x.pxs_conductor.argtypes = [P, I32, I64, I64, I64]
        x.pxs_medium.argtypes = [P, D, I32, DP, C.POINTER(C.c_uint8), C.POINTER(Geometry)]
        x.pxs_add_source.argtypes = [P, I32, I32, I64, I64, I64, DP]
        x.pxs_add_current.argtypes = [P, I32, I64, I32P, I64P, DP, DP]
        x.pxs_add_dipole.argtypes = [P, I32, I32, DP, D, D, DP]
        x.pxs_add_probe.argtypes = [P, I32, I32, I64, I64, I64]
        x.pxs_add_dft.argtypes = [P, I64P, I64P, I32, DP]
        x.pxs_add_flux.argtypes = [P, I32, I64, I64P, I32, DP]
        x.pxs_add_flux_box.argtypes = [P, I64P, I32, DP]
        x.pxs_run.argtypes = [P, I64]
        x.pxs_dt.argtypes = [P]
        x.pxs_dt.restype = D
        x.pxs_steps.argtypes = [P]
        x.pxs_steps.restype = I64
        x.pxs_get_field.argtypes = [P, I32, I32, DP]
        x.pxs_set_field.argtypes = [P, I32, I32, DP]
        x.pxs_probe.argtypes = [P, I32, DP]
        x.pxs_probe.restype = I64
        x.pxs_transforms.argtypes = [P, DP]
        x.pxs_transforms.restype = I64
        x.pxs_flux.argtypes = [P, I32, DP]
        x.pxs_tables.argtypes = [P, I32, DP]
        x.pxs_tables.restype = I64
        x.pxs_engine.argtypes = [P]
        x.pxs_time.argtypes = [P]
        x.pxs_time.restype = D
        x.pxs_run_until.argtypes = [P, D]
        x.pxs_run_until_decayed.argtypes = [P, I32, I32P, D, D, D, I32P, DP]
        x.pxs_waveform_spectrum.argtypes = [DP, I32, D, I64, I32, DP, DP]
        x.pxs_add_plane_wave.argtypes = [P, I64P, I64P, I64P, DP, D, DP]
        x.pxs_incident.argtypes = [P, I32, I32, I32, I64, I64, I64, DP]
        x.pxs_add_beam.argtypes = [P, I32, I64, I32, DP, D, D, I32, D, I32, D, DP]
        x.pxs_create_bloch.restype = P
        x.pxs_create_bloch.argtypes = [I64P, DP, DP, I32P, I64P, I64P, DP, DP, D, DP,
                                       C.POINTER(Geometry), I32, C.c_size_t, C.c_char_p, I32]
        x.pxs_is_complex.argtypes = [P]
        x.pxs_get_field_imag.argtypes = [P, I32, I32, DP]
        x.pxs_set_field_imag.argtypes = [P, I32, I32, DP]
        x.pxs_probe_imag.argtypes = [P, I32, DP]
        x.pxs_probe_imag.restype = I64
        x.pxs_engine.restype = P
        _lib = x
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(DP)


def _i64(a):
    a = np.ascontiguousarray(a, dtype=np.int64)
    return a, a.ctypes.data_as(I64P)


def _i32(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(I32P)


def _geometry(g: Boxes):
    arr = np.ascontiguousarray(g.as_array(), dtype=np.float64)
    return arr, Geometry(float(g.background), len(g.boxes), arr.ctypes.data_as(DP))


def average(grid: Grid3d, geometry: Boxes, device: bool = False) -> np.ndarray:
    """FDFD's cell average of a box geometry at each value of E, (3, cells): what
    ``Simulation::new`` takes from ``eps(x, y, z)`` (``src/fdtd.rs:570-604``). ``device``: on
    the current CUDA device, one thread per value (the same bits as on the host)."""
    n, d, o = grid.as_arrays()
    out = np.empty(3 * grid.cells())
    keep = [_i64(n), _d(d), _d(o)]
    arr, geo = _geometry(geometry)
    x = library()
    if device:
        x.pxs_average_device.argtypes = [I64P, DP, DP, C.POINTER(Geometry), DP]
        code = x.pxs_average_device(keep[0][1], keep[1][1], keep[2][1], C.byref(geo),
                                    out.ctypes.data_as(DP))
        if code != 0:
            raise GpuError(f"the cell average on the device failed ({code})")
    else:
        x.pxs_average(keep[0][1], keep[1][1], keep[2][1], C.byref(geo), out.ctypes.data_as(DP))
    return out.reshape(3, -1)


def cpml_tables(grid: Grid3d, boundaries, dt: float, which: int) -> np.ndarray:
    """The CPML's tables (``Simulation::build_cpml``, ``src/fdtd.rs:799-869``) made on the
    current CUDA device, one thread per node, with the host library's functions (the same bits):
    ``which`` 2 the kappa factors over the step at the nodes, 3 at the half-steps, 4 the slabs,
    laid out as :meth:`Simulation.tables` lays them out."""
    n, d, _ = grid.as_arrays()
    kind, low, high = boundaries.as_arrays()
    keep = [_i64(n), _d(d), _i32(kind), _i64(low), _i64(high), _d(boundaries.cpml.as_array())]
    x = library()
    x.pxs_cpml_device.argtypes = [I64P, DP, I32P, I64P, I64P, DP, D, I32, DP]
    x.pxs_cpml_device.restype = I64
    args = [k[1] for k in keep] + [float(dt), int(which)]
    count = x.pxs_cpml_device(*args, None)
    if count < 0:
        raise InvalidValue(f"the CPML's tables need a grid and CPMLs that fit it ({count})")
    out = np.empty(count)
    code = x.pxs_cpml_device(*args, out.ctypes.data_as(DP))
    if code != count:
        raise GpuError(f"the CPML's tables on the device failed ({code})")
    return out


def waveform_spectrum(waveform, field, dt: float, steps: int, frequencies) -> np.ndarray:
    """``Waveform::spectrum`` (``src/fdtd.rs:361-396``): sum over n < steps of w(t_n)
    e^(i omega t_n) dt, t_n = n dt (+ dt/2 for E), at each frequency (c/um), with the
    reference's exp and sin/cos; complex, one per frequency."""
    w, wp = _d(waveform.as_array())
    f, fp = _d(np.asarray(frequencies, dtype=np.float64).reshape(-1))
    out = np.zeros(2 * f.size)
    code = library().pxs_waveform_spectrum(wp, int(field), float(dt), int(steps), f.size, fp,
                                           out.ctypes.data_as(DP))
    if code != 0:
        raise InvalidValue(f"a waveform's spectrum needs dt > 0 and steps >= 0 ({code})")
    return out[0::2] + 1j * out[1::2]


class Simulation:
    """An FDTD problem on the B200: ``Simulation::new(grid, eps, boundaries, courant)``.

    ``eps`` is a :class:`Boxes` geometry (averaged over each value's cell as the reference
    averages its closure) or an array (3, cells) of per-value permittivities. ``precision`` 32
    steps in f32 (the engine's product precision), 64 in f64 (for checking against the CPU).
    ``hbm_budget`` (bytes, 0 for none) refuses a problem that would need more device memory.
    """

    def __init__(self, grid: Grid3d, eps, boundaries, courant: float, precision: int = 32,
                 hbm_budget: int = 0):
        lib = library()
        self.grid = grid
        self.boundaries = boundaries
        self.precision = precision
        n, d, o = grid.as_arrays()
        kind, low, high = boundaries.as_arrays()
        keep = [_i64(n), _d(d), _d(o), _i32(kind), _i64(low), _i64(high),
                _d(boundaries.cpml.as_array())]
        eps_p, geo_p = None, None
        if isinstance(eps, Boxes):
            arr, geo = _geometry(eps)
            keep.append((arr, geo))
            geo_p = C.byref(geo)
        else:
            e = np.ascontiguousarray(np.asarray(eps, dtype=np.float64).reshape(-1))
            if e.size != 3 * grid.cells():
                raise InvalidValue(f"eps needs 3 x {grid.cells()} values, got {e.size}")
            keep.append(e)
            eps_p = e.ctypes.data_as(DP)
        err = C.create_string_buffer(1024)
        bloch = _d(boundaries.bloch() if hasattr(boundaries, "bloch") else [0.0, 0.0, 0.0])
        h = lib.pxs_create_bloch(keep[0][1], keep[1][1], keep[2][1], keep[3][1], keep[4][1],
                                 keep[5][1], keep[6][1], bloch[1], float(courant), eps_p, geo_p,
                                 int(precision), int(hbm_budget), err, 1024)
        if not h:
            raise InvalidValue(err.value.decode())
        self._h = h
        self._nflux = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.pxs_destroy(h)
            self._h = None

    def _check(self, code):
        if code is None or code >= 0:
            return code
        msg = library().pxs_last_error(self._h).decode()
        if code == FDTD_E_INVALID:
            raise InvalidValue(msg)
        raise GpuError(msg)

    # -- the medium ---------------------------------------------------------------------------
    def with_conductivity(self, sigma) -> "Simulation":
        """``Simulation::with_conductivity``: sigma (1/um with eta0 = 1) sampled at each value
        of E, as a :class:`Boxes` geometry or an array (3, cells)."""
        if isinstance(sigma, Boxes):
            arr, geo = _geometry(sigma)
            self._check(library().pxs_conductivity(self._h, None, C.byref(geo)))
        else:
            a, p = _d(np.asarray(sigma).reshape(-1))
            self._check(library().pxs_conductivity(self._h, p, None))
        return self

    def with_medium(self, medium: Dispersive, inside) -> "Simulation":
        """``Simulation::with_medium``: the dispersive medium wherever ``inside`` (a
        :class:`Boxes` whose nonzero values mark it, or a mask (3, cells)) holds at a value of
        E, refused unless it steps stably at this time step."""
        medium.check()
        poles, pp = _d([v for q in medium.poles for v in q.as_array()] or [0.0])
        if isinstance(inside, Boxes):
            arr, geo = _geometry(inside)
            self._check(library().pxs_medium(self._h, medium.eps_inf, len(medium.poles), pp,
                                             None, C.byref(geo)))
        else:
            mask = np.ascontiguousarray(np.asarray(inside).reshape(-1), dtype=np.uint8)
            self._check(library().pxs_medium(self._h, medium.eps_inf, len(medium.poles), pp,
                                             mask.ctypes.data_as(C.POINTER(C.c_uint8)), None))
        return self

    def conductor(self, component, at):
        self._check(library().pxs_conductor(self._h, int(component), *[int(v) for v in at]))

    # -- sources, probes, monitors ------------------------------------------------------------
    def add_source(self, s: Source):
        w, wp = _d(s.waveform.as_array())
        self._check(library().pxs_add_source(self._h, int(s.field), int(s.component),
                                             *[int(v) for v in s.at], wp))

    def add_current(self, c: Current):
        comps, cp = _i32([int(v[0]) for v in c.values])
        at, ap = _i64([int(x) for v in c.values for x in v[1]])
        amps, mp = _d([x for v in c.values for x in (complex(v[2]).real, complex(v[2]).imag)])
        w, wp = _d(c.waveform.as_array())
        self._check(library().pxs_add_current(self._h, int(c.field), len(c.values), cp, ap, mp,
                                              wp))

    def add_dipole(self, d: Dipole):
        pos, pp = _d(d.position)
        w, wp = _d(d.waveform.as_array())
        a = complex(d.amplitude)
        self._check(library().pxs_add_dipole(self._h, int(d.field), int(d.component), pp, a.real,
                                             a.imag, wp))

    def add_plane_wave(self, wave: PlaneWave) -> int:
        """``Simulation::add_plane_wave``: a total-field/scattered-field box whose incident
        field an auxiliary 1D run along the direction gives (stepped on the device with the
        grid); its number, for :meth:`incident`."""
        lo, lp = _i64(wave.low)
        hi, hp = _i64(wave.high)
        dr, dp = _i64(wave.direction)
        po, pp = _d(wave.polarization)
        w, wp = _d(wave.waveform.as_array())
        return self._check(library().pxs_add_plane_wave(self._h, lp, hp, dp, pp, float(wave.eps),
                                                        wp))

    def add_beam(self, beam: GaussianBeam, waveform) -> None:
        """``Simulation::add_beam``: the beam's plane waves on its surface become currents
        with ``waveform`` (which needs a carrier)."""
        c, cp = _d(beam.centre)
        w, wp = _d(waveform.as_array())
        self._check(library().pxs_add_beam(self._h, int(beam.axis), int(beam.plane),
                                           1 if beam.forward else -1, cp, float(beam.waist),
                                           float(beam.focus), int(beam.tilt), float(beam.angle),
                                           1 if beam.parallel else 0, float(beam.eps), wp))

    def incident(self, n: int, field, component, at) -> float:
        """``Simulation::incident``: plane wave n's incident field now at a value."""
        out = C.c_double(0.0)
        self._check(library().pxs_incident(self._h, int(n), int(field), int(component),
                                           *[int(v) for v in at], C.byref(out)))
        return out.value

    def add_probe(self, field, component, at) -> int:
        return self._check(library().pxs_add_probe(self._h, int(field), int(component),
                                                   *[int(v) for v in at]))

    def add_dft(self, low, high, frequencies) -> int:
        lo, lp = _i64(low)
        hi, hp = _i64(high)
        f, fp = _d(frequencies)
        return self._check(library().pxs_add_dft(self._h, lp, hp, len(f), fp))

    def add_flux(self, plane: FluxPlane, frequencies) -> int:
        w, wp = _i64(plane.window_array())
        f, fp = _d(frequencies)
        return self._check(library().pxs_add_flux(self._h, int(plane.axis), int(plane.plane), wp,
                                                  len(f), fp))

    def add_flux_box(self, planes, frequencies) -> int:
        p, pp = _i64([int(v) for pr in planes for v in pr])
        f, fp = _d(frequencies)
        return self._check(library().pxs_add_flux_box(self._h, pp, len(f), fp))

    # -- stepping and reading -----------------------------------------------------------------
    def run(self, steps: int):
        """``Simulation::run``: ``steps`` steps on the device."""
        self._check(library().pxs_run(self._h, int(steps)))

    def step(self):
        self.run(1)

    def time(self) -> float:
        """``Simulation::time``: steps x dt (um/c)."""
        return float(library().pxs_time(self._h))

    def run_until(self, time: float) -> "Simulation":
        """``Simulation::run_until`` (src/fdtd.rs:1161-1167): the steps that bring the time to
        ``time``."""
        self._check(library().pxs_run_until(self._h, float(time)))
        return self

    def run_until_decayed(self, probes, fraction: float, interval: float, limit: float) -> bool:
        """``Simulation::run_until_decayed`` (src/fdtd/monitors.rs:742-838): runs in blocks of
        ``interval`` until |F|^2 at every probe stayed within ``fraction`` of its peak over a
        block (True) or the time reaches ``limit`` (False). Raises :class:`Growing` when the
        fields grow again after the sources end."""
        ps = (C.c_int32 * len(probes))(*[int(p) for p in probes])
        done = C.c_int32(0)
        info = (C.c_double * 3)()
        code = library().pxs_run_until_decayed(self._h, len(probes), ps, float(fraction),
                                               float(interval), float(limit), C.byref(done), info)
        if code == FDTD_E_GROWING:
            raise Growing(library().pxs_last_error(self._h).decode(), info[0], int(info[1]),
                          info[2])
        self._check(code)
        return bool(done.value)

    @property
    def dt(self) -> float:
        return library().pxs_dt(self._h)

    @property
    def steps(self) -> int:
        return library().pxs_steps(self._h)

    def _field(self, field, component) -> np.ndarray:
        out = np.empty(self.grid.cells())
        self._check(library().pxs_get_field(self._h, int(field), int(component),
                                            out.ctypes.data_as(DP)))
        return out

    def e(self, component) -> np.ndarray:
        return self._field(Field.E, component)

    def h(self, component) -> np.ndarray:
        return self._field(Field.H, component)

    def set_field(self, field, component, values):
        a, p = _d(np.asarray(values).reshape(-1))
        self._check(library().pxs_set_field(self._h, int(field), int(component), p))

    @property
    def is_complex(self) -> bool:
        """``Simulation::is_complex``: a Bloch phase on a side makes the fields complex."""
        return bool(library().pxs_is_complex(self._h))

    def _imag(self, field, component) -> np.ndarray:
        out = np.empty(self.grid.cells())
        self._check(library().pxs_get_field_imag(self._h, int(field), int(component),
                                                 out.ctypes.data_as(DP)))
        return out

    def e_imaginary(self, component) -> np.ndarray:
        """``Simulation::e_imaginary``: E's imaginary part in a complex run."""
        return self._imag(0, component)

    def h_imaginary(self, component) -> np.ndarray:
        return self._imag(1, component)

    def set_field_imaginary(self, field, component, values):
        a, p = _d(np.asarray(values).reshape(-1))
        self._check(library().pxs_set_field_imag(self._h, int(field), int(component), p))

    def probe_complex(self, n: int) -> np.ndarray:
        """``Simulation::probe_complex``: the probe's values with their imaginary part."""
        re = self.probe(n)
        if not self.is_complex:
            return re + 0j
        lib = library()
        count = self._check(lib.pxs_probe_imag(self._h, int(n), None))
        im = np.empty(count)
        self._check(lib.pxs_probe_imag(self._h, int(n), im.ctypes.data_as(DP)))
        return re + 1j * im

    def probe(self, n: int) -> np.ndarray:
        count = self._check(library().pxs_probe(self._h, int(n), None))
        out = np.empty(count)
        library().pxs_probe(self._h, int(n), out.ctypes.data_as(DP))
        return out

    def transforms(self) -> np.ndarray:
        """Every transform's sums in ``Monitors::layout`` order, complex."""
        count = self._check(library().pxs_transforms(self._h, None))
        out = np.empty(2 * count)
        self._check(library().pxs_transforms(self._h, out.ctypes.data_as(DP)))
        return out.view(np.complex128)

    def flux(self, n: int) -> np.ndarray:
        """``Simulation::flux``: the flux at each frequency of flux monitor ``n``."""
        out = np.empty(4096)
        count = self._check(library().pxs_flux(self._h, int(n), out.ctypes.data_as(DP)))
        return out[:count].copy()

    def tables(self, which: int) -> np.ndarray:
        count = library().pxs_tables(self._h, int(which), None)
        out = np.empty(count)
        library().pxs_tables(self._h, int(which), out.ctypes.data_as(DP))
        return out

    def engine(self) -> Optional[int]:
        """The device engine's context pointer (a ``fdtd_ctx*``), once the run has started."""
        return library().pxs_engine(self._h)
