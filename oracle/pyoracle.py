"""ORACLE (test infrastructure only): Python access to the CPU restatement of photonoxide's FDTD
step in ``liboracle_fdtd.so``. Only the tests, the smoke check and the benchmark's CPU-baseline leg
use it, to check the CUDA engine; the product never imports it.

``OracleSimulation`` takes the same calls as the reference's ``Simulation`` (``src/fdtd.rs``) with
the plain types of ``photonoxide_b200.types``. ``precision=64`` is the reference's own arithmetic
(the parity target); ``precision=32`` is its ``Yee<f32>`` kernel arithmetic.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from photonoxide_b200.types import (Boxes, Current, Dipole, Dispersive, Field, FluxPlane,
                                    Grid3d, InvalidValue, PlaneWave, Source)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_fdtd.so")

_lib = None

D = C.c_double
L = C.c_long
P = C.c_void_p
DP = C.POINTER(C.c_double)
LP = C.POINTER(C.c_long)
IP = C.POINTER(C.c_int)


def build():
    """Compiles the oracle with its Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        x = C.CDLL(LIB_PATH)
        x.orc_create.restype = P
        x.orc_create.argtypes = [C.c_int, LP, DP, DP, IP, LP, LP, DP, D, DP, C.c_char_p, C.c_int]
        x.orc_destroy.argtypes = [P]
        x.orc_average_boxes.argtypes = [LP, DP, DP, DP, C.c_int, D, C.c_int, DP]
        x.orc_sample_boxes.argtypes = [LP, DP, DP, DP, C.c_int, D, DP]
        x.orc_conductivity.argtypes = [P, DP, C.c_char_p, C.c_int]
        x.orc_conductor.argtypes = [P, C.c_int, L, L, L]
        x.orc_add_source.argtypes = [P, C.c_int, C.c_int, L, L, L, DP]
        x.orc_add_current.argtypes = [P, C.c_int, L, IP, LP, DP, DP]
        x.orc_add_dipole.argtypes = [P, C.c_int, C.c_int, DP, D, D, DP]
        x.orc_add_probe.argtypes = [P, C.c_int, C.c_int, L, L, L]
        x.orc_add_dft.argtypes = [P, LP, LP, C.c_int, DP]
        x.orc_add_flux.argtypes = [P, C.c_int, L, LP, C.c_int, DP]
        x.orc_add_flux_box.argtypes = [P, LP, C.c_int, DP]
        x.orc_add_medium.argtypes = [P, D, C.c_int, DP, C.POINTER(C.c_ubyte), C.c_int,
                                     C.c_char_p, C.c_int]
        x.orc_run.argtypes = [P, L]
        x.orc_dt.argtypes = [P]
        x.orc_dt.restype = D
        x.orc_steps.argtypes = [P]
        x.orc_steps.restype = L
        x.orc_get_field.argtypes = [P, C.c_int, C.c_int, DP]
        x.orc_set_field.argtypes = [P, C.c_int, C.c_int, DP]
        x.orc_probe.argtypes = [P, C.c_int, DP]
        x.orc_probe.restype = L
        x.orc_transforms.argtypes = [P, DP]
        x.orc_transforms.restype = L
        x.orc_flux.argtypes = [P, C.c_int, DP]
        x.orc_tables.argtypes = [P, C.c_int, DP]
        x.orc_tables.restype = L
        x.orc_medium_stable.argtypes = [D, C.c_int, DP, D, D, D]
        x.orc_triad.argtypes = [L, C.c_int]
        x.orc_triad.restype = D
        x.orc_waveform_spectrum.argtypes = [DP, C.c_int, D, L, C.c_int, DP, DP]
        x.orc_add_plane_wave.argtypes = [P, LP, LP, LP, DP, D, DP, C.c_char_p, C.c_int]
        x.orc_create_bloch.restype = P
        x.orc_create_bloch.argtypes = [C.c_int, LP, DP, DP, IP, LP, LP, DP, DP, D, DP,
                                       C.c_char_p, C.c_int]
        x.orc_is_complex.argtypes = [P]
        x.orc_threads.argtypes = [C.c_int]
        x.orc_get_field_imag.argtypes = [P, C.c_int, C.c_int, DP]
        x.orc_probe_imag.argtypes = [P, C.c_int, DP]
        x.orc_probe_imag.restype = L
        x.orc_incident.argtypes = [P, C.c_int, C.c_int, C.c_int, L, L, L]
        x.orc_incident.restype = D
        _lib = x
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(DP)


def _l(a):
    a = np.ascontiguousarray(a, dtype=np.int64)
    return a, a.ctypes.data_as(LP)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(IP)


def average_boxes(grid: Grid3d, geometry: Boxes, samples: int = 8) -> np.ndarray:
    """FDFD's cell average of a box geometry at every value of E: (3, cells)."""
    n, d, o = grid.as_arrays()
    out = np.empty(3 * grid.cells())
    na, nap = _l(n)
    da, dap = _d(d)
    oa, oap = _d(o)
    b, bp = _d(geometry.as_array())
    lib().orc_average_boxes(nap, dap, oap, bp, len(geometry.boxes), geometry.background, samples,
                            out.ctypes.data_as(DP))
    return out.reshape(3, -1)


def sample_boxes(grid: Grid3d, geometry: Boxes) -> np.ndarray:
    n, d, o = grid.as_arrays()
    out = np.empty(3 * grid.cells())
    na, nap = _l(n)
    da, dap = _d(d)
    oa, oap = _d(o)
    b, bp = _d(geometry.as_array())
    lib().orc_sample_boxes(nap, dap, oap, bp, len(geometry.boxes), geometry.background,
                           out.ctypes.data_as(DP))
    return out.reshape(3, -1)


class OracleSimulation:
    """The reference's ``Simulation`` restated on the CPU (``src/fdtd.rs:469-1590``)."""

    def __init__(self, grid: Grid3d, eps, boundaries, courant: float, precision: int = 64):
        self.grid = grid
        self.boundaries = boundaries
        if isinstance(eps, Boxes):
            eps = average_boxes(grid, eps)
        eps = np.asarray(eps, dtype=np.float64).reshape(3, grid.cells())
        n, d, o = grid.as_arrays()
        kind, low, high = boundaries.as_arrays()
        err = C.create_string_buffer(512)
        keep = [_l(n), _d(d), _d(o), _i(kind), _l(low), _l(high), _d(boundaries.cpml.as_array()),
                _d(eps)]
        bloch = _d(boundaries.bloch() if hasattr(boundaries, "bloch") else [0.0, 0.0, 0.0])
        h = lib().orc_create_bloch(precision, keep[0][1], keep[1][1], keep[2][1], keep[3][1],
                                   keep[4][1], keep[5][1], keep[6][1], bloch[1], float(courant),
                                   keep[7][1], err, 512)
        if not h:
            raise InvalidValue(err.value.decode())
        self._h = h
        self.precision = precision
        self._fluxes = 0

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    # -- the medium ---------------------------------------------------------------------------
    def with_conductivity(self, sigma):
        if isinstance(sigma, Boxes):
            sigma = sample_boxes(self.grid, sigma)
        a, p = _d(np.asarray(sigma).reshape(-1))
        err = C.create_string_buffer(512)
        if lib().orc_conductivity(self._h, p, err, 512):
            raise InvalidValue(err.value.decode())
        return self

    def with_medium(self, medium: Dispersive, inside, check_stability: bool = True):
        if isinstance(inside, Boxes):
            inside = sample_boxes(self.grid, inside) != 0
        mask = np.ascontiguousarray(np.asarray(inside).reshape(-1), dtype=np.uint8)
        poles, pp = _d([v for p in medium.poles for v in p.as_array()] or [0.0])
        err = C.create_string_buffer(512)
        if lib().orc_add_medium(self._h, medium.eps_inf, len(medium.poles), pp,
                                mask.ctypes.data_as(C.POINTER(C.c_ubyte)), int(check_stability),
                                err, 512):
            raise InvalidValue(err.value.decode())
        return self

    def conductor(self, component, at):
        lib().orc_conductor(self._h, int(component), *[int(v) for v in at])

    # -- sources, probes, monitors ------------------------------------------------------------
    def add_source(self, s: Source):
        w, wp = _d(s.waveform.as_array())
        if lib().orc_add_source(self._h, int(s.field), int(s.component), *[int(v) for v in s.at],
                                wp):
            raise InvalidValue(f"{s.at} is outside the grid")

    def add_current(self, c: Current):
        comps, cp = _i([int(v[0]) for v in c.values])
        at, ap = _l([int(x) for v in c.values for x in v[1]])
        amps, mp = _d([x for v in c.values for x in (complex(v[2]).real, complex(v[2]).imag)])
        w, wp = _d(c.waveform.as_array())
        if lib().orc_add_current(self._h, int(c.field), len(c.values), cp, ap, mp, wp):
            raise InvalidValue("a current's value is outside the grid or not finite")

    def add_dipole(self, d: Dipole):
        pos, pp = _d(d.position)
        w, wp = _d(d.waveform.as_array())
        a = complex(d.amplitude)
        if lib().orc_add_dipole(self._h, int(d.field), int(d.component), pp, a.real, a.imag, wp):
            raise InvalidValue(f"the dipole {d} is outside its component's values")

    def add_plane_wave(self, wave: PlaneWave) -> int:
        lo, lp = _l(wave.low)
        hi, hp = _l(wave.high)
        dr, dp = _l(wave.direction)
        po, pp = _d(wave.polarization)
        w, wp = _d(wave.waveform.as_array())
        err = C.create_string_buffer(512)
        r = lib().orc_add_plane_wave(self._h, lp, hp, dp, pp, float(wave.eps), wp, err, 512)
        if r < 0:
            raise InvalidValue(err.value.decode())
        return r

    def incident(self, n: int, field, component, at) -> float:
        return float(lib().orc_incident(self._h, int(n), int(field), int(component),
                                        *[int(v) for v in at]))

    @property
    def is_complex(self) -> bool:
        return bool(lib().orc_is_complex(self._h))

    def _imag(self, field, component):
        out = np.empty(self.grid.cells())
        if lib().orc_get_field_imag(self._h, int(field), int(component),
                                    out.ctypes.data_as(DP)):
            raise InvalidValue("the fields are real: no Bloch phase")
        return out

    def e_imaginary(self, component) -> np.ndarray:
        return self._imag(0, component)

    def h_imaginary(self, component) -> np.ndarray:
        return self._imag(1, component)

    def probe_complex(self, n: int) -> np.ndarray:
        re = self.probe(n)
        if not self.is_complex:
            return re + 0j
        count = lib().orc_probe_imag(self._h, int(n), None)
        im = np.empty(count)
        lib().orc_probe_imag(self._h, int(n), im.ctypes.data_as(DP))
        return re + 1j * im

    def add_probe(self, field, component, at) -> int:
        r = lib().orc_add_probe(self._h, int(field), int(component), *[int(v) for v in at])
        if r < 0:
            raise InvalidValue(f"{at} is outside the grid")
        return r

    def add_dft(self, low, high, frequencies) -> int:
        lo, lp = _l(low)
        hi, hp = _l(high)
        f, fp = _d(frequencies)
        r = lib().orc_add_dft(self._h, lp, hp, len(f), fp)
        if r < 0:
            raise InvalidValue("bad transform box or frequencies")
        return r

    def add_flux(self, plane: FluxPlane, frequencies) -> int:
        w, wp = _l(plane.window_array())
        f, fp = _d(frequencies)
        r = lib().orc_add_flux(self._h, int(plane.axis), int(plane.plane), wp, len(f), fp)
        if r < 0:
            raise InvalidValue("bad flux plane or frequencies")
        return r

    def add_flux_box(self, planes, frequencies) -> int:
        p, pp = _l([int(v) for pr in planes for v in pr])
        f, fp = _d(frequencies)
        r = lib().orc_add_flux_box(self._h, pp, len(f), fp)
        if r < 0:
            raise InvalidValue("bad flux box or frequencies")
        return r

    # -- stepping and reading -----------------------------------------------------------------
    def run(self, steps: int):
        lib().orc_run(self._h, int(steps))

    def step(self):
        self.run(1)

    @property
    def dt(self) -> float:
        return lib().orc_dt(self._h)

    @property
    def steps(self) -> int:
        return lib().orc_steps(self._h)

    def _field(self, field, component):
        out = np.empty(self.grid.cells())
        lib().orc_get_field(self._h, int(field), int(component), out.ctypes.data_as(DP))
        return out

    def e(self, component) -> np.ndarray:
        return self._field(Field.E, component)

    def h(self, component) -> np.ndarray:
        return self._field(Field.H, component)

    def set_field(self, field, component, values):
        a, p = _d(np.asarray(values).reshape(-1))
        lib().orc_set_field(self._h, int(field), int(component), p)

    def probe(self, n: int) -> np.ndarray:
        count = lib().orc_probe(self._h, n, None)
        out = np.empty(count)
        lib().orc_probe(self._h, n, out.ctypes.data_as(DP))
        return out

    def transforms(self) -> np.ndarray:
        count = lib().orc_transforms(self._h, None)
        out = np.empty(2 * count)
        lib().orc_transforms(self._h, out.ctypes.data_as(DP))
        return out.view(np.complex128)

    def flux(self, n: int) -> np.ndarray:
        out = np.empty(256)
        count = lib().orc_flux(self._h, n, out.ctypes.data_as(DP))
        return out[:count].copy()

    def tables(self, which: int) -> np.ndarray:
        count = lib().orc_tables(self._h, which, None)
        out = np.empty(count)
        lib().orc_tables(self._h, which, out.ctypes.data_as(DP))
        return out


def medium_stable(medium: Dispersive, sigma: float, dt: float, top: float) -> bool:
    p, pp = _d([v for q in medium.poles for v in q.as_array()] or [0.0])
    return bool(lib().orc_medium_stable(medium.eps_inf, len(medium.poles), pp, sigma, dt, top))


def triad(length: int = 1 << 26, repeats: int = 5) -> float:
    """The host's STREAM triad bandwidth, GB/s, as the reference measures it (src/traffic.rs)."""
    return float(lib().orc_triad(int(length), int(repeats)))


def waveform_spectrum(waveform, field, dt: float, steps: int, frequencies) -> np.ndarray:
    """``Waveform::spectrum`` (src/fdtd.rs:361-396) at each frequency: complex."""
    w, wp = _d(waveform.as_array())
    f, fp = _d(np.asarray(frequencies, dtype=np.float64).reshape(-1))
    out = np.zeros(2 * f.size)
    if lib().orc_waveform_spectrum(wp, int(field), float(dt), int(steps), f.size, fp,
                                   out.ctypes.data_as(DP)) != 0:
        raise InvalidValue("a waveform's spectrum needs dt > 0 and steps >= 0")
    return out[0::2] + 1j * out[1::2]


def threads(n: int) -> int:
    """Sets the host threads the oracle's loops use; returns the number before."""
    return int(lib().orc_threads(int(n)))
