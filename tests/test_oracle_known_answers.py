"""The oracle against the measured values photonoxide publishes for its FDTD (docs/validation.md,
rows fdtd/cpml-thickness, fdtd/drude-fresnel and fdtd/lorentz-group-delay), each fixture restated
from the reference's own checks and run on the oracle in f64: the same numbers to the digits the
reference prints. These pin the parts of the step the canary hash does not reach: the CPML's
grading and recursion (three thicknesses), and the Drude and Lorentz ADE updates (three
resolutions each, second order in the cells)."""
import math

import numpy as np
import pytest

from photonoxide_b200.types import (Axis, Boundaries, Cpml, Dispersive, Field, Grid3d, Periodic,
                                    Pml, Pole, Source, Waveform)
from pyoracle import OracleSimulation

TAU = 2.0 * math.pi


def printed(x: float) -> str:
    """x to two significant digits, as the reference's report prints it."""
    return f"{x:.1e}"


def steps_until(dt: float, time: float) -> int:
    """Simulation::run_until's count (src/fdtd.rs:1161-1167): steps while n dt < time."""
    n = 0
    while n * dt < time:
        n += 1
    return n


# -- fdtd/cpml-thickness: src/fdtd/checks.rs:135-200 ------------------------------------------

def cpml_record(pad: int, cells: int, interior: int = 40, gap: int = 2, h: float = 0.05):
    n = interior + 2 * pad
    g = Grid3d(n, n, 1, h, h, h, -n * h / 2, -n * h / 2, -h / 2)
    b = Boundaries(Pml(cells, cells), Pml(cells, cells), Periodic(), Cpml())
    s = OracleSimulation(g, np.ones((3, g.cells())), b, 0.7, precision=64)
    c = n // 2
    s.add_source(Source(Field.E, Axis.Z, (c, c, 0), Waveform.gaussian(1.0, 0.5, 1.6)))
    near = pad + gap
    p = s.add_probe(Field.E, Axis.Z, (near, c, 0))
    q = s.add_probe(Field.E, Axis.Z, (near, near, 0))
    s.run(steps_until(s.dt, 9.0))
    return np.concatenate([s.probe(p), s.probe(q)])


@pytest.mark.parametrize("thickness,published", [(4, "2.6e-02"), (8, "1.2e-04"), (16, "6.1e-06")])
def test_cpml_thickness(thickness, published):
    small = cpml_record(thickness, thickness)
    reference = cpml_record(thickness + 120, 20)
    error = float(np.max(np.abs(small - reference)) / np.max(np.abs(reference)))
    assert printed(error) == published, error


# -- the columns of src/fdtd/media_checks.rs:92-157 ---------------------------------------------

def column(h: float, nz: int, cpml: int):
    g = Grid3d(1, 1, nz, h, h, h, 0.0, 0.0, 0.0)
    return g, Boundaries(Periodic(), Periodic(), Pml(cpml, cpml), Cpml())


def inside_z(g: Grid3d, test) -> np.ndarray:
    """Which E values' positions (E_c half a step along c) satisfy test(z)."""
    k = np.arange(g.nz, dtype=np.float64)
    mask = np.zeros((3, g.cells()), dtype=bool)
    for c in range(3):
        z = g.z0 + (k + (0.5 if c == 2 else 0.0)) * g.dz
        mask[c] = test(z)
    return mask


def transforms(series, dt, frequencies):
    """sum_n v_n e^{i w t_n} and sum_n t_n v_n e^{i w t_n}, t_n = (n + 1) dt (the probe's time)."""
    t = (np.arange(len(series)) + 1) * dt
    out = []
    for f in frequencies:
        w = np.exp(1j * TAU * f * t) * series
        out.append((w.sum(), (w * t).sum()))
    return out


def permittivity(medium: Dispersive, f: float) -> complex:
    w = TAU * f
    eps = complex(medium.eps_inf)
    for p in medium.poles:
        a, w0sq, gamma = p.parts()
        eps += a / complex(w0sq - w * w, -gamma * w)
    return eps


def column_run(g, b, medium, mask, source, probe, pulse, until):
    s = OracleSimulation(g, np.ones((3, g.cells())), b, 0.9, precision=64)
    if medium is not None:
        s.with_medium(medium, mask)
    s.add_source(Source(Field.E, Axis.X, (0, 0, source), pulse))
    p = s.add_probe(Field.E, Axis.X, (0, 0, probe))
    s.run(steps_until(s.dt, until))
    return s.probe(p), s.dt


# -- fdtd/drude-fresnel: src/fdtd/media_checks.rs:159-234 ---------------------------------------

@pytest.mark.parametrize("h,published", [(0.02, "6.9e-03"), (0.01, "1.6e-03"), (0.005, "3.0e-04")])
def test_drude_fresnel(h, published):
    cells = lambda x: int(round(x / h))  # noqa: E731
    cpml = cells(0.5)
    nz = 2 * cpml + cells(4.0)
    g, b = column(h, nz, cpml)
    face_node = cpml + cells(2.0)
    face = g.z0 + face_node * h - h / 2.0
    source, probe = cpml + cells(0.5), cpml + cells(1.5)
    metal = Dispersive(1.0, [Pole.drude(1.0, 0.05)])
    pulse = Waveform.pulse(1.0, 1.2)
    full, dt = column_run(g, b, metal, inside_z(g, lambda z: z > face), source, probe, pulse, 150.0)
    empty, _ = column_run(g, b, None, None, source, probe, pulse, 150.0)
    band = [0.4, 0.6, 0.8, 1.0, 1.2, 1.4, 1.6]
    s = transforms(full - empty, dt, band)
    i = transforms(empty, dt, band)
    distance = face - (g.z0 + probe * h)
    worst = 0.0
    for f, (sf, _), (ifq, _) in zip(band, s, i):
        w = TAU * f
        k = 2.0 / h * math.asin(math.sin(w * dt / 2.0) * h / dt)  # the grid's wavenumber
        r = sf / ifq * np.exp(-2j * k * distance)
        n = np.sqrt(permittivity(metal, f))
        worst = max(worst, abs(r - (1 - n) / (1 + n)))
    assert printed(worst) == published, worst


# -- fdtd/lorentz-group-delay: src/fdtd/media_checks.rs:236-329 ---------------------------------

@pytest.mark.parametrize("h,published", [(0.01, "3.0e-03"), (0.005, "8.8e-04"), (0.0025, "3.6e-04")])
def test_lorentz_group_delay(h, published):
    d = 10.0
    cells = lambda x: int(round(x / h))  # noqa: E731
    cpml = cells(0.5)
    nz = 2 * cpml + cells(d + 3.0)
    g, b = column(h, nz, cpml)
    front = g.z0 + (cpml + cells(1.5)) * h - h / 2.0
    back = front + d
    source, probe = cpml + cells(0.5), nz - cpml - cells(0.5)
    glass = Dispersive(2.25, [Pole.lorentz(1.0, 2.0, 0.02)])
    pulse = Waveform.pulse(1.0, 0.3)

    def n_of(f):
        return np.sqrt(permittivity(glass, f))

    def group_index(f):
        df = 1e-5 * f
        return (n_of(f) + f * (n_of(f + df) - n_of(f - df)) / (2 * df)).real

    ng = group_index(1.0)
    delay = pulse.params[2]  # the Gaussian's peak
    vacuum = delay + (g.z0 + probe * h) - (g.z0 + source * h)
    cut = vacuum + (ng - 1.0) * d + ng * d  # halfway to the first echo
    mask = inside_z(g, lambda z: (z > front) & (z < back))
    full, dt = column_run(g, b, glass, mask, source, probe, pulse, cut)
    empty, _ = column_run(g, b, None, None, source, probe, pulse, cut)
    band = [0.8, 0.9, 1.0, 1.1, 1.2]
    a, e = transforms(full, dt, band), transforms(empty, dt, band)

    def slope(dd, td):
        return (1j * td / dd).imag

    def first_pass(f):
        n = n_of(f)
        return 4 * n / ((1 + n) * (1 + n)) * np.exp(1j * TAU * f * d * (n - 1))

    worst = 0.0
    for f, (d1, t1), (d0, t0) in zip(band, a, e):
        measured = 1.0 + (slope(d1, t1) - slope(d0, t0)) / d
        df = 1e-5 * f
        exact = 1.0 + np.angle(first_pass(f + df) / first_pass(f - df)) / (TAU * 2 * df) / d
        worst = max(worst, abs(measured - exact))
    assert printed(worst) == published, worst
