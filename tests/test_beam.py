"""Gaussian beams (Simulation::add_beam, src/fdtd/sources.rs:598-714): the plane's paraxial E
decomposed into the grid's own plane waves, launched one way by currents on the surface.

CPU: the refusals of src/fdtd/tests.rs:402-434. GPU: the reference's beam fixture
(src/fdtd/checks.rs:845-913, test src/fdtd/tests.rs:306-346) against its published figures
(docs/validation.md, rows fdtd/beam-waist, fdtd/beam-divergence, fdtd/beam-tilt): a 2D beam of
1 um in vacuum, w0 = 1.5 um, its focus 2 um ahead, on 50 nm cells: the fitted waist 1.49999, the
divergence against the grid's own prediction within 1e-4 (measured 2.7e-6), almost nothing behind
the plane (< 1e-5), and tilted by 10 degrees, its centre's slope against the prediction within
1e-3 (measured 1.5e-4).
"""
import math

import numpy as np
import pytest

from photonoxide_b200.fdtd import Simulation
from photonoxide_b200.types import (Axis, Boundaries, Boxes, GaussianBeam, Grid3d, InvalidValue,
                                    Waveform)


def test_a_beam_that_cant_be_launched_as_asked_is_refused():
    g = Grid3d(40, 40, 1, 0.05, 0.05, 0.05, -1.0, -1.0, -0.025)
    block = Boxes(1.0).add((0.4, -math.inf, -math.inf), (math.inf, math.inf, math.inf), 4.0)
    s = Simulation(g, block, Boundaries.cpml_2d(6), 0.9)
    pulse = Waveform.pulse(1.0, 0.5)
    beam = GaussianBeam(Axis.Y, 10, True, (0.0, -0.5), 0.4, 0.0, Axis.Z, 0.0, False, 1.0)
    with pytest.raises(InvalidValue):  # no carrier
        s.add_beam(beam, Waveform.differentiated_gaussian(0.3, 1.5))
    with pytest.raises(InvalidValue):  # its plane crosses the block
        s.add_beam(beam, pulse)
    along_x = GaussianBeam(Axis.X, 10, True, (0.0, -0.5), 0.4, 0.0, Axis.Y, 0.0, False, 1.0)
    s.add_beam(along_x, pulse)
    towards_z = GaussianBeam(Axis.X, 10, True, (0.0, -0.5), 0.4, 0.0, Axis.Z, 0.2, False, 1.0)
    with pytest.raises(InvalidValue):  # tilted towards the axis that doesn't vary
        s.add_beam(towards_z, pulse)


def beam(angle, precision):
    """src/fdtd/checks.rs:845-913: the beam's width and centre at 2 to 14 um, and the largest
    |E_z| behind the plane relative to ahead of it."""
    h = 0.05
    g = Grid3d.centred((10 + 2 + 320 + 10, 460, 1), h)
    steps_per_period = 32
    courant = 1.0 / steps_per_period * math.sqrt(2.0) / h
    s = Simulation(g, Boxes(1.0), Boundaries.cpml_2d(10), courant, precision=precision)
    plane = 12
    s.add_beam(GaussianBeam(Axis.X, plane, True, (0.0, 0.0), 1.5, 2.0, Axis.Y, angle, False, 1.0),
               Waveform.continuous(1.0, 1.0, 4.0))
    s.run(32 * steps_per_period)
    # steady_amplitude (src/fdtd/checks.rs:646-667): 2/N sum of E e^(i omega t) over two periods
    omega = 2 * math.pi
    amp = np.zeros(g.cells(), complex)
    for _ in range(2 * steps_per_period):
        s.run(1)
        amp += s.e(2) * np.exp(1j * omega * s.steps * s.dt)
    ez = np.abs(amp * (2.0 / (2 * steps_per_period))).reshape(g.ny, g.nx)
    columns = []
    y = g.y0 + np.arange(g.ny) * h
    for d in (2.0, 5.0, 8.0, 11.0, 14.0):
        i = plane + int(round(d / h))
        p = ez[:, i] ** 2
        total, first, second = p.sum(), (p * y).sum(), (p * y * y).sum()
        centre = first / total
        columns.append((d, 2.0 * math.sqrt(second / total - centre * centre), centre))
    inner = ez[10:g.ny - 10, 10:g.nx - 10]
    behind = inner[:, :plane - 10].max()
    ahead = inner[:, plane - 10:].max()
    return columns, behind / ahead, s.dt


def beam_fit(columns):
    """src/fdtd/checks.rs:915-951: w^2 = w0^2 + theta^2 (d - d0)^2 by least squares."""
    a = np.zeros((3, 3))
    rhs = np.zeros(3)
    for d, w, _ in columns:
        p = np.array([1.0, d, d * d])
        a += np.outer(p, p)
        rhs += p * w * w
    c0, c1, c2 = np.linalg.solve(a, rhs)
    focus = -c1 / (2.0 * c2)
    return math.sqrt(c0 - c2 * focus * focus), focus, math.sqrt(c2)


def simpson(f, span, points=20000):
    step = 2.0 * span / points
    weighted = total = 0.0
    for i in range(points + 1):
        x = -span + i * step
        factor = 1.0 if i in (0, points) else (4.0 if i % 2 else 2.0)
        w, v = f(x)
        if v is not None:
            weighted += w * factor * v
        total += w * factor
    return weighted / total


def beam_divergence(waist, wavelength, h, dt):
    """src/fdtd/checks.rs:953-998 with the grid's dispersion."""
    omega = 2 * math.pi / wavelength
    tilde = 2.0 / dt * math.sin(omega * dt / 2.0)

    def f(ky):
        s = (tilde * h / 2.0) ** 2 - math.sin(ky * h / 2.0) ** 2
        v = None
        if s > 0.0:
            kx = 2.0 / h * math.asin(math.sqrt(s))
            v = (math.sin(ky * h) / math.sin(kx * h)) ** 2
        return math.exp(-ky * ky * waist * waist / 2.0), v
    return 2.0 * math.sqrt(simpson(f, 10.0 / waist))


def beam_centre_slope(waist, angle, wavelength, h, dt):
    """src/fdtd/checks.rs:1000-1036"""
    omega = 2 * math.pi / wavelength
    tilde = 2.0 / dt * math.sin(omega * dt / 2.0)
    span = min(10.0 / waist, 0.999 * tilde)
    weighted = total = 0.0
    points = 20000
    step = 2.0 * span / points
    for i in range(points + 1):
        kappa = -span + i * step
        phi = angle + math.asin(kappa / tilde)
        ky = tilde * math.sin(phi)
        s = (tilde * h / 2.0) ** 2 - math.sin(ky * h / 2.0) ** 2
        if s <= 0.0 or math.cos(phi) <= 0.0:
            continue
        kx = 2.0 / h * math.asin(math.sqrt(s))
        factor = 1.0 if i in (0, points) else (4.0 if i % 2 else 2.0)
        weight = (math.exp(-kappa * kappa * waist * waist / 2.0) * math.cos(phi - angle)
                  / math.cos(phi) * factor)
        weighted += weight * math.sin(ky * h) / math.sin(kx * h)
        total += weight
    return weighted / total


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [64, 32])
def test_a_gaussian_beam_keeps_its_waist_and_divergence(precision):
    columns, backward, dt = beam(0.0, precision)
    waist, focus, divergence = beam_fit(columns)
    on_grid = beam_divergence(1.5, 1.0, 0.05, dt)
    print(f"f{precision}: waist {waist:.6f}, focus {focus:.4f}, divergence {divergence:.6f} "
          f"(grid {on_grid:.6f}, relative {abs(divergence - on_grid) / on_grid:.2e}), "
          f"backward {backward:.2e}")
    assert abs(waist - 1.5) < 1e-3 and f"{waist:.5f}" == "1.49999"
    assert abs(focus - 2.0) < 0.1 and f"{focus:.2f}" == "1.94"
    assert abs(divergence - on_grid) < 1e-4 * on_grid
    assert f"{divergence:.6f}" == "0.218825"
    assert backward < 1e-5
    tilted, back, dt = beam(math.radians(10.0), precision)
    (d0, _, y0), (d1, _, y1) = tilted[0], tilted[4]
    slope = (y1 - y0) / (d1 - d0)
    predicted = beam_centre_slope(1.5, math.radians(10.0), 1.0, 0.05, dt)
    print(f"f{precision}: tilted slope {slope:.6f}, predicted {predicted:.6f} "
          f"({abs(slope - predicted) / predicted:.2e}), backward {back:.2e}")
    assert abs(slope - predicted) < 1e-3 * predicted and f"{slope:.4f}" == "0.1825"
