"""The oracle's Bloch sides (src/fdtd/bloch.rs): the fields' imaginary part stepped alongside,
the two parts coupled across the sides by e^(+-ikL), against the reference's published known
answer (docs/validation.md, row fdtd/bloch-multilayer; fixture src/cases/fdtd/bloch_checks.rs:
141-231): a pulse at a fixed k_x = 2 pi x 0.2 rad/um through 4 pairs of n = 2 (0.12 um) and
n = 1.5 (0.16 um), in a column one cell across, its transmittance at 0.7 to 1.3 c/um (each at
its own angle) against the transfer matrices': TE 2.0e-2, 4.9e-3, 1.2e-3 and TM 2.0e-2, 5.0e-3,
1.3e-3 at 20, 10 and 5 nm, second order in the cells.
"""
import math

import numpy as np
import pytest

from photonoxide_b200.types import (Axis, Bloch, Boundaries, Boxes, Cpml, Current, Field,
                                    Grid3d, InvalidValue, Pml, Waveform)

import pyoracle

STACK = [(2.0, 0.12), (1.5, 0.16)]
PAIRS = 4
KX = 2 * math.pi * 0.2
BAND = [0.7, 0.8, 0.9, 1.0, 1.1, 1.2, 1.3]


def transmittance(f, tm):
    """A lossless stack in vacuum at the angle sin(theta) = k_x / omega: the characteristic
    matrices' transmittance (J. Chilwell, I. Hodgkinson, JOSA A 1, 742 (1984))."""
    k = 2 * math.pi * f
    beta = KX / k  # the in-plane index in the vacuum cover
    cos0 = math.sqrt(1.0 - beta * beta)

    def admittance(n):
        c = np.sqrt(complex(n * n - beta * beta)) / n
        return n / c if tm else n * c

    m = np.eye(2, dtype=complex)
    for _ in range(PAIRS):
        for n, d in STACK:
            delta = k * d * np.sqrt(complex(n * n - beta * beta))
            y = admittance(n)
            m = m @ np.array([[np.cos(delta), 1j * np.sin(delta) / y],
                              [1j * y * np.sin(delta), np.cos(delta)]])
    y0 = 1.0 / cos0 if tm else cos0
    b, c = m @ np.array([1.0, y0])
    t = 2 * y0 / (y0 * b + c)
    return abs(t) ** 2


def multilayer(h, tm):
    """src/cases/fdtd/bloch_checks.rs:154-231 on the oracle: the largest |T - T_exact|."""
    cells = lambda x: int(round(x / h))  # noqa: E731
    cpml = cells(0.5)
    thickness = PAIRS * (STACK[0][1] + STACK[1][1])
    nz = 2 * cpml + cells(thickness + 2.0)
    g = Grid3d(1, 1, nz, h, h, h, 0.0, 0.0, 0.0)
    b = Boundaries(Bloch(KX), Bloch(0.0), Pml(cpml, cpml), Cpml())
    front = g.node(2, cpml + cells(1.0))
    # each layer's n^2 where front <= z < front + thickness (a closed face at v is the open
    # face at the double below v); the oracle averages it over each value's cell
    eps = Boxes(1.0)
    below = lambda v: math.nextafter(v, -math.inf)  # noqa: E731
    period = STACK[0][1] + STACK[1][1]
    for q in range(PAIRS):
        z0 = front + q * period
        eps.add((-math.inf, -math.inf, below(z0)), (math.inf, math.inf, z0 + STACK[0][1]),
                STACK[0][0] ** 2)
        eps.add((-math.inf, -math.inf, below(z0 + STACK[0][1])),
                (math.inf, math.inf, z0 + period), STACK[1][0] ** 2)
    comp = Axis.X if tm else Axis.Y
    source, probe = cpml + cells(0.4), nz - cpml - cells(0.4)
    pulse = Waveform.pulse(1.0, 0.3)

    def run(with_stack):
        s = pyoracle.OracleSimulation(g, eps if with_stack else Boxes(1.0), b, 0.9)
        assert s.is_complex
        s.add_current(Current(Field.E, [(comp, (0, 0, source), 1.0 + 0.0j)], pulse))
        p = s.add_probe(Field.E, comp, (0, 0, probe))
        steps = 0
        while steps * s.dt < 300.0:
            steps += 1
        s.run(steps)
        return s.probe_complex(p), s.dt

    (full, dt), (empty, _) = run(True), run(False)
    t = (np.arange(len(full)) + 1) * dt
    worst = 0.0
    for f in BAND:
        w = np.exp(1j * 2 * math.pi * f * t)
        measured = abs((full * w).sum() / (empty * w).sum()) ** 2
        worst = max(worst, abs(measured - transmittance(f, tm)))
    return worst


@pytest.mark.parametrize("tm, published", [(False, [2.0e-2, 4.9e-3, 1.2e-3]),
                                           (True, [2.0e-2, 5.0e-3, 1.3e-3])])
def test_a_multilayer_at_oblique_incidence_through_bloch_sides(tm, published):
    before = pyoracle.threads(1)  # a column of a few hundred cells: one thread is fastest
    try:
        errors = [multilayer(h, tm) for h in (0.02, 0.01, 0.005)]
    finally:
        pyoracle.threads(before)
    print(("TM" if tm else "TE"), ", ".join(f"{e:.2g}" for e in errors))
    assert [float(f"{e:.2g}") for e in errors] == published


def test_a_complex_run_refuses_a_plane_wave_and_a_real_run_is_real():
    from photonoxide_b200.types import PlaneWave
    g = Grid3d(20, 1, 30, 0.05, 0.05, 0.05)
    s = pyoracle.OracleSimulation(g, Boxes(1.0), Boundaries(Bloch(1.3), Bloch(0.0), Pml(5, 5),
                                                            Cpml()), 0.9)
    assert s.is_complex
    with pytest.raises(InvalidValue):
        s.add_plane_wave(PlaneWave((0, 0, 8), (20, 1, 20), (0, 0, 1), (1.0, 0.0, 0.0), 1.0,
                                   Waveform.pulse(1.0, 0.5)))
    real = pyoracle.OracleSimulation(g, Boxes(1.0), Boundaries(Bloch(0.0), Bloch(0.0),
                                                               Pml(5, 5), Cpml()), 0.9)
    assert not real.is_complex
