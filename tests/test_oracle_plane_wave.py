"""The oracle's total-field/scattered-field plane wave (src/fdtd/sources.rs:716-1041) against the
reference's published known answers (docs/validation.md, rows fdtd/tfsf-leakage and
fdtd/tfsf-slab; fixtures src/fdtd/checks.rs:511-640, tests src/fdtd/tests.rs:251-274):

- an empty box in vacuum leaks nothing but round-off at normal and oblique incidence, 2D and 3D
  (the largest scattered field over the run relative to the largest incident one: <= 1e-12,
  measured 1.3e-15);
- a slab of eps = 4, 0.3 um thick, in a box at normal incidence reflects as Airy's formula says,
  to second order in the cells: 5.4e-3, 1.3e-3 and 3.3e-4 at 20, 10 and 5 nm.

And the refusals of src/fdtd/tests.rs:346-400.
"""
import math

import numpy as np
import pytest

from photonoxide_b200.types import (Axis, Boundaries, Boxes, Cpml, Field, Grid3d, InvalidValue,
                                    Periodic, PlaneWave, Pml, Waveform)

import pyoracle


def twice(field, comp, axis, m):
    half = (comp == axis) if field == Field.E else (comp != axis)
    return 2 * m + (1 if half else 0)


def in_box_mask(field, comp, n, low, high):
    """src/fdtd/checks.rs:495-509 over every value of a component (an axis of one cell is whole)."""
    idx = np.indices((n[2], n[1], n[0]))  # k, j, i
    at = [idx[2], idx[1], idx[0]]
    mask = np.ones((n[2], n[1], n[0]), dtype=bool)
    for a in range(3):
        if n[a] == 1:
            continue
        half = (comp == a) if field == Field.E else (comp != a)
        t = 2 * at[a] + (1 if half else 0)
        mask &= (t >= 2 * low[a]) & (t <= 2 * high[a])
    return mask.reshape(-1)


def tfsf_leakage(direction, polarization, three_d):
    """src/fdtd/checks.rs:511-562"""
    h = 0.05
    if three_d:
        n, low, high, cpml = (36, 36, 36), (12, 12, 12), (24, 24, 24), 8
        b = Boundaries.with_cpml(cpml)
    else:
        n, low, high, cpml = (80, 80, 1), (25, 25, 0), (55, 55, 1), 10
        b = Boundaries.cpml_2d(cpml)
    g = Grid3d.centred(n, h)
    s = pyoracle.OracleSimulation(g, Boxes(1.0), b, 0.9)
    s.add_plane_wave(PlaneWave(low, high, direction, polarization, 1.0,
                               Waveform.pulse(1.0, 0.6)))
    masks = {(f, c): in_box_mask(f, c, n, low, high) for f in (Field.E, Field.H) for c in range(3)}
    leak = largest = 0.0
    for _ in range(int(12.0 / s.dt)):
        s.run(1)
        for (f, c), m in masks.items():
            v = np.abs(s.e(c) if f == Field.E else s.h(c))
            largest = max(largest, float(v[m].max()))
            if (~m).any():
                leak = max(leak, float(v[~m].max()))
    return leak / largest


@pytest.mark.parametrize("direction, polarization, three_d", [
    ((1, 0, 0), (0.0, 0.0, 1.0), False),
    ((2, 1, 0), (0.0, 0.0, 1.0), False),
    ((1, -3, 0), (1.0, 0.0, 0.0), False),
    ((0, 0, 1), (1.0, 0.0, 0.0), True),
    ((2, 1, 1), (1.0, -1.0, 0.0), True),
])
def test_an_empty_box_leaks_only_round_off(direction, polarization, three_d):
    leak = tfsf_leakage(direction, polarization, three_d)
    print(f"{direction} {polarization}: leakage {leak:.2e}")
    assert leak < 1e-12


def tfsf_slab(h):
    """src/fdtd/checks.rs:568-640: the largest |R_measured - R_Airy| at 0.8, 1 and 1.2 c/um."""
    thickness, eps_slab = 0.3, 4.0
    cells = lambda x: int(round(x / h))  # noqa: E731 (x / h > 0: half-way cases don't arise)
    cpml = cells(0.5)
    nz = 2 * cpml + cells(2.4)
    g = Grid3d(1, 1, nz, h, h, h, 0.0, 0.0, 0.0)
    low, high = cpml + cells(0.4), nz - cpml - cells(0.4)
    za = g.node(2, low + cells(0.5))
    zb = za + thickness
    b = Boundaries(Periodic(), Periodic(), Pml(cpml, cpml), Cpml())
    # z >= za and z < zb: the open box from the double below za
    eps = Boxes(1.0).add((-math.inf, -math.inf, math.nextafter(za, -math.inf)),
                         (math.inf, math.inf, zb), eps_slab)
    s = pyoracle.OracleSimulation(g, eps, b, 0.9)
    wave = s.add_plane_wave(PlaneWave((0, 0, low), (1, 1, high), (0, 0, 1), (1.0, 0.0, 0.0), 1.0,
                                      Waveform.pulse(1.0, 0.8)))
    front, inside = low - cells(0.2), (0, 0, low + 2)
    freqs = np.array([0.8, 1.0, 1.2])
    scattered = np.zeros(3, complex)
    incident = np.zeros(3, complex)
    for _ in range(int(30.0 / s.dt)):
        s.run(1)
        t = s.steps * s.dt
        es = s.e(0)[front]
        ei = s.incident(wave, Field.E, Axis.X, inside)
        w = np.exp(1j * 2 * math.pi * freqs * t)
        scattered += es * w
        incident += ei * w
    measured = np.abs(scattered / incident) ** 2
    n2 = math.sqrt(eps_slab)
    r12 = (1.0 - n2) / (1.0 + n2)
    phase = np.exp(1j * 2.0 * n2 * 2 * math.pi * freqs * thickness)
    r = r12 * (1.0 - phase) / (1.0 - r12 * r12 * phase)
    return float(np.max(np.abs(measured - np.abs(r) ** 2)))


def test_a_slab_reflects_as_airys_formula_to_second_order():
    errors = [tfsf_slab(h) for h in (0.02, 0.01, 0.005)]
    print("slab:", ", ".join(f"{e:.2g}" for e in errors))
    # the reference's measured 5.4e-3, 1.3e-3 and 3.3e-4, to the digits it prints
    assert [float(f"{e:.2g}") for e in errors] == [5.4e-3, 1.3e-3, 3.3e-4]
    assert errors[1] < errors[0] / 3.0 and errors[2] < errors[1] / 3.0


def test_sources_that_cant_be_launched_as_asked_are_refused():
    """src/fdtd/tests.rs:346-400"""
    g = Grid3d(40, 40, 1, 0.05, 0.05, 0.05, -1.0, -1.0, -0.025)
    block = Boxes(1.0).add((0.4, -math.inf, -math.inf), (math.inf, math.inf, math.inf), 4.0)
    s = pyoracle.OracleSimulation(g, block, Boundaries.cpml_2d(6), 0.9)
    pulse = Waveform.pulse(1.0, 0.5)

    def wave(low, high, direction, pol=(0.0, 0.0, 1.0)):
        return PlaneWave(low, high, direction, pol, 1.0, pulse)

    assert s.add_plane_wave(wave((10, 10, 0), (25, 25, 1), (2, 1, 0))) == 0
    for bad in [wave((5, 10, 0), (25, 25, 1), (1, 0, 0)), wave((6, 10, 0), (25, 25, 1), (1, 0, 0)),
                wave((10, 10, 0), (25, 25, 0), (1, 0, 0)), wave((10, 10, 0), (25, 25, 1), (1, 0, 1)),
                wave((10, 10, 0), (30, 25, 1), (1, 0, 0)),
                wave((10, 10, 0), (25, 25, 1), (1, 0, 0), (1.0, 0.0, 0.0)),
                wave((10, 10, 0), (25, 25, 1), (0, 0, 0))]:
        with pytest.raises(InvalidValue):
            s.add_plane_wave(bad)
