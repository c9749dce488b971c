"""Total-field/scattered-field plane waves on the engine (Simulation::add_plane_wave,
src/fdtd/sources.rs:716-1041): the box's couplings are injections whose incident values an
auxiliary 1D run, stepped on the device with the grid, records each step.

CPU: the host library refuses what the reference refuses (src/fdtd/tests.rs:346-400) and accepts
the rest, with no GPU. GPU: in f64 the fields, the incident field and the slab's reflection are
the oracle's bits (itself pinned to the reference's published leakage and Airy numbers); in f32
an empty box in vacuum leaks at f32 round-off and the slab reflects as the oracle's within 1e-4.
"""
import math

import numpy as np
import pytest

from photonoxide_b200.fdtd import Simulation
from photonoxide_b200.types import (Axis, Boundaries, Boxes, Cpml, Dipole, Field, Grid3d,
                                    InvalidValue, Periodic, PlaneWave, Pml, Waveform)

import pyoracle


def test_the_host_refuses_what_the_reference_refuses():
    g = Grid3d(40, 40, 1, 0.05, 0.05, 0.05, -1.0, -1.0, -0.025)
    block = Boxes(1.0).add((0.4, -math.inf, -math.inf), (math.inf, math.inf, math.inf), 4.0)
    s = Simulation(g, block, Boundaries.cpml_2d(6), 0.9)
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
    assert s.incident(0, Field.E, Axis.Z, (12, 12, 0)) == 0.0  # nothing launched yet


def box_case(three_d, direction, polarization):
    """The reference's leakage fixture (src/fdtd/checks.rs:511-562) with a dipole outside the
    box and a dielectric block inside it, so that both sides carry fields."""
    h = 0.05
    if three_d:
        n, low, high, b = (36, 36, 36), (12, 12, 12), (24, 24, 24), Boundaries.with_cpml(8)
    else:
        n, low, high, b = (80, 80, 1), (25, 25, 0), (55, 55, 1), Boundaries.cpml_2d(10)
    g = Grid3d.centred(n, h)
    inner = 0.15 if three_d else 0.4
    eps = Boxes(1.0).add((-inner, -inner, -inner if three_d else -math.inf),
                         (inner, inner, inner if three_d else math.inf), 2.25)
    wave = PlaneWave(low, high, direction, polarization, 1.0, Waveform.pulse(1.0, 0.6))
    return g, eps, b, wave


def run_pair(cls, precision, g, eps, b, wave, steps):
    s = cls(g, eps, b, 0.9, precision=precision)
    n = s.add_plane_wave(wave)
    at = (0.4, 0.38, 0.02) if g.nz > 1 else (1.0, 0.9, 0.0)
    s.add_dipole(Dipole(Field.E, Axis.Y, at, 0.01 + 0.002j, Waveform.pulse(0.9, 0.4)))
    s.run(steps)
    return s, n


@pytest.mark.gpu
@pytest.mark.parametrize("three_d, direction, polarization", [
    (False, (1, -3, 0), (1.0, 0.0, 0.0)),
    (True, (2, 1, 1), (1.0, -1.0, 0.0)),
    (True, (0, 0, 1), (1.0, 0.0, 0.0)),
])
def test_a_box_on_the_engine_is_the_oracles_bits(three_d, direction, polarization):
    g, eps, b, wave = box_case(three_d, direction, polarization)
    steps = 300
    ours, n = run_pair(Simulation, 64, g, eps, b, wave, steps)
    ref, m = run_pair(pyoracle.OracleSimulation, 64, g, eps, b, wave, steps)
    for c in range(3):
        assert np.array_equal(ours.e(c), ref.e(c)), ("E", c)
        assert np.array_equal(ours.h(c), ref.h(c)), ("H", c)
    for at in [(g.nx // 2, g.ny // 2, g.nz // 2), (14, 20, 0 if not three_d else 13)]:
        for f in (Field.E, Field.H):
            for c in range(3):
                assert ours.incident(n, f, c, at) == ref.incident(m, f, c, at)
    # the run goes on from where it stopped: a second run, and a re-configuration (a probe
    # added) that carries the auxiliary run's state to the engine again
    ours.add_probe(Field.E, Axis.X, (g.nx // 2, g.ny // 2, g.nz // 2))
    ref.add_probe(Field.E, Axis.X, (g.nx // 2, g.ny // 2, g.nz // 2))
    ours.run(100)
    ref.run(100)
    assert np.array_equal(ours.probe(0), ref.probe(0))
    for c in range(3):
        assert np.array_equal(ours.e(c), ref.e(c))


@pytest.mark.gpu
def test_an_empty_box_in_f32_leaks_at_f32_round_off():
    g = Grid3d.centred((36, 36, 36), 0.05)
    low, high = (12, 12, 12), (24, 24, 24)
    s = Simulation(g, Boxes(1.0), Boundaries.with_cpml(8), 0.9, precision=32)
    s.add_plane_wave(PlaneWave(low, high, (2, 1, 1), (1.0, -1.0, 0.0), 1.0,
                               Waveform.pulse(1.0, 0.6)))
    idx = np.indices((36, 36, 36))
    leak = largest = 0.0
    for _ in range(int(12.0 / s.dt) // 40):
        s.run(40)
        for f in (Field.E, Field.H):
            for c in range(3):
                v = np.abs(s.e(c) if f == Field.E else s.h(c)).reshape(36, 36, 36)
                mask = np.ones((36, 36, 36), bool)
                for a, ax in enumerate((2, 1, 0)):  # idx[0] is k (z), idx[2] is i (x)
                    half = (c == a) if f == Field.E else (c != a)
                    t = 2 * idx[ax] + (1 if half else 0)
                    mask &= (t >= 2 * low[a]) & (t <= 2 * high[a])
                largest = max(largest, float(v[mask].max()))
                leak = max(leak, float(v[~mask].max()))
    print(f"f32 leakage {leak / largest:.2e}")
    assert leak / largest < 1e-5


def slab(cls, precision, h):
    """src/fdtd/checks.rs:568-640 at cells of h: the scattered and incident fields' transforms at
    0.8, 1 and 1.2 c/um."""
    cells = lambda x: int(round(x / h))  # noqa: E731
    cpml = cells(0.5)
    nz = 2 * cpml + cells(2.4)
    g = Grid3d(1, 1, nz, h, h, h, 0.0, 0.0, 0.0)
    low, high = cpml + cells(0.4), nz - cpml - cells(0.4)
    za = g.node(2, low + cells(0.5))
    eps = Boxes(1.0).add((-math.inf, -math.inf, math.nextafter(za, -math.inf)),
                         (math.inf, math.inf, za + 0.3), 4.0)
    s = cls(g, eps, Boundaries(Periodic(), Periodic(), Pml(cpml, cpml), Cpml()), 0.9,
            precision=precision)
    n = s.add_plane_wave(PlaneWave((0, 0, low), (1, 1, high), (0, 0, 1), (1.0, 0.0, 0.0), 1.0,
                                   Waveform.pulse(1.0, 0.8)))
    front = s.add_probe(Field.E, Axis.X, (0, 0, low - cells(0.2)))
    steps = int(30.0 / s.dt)
    inc = np.empty(steps)
    for q in range(steps):  # the incident field at a value inside, after each step
        s.run(1)
        inc[q] = s.incident(n, Field.E, Axis.X, (0, 0, low + 2))
    es = np.asarray(s.probe(front))
    t = (np.arange(steps) + 1) * s.dt
    w = np.exp(1j * 2 * math.pi * np.array([0.8, 1.0, 1.2])[:, None] * t[None, :])
    return es, inc, np.abs((w * es).sum(1) / (w * inc).sum(1)) ** 2


@pytest.mark.gpu
def test_the_slab_is_the_oracles_bits_and_reflects_as_airy():
    es, inc, r = slab(Simulation, 64, 0.02)
    es_ref, inc_ref, r_ref = slab(pyoracle.OracleSimulation, 64, 0.02)
    assert np.array_equal(es, es_ref) and np.array_equal(inc, inc_ref)
    es32, _, r32 = slab(Simulation, 32, 0.02)
    print("slab reflection f64", r, "f32", r32)
    assert np.max(np.abs(r32 - r)) < 1e-4
