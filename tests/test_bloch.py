"""Bloch sides on the engine (src/fdtd/bloch.rs): a complex run's real and imaginary parts as two
contexts stepped together, coupled across the sides after each half step (H's couplings as
injections in the step kernels, E's by a pass after them), the monitors transforming both parts.

CPU: the host library's complex set-up (the time step's Bloch bound, the refusals) against the
oracle's. GPU: the f64 engine against the f64 oracle (itself pinned to the reference's published
multilayer transmittance), bit for bit: the reference's Bloch fixture (src/cases/fdtd/
bloch_checks.rs:47-139: two Bloch sides, walls, conductivity, a continuous current and a dipole
restricted across the sides, with and without Drude and Lorentz media), a transform monitor, and
the multilayer column; and the f32 engine near the f64 one.
"""
import math

import numpy as np
import pytest

from photonoxide_b200.fdtd import Simulation
from photonoxide_b200.types import (Axis, Bloch, Boundaries, Boxes, Cpml, Current, Dipole,
                                    Dispersive, Field, GaussianBeam, Grid3d, InvalidValue, Pml,
                                    PlaneWave, Pole, Waveform)

import pyoracle


def fixture():
    h, n = 0.05, (16, 14, 12)
    g = Grid3d.centred(n, h)
    b = Boundaries(Bloch(1.3), Bloch(-2.1), Pml(0, 0), Cpml())
    dt = 1.55 / 64
    courant = dt * math.sqrt(3.0 / (h * h))
    return g, b, courant


def test_the_host_builds_a_complex_run_as_the_oracle_does():
    g, b, courant = fixture()
    s = Simulation(g, Boxes(2.1), b, courant)
    o = pyoracle.OracleSimulation(g, Boxes(2.1), b, courant)
    assert s.is_complex and o.is_complex
    assert s.dt == o.dt
    for which in (0, 1, 2, 3, 4):
        assert np.array_equal(s.tables(which), o.tables(which)), which
    # one cell along a Bloch axis: the time step counts sin^2(k h / 2)
    col = Grid3d(1, 1, 40, 0.01, 0.01, 0.01)
    cb = Boundaries(Bloch(1.2566), Bloch(0.0), Pml(5, 5), Cpml())
    assert Simulation(col, Boxes(1.0), cb, 0.9).dt == pyoracle.OracleSimulation(
        col, Boxes(1.0), cb, 0.9).dt
    pulse = Waveform.pulse(1.0, 0.5)
    with pytest.raises(InvalidValue):
        s.add_plane_wave(PlaneWave((0, 0, 3), (16, 14, 8), (0, 0, 1), (1.0, 0.0, 0.0), 1.0,
                                   pulse))
    with pytest.raises(InvalidValue):
        s.add_beam(GaussianBeam(Axis.Z, 3, True, (0.0, 0.0), 0.3, 0.0, Axis.X, 0.0, False, 1.0),
                   pulse)
    real = Simulation(g, Boxes(2.1), Boundaries(Bloch(0.0), Bloch(0.0), Pml(0, 0), Cpml()),
                      courant)
    assert not real.is_complex


def drude_lorentz():
    return Dispersive(2.0, [Pole.drude(0.8, 0.05), Pole.lorentz(1.5, 0.7, 0.08)])


def setup(cls, precision, dispersive):
    g, b, courant = fixture()
    s = cls(g, Boxes(2.1), b, courant, precision=precision)
    s.with_conductivity(Boxes(2.0))
    if dispersive:
        s.with_medium(drude_lorentz(), Boxes(0.0).add((-1, -1, -1), (1, 1, 1), 1.0))
    wave = Waveform.continuous(1.0 / 1.55, 1.0, 6.0 * 1.55)
    at = (g.nx // 2 + 1, g.ny // 2, g.nz // 2)
    s.add_current(Current(Field.E, [(Axis.Y, at, 1.0 + 0.0j)], wave))
    s.add_dipole(Dipole(Field.E, Axis.Z, (g.x0 + (g.nx - 0.3) * g.dx, g.y0 - 0.2 * g.dy, 0.017),
                        0.002 + 0.001j, wave))
    p = s.add_probe(Field.E, Axis.Z, (g.nx - 1, 0, g.nz // 2))
    return s, p


@pytest.mark.gpu
@pytest.mark.parametrize("dispersive", [False, True])
def test_the_bloch_fixture_is_the_oracles_bits(dispersive):
    ours, p = setup(Simulation, 64, dispersive)
    ref, q = setup(pyoracle.OracleSimulation, 64, dispersive)
    for chunk in (70, 130):
        ours.run(chunk)
        ref.run(chunk)
        for c in range(3):
            assert np.array_equal(ours.e(c), ref.e(c)), ("E", c)
            assert np.array_equal(ours.h(c), ref.h(c)), ("H", c)
            assert np.array_equal(ours.e_imaginary(c), ref.e_imaginary(c)), ("E im", c)
            assert np.array_equal(ours.h_imaginary(c), ref.h_imaginary(c)), ("H im", c)
        assert np.array_equal(ours.probe_complex(p), ref.probe_complex(q))
    assert np.max(np.abs(ours.e_imaginary(1))) > 0.0


@pytest.mark.gpu
def test_a_complex_runs_transforms_are_the_oracles_bits():
    g, b, courant = fixture()
    runs = []
    for cls in (Simulation, pyoracle.OracleSimulation):
        s, _ = setup(cls, 64, False)
        s.add_dft((0, 0, 0), (g.nx - 1, g.ny - 1, g.nz - 1), [1.0 / 1.55, 0.7])
        s.run(150)
        runs.append(np.asarray(s.transforms()))
    assert np.array_equal(runs[0], runs[1])


@pytest.mark.gpu
def test_f32_stays_near_f64():
    ours, p = setup(Simulation, 32, True)
    ref, q = setup(Simulation, 64, True)
    ours.run(300)
    ref.run(300)
    for c in range(3):
        for a, b in ((ours.e(c), ref.e(c)), (ours.e_imaginary(c), ref.e_imaginary(c))):
            assert np.max(np.abs(a - b)) <= 1e-4 * np.max(np.abs(b))


@pytest.mark.gpu
def test_the_multilayer_column_is_the_oracles_bits():
    h = 0.02
    from test_oracle_bloch import KX, STACK, PAIRS
    cells = lambda x: int(round(x / h))  # noqa: E731
    cpml = cells(0.5)
    nz = 2 * cpml + cells(PAIRS * (STACK[0][1] + STACK[1][1]) + 2.0)
    g = Grid3d(1, 1, nz, h, h, h, 0.0, 0.0, 0.0)
    b = Boundaries(Bloch(KX), Bloch(0.0), Pml(cpml, cpml), Cpml())
    eps = Boxes(1.0).add((-1, -1, 1.5), (1, 1, 2.2), 4.0)
    series = []
    for cls in (Simulation, pyoracle.OracleSimulation):
        s = cls(g, eps, b, 0.9, precision=64)
        s.add_current(Current(Field.E, [(Axis.Y, (0, 0, cpml + cells(0.4)), 1.0 + 0.0j)],
                              Waveform.pulse(1.0, 0.3)))
        p = s.add_probe(Field.E, Axis.Y, (0, 0, nz - cpml - cells(0.4)))
        s.run(3000)
        series.append(s.probe_complex(p))
    assert np.array_equal(series[0], series[1])
    assert np.max(np.abs(series[0].imag)) > 0.0
