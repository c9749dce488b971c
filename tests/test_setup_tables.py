"""The engine's host library builds the reference's setup tables bit for bit: the averaged
permittivity, the time step, ca/cb with walls, conductivity and conductors, kappa/h and the CPML
slabs' recursions (src/fdtd.rs:570-869, 945-1008). No device is touched before the first run."""
import numpy as np
import pytest

from photonoxide_b200.fdtd import Simulation, average
from photonoxide_b200.types import (INF, Axis, Boundaries, Boxes, Cpml, Dispersive, Grid3d, Pml,
                                    Periodic, Pole)
from pyoracle import OracleSimulation, average_boxes
from scenarios import busy, closed, stirred


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a, b)


@pytest.mark.parametrize("two_d", [False, True])
def test_busy_tables_bitwise(two_d):
    p = busy(lambda *a: Simulation(*a, precision=64), two_d)
    o = busy(lambda *a: OracleSimulation(*a, precision=64), two_d)
    assert p.dt == o.dt
    for which in range(5):
        assert same(p.tables(which), o.tables(which)), which


def test_stirred_and_closed_tables_bitwise():
    for make_p, make_o in [
        (lambda m: stirred(m, periodic_axes=(0,)), lambda m: stirred(m, periodic_axes=(0,))),
        (lambda m: stirred(m, periodic_axes=(1, 2)), lambda m: stirred(m, periodic_axes=(1, 2))),
        (closed, closed),
    ]:
        p = make_p(lambda *a: Simulation(*a))
        o = make_o(lambda *a: OracleSimulation(*a))
        assert p.dt == o.dt
        for which in range(5):
            assert same(p.tables(which), o.tables(which)), which


def test_average_fast_path_is_the_full_average():
    """The host averages only the cells a box's face crosses; every other cell's value is the
    full 8^3-sample average's, bit for bit."""
    g = Grid3d(41, 23, 9, 0.02, 0.025, 0.03, -0.4, -0.3, -0.12)
    geo = (Boxes(1.444 ** 2)
           .add((-INF, -0.11, -0.05), (0.1, 0.11, 0.06), 3.48 ** 2)
           .add((0.0, -0.2, -INF), (0.31, 0.2, 0.0), 2.1)
           .add((0.02, 0.02, 0.02), (0.04, 0.04, 0.04), 7.0))
    assert same(average(g, geo), average_boxes(g, geo))


def test_refusals_as_the_reference():
    g = Grid3d.centred((10, 10, 10), 0.05)
    eps = np.ones((3, g.cells()))
    from photonoxide_b200.types import InvalidValue
    with pytest.raises(InvalidValue):
        Simulation(g, eps, Boundaries.with_cpml(5), 0.9)  # CPMLs fill the axis
    with pytest.raises(InvalidValue):
        Simulation(g, eps, Boundaries.walls(), 1.5)  # Courant number above 1
    with pytest.raises(InvalidValue):
        Simulation(g, -eps, Boundaries.walls(), 0.9)  # permittivity not positive
    with pytest.raises(InvalidValue):
        Simulation(g, eps, Boundaries(Pml(1, 1), Pml(1, 1), Pml(1, 1), Cpml(kappa=0.5)), 0.9)
    s = Simulation(g, eps, Boundaries.walls(), 0.9)
    with pytest.raises(InvalidValue):
        s.add_probe(0, 0, (10, 0, 0))
    with pytest.raises(InvalidValue):
        s.add_dft((0, 0, 0), (3, 3, 3), [1.0 / s.dt])  # beyond Nyquist


def overlapping_media(make):
    """Seeded random Drude and two-pole Lorentz boxes that overlap one another and a conductivity
    region, a conductor, and a medium given by a mask: every value a later medium takes leaves the
    group it was in (src/fdtd/media.rs:641-653, 749-825)."""
    rng = np.random.default_rng(3)
    g = Grid3d.centred((40, 34, 22), 0.02)
    s = make(g, Boxes(1.0).add((-0.1, -0.1, -INF), (0.12, 0.08, INF), 2.5), Boundaries.with_cpml(4),
             0.5)
    s.with_conductivity(Boxes(0.0).add((0.0, -INF, -INF), (INF, 0.05, INF), 0.7))
    drude, lorentz = Boxes(0.0), Boxes(0.0)
    for q in range(14):
        lo = rng.uniform(-0.4, 0.2, 3) * np.array([1.0, 1.0, 0.5])
        hi = lo + rng.uniform(0.05, 0.3, 3)
        (drude if q % 2 else lorentz).add(tuple(lo), tuple(hi), 1.0)
    s.with_medium(Dispersive(1.0, [Pole.drude(7.27, 0.0531)]), drude)
    s.with_medium(Dispersive(2.25, [Pole.lorentz(1.2, 0.7, 0.01), Pole.lorentz(0.6, 0.45, 0.02)]),
                  lorentz)
    mask = np.zeros((3, g.cells()), dtype=np.uint8)
    mask[1, ::7] = 1
    s.with_medium(Dispersive(1.5, [Pole.lorentz(0.8, 0.9, 0.03)]), mask)
    s.conductor(Axis.Y, (20, 17, 11))
    return s


def test_media_tables_bitwise():
    p = overlapping_media(lambda *a: Simulation(*a, precision=64))
    o = overlapping_media(lambda *a: OracleSimulation(*a, precision=64))
    for which in (0, 1, 5):
        assert same(p.tables(which), o.tables(which)), which
    assert len(p.tables(5)) > 1000
