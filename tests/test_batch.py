"""The batch of 2D TE grids (photonoxide_b200.batch) against the oracle and against each grid run
alone: a grid stepped in a batch has the bits it has alone, which in f32 and f64 are the
oracle's (the reference's CPU step, src/fdtd/kernel/reference.rs)."""
import numpy as np
import pytest

from photonoxide_b200.batch import Batch
from photonoxide_b200.fdtd import Simulation
from photonoxide_b200.types import (INF, Axis, Boundaries, Boxes, Cpml, Current, Field,
                                    FluxPlane, Grid3d, InvalidValue, Periodic, Pml, Source,
                                    Waveform)
from pyoracle import OracleSimulation
from scenarios import noise, pulse

pytestmark = pytest.mark.gpu

# grids of uneven sizes and every edge kind along x and y
CASES = [
    ((70, 45), Boundaries(Pml(6, 5), Pml(4, 6), Periodic(), Cpml(kappa=2.0, alpha=0.3))),
    ((53, 29), Boundaries(Periodic(), Pml(6, 6), Periodic(), Cpml(kappa=2.0, alpha=0.3))),
    ((130, 40), Boundaries(Pml(8, 8), Periodic(), Periodic(), Cpml())),
    ((33, 70), Boundaries(Pml(0, 0), Pml(5, 0), Periodic(), Cpml(kappa=1.5, alpha=0.1))),
]


def te_busy(make, n, b, seed, precision):
    """A dielectric block and a lossy one, a conductor, TE random fields, point sources on H_z
    and E_y, a current on E_x and E_y, probes, a transform box and a flux plane."""
    g = Grid3d.centred((n[0], n[1], 1), 0.05)
    eps = Boxes(1.0).add((-0.4, -0.2, -INF), (0.3, 0.25, INF), 12.0)
    s = make(g, eps, b, 0.9, precision=precision)
    s.with_conductivity(Boxes(0.0).add((0.5, 0.3, -INF), (INF, INF, INF), 2.0))
    nx, ny = n
    r = np.arange(g.cells())
    s.set_field(Field.E, 0, 0.01 * noise(r + seed))
    s.set_field(Field.E, 1, 0.01 * noise(r + seed + 17))
    s.set_field(Field.H, 2, 0.01 * noise(r + seed + 50_000))
    s.conductor(Axis.X, (nx // 3, ny // 3, 0))
    mid = (nx // 2, ny // 2, 0)
    s.add_source(Source(Field.H, Axis.Z, mid, pulse()))
    s.add_source(Source(Field.E, Axis.Y, (nx // 4, ny // 2, 0),
                        Waveform.differentiated_gaussian(0.3, 1.2)))
    s.add_current(Current(Field.E, [(Axis.X, (nx // 2 + 2, ny // 2, 0), complex(0.5, -0.25)),
                                    (Axis.Y, (nx // 2 + 2, ny // 2, 0), complex(-0.3, 0.7))],
                          pulse()))
    # an H source on a tile's low edge and on the grid's last column and row (halo cases)
    s.add_source(Source(Field.H, Axis.Z, (31, ny - 1, 0), pulse()))
    s.add_source(Source(Field.H, Axis.Z, (nx - 1, 7, 0), pulse()))
    if nx > 124:  # the last column and row of a 124 x 7 tile
        s.add_source(Source(Field.H, Axis.Z, (123, 6, 0), pulse()))
    for at in [(3, 3, 0), (nx - 8, ny // 3, 0), mid]:
        s.add_probe(Field.E, Axis.Y, at)
        s.add_probe(Field.H, Axis.Z, at)
    freqs = [0.8, 1.0, 1.3]
    s.add_dft((nx // 2 - 6, ny // 2 - 4, 0), (nx // 2 + 6, ny // 2 + 4, 0), freqs)
    s.add_flux(FluxPlane(Axis.Y, ny - 12), freqs)
    return s


def fields(s):
    return [s.e(0), s.e(1), s.e(2), s.h(0), s.h(1), s.h(2)]


def same(a, b):
    for x, y in zip(fields(a), fields(b)):
        assert np.array_equal(x, y)
    for p in range(6):
        assert np.array_equal(a.probe(p), b.probe(p)), p
    assert np.array_equal(a.transforms(), b.transforms())
    assert np.array_equal(a.flux(0), b.flux(0))


# grids of widths a multiple of 4 (the row kernel's 16-byte path), over more than one tile
CASES4 = [
    ((136, 50), Boundaries(Periodic(), Pml(5, 5), Periodic(), Cpml())),
    ((252, 30), Boundaries(Pml(7, 6), Pml(4, 4), Periodic(), Cpml(kappa=2.0, alpha=0.3))),
    ((128, 23), Boundaries(Pml(5, 4), Periodic(), Periodic(), Cpml(kappa=1.5, alpha=0.1))),
]


@pytest.mark.parametrize("precision", [32, 64])
def test_batch_matches_the_oracle_and_each_grid_alone(precision):
    """500 steps: the first run times the seven tile shapes on 448 of them."""
    batch = [te_busy(Simulation, n, b, 100 * i, precision) for i, (n, b) in enumerate(CASES)]
    alone = [te_busy(Simulation, n, b, 100 * i, precision) for i, (n, b) in enumerate(CASES)]
    oracle = [te_busy(OracleSimulation, n, b, 100 * i, precision) for i, (n, b) in enumerate(CASES)]
    B = Batch(batch)
    B.run(500)
    assert B.tile != (0, 0)
    for s in alone + oracle:
        s.run(500)
    for x, y, z in zip(batch, alone, oracle):
        same(x, y)
        same(x, z)


@pytest.mark.parametrize("tile", [(32, 8), (32, 16), (64, 4), (64, 8), (128, 2), (128, 4),
                                  (124, 7)])
def test_every_tile_shape_gives_the_same_bits(tile):
    a = [te_busy(Simulation, n, b, 7 * i, 32) for i, (n, b) in enumerate(CASES)]
    o = [te_busy(Simulation, n, b, 7 * i, 32) for i, (n, b) in enumerate(CASES)]
    Batch(a, tile=tile).run(101)
    for s in o:
        s.run(101)
    for x, y in zip(a, o):
        same(x, y)


@pytest.mark.parametrize("precision", [32, 64])
def test_row_kernel_matches_the_oracle(precision):
    """The 124 x 7 row tiles on grids of every edge kind, with widths a multiple of 4 or not."""
    cases = CASES + CASES4
    a = [te_busy(Simulation, n, b, 11 * i, precision) for i, (n, b) in enumerate(cases)]
    o = [te_busy(OracleSimulation, n, b, 11 * i, precision) for i, (n, b) in enumerate(cases)]
    Batch(a, tile=(124, 7)).run(203)
    for s in o:
        s.run(203)
    for x, y in zip(a, o):
        same(x, y)


def test_runs_in_pieces_and_single_runs_in_between():
    """Batch runs of odd lengths (graph chunks and a remainder), then a grid on its own, then the
    batch again: the same bits as one grid run straight through."""
    a = [te_busy(Simulation, n, b, 3 * i, 32) for i, (n, b) in enumerate(CASES)]
    o = [te_busy(Simulation, n, b, 3 * i, 32) for i, (n, b) in enumerate(CASES)]
    B = Batch(a, tile=(64, 8))
    B.run(77)
    B.run(64)
    a[1].run(5)   # one grid alone for a while: its step count moves on
    for s in a[:1] + a[2:]:
        s.run(5)
    B.run(33)
    for s in o:
        s.run(179)
    for x, y in zip(a, o):
        same(x, y)


def test_refusals():
    g3 = Grid3d.centred((20, 20, 8), 0.05)
    s3 = Simulation(g3, Boxes(1.0), Boundaries.with_cpml(3), 0.9)
    with pytest.raises(InvalidValue):
        Batch([s3])
    g = Grid3d.centred((40, 30, 1), 0.05)
    tm = Simulation(g, Boxes(1.0), Boundaries.cpml_2d(4), 0.9)
    tm.set_field(Field.E, 2, np.ones(g.cells()))
    with pytest.raises(InvalidValue):
        Batch([tm]).run(4)
    src = Simulation(g, Boxes(1.0), Boundaries.cpml_2d(4), 0.9)
    src.add_source(Source(Field.E, Axis.Z, (20, 15, 0), pulse()))
    with pytest.raises(InvalidValue):
        Batch([src]).run(4)
    a = Simulation(g, Boxes(1.0), Boundaries.cpml_2d(4), 0.9)
    with pytest.raises(InvalidValue):
        Batch([a], tile=(48, 8))
