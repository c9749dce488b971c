"""The CUDA engine against the oracle on the same inputs.

- Without sources, the engine's f64 and f32 arithmetic IS the oracle's (the reference's CPU
  kernel, src/fdtd/kernel/reference.rs, and its f32 `Yee<f32>`): fields equal bit for bit, on
  every boundary kind (CPML with kappa and alpha, walls, periodic sides, 2D).
- With sources and monitors too: the device evaluates the waveforms and the transforms' phases
  in f64 with the reference's own exp and sincos algorithms (photonoxide_b200/csrc/portable.h),
  accumulates the transforms in f64 in time order, and adds each source's amount where the CPU
  step does. So the f64 engine's fields, probes, transforms and fluxes are the oracle's bits, and
  the f32 engine's are the oracle's f32 bits; against the f64 oracle the f32 engine is within the
  reference's GPU tolerance, 2e-5 over 800 steps (src/fdtd/gpu/tests.rs:51-66).
"""
import numpy as np
import pytest

from photonoxide_b200.fdtd import Simulation
from photonoxide_b200.types import (INF, Axis, Boundaries, Boxes, Dispersive, Field, Grid3d,
                                    Periodic, Pole, Source, Waveform)
from pyoracle import OracleSimulation
from scenarios import busy, closed, noise, stirred

pytestmark = pytest.mark.gpu


def relative(a, b):
    """The largest difference of a from b, relative to the largest of b (gpu/checks.rs:16-23)."""
    a, b = np.asarray(a), np.asarray(b)
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a)))


def fields(s):
    return [s.e(c) for c in range(3)] + [s.h(c) for c in range(3)]


# grid sizes: 33 along x takes the plain kernel; 36 and 68 (multiples of 4) the staged one, with
# partial tiles along x and y, and several tiles and planes split among CTAs
SIZES = [(33, 18, 11), (36, 18, 11), (68, 35, 12)]


@pytest.mark.parametrize("precision", [32, 64])
@pytest.mark.parametrize("periodic", [(), (0,), (1,), (2,), (0, 1), (0, 1, 2)])
@pytest.mark.parametrize("n", SIZES)
def test_stirred_bit_for_bit(precision, periodic, n):
    p = stirred(lambda *a: Simulation(*a, precision=precision), periodic_axes=periodic, n=n)
    o = stirred(lambda *a: OracleSimulation(*a, precision=precision), periodic_axes=periodic, n=n)
    p.run(37)
    o.run(37)
    for c, (x, y) in enumerate(zip(fields(p), fields(o))):
        assert np.array_equal(x, y), (c, relative(x, y))


@pytest.mark.parametrize("precision", [32, 64])
@pytest.mark.parametrize("n,cpml,periodic", [((260, 24, 23), 10, ()), ((252, 23, 22), 10, ()),
                                             ((256, 8, 6), 15, (1, 2)), ((264, 9, 6), 20, (1, 2))])
def test_long_rows_bit_for_bit(precision, n, cpml, periodic):
    """Rows longer than one tile: the x CPML's places of a tile's row shared out over a warp's
    lanes (one side's, at most 16: 10 and 11, 15 and 16 places), a high slab straddling two tiles
    (252), and slabs of 20 and 21 places (each lane its own)."""
    p = stirred(lambda *a: Simulation(*a, precision=precision), periodic, cpml, n)
    o = stirred(lambda *a: OracleSimulation(*a, precision=precision), periodic, cpml, n)
    p.run(37)
    o.run(37)
    for c, (x, y) in enumerate(zip(fields(p), fields(o))):
        assert np.array_equal(x, y), (c, relative(x, y))


@pytest.mark.parametrize("precision", [32, 64])
def test_two_d_bit_for_bit(precision):
    """A grid one cell thick and periodic along z (Boundaries::cpml_2d), odd sizes."""
    def make(cls):
        g = Grid3d.centred((53, 29, 1), 0.05)
        eps = np.ones((3, g.cells())) * 2.25
        s = cls(g, eps, Boundaries.cpml_2d(6), 0.7, precision=precision)
        r = np.arange(g.cells())
        for c in range(3):
            s.set_field(Field.E, c, noise(r + 5 * c))
            s.set_field(Field.H, c, noise(r + 9 * c + 123))
        return s
    p, o = make(Simulation), make(OracleSimulation)
    p.run(120)
    o.run(120)
    for x, y in zip(fields(p), fields(o)):
        assert np.array_equal(x, y)


def test_closed_box_f32_bit_for_bit_over_300_steps():
    p = closed(lambda *a: Simulation(*a, precision=32), n=(40, 36, 32))
    o = closed(lambda *a: OracleSimulation(*a, precision=32), n=(40, 36, 32))
    p.run(300)
    o.run(300)
    for x, y in zip(fields(p), fields(o)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("runs", [5, 9, 13])
def test_runs_of_planes_give_the_oracles_bits(runs, monkeypatch):
    """The quad kernel's z cut into runs of planes (each recomputing its first plane of H): the
    z CPMLs' runs, equal interior runs and, from four interior runs on, two short ones; every
    cut the oracle's bits."""
    monkeypatch.setenv("PHOTONOXIDE_FDTD_ZCHUNKS", str(runs))
    p = stirred(lambda *a: Simulation(*a, precision=32), (), 4, (132, 20, 40))
    o = stirred(lambda *a: OracleSimulation(*a, precision=32), (), 4, (132, 20, 40))
    p.run(29)
    o.run(29)
    for c, (x, y) in enumerate(zip(fields(p), fields(o))):
        assert np.array_equal(x, y), (c, relative(x, y))


@pytest.mark.parametrize("precision", [32, 64])
@pytest.mark.parametrize("periodic_x", [False, True])
def test_lossless_conductors_bit_for_bit(precision, periodic_x):
    """A lossless grid (ca 1, and 0 where cb is 0) with conductors inside tiles, on a tile's
    first row and column and in its last row, walls, and random fields, so that E at a zero cb
    starts non-zero and must come out as the oracle's zero of the right sign."""
    from photonoxide_b200.types import Pml, Cpml
    n = (132, 30, 12)

    def make(cls):
        g = Grid3d.centred(n, 0.05)
        b = Boundaries(Periodic() if periodic_x else Pml(0, 0), Pml(4, 0), Pml(0, 0), Cpml())
        eps = Boxes(1.0).add((-0.5, -0.3, -INF), (0.5, 0.3, INF), 6.0)
        s = cls(g, eps, b, 0.9, precision=precision)
        r = np.arange(g.cells())
        for c in range(3):
            s.set_field(Field.E, c, 0.01 * noise(r + 3 * c))
            s.set_field(Field.H, c, 0.01 * noise(r + 7 * c + 50_000))
        for comp, at in [(Axis.X, (5, 9, 4)), (Axis.Y, (124, 14, 6)), (Axis.Z, (60, 7, 8)),
                         (Axis.Z, (131, 29, 11)), (Axis.Y, (0, 20, 3)), (Axis.X, (70, 13, 0))]:
            s.conductor(comp, at)
        return s

    p, o = make(Simulation), make(OracleSimulation)
    p.run(61)
    o.run(61)
    for c, (x, y) in enumerate(zip(fields(p), fields(o))):
        assert np.array_equal(x, y), (c, relative(x, y))


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("two_d,n", [(False, None), (True, None), (False, (40, 21, 19)),
                                     (True, (72, 45, 1)), (False, (96, 37, 14)),
                                     (False, (256, 21, 19))])
def test_busy_bit_for_bit(two_d, n, precision):
    p = busy(lambda *a: Simulation(*a, precision=precision), two_d, n=n)
    o = busy(lambda *a: OracleSimulation(*a, precision=precision), two_d, n=n)
    p.run(800)
    o.run(800)
    for c, (x, y) in enumerate(zip(fields(p), fields(o))):
        assert np.array_equal(x, y), (c, relative(x, y))
    for n in range(6):
        assert np.array_equal(p.probe(n), o.probe(n)), n
    assert np.array_equal(p.transforms(), o.transforms()), relative(p.transforms(), o.transforms())
    assert np.array_equal(p.flux(0), o.flux(0))


@pytest.mark.parametrize("two_d", [False, True])
def test_busy_f32_within_the_reference_tolerance(two_d):
    """The reference's Agreement (src/fdtd/gpu/checks.rs:148-205): every output of each kind
    together, E and H of all components, all probes, all transforms, all fluxes, each kind's
    largest difference relative to its largest value; within 2e-5 after 800 steps."""
    p = busy(lambda *a: Simulation(*a, precision=32), two_d)
    o = busy(lambda *a: OracleSimulation(*a, precision=64), two_d)
    p.run(800)
    o.run(800)
    assert relative(np.concatenate(fields(p)), np.concatenate(fields(o))) < 2e-5
    assert relative(np.concatenate([p.probe(n) for n in range(6)]),
                    np.concatenate([o.probe(n) for n in range(6)])) < 2e-5
    assert relative(p.transforms(), o.transforms()) < 2e-5
    assert relative(p.flux(0), o.flux(0)) < 2e-5


def test_runs_in_pieces_give_the_same_bits():
    """Simulation::run gives the same bits however the steps are split (src/fdtd.rs:1169-1190),
    and a run repeats bit for bit (src/fdtd/gpu/tests.rs:93-115)."""
    a = busy(lambda *x: Simulation(*x), False)
    b = busy(lambda *x: Simulation(*x), False)
    c = busy(lambda *x: Simulation(*x), False)
    a.run(800)
    for _ in range(6):
        b.run(130)
    b.run(20)
    c.run(800)
    for x, y, z in zip(fields(a), fields(b), fields(c)):
        assert np.array_equal(x, y) and np.array_equal(x, z)
    assert np.array_equal(a.transforms(), b.transforms())
    assert np.array_equal(a.probe(3), b.probe(3))


@pytest.mark.parametrize("kind", ["plain", "staged", "row"])
def test_every_kernel_gives_the_same_bits(kind, monkeypatch):
    """The same grid (nx a multiple of 4, partial tiles) stepped by the default kernel and,
    forced, by each other one: the same bits, fields and transforms."""
    default = busy(lambda *a: Simulation(*a), False, n=(40, 21, 19))
    monkeypatch.setenv("PHOTONOXIDE_FDTD_KERNEL", kind)
    other = busy(lambda *a: Simulation(*a), False, n=(40, 21, 19))
    default.run(300)
    other.run(300)
    for x, y in zip(fields(default), fields(other)):
        assert np.array_equal(x, y)
    assert np.array_equal(default.transforms(), other.transforms())


def dispersive(cls, precision, n):
    """Drude and two-pole Lorentz boxes (src/fdtd/media_checks.rs:12 kind) with a conductivity
    under part of one, CPML all round, random fields and a point source."""
    g = Grid3d.centred(n, 0.02)
    s = cls(g, Boxes(1.0).add((-0.1, -0.1, -INF), (0.1, 0.1, INF), 2.0), Boundaries.with_cpml(4),
            0.5, precision=precision)
    s.with_conductivity(Boxes(0.0).add((0.0, -INF, -INF), (INF, 0.0, INF), 0.5))
    drude = Dispersive(1.0, [Pole.drude(7.27, 0.0531)])
    lorentz = Dispersive(2.25, [Pole.lorentz(1.2, 0.7, 0.01), Pole.lorentz(0.6, 0.45, 0.02)])
    s.with_medium(drude, Boxes(0.0).add((-0.3, -0.2, -INF), (-0.05, 0.25, INF), 1.0))
    s.with_medium(lorentz, Boxes(0.0).add((-0.08, -0.3, -0.1), (0.3, 0.05, 0.12), 1.0))
    r = np.arange(g.cells())
    for c in range(3):
        s.set_field(Field.E, c, 0.01 * noise(r + 5 * c))
    s.add_source(Source(Field.E, Axis.Z, (g.nx // 2, g.ny // 2, g.nz // 2), Waveform.pulse(1.0, 0.5)))
    p = s.add_probe(Field.E, Axis.Z, (g.nx // 3, g.ny // 2, g.nz // 2))
    return s, p


@pytest.mark.parametrize("precision", [32, 64])
@pytest.mark.parametrize("n", [(37, 29, 17), (40, 28, 16)])
def test_dispersive_media_bit_for_bit(precision, n):
    """The ADE currents (src/fdtd/media.rs:661-705) stepped in the same pass as E."""
    p, pp = dispersive(Simulation, precision, n)
    o, op = dispersive(OracleSimulation, precision, n)
    p.run(300)
    o.run(300)
    for x, y in zip(fields(p), fields(o)):
        assert np.array_equal(x, y), relative(x, y)
    assert np.array_equal(p.probe(pp), o.probe(op))


@pytest.mark.parametrize("h", [0.02, 0.04, 0.05])
def test_fast_division_is_checked_and_on(h):
    """The slabs' d/h in f32 goes through the product form only where the engine found it equal to
    division for every finite float; for the steps these tests use (and the MMI's 20 nm) it is,
    so the bit-for-bit tests above run through it. In f64 the division stays."""
    import ctypes
    from photonoxide_b200.fdtd import library
    flags = {}
    for precision in (32, 64):
        s = Simulation(Grid3d.centred((24, 20, 12), h), Boxes(1.0), Boundaries.with_cpml(3), 0.9,
                       precision=precision)
        s.run(1)
        out = (ctypes.c_int32 * 3)()
        lib = library()
        lib.fdtd_fast_division.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]
        assert lib.fdtd_fast_division(s.engine(), out) == 0
        flags[precision] = list(out)
    assert flags[32] == [1, 1, 1]
    assert flags[64] == [0, 0, 0]


@pytest.mark.parametrize("precision", [32, 64])
def test_captured_batches_give_the_same_bits(precision):
    """Without probes, whole batches of 64 steps replay a captured CUDA graph (after one direct
    batch): 330 steps with sources and transforms, split 200 + 130, equal the oracle's bits."""
    def make(cls):
        s = stirred(lambda *a: cls(*a, precision=precision), periodic_axes=(1,), n=(36, 18, 11))
        s.add_source(Source(Field.E, Axis.Z, (18, 9, 5), Waveform.pulse(1.0, 0.6)))
        s.add_source(Source(Field.H, Axis.X, (10, 9, 5), Waveform.differentiated_gaussian(0.3, 1.2)))
        s.add_dft((10, 4, 2), (25, 14, 8), [0.8, 1.0, 1.3])
        return s
    p, o = make(Simulation), make(OracleSimulation)
    p.run(200)
    p.run(130)
    o.run(330)
    for x, y in zip(fields(p), fields(o)):
        assert np.array_equal(x, y)
    assert np.array_equal(p.transforms(), o.transforms())
