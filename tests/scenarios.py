"""Problems the tests step on the engine and on the oracle alike, restating the reference's own
fixtures: ``noise`` (src/fdtd/checks.rs:84-90), ``busy`` (src/fdtd/gpu/checks.rs:36-147) and
``closed`` (src/fdtd/gpu/checks.rs:282-306). Each takes ``make(grid, eps, boundaries, courant)``,
the constructor of either simulation."""
import numpy as np

from photonoxide_b200.types import (INF, Axis, Boundaries, Boxes, Cpml, Current, Dipole, Field,
                                    FluxPlane, Grid3d, Periodic, Pml, Source, Waveform)


def noise(r) -> np.ndarray:
    """A pseudo-random value in [-1, 1) from an integer, the reference's bits."""
    x = np.asarray(r, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = (x * np.uint64(0x9E3779B97F4A7C15)) ^ np.uint64(0x5DEECE66)
        x ^= x >> np.uint64(31)
        x = x * np.uint64(0xBF58476D1CE4E5B9)
        x ^= x >> np.uint64(29)
    return (x >> np.uint64(11)).astype(np.float64) / float(1 << 52) - 1.0


def pulse() -> Waveform:
    return Waveform.pulse(1.0, 0.6)


def busy(make, two_d: bool, sources: bool = True, scale: float = 0.01, n=None):
    """A dielectric block and a lossy one, a conductor, CPMLs with kappa and alpha, a wall and (in
    2D) periodic sides, random fields, point sources on E and H, a current sharing a value with
    one, a dipole, probes, a transform box and a flux box (3D) or plane (2D). 3D: 37 x 21 x 19
    cells of 50 nm, sizes that leave tiles part-filled."""
    if two_d:
        b = Boundaries(Periodic(), Pml(6, 6), Periodic(), Cpml(kappa=2.0, alpha=0.3))
        g = Grid3d.centred(n or (70, 45, 1), 0.05)
    else:
        b = Boundaries(Pml(4, 5), Pml(4, 0), Pml(3, 3), Cpml(kappa=3.0, alpha=0.2))
        g = Grid3d.centred(n or (37, 21, 19), 0.05)
    eps = Boxes(1.0).add((-0.3, -0.2, -INF), (0.3, 0.2, INF), 12.0)
    s = make(g, eps, b, 0.9)
    s.with_conductivity(Boxes(0.0).add((0.6, 0.3, -INF), (INF, INF, INF), 2.0))
    n = g.cells()
    r = np.arange(n)
    for c in range(3):
        s.set_field(Field.E, c, scale * noise(r + 3 * c))
        s.set_field(Field.H, c, scale * noise(r + 7 * c + 50_000))
    nx, ny, nz = g.nx, g.ny, g.nz
    mid = (nx // 2, ny // 2, nz // 2)
    s.conductor(Axis.X, (nx // 3, ny // 3, nz // 2))
    if sources:
        s.add_source(Source(Field.E, Axis.Z, mid, pulse()))
        s.add_source(Source(Field.H, Axis.X, (nx // 4, ny // 2, nz // 2),
                            Waveform.differentiated_gaussian(0.3, 1.2)))
        s.add_current(Current(Field.E, [(Axis.Z, mid, complex(0.5, -0.25)),
                                        (Axis.Y, (nx // 2 + 3, ny // 2, nz // 2),
                                         complex(-0.3, 0.7))], pulse()))
        centre = [g.x0 + 0.5 * nx * 0.05, g.y0 + 0.5 * ny * 0.05, g.z0 + 0.5 * nz * 0.05]
        s.add_dipole(Dipole(Field.H, Axis.Z, (centre[0] + 0.33, centre[1] - 0.21, centre[2]),
                            complex(1.0, 0.5), pulse()))
    for at in [(3, 3, 0), (nx - 8, ny // 3, nz // 3), mid]:
        s.add_probe(Field.E, Axis.Z, at)
        s.add_probe(Field.H, Axis.Y, at)
    freqs = [0.8, 1.0, 1.3]
    s.add_dft((nx // 2 - 6, ny // 2 - 4, 0), (nx // 2 + 6, ny // 2 + 4, nz - 1), freqs)
    if two_d:
        s.add_flux(FluxPlane(Axis.Y, ny - 12), freqs)
    else:
        box = lambda n: (n // 2 - 5, n // 2 + 5)  # noqa: E731
        s.add_flux_box([box(nx), box(ny), box(nz)], freqs)
    return s


def closed(make, n=(40, 36, 32)):
    """A closed box of walls with a block of eps = 12 and random fields: nothing leaves it."""
    g = Grid3d.centred(n, 0.05)
    eps = Boxes(1.0).add((-0.3, -0.2, -INF), (0.3, 0.2, INF), 12.0)
    s = make(g, eps, Boundaries.walls(), 0.9)
    r = np.arange(g.cells())
    for c in range(3):
        s.set_field(Field.E, c, noise(r + 3 * c))
        s.set_field(Field.H, c, noise(r + 7 * c + 50_000))
    return s


def stirred(make, periodic_axes=(), cpml=4, n=(33, 18, 11)):
    """Random fields in a dielectric with CPMLs (kappa, alpha) on the non-periodic axes: every
    boundary kind the kernel treats, and no source (the f32 arithmetic is then exactly the
    oracle's)."""
    edges = [Periodic() if a in periodic_axes else Pml(cpml, cpml + 1) for a in range(3)]
    b = Boundaries(edges[0], edges[1], edges[2], Cpml(kappa=2.5, alpha=0.25))
    g = Grid3d.centred(n, 0.04)
    eps = Boxes(2.0).add((-0.2, -0.1, -INF), (0.25, 0.15, INF), 9.0)
    s = make(g, eps, b, 0.8)
    r = np.arange(g.cells())
    for c in range(3):
        s.set_field(Field.E, c, noise(r + 11 * c))
        s.set_field(Field.H, c, noise(r + 13 * c + 7_000))
    return s
