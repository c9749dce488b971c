"""The oracle against the reference's own known answers: what pins the CPU restatement to
photonoxide's FDTD before it is trusted to check the CUDA engine."""
import math
import struct

import numpy as np

from photonoxide_b200.types import (INF, Axis, Boundaries, Boxes, Field, Grid3d, Periodic, Pml,
                                    Source, Waveform)
from pyoracle import OracleSimulation


def fold(h: int, v: float) -> int:
    """The canary's order-sensitive hash of a value's bits (tests/canary.rs:138-140)."""
    bits = struct.unpack("<Q", struct.pack("<d", v))[0]
    h = ((h << 7) | (h >> 57)) & 0xFFFFFFFFFFFFFFFF
    return h ^ bits


def canary_run():
    """tests/canary.rs:1007-1062: 200 steps of a 2D run (walls across x and y, periodic along z)
    of a dielectric strip lit by a Gaussian pulse on E_z."""
    g = Grid3d(48, 40, 1, 0.05, 0.05, 0.05, -1.2, -1.0, -0.025)
    b = Boundaries(Pml(0, 0), Pml(0, 0), Periodic())
    eps = Boxes(1.0).add((-0.3, -0.2, -INF), (INF, 0.2, INF), 6.25)  # |y| < 0.2 and x > -0.3
    s = OracleSimulation(g, eps, b, 0.9)
    s.add_source(Source(Field.E, Axis.Z, (12, 20, 0), Waveform.gaussian(1.0, 0.6, 1.8)))
    s.run(200)
    return s


def test_canary_fdtd_2d_bit_hash():
    s = canary_run()
    h = 0
    for v in np.concatenate([s.e(Axis.Z), s.h(Axis.X), s.h(Axis.Y)]):
        h = fold(h, float(v))
    peak = np.abs(s.e(Axis.Z)).max()
    assert 1e-6 < peak < math.inf
    assert h == 0x7C8DB7AE69980888, hex(h)


def test_dispersion_relation_exact():
    """src/fdtd/checks.rs:35-81: E_z of a plane wave on a periodic box steps as cos(n theta)
    with sin^2(theta/2) = (dt^2/4) sum (4/d^2) sin^2(k d/2), to round-off."""
    g = Grid3d(24, 18, 1, 0.05, 0.04, 0.05)
    per = Boundaries(Periodic(), Periodic(), Periodic())
    for (mx, my), courant in [((1, 0), 0.9), ((2, 3), 0.5), ((5, 4), 0.99)]:
        kx = 2 * math.pi * mx / (g.nx * g.dx)
        ky = 2 * math.pi * my / (g.ny * g.dy)
        s = OracleSimulation(g, np.ones((3, g.cells())), per, courant)
        ez = np.zeros(g.cells())
        for j in range(g.ny):
            for i in range(g.nx):
                x, y, _ = g.e_position(2, (i, j, 0))
                ez[j * g.nx + i] = math.cos(kx * x + ky * y)
        s.set_field(Field.E, Axis.Z, ez)
        at = int(np.argmax(np.abs(ez)))
        p = s.add_probe(Field.E, Axis.Z, (at % g.nx, at // g.nx, 0))
        s.run(400)
        series = np.concatenate([[ez[at]], s.probe(p)])
        num = np.sum(series[1:-1] * (series[2:] + series[:-2]))
        den = np.sum(2 * series[1:-1] ** 2)
        measured = math.acos(num / den)
        lam = 4 / g.dx ** 2 * math.sin(kx * g.dx / 2) ** 2 + 4 / g.dy ** 2 * math.sin(ky * g.dy / 2) ** 2
        theory = 2 * math.asin(s.dt * math.sqrt(lam) / 2)
        assert abs(measured - theory) < 1e-12 * max(1.0, theory), (measured, theory)
