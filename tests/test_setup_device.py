"""The cell average on the device (pxs_average_device, one thread per E value) against the host
library's (pxs_average, itself the oracle's bit for bit): the same functions, so the same bits,
on the 3D MMI's geometry and on boxes whose faces fall on the averaging's sample points."""
import numpy as np
import pytest

from photonoxide_b200 import configs
from photonoxide_b200.fdtd import average
from photonoxide_b200.types import INF, Boxes, Grid3d

pytestmark = pytest.mark.gpu


def test_mmi_geometry():
    g = Grid3d(600, 200, 100, 0.02, 0.02, 0.02, -6.0, -2.0, -1.0)
    geo = configs.mmi_geometry()
    assert np.array_equal(average(g, geo, device=True), average(g, geo))


def test_faces_on_samples_overlaps_and_two_d():
    h = 0.05
    g = Grid3d(48, 40, 24, h, h, h, 0.0, 0.0, 0.0)
    # faces on the nodes, on half steps (the E positions) and on the samples' sixteenths
    b = (Boxes(1.7)
         .add((0.25, 0.1, -INF), (1.0, 0.6, 0.4), 12.0)
         .add((0.5 + h / 16, 0.35 + 3 * h / 16, 0.2), (1.9, 1.2, INF), 2.25)
         .add((0.0, 0.0, 0.5 - h / 2), (0.3 + 5 * h / 16, INF, 0.75), 12.0)
         .add((-INF, 0.85, -INF), (INF, 0.85 + h / 32, INF), 4.0))
    assert np.array_equal(average(g, b, device=True), average(g, b))
    g2 = Grid3d(70, 45, 1, h, h, h, -1.75, -1.1, -h / 2)
    assert np.array_equal(average(g2, b, device=True), average(g2, b))
    assert np.array_equal(average(g2, Boxes(2.1), device=True), average(g2, Boxes(2.1)))


@pytest.mark.parametrize("edges", [
    "mmi", "mixed", "graded",
])
def test_cpml_tables_on_the_device_are_the_hosts(edges):
    """The CPML's kappa factors and slabs made on the device (one thread per node) against the
    host library's, which equal the oracle's (test_setup_tables.py): the same bits."""
    from photonoxide_b200.fdtd import Simulation, cpml_tables
    from photonoxide_b200.types import Boundaries, Cpml, Periodic, Pml
    if edges == "mmi":
        g = Grid3d(600, 200, 100, 0.02, 0.02, 0.02, -6.0, -2.0, -1.0)
        b = Boundaries.with_cpml(10)
    elif edges == "mixed":
        g = Grid3d(40, 33, 27, 0.05, 0.04, 0.03)
        b = Boundaries(Pml(6, 9), Periodic(), Pml(0, 5), Cpml())
    else:  # a given sigma, kappa > 1, alpha > 0, order 4
        g = Grid3d(31, 29, 24, 0.05, 0.05, 0.05)
        b = Boundaries(Pml(7, 7), Pml(5, 0), Pml(4, 6), Cpml(1e-6, 12.0, 4.0, 3.5, 0.2))
    s = Simulation(g, Boxes(2.25), b, 0.9)
    for which in (2, 3, 4):
        assert np.array_equal(cpml_tables(g, b, s.dt, which), s.tables(which)), which
