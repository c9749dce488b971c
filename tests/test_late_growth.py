"""Late growth stops a run (src/fdtd/monitors.rs:663-838, Error::Growing): the strip of the
reference's issue #251 (src/fdtd/checks.rs:257-300), a guide of eps = 6 running into CPMLs of 6
cells on cells of 50 nm, whose fields fall after the pulse and then grow again from about
250 um/c as a wave of the grid amplified in the CPML. Run until |E_y|^2 at a monitor's point has
decayed below 1e-30 of its peak, checked every 10 um/c up to 2000 um/c, the engine stops on the
growth with the reference's count of rises (src/fdtd/tests.rs:560-603); and the steps it took
before are the plain run's, the oracle's bits."""
import numpy as np
import pytest

from photonoxide_b200.fdtd import Simulation
from photonoxide_b200.types import (INF, Axis, Boundaries, Boxes, Field, Grid3d, Growing,
                                    Source, Waveform)
from pyoracle import OracleSimulation

pytestmark = pytest.mark.gpu


def late_strip(make, h=0.05, cells=6):
    scale = int(round(0.05 / h))
    n = (36 * scale, 20 * scale, 20 * scale)
    g = Grid3d(n[0], n[1], n[2], h, h, h, -n[0] * h / 2, -n[1] * h / 2, -n[2] * h / 2)
    strip = Boxes(1.0).add((-INF, -0.15, -0.15), (INF, 0.15, 0.15), 6.0)
    s = make(g, strip, Boundaries.with_cpml(cells), 0.99)
    j = int(round(8.5 * scale - 0.5))
    s.add_source(Source(Field.E, Axis.Y, (10 * scale, j, 11 * scale), Waveform.pulse(1.0, 0.25)))
    j, k = n[1] // 2 + scale, n[2] // 2 + scale
    s.add_probe(Field.E, Axis.Y, (n[0] - cells // 2, j, k))
    inside = s.add_probe(Field.E, Axis.Y, (26 * scale, j, k))
    return s, inside


def test_late_growth_stops_the_run():
    s, inside = late_strip(lambda *a: Simulation(*a, precision=64))
    with pytest.raises(Growing) as err:
        s.run_until_decayed([inside], 1e-30, 10.0, 2000.0)
    e = err.value
    assert e.checks == 4
    assert 250.0 <= e.time_um < 500.0, e.time_um
    assert e.factor >= 1e3, e.factor
    assert "grew again" in str(e)
    # its first 2000 steps are the plain run's, the oracle's bits (it reads the probes only
    # between blocks of about 350 steps, so these cross five of its checks)
    prefix = 2000
    assert s.steps > prefix
    o, q = late_strip(lambda *a: OracleSimulation(*a, precision=64))
    o.run(prefix)
    assert np.array_equal(s.probe(inside)[:prefix], o.probe(q))


def test_late_growth_stops_the_f32_run_too():
    s, inside = late_strip(lambda *a: Simulation(*a, precision=32))
    with pytest.raises(Growing) as err:
        s.run_until_decayed([inside], 1e-30, 10.0, 2000.0)
    assert 250.0 <= err.value.time_um < 500.0, err.value.time_um
