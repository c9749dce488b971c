"""The stopping rules (src/fdtd/monitors.rs:663-838, src/fdtd.rs:1161-1167) on the engine:
run_until's step count, and run_until_decayed against the rule restated here over a twin run
(block by block, the same probes): the same answer, the same steps, the same bits."""
import numpy as np
import pytest

from photonoxide_b200.fdtd import Simulation
from photonoxide_b200.types import (INF, Axis, Boundaries, Boxes, Field, Grid3d, InvalidValue,
                                    Source, Waveform)

pytestmark = pytest.mark.gpu


def lossy_box():
    g = Grid3d.centred((60, 50, 1), 0.05)
    s = Simulation(g, Boxes(1.0).add((-0.5, -0.5, -INF), (0.5, 0.5, INF), 4.0),
                   Boundaries.cpml_2d(8), 0.7)
    s.with_conductivity(Boxes(0.3))
    s.add_source(Source(Field.H, Axis.Z, (30, 25, 0), Waveform.pulse(1.0, 0.8)))
    p = [s.add_probe(Field.H, Axis.Z, (20, 20, 0)), s.add_probe(Field.E, Axis.Y, (40, 30, 0))]
    return s, p


def decayed_restated(s, probes, fraction, interval, limit):
    while s.time() < limit:
        start = len(s.probe(probes[0]))
        s.run_until(min(s.time() + interval, limit))
        ok = True
        for n in probes:
            v = np.asarray(s.probe(n)) ** 2
            peak, recent = v.max(initial=0.0), v[start:].max(initial=0.0)
            ok &= bool(peak > 0 and recent <= fraction * peak)
        if ok:
            return True
    return False


def test_run_until_takes_the_reference_count():
    s, _ = lossy_box()
    s.run_until(1.0)
    n = 0
    while n * s.dt < 1.0:
        n += 1
    assert s.steps == n and s.time() >= 1.0


@pytest.mark.parametrize("fraction,limit", [(1e-3, 60.0), (1e-9, 6.0)])
def test_run_until_decayed_as_the_rule_says(fraction, limit):
    a, pa = lossy_box()
    b, pb = lossy_box()
    got = a.run_until_decayed(pa, fraction, 0.5, limit)
    want = decayed_restated(b, pb, fraction, 0.5, limit)
    assert got == want
    assert a.steps == b.steps
    for c in range(3):
        assert np.array_equal(a.e(c), b.e(c)) and np.array_equal(a.h(c), b.h(c))


def test_refusals():
    s, p = lossy_box()
    with pytest.raises(InvalidValue):
        s.run_until_decayed([], 1e-3, 0.5, 10.0)
    with pytest.raises(InvalidValue):
        s.run_until_decayed(p, 1.5, 0.5, 10.0)
    with pytest.raises(InvalidValue):
        s.run_until_decayed(p, 1e-3, 0.0, 10.0)
    with pytest.raises(InvalidValue):
        s.run_until_decayed([7], 1e-3, 0.5, 10.0)
