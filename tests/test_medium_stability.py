"""Media that would grow, or that the step can't take, are refused when they are set, as the
reference refuses them (src/fdtd/media.rs:261-309, media_tests.rs:57-127): the engine's host
(photonoxide_b200.fdtd.Simulation) and the oracle alike. No GPU: the refusals come before any
device work."""
import math

import numpy as np
import pytest

from photonoxide_b200.fdtd import Simulation
from photonoxide_b200.types import Boundaries, Dispersive, Grid3d, InvalidValue, Pole
from pyoracle import OracleSimulation, medium_stable

TAU = 2.0 * math.pi


def grid(n, h):
    return Grid3d(n[0], n[1], n[2], h, h, h, -n[0] * h / 2, -n[1] * h / 2, -n[2] * h / 2)


def lorentz(eps_inf, w0dt, damping):
    return Dispersive(eps_inf, [Pole.lorentz(1.0, w0dt / TAU, damping)])


def test_stability_at_courant_one_in_one_dimension():
    """At C = 1 in 1D (dt = h = 1, (K dt)^2 up to 4): a Lorentz term steps stably only with
    w0 dt below 2 and eps_inf at least 1; a Drude term at any wp dt (media_tests.rs:57-82)."""
    assert medium_stable(lorentz(1.0, 1.99, 0.0), 0.0, 1.0, 4.0)
    assert medium_stable(lorentz(1.0, 1.99, 0.05), 2.0, 1.0, 4.0)
    assert not medium_stable(lorentz(1.0, 2.01, 0.0), 0.0, 1.0, 4.0)
    assert not medium_stable(lorentz(0.99, 1.0, 0.0), 0.0, 1.0, 4.0)
    for wpdt in (1.0, 5.0, 50.0):
        drude = Dispersive(1.0, [Pole.drude(wpdt / TAU, 0.1)])
        assert medium_stable(drude, 0.0, 1.0, 4.0), wpdt


REFUSED = {
    "gain": Dispersive(1.0, [Pole.lorentz(-0.5, 1.0, 0.1)]),
    "negative damping": Dispersive(1.0, [Pole.drude(1.0, -0.1)]),
    # w0 dt = 2 pi x 40 x 0.026 = 6.5
    "fast resonance": Dispersive(1.0, [Pole.lorentz(1.0, 40.0, 0.0)]),
    "eps_inf below the Courant number squared": Dispersive(0.5, []),
}


@pytest.mark.parametrize("name", sorted(REFUSED))
@pytest.mark.parametrize("cls", [Simulation, OracleSimulation], ids=["engine", "oracle"])
def test_media_that_would_grow_are_refused(cls, name):
    """media_tests.rs:84-122: a gain, a negative damping, a resonance the step can't resolve and
    an eps_inf the Courant number needs more of, on a 10 x 9 x 8 grid of 50 nm at Courant 0.9."""
    g = grid((10, 9, 8), 0.05)
    s = cls(g, np.ones((3, g.cells())), Boundaries.walls(), 0.9)
    with pytest.raises(InvalidValue):
        s.with_medium(REFUSED[name], np.ones((3, g.cells()), dtype=bool))


@pytest.mark.parametrize("cls", [Simulation, OracleSimulation], ids=["engine", "oracle"])
def test_a_stable_medium_is_taken(cls):
    g = grid((10, 9, 8), 0.05)
    s = cls(g, np.ones((3, g.cells())), Boundaries.walls(), 0.9)
    s.with_medium(Dispersive(1.0, [Pole.drude(1.0, 0.05)]), np.ones((3, g.cells()), dtype=bool))
