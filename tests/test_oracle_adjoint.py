"""The reference's frequency-domain adjoint, restated on the oracle (oracle/fd_adjoint.py,
src/fdtd/adjoint.rs:480-883), against central differences of the oracle's own runs, as the
reference checks its adjoint (src/fdtd/adjoint_checks.rs:288-316): the gradient of a 2D TE arm's
flux at 1550 nm with respect to the design cells' permittivities. This pins the restatement
the engine's time-reversed adjoint is compared with (tests/test_adjoint_reference.py)."""
import numpy as np

from photonoxide_b200 import configs
from photonoxide_b200.types import Boundaries
from pyoracle import OracleSimulation
from fd_adjoint import reference_gradient

EPS0, EPS1 = configs.N_SIO2 ** 2, configs.N_SI ** 2


def test_reference_adjoint_matches_central_differences():
    steps, dc = 3000, 24
    rho = np.random.default_rng(1).uniform(0.0, 1.0, (dc, dc))
    eps_cells = EPS0 + rho * (EPS1 - EPS0)
    o = configs.te_design(150, 110, precision=64, steps=steps, segment=500, design_cells=dc,
                          cls=lambda *a, precision=64: OracleSimulation(*a, precision=64))

    def make(cells=eps_cells, at_rest=False):
        if at_rest:
            return OracleSimulation(o.grid, o.permittivity(cells), Boundaries.cpml_2d(12), 0.5,
                                    precision=64)
        return o.simulation(cells)

    d = o.design
    box = ((d.x0, d.y0, 0), (d.x0 + d.nx, d.y0 + d.ny, 0))
    _, per_value = reference_gradient(lambda at_rest=False: make(at_rest=at_rest), box,
                                      list(zip(o.comp, o.r)), 1.0 / 1.55, steps)
    grad = o.S.T @ per_value

    def flux(cells):
        s = make(cells)
        s.run(steps)
        return float(s.flux(0)[0])

    delta = 1e-3
    for p in np.random.default_rng(7).choice(dc * dc, 4, replace=False):
        up, down = eps_cells.copy().reshape(-1), eps_cells.copy().reshape(-1)
        up[p] += delta
        down[p] -= delta
        fd = (flux(up.reshape(dc, dc)) - flux(down.reshape(dc, dc))) / (2 * delta)
        assert abs(grad[p] - fd) <= 1e-3 * abs(fd), (p, grad[p], fd)
