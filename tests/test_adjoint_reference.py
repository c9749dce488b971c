"""The engine's time-reversed adjoint against the reference's own adjoint method: photonoxide
computes design gradients in the frequency domain (src/fdtd/adjoint.rs:480-883: a design monitor
of the forward run, adjoint currents from the objective's derivative on two Gaussian pulses whose
amplitudes are solved for, dF/deps = sum_f 2 Re(i w~ E_adj E)), restated on the oracle in
oracle/fd_adjoint.py (f64). On a 2D TE instance of the batched-and-adjoint workload (150 x 110
cells, a 24 x 24 design, 3000 steps, long enough for both runs' fields to die away), the engine's
gradient of the arm's flux at 1550 nm with respect to the design cells' permittivities agrees
with it to 1e-3 (relative L2), the bound the engine's gradient is held to."""
import numpy as np
import pytest
import torch

from photonoxide_b200 import configs
from photonoxide_b200.adjoint import TeFlux
from photonoxide_b200.types import Boundaries
from pyoracle import OracleSimulation
from fd_adjoint import reference_gradient

pytestmark = pytest.mark.gpu

EPS0, EPS1 = configs.N_SIO2 ** 2, configs.N_SI ** 2


def test_time_reversed_adjoint_matches_the_references_frequency_domain_adjoint():
    steps, dc = 3000, 24
    rho = np.random.default_rng(1).uniform(0.0, 1.0, (dc, dc))
    eps_cells = EPS0 + rho * (EPS1 - EPS0)
    p = configs.te_design(150, 110, precision=64, steps=steps, segment=500, design_cells=dc)
    e = torch.tensor(eps_cells, requires_grad=True)
    t = TeFlux.apply(e, p)
    t[0].backward()
    engine = e.grad.numpy().reshape(-1)

    o = configs.te_design(150, 110, precision=64, steps=steps, segment=500, design_cells=dc,
                          cls=lambda *a, precision=64: OracleSimulation(*a, precision=64))

    def make(at_rest=False):
        if at_rest:
            return OracleSimulation(o.grid, o.permittivity(eps_cells), Boundaries.cpml_2d(12), 0.5,
                                    precision=64)
        return o.simulation(eps_cells)

    d = o.design
    box = ((d.x0, d.y0, 0), (d.x0 + d.nx, d.y0 + d.ny, 0))
    F, per_value = reference_gradient(make, box, list(zip(o.comp, o.r)), 1.0 / 1.55, steps)
    reference = o.S.T @ per_value
    assert abs(F - float(t[0].detach())) <= 1e-12 * abs(F)  # the same forward run
    rel = np.linalg.norm(engine - reference) / np.linalg.norm(reference)
    print(f"engine adjoint against the reference's method: relative L2 {rel:.3g}")
    assert rel <= 1e-3
