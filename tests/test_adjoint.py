"""The time-reversed adjoint of 2D TE runs (photonoxide_b200.adjoint): the gradient of the arm's
flux with respect to the design's densities against central finite differences of the engine's
own forward runs (the reference checks its adjoint the same way, src/fdtd/adjoint_checks.rs:
288-316), and the adjoint's bookkeeping: its forward run is a plain run, its reverse run leaves
the simulation as it was, checkpoint segments do not change the gradient."""
import numpy as np
import pytest
import torch

from photonoxide_b200 import configs
from photonoxide_b200.adjoint import central_differences, transmission

pytestmark = pytest.mark.gpu

EPS0, EPS1 = configs.N_SIO2 ** 2, configs.N_SI ** 2


def problem(precision=64, segment=200, steps=1400):
    return configs.te_design(150, 110, precision=precision, steps=steps, segment=segment,
                             design_cells=24)


def density(seed=1):
    return np.random.default_rng(seed).uniform(0.0, 1.0, (24, 24))


def gradient(p, rho):
    r = torch.tensor(rho, requires_grad=True)
    t = transmission(r, p, EPS0, EPS1, sigma=2.0)
    t[0].backward()
    return float(t[0].detach()), r.grad.numpy().copy()


def objective(p):
    def f(rho):
        with torch.no_grad():
            return float(transmission(torch.tensor(rho), p, EPS0, EPS1, sigma=2.0)[0])
    return f


def test_gradient_matches_central_differences():
    p = problem()
    rho = density()
    J, g = gradient(p, rho)
    assert abs(J) > 0
    pixels = np.random.default_rng(7).choice(rho.size, 8, replace=False)
    fd = central_differences(objective(p), rho, pixels, 1e-3)
    ga = g.reshape(-1)[pixels]
    assert np.linalg.norm(ga - fd) <= 1e-3 * np.linalg.norm(fd), (ga, fd)
    assert np.max(np.abs(ga - fd)) <= 1e-3 * np.max(np.abs(fd))


def test_segments_do_not_change_the_gradient():
    rho = density(3)
    _, a = gradient(problem(segment=100), rho)
    _, b = gradient(problem(segment=1400), rho)
    # the same bits: the reverse run injects without atomics and recomputes each segment exactly
    assert np.array_equal(a, b)


def test_the_gradient_is_deterministic():
    rho = density(4)
    _, a = gradient(problem(precision=32), rho)
    _, b = gradient(problem(precision=32), rho)
    assert np.array_equal(a, b)


def test_f32_gradient_near_f64():
    rho = density(5)
    _, a = gradient(problem(precision=32), rho)
    _, b = gradient(problem(precision=64), rho)
    assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b)


def test_forward_is_a_plain_run_and_the_reverse_run_restores_it():
    from photonoxide_b200.adjoint import TeFlux
    p = problem(precision=32)
    rho = density(2)
    eps = EPS0 + configs_blur(rho) * (EPS1 - EPS0)
    plain = p.simulation(eps)
    plain.run(p.steps)
    e = torch.tensor(eps, requires_grad=True)
    t = TeFlux.apply(e, p)
    assert np.array_equal(t.detach().numpy(), plain.flux(0))


def configs_blur(rho):
    from photonoxide_b200.adjoint import gaussian_blur
    return gaussian_blur(torch.tensor(rho), 2.0).numpy()


def test_flux_gradient_is_the_bilinear_form():
    """The flux is bilinear in the transforms, so sum(sums . dflux/dsums) = 2 flux."""
    import ctypes as C
    from photonoxide_b200.adjoint import _lib, _dp
    p = problem(precision=64, steps=600)
    s = p.simulation(EPS0 + 0.5 * (EPS1 - EPS0) * np.ones((24, 24)))
    s.run(600)
    sums = s.transforms()
    grad = np.zeros(2 * sums.size)
    assert _lib().pxs_flux_gradient(s._h, 0, 0, 1.0, _dp(grad)) == 0
    flux = s.flux(0)[0]
    both = np.stack([sums.real, sums.imag], axis=-1).reshape(-1)
    assert abs(float(both @ grad) - 2 * flux) <= 1e-12 * abs(flux)
