"""Gradients of 2D TE transmission with respect to a design region's permittivity, by the
engine's time-reversed adjoint (include/photonoxide_adjoint.h), behind a
``torch.autograd.Function``.

The reference's adjoint (src/fdtd/adjoint.rs) works in the frequency domain. Its design is a box
of grid cells, each with a permittivity eps(rho) = eps0 + rho (eps1 - eps0) (``Design``,
adjoint.rs:70-110), and each E value whose averaging cell reaches the design takes a share of
each design cell it covers (``Design::values``, adjoint.rs:199-259). The same shares are used
here. On a 2D grid (one cell along z), E_x at (i + 1/2, j) averages over y from j - 1/2 to
j + 1/2, so it takes half of design cell (i, j - 1) and half of (i, j); E_y at (i, j + 1/2)
takes half of (i - 1, j) and half of (i, j). A value's permittivity is its share-weighted sum of
design cells plus the rest of the background's average there.

The gradient itself is the exact derivative of the engine's discrete time stepping: reverse mode
through every step, with the forward fields recomputed segment by segment from checkpoints.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np
import torch

from .fdtd import FDTD_E_INVALID, Simulation, library
from .types import GpuError, Grid3d, InvalidValue

_bound = False


def _lib():
    global _bound
    x = library()
    if not _bound:
        P, I32, I64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        DP, I32P, I64P = C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int64)
        x.pxs_flux_gradient.argtypes = [P, I32, I32, D, DP]
        x.pxs_adjoint_create.argtypes = [P, I64, I32, I64, I32P, I64P, C.POINTER(P)]
        x.pxs_adjoint_last_error.argtypes = [P]
        x.pxs_adjoint_last_error.restype = C.c_char_p
        x.pxs_adjoint_forward.argtypes = [P]
        x.pxs_adjoint_backward.argtypes = [P, DP, DP]
        x.pxs_adjoint_destroy.argtypes = [P]
        _bound = True
    return x


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass(frozen=True)
class Design2d:
    """A design region of a 2D grid: cells x0 .. x0+nx-1 and y0 .. y0+ny-1 (cell i spans nodes i
    to i+1), whose permittivities are the variables."""

    x0: int
    y0: int
    nx: int
    ny: int

    def cells(self) -> int:
        return self.nx * self.ny

    def shares(self, grid: Grid3d):
        """Every E value the design reaches: (component (0 E_x, 1 E_y), index r, [(design cell,
        share)]), design cells numbered x fastest."""
        out = []
        for comp in (0, 1):
            ys = range(self.y0, self.y0 + self.ny + (1 if comp == 0 else 0))
            xs = range(self.x0, self.x0 + self.nx + (1 if comp == 1 else 0))
            for j in ys:
                for i in xs:
                    if i >= grid.nx or j >= grid.ny:
                        continue
                    # the two cells the value's averaging cell spans across the component
                    cand = [(i, j - 1), (i, j)] if comp == 0 else [(i - 1, j), (i, j)]
                    sh = []
                    for (ci, cj) in cand:
                        if self.x0 <= ci < self.x0 + self.nx and self.y0 <= cj < self.y0 + self.ny:
                            sh.append(((cj - self.y0) * self.nx + (ci - self.x0), 0.5))
                    if sh:
                        out.append((comp, j * grid.nx + i, sh))
        return out


class TeProblem:
    """A 2D TE simulation whose design region's permittivities vary: ``build(eps)`` makes the
    simulation from per-value permittivities (3, cells), with its sources and a flux monitor
    (number 0) whose transmission is the objective."""

    def __init__(self, grid: Grid3d, background: np.ndarray, design: Design2d,
                 build: Callable[[np.ndarray, int], Simulation], steps: int,
                 precision: int = 32, segment: int = 500):
        self.grid = grid
        self.background = np.asarray(background, dtype=np.float64).reshape(3, grid.cells())
        self.design = design
        self._build = build
        self.steps = int(steps)
        self.precision = int(precision)
        self.segment = int(segment)
        touched = design.shares(grid)
        self.comp = np.array([t[0] for t in touched], dtype=np.int32)
        self.r = np.array([t[1] for t in touched], dtype=np.int64)
        # shares as a dense (values x cells) matrix: designs are small (100 x 100 cells)
        S = np.zeros((len(touched), design.cells()))
        for q, (_, _, sh) in enumerate(touched):
            for cell, w in sh:
                S[q, cell] += w
        self.S = S
        # the background's part of each touched value: its average times the share left over
        base = self.background[self.comp, self.r]
        self.rest = base * (1.0 - S.sum(axis=1))

    def permittivity(self, eps_cells: np.ndarray) -> np.ndarray:
        """Per-value permittivities (3, cells) with the design cells at eps_cells (ny, nx)."""
        eps = self.background.copy()
        eps[self.comp, self.r] = self.rest + self.S @ np.asarray(eps_cells, np.float64).reshape(-1)
        return eps

    def simulation(self, eps_cells: np.ndarray) -> Simulation:
        return self._build(self.permittivity(eps_cells), self.precision)


def _check(x, a, code):
    if code is None or code >= 0:
        return code
    msg = x.pxs_adjoint_last_error(a).decode() if a else "adjoint"
    if code == FDTD_E_INVALID:
        raise InvalidValue(msg)
    raise GpuError(msg)


class _Handle:
    """An engine adjoint, destroyed with the last reference to it (a forward run whose gradient
    is never asked for still frees its checkpoints)."""

    def __init__(self, h, sim):
        self.h = h
        self.sim = sim  # the simulation the adjoint steps outlives it

    def __del__(self):
        if self.h:
            _lib().pxs_adjoint_destroy(self.h)
            self.h = None


class TeFlux(torch.autograd.Function):
    """eps of the design cells (ny, nx, float64) -> the flux of monitor 0 at each of its
    frequencies, after ``problem.steps`` steps. Backward: the engine's adjoint."""

    @staticmethod
    def forward(ctx, eps_cells: torch.Tensor, problem: TeProblem):
        x = _lib()
        e = eps_cells.detach().cpu().numpy().astype(np.float64)
        sim = problem.simulation(e)
        h = C.c_void_p()
        code = x.pxs_adjoint_create(sim._h, problem.steps, problem.segment, len(problem.r),
                                    problem.comp.ctypes.data_as(C.POINTER(C.c_int32)),
                                    problem.r.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(h))
        adj = _Handle(h.value, sim)
        _check(x, adj.h, code)
        _check(x, adj.h, x.pxs_adjoint_forward(adj.h))
        flux = sim.flux(0)
        if ctx.needs_input_grad[0]:
            ctx.sim, ctx.adj, ctx.problem = sim, adj, problem
            ctx.eps_values = problem.permittivity(e)[problem.comp, problem.r]
        return torch.as_tensor(np.asarray(flux, dtype=np.float64))

    @staticmethod
    def backward(ctx, grad_flux: torch.Tensor):
        x = _lib()
        sim, adj, problem = ctx.sim, ctx.adj, ctx.problem
        g = grad_flux.detach().cpu().numpy().astype(np.float64)
        nsums = sim.transforms().size
        grad_sums = np.zeros(2 * nsums)
        for f, w in enumerate(g):
            if w != 0.0:
                sim._check(x.pxs_flux_gradient(sim._h, 0, f, float(w), _dp(grad_sums)))
        grad_cb = np.zeros(len(problem.r))
        _check(x, adj.h, x.pxs_adjoint_backward(adj.h, _dp(grad_sums), _dp(grad_cb)))
        ctx.adj = None
        # cb = dt / eps at each value; eps of a value is rest + shares . eps_cells
        grad_eps_values = grad_cb * (-sim.dt / ctx.eps_values ** 2)
        grad_cells = problem.S.T @ grad_eps_values
        return torch.as_tensor(grad_cells.reshape(problem.design.ny, problem.design.nx)), None


def gaussian_blur(rho: torch.Tensor, sigma: float) -> torch.Tensor:
    """A Gaussian blur of a 2D density (pixels), truncated at 4 sigma, with the edge pixels
    repeated beyond the region. The reference has none (its filters are Helmholtz filters,
    src/topology/helmholtz.rs); written here as a separable convolution, differentiable by
    torch."""
    radius = max(1, int(np.ceil(4.0 * sigma)))
    t = torch.arange(-radius, radius + 1, dtype=rho.dtype)
    k = torch.exp(-0.5 * (t / sigma) ** 2)
    k = k / k.sum()
    x = rho[None, None]
    x = torch.nn.functional.pad(x, (radius, radius, radius, radius), mode="replicate")
    x = torch.nn.functional.conv2d(x, k.view(1, 1, 1, -1))
    x = torch.nn.functional.conv2d(x, k.view(1, 1, -1, 1))
    return x[0, 0]


def transmission(rho: torch.Tensor, problem: TeProblem, eps0: float, eps1: float,
                 sigma: float = 2.0) -> torch.Tensor:
    """The flux through monitor 0 for densities rho (ny, nx) in [0, 1]: blurred by a Gaussian
    of `sigma` pixels, then eps = eps0 + rho~ (eps1 - eps0) (``Design::permittivity``)."""
    smooth = gaussian_blur(rho, sigma) if sigma > 0 else rho
    eps = eps0 + smooth * (eps1 - eps0)
    return TeFlux.apply(eps, problem)


def central_differences(f: Callable[[np.ndarray], float], rho: np.ndarray,
                        pixels: Sequence[int], delta: float) -> np.ndarray:
    """(f(rho + delta e_p) - f(rho - delta e_p)) / (2 delta) at each pixel p (flat index)."""
    out = []
    for p in pixels:
        up, down = rho.copy().reshape(-1), rho.copy().reshape(-1)
        up[p] += delta
        down[p] -= delta
        out.append((f(up.reshape(rho.shape)) - f(down.reshape(rho.shape))) / (2.0 * delta))
    return np.array(out)
