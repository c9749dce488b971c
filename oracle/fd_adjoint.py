"""ORACLE (test infrastructure only): the reference's own adjoint gradient, restated on the oracle.

photonoxide's adjoint works in the frequency domain (src/fdtd/adjoint.rs:480-883): a forward run
records the design's values of E at the objective's frequency (a design monitor), the objective's
derivative with respect to the transforms it reads becomes currents of an adjoint run of the same
problem at rest (J = -g for E, M = g for H, divided by the CPMLs' symmetrizer, 1 away from them),
each a sum of two Gaussian pulses on the frequency whose real amplitudes are solved so that the
currents' transforms are those targets (``basis``, ``amplitudes``), and once both runs have died
away the gradient is dF/deps = sum_f 2 Re(i w~ E_adj E) at each design value
(``permittivity_gradient``, w~ the leapfrog's wavenumber). This module takes those steps with the
oracle's runs (f64, the reference's arithmetic), for a flux objective (``Term::Flux``) on a grid
whose flux plane lies outside the CPMLs. The engine's time-reversed adjoint is compared with it:
two derivatives of the same objective, the reference's method against the engine's.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from photonoxide_b200.types import Current, Field, Waveform
from pyoracle import lib

TAU = 2.0 * math.pi


def _bind():
    x = lib()
    LP, DP = C.POINTER(C.c_long), C.POINTER(C.c_double)
    x.orc_dft_value.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, LP, C.c_int, DP]
    x.orc_dft_value.restype = C.c_int
    x.orc_flux_derivatives.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, LP, DP, C.c_long]
    x.orc_flux_derivatives.restype = C.c_long
    return x


def dft_value(sim, monitor: int, field: int, comp: int, at, f: int) -> complex:
    x = _bind()
    a = (C.c_long * 3)(*[int(v) for v in at])
    out = (C.c_double * 2)()
    if not x.orc_dft_value(sim._h, monitor, field, comp, a, f, out):
        raise KeyError((monitor, field, comp, tuple(at)))
    return complex(out[0], out[1])


def flux_derivatives(sim, monitor: int, f: int, scale: float = 1.0):
    """[(field, comp, r, g)]: the flux's derivative g with respect to each transform it reads."""
    x = _bind()
    n = x.orc_flux_derivatives(sim._h, monitor, f, scale, None, None, 0)
    keys = (C.c_long * (3 * n))()
    vals = (C.c_double * (2 * n))()
    x.orc_flux_derivatives(sim._h, monitor, f, scale, keys, vals, n)
    return [(keys[3 * q], keys[3 * q + 1], keys[3 * q + 2], complex(vals[2 * q], vals[2 * q + 1]))
            for q in range(n)]


def basis(frequency: float, bandwidth: float):
    """Two Gaussian pulses on the frequency, the second a quarter period after the first
    (adjoint.rs:1005-1033, ``basis``)."""
    w = Waveform.pulse(frequency, bandwidth)
    f, width, delay = w.params[:3]
    return [Waveform.gaussian(f, width, delay), Waveform.gaussian(f, width, delay + 0.25 / f)]


def spectrum(w: Waveform, field: int, dt: float, steps: int, frequency: float) -> complex:
    """sum_n w(t_n) e^{i w t_n} dt with t_n = n dt (+ dt/2 for E), as a current enters
    (src/fdtd.rs:361-396, ``Waveform::spectrum``)."""
    f, width, delay = w.params[:3]
    t = np.arange(steps) * dt + (0.5 * dt if field == 0 else 0.0)
    u = (t - delay) / width
    vals = np.exp(-u * u) * np.sin(TAU * f * (t - delay))
    return complex(np.sum(vals * np.exp(1j * TAU * frequency * t) * dt))


def amplitudes(waves, field: int, dt: float, frequency: float, targets):
    """Each target's real amplitudes on the basis waveforms, solving W beta = target at the
    frequency in real and imaginary parts (adjoint.rs:575-621, ``amplitudes``; the transforms
    summed until each pulse has died, to e^-64 of its peak)."""
    steps = max(int(math.ceil((w.params[2] + 8.0 * w.params[1]) / dt)) + 1 for w in waves)
    W = [spectrum(w, field, dt, steps, frequency) for w in waves]
    M = np.array([[W[0].real, W[1].real], [W[0].imag, W[1].imag]])
    rhs = np.array([[t.real for t in targets], [t.imag for t in targets]])
    return np.linalg.solve(M, rhs).T  # (targets, 2)


def reference_gradient(make, box, touched, frequency: float, steps: int,
                       bandwidth: float = 0.3):
    """dF/deps at each touched design value (comp, r) of the flux monitor 0's flux F at
    `frequency` (its only frequency), by the reference's frequency-domain adjoint.

    make(): the oracle simulation with its sources and flux monitor 0; make(at_rest=True): the
    same grid, medium and boundaries without sources or monitors. box = (low, high) the design
    region's index box for the design monitor; both runs take `steps` steps (long enough for
    their fields to die away). `bandwidth` is the adjoint pulses' (c/um)."""
    fwd = make()
    nd = fwd.add_dft(box[0], box[1], [frequency])
    fwd.run(steps)
    F = float(fwd.flux(0)[0])
    g = flux_derivatives(fwd, 0, 0)
    grid = fwd.grid
    dt = fwd.dt
    # the adjoint's sources: J = -g on E, M = g on H (the symmetrizer is 1 off the CPMLs)
    waves = basis(frequency, bandwidth)
    adj = make(at_rest=True)
    for field in (0, 1):
        mine = {}
        for (fd, comp, r, d) in g:
            if fd == field:
                mine[(comp, r)] = mine.get((comp, r), 0.0) + (-d if field == 0 else d)
        if not mine:
            continue
        keys = sorted(mine)
        beta = amplitudes(waves, field, dt, frequency, [mine[k] for k in keys])
        for m, w in enumerate(waves):
            values = []
            for (comp, r), b in zip(keys, beta):
                if b[m] != 0.0:
                    at = (r % grid.nx, (r // grid.nx) % grid.ny, r // (grid.nx * grid.ny))
                    values.append((comp, at, complex(b[m], 0.0)))
            adj.add_current(Current(Field.E if field == 0 else Field.H, values, w))
    na = adj.add_dft(box[0], box[1], [frequency])
    adj.run(steps)
    tilde = 2.0 / dt * math.sin(TAU * frequency * dt / 2.0)
    out = np.empty(len(touched))
    for q, (comp, r) in enumerate(touched):
        at = (r % grid.nx, (r // grid.nx) % grid.ny, r // (grid.nx * grid.ny))
        e_f = dft_value(fwd, nd, 0, comp, at, 0)
        e_a = dft_value(adj, na, 0, comp, at, 0)
        out[q] = 2.0 * (1j * tilde * e_a * e_f).real
    return F, out
