"""Makes the full-size golden fixtures of this directory with the oracle (the f64 CPU restatement
of photonoxide's FDTD step, oracle/): runs the measured workloads at their full sizes and step
counts on the host's cores and keeps the results the parity tests compare the CUDA engine with.

    python tests/golden/make_golden.py [mmi] [dispersive]

- ``mmi_20000.npz``: the 3D MMI (600 x 200 x 100, CPML 10, Gaussian-profile current at 1550 nm)
  after 20 000 steps: both arms' flux spectra at 51 wavelengths and the probe's time series.
- ``dispersive_10000.npz``: the dispersive grid (256 x 256 x 128, Drude and two-pole Lorentz
  boxes, seed 7) after 10 000 steps: the probe's time series and the final E_z plane through the
  source; ``dispersive_10000_f32.npz`` the same from the oracle's f32 arithmetic
  (``dispersive32``).

Each takes tens of minutes on 8 host threads; the fixtures are small (the spectra and series).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

from photonoxide_b200 import configs  # noqa: E402
from pyoracle import OracleSimulation  # noqa: E402


def oracle(*a, precision=64, **kw):
    return OracleSimulation(*a, precision=64, **kw)


def mmi():
    s, info = configs.mmi_3d(oracle)
    t0 = time.perf_counter()
    s.run(info["steps"])
    seconds = time.perf_counter() - t0
    np.savez_compressed(os.path.join(HERE, "mmi_20000.npz"),
                        flux=np.array([s.flux(n) for n in info["fluxes"]]),
                        probe=s.probe(info["probe"]), steps=info["steps"], seconds=seconds)
    print(f"mmi: {info['steps']} steps in {seconds:.0f} s", flush=True)


def dispersive(precision=64):
    s, info = configs.dispersive_3d(
        lambda *a, **kw: OracleSimulation(*a, **{**kw, "precision": precision}), 7)
    t0 = time.perf_counter()
    s.run(info["steps"])
    seconds = time.perf_counter() - t0
    g = s.grid
    ez = s.e(2).reshape(g.nz, g.ny, g.nx)[g.nz // 2]
    name = "dispersive_10000.npz" if precision == 64 else "dispersive_10000_f32.npz"
    np.savez_compressed(os.path.join(HERE, name), probe=s.probe(info["probe"]),
                        ez_mid=ez, steps=info["steps"], seconds=seconds)
    print(f"dispersive (f{precision}): {info['steps']} steps in {seconds:.0f} s", flush=True)


if __name__ == "__main__":
    which = sys.argv[1:] or ["mmi", "dispersive"]
    for name in which:
        {"mmi": mmi, "dispersive": dispersive,
         "dispersive32": lambda: dispersive(32)}[name]()
