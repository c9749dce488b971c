"""Batched 2D TE simulations: several :class:`~photonoxide_b200.fdtd.Simulation` grids stepped
together on the GPU, one persistent launch per step for all of them (include/photonoxide_batch.h).

Each simulation keeps its own setup, sources and monitors; after ``Batch.run(n)`` it reads out
(fields, probes, transforms, fluxes) exactly as if ``Simulation.run(n)`` had taken the steps,
with the same bits. The grids must be 2D TE: one cell along z and periodic there
(``Boundaries.cpml_2d``), fields on E_x, E_y and H_z only, sources on those components, no
dispersive media, all in one precision.

The reference has no batch: its ``Simulation::run`` (src/fdtd.rs:1134-1190) steps one grid.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence, Tuple

from .fdtd import FDTD_E_INVALID, Simulation, library
from .types import GpuError, InvalidValue

_bound = False


def _lib():
    global _bound
    x = library()
    if not _bound:
        P, I32, I64 = C.c_void_p, C.c_int32, C.c_int64
        x.pxs_batch_create.argtypes = [I32, C.POINTER(P), C.POINTER(P)]
        x.pxs_batch_last_error.argtypes = [P]
        x.pxs_batch_last_error.restype = C.c_char_p
        x.pxs_batch_run.argtypes = [P, I64]
        x.pxs_batch_tile.argtypes = [P, C.POINTER(I32), C.POINTER(I32)]
        x.pxs_batch_set_tile.argtypes = [P, I32, I32]
        x.pxs_batch_launches.argtypes = [P]
        x.pxs_batch_launches.restype = I64
        x.pxs_batch_destroy.argtypes = [P]
        _bound = True
    return x


class Batch:
    """2D TE simulations stepped together. The batch holds references to its simulations, which
    must not be run on their own while the batch is in use (their steps would not be its)."""

    def __init__(self, sims: Sequence[Simulation], tile: Tuple[int, int] | None = None):
        if not sims:
            raise InvalidValue("a batch needs simulations")
        self.sims = list(sims)
        x = _lib()
        arr = (C.c_void_p * len(self.sims))(*[s._h for s in self.sims])
        h = C.c_void_p()
        code = x.pxs_batch_create(len(self.sims), arr, C.byref(h))
        self._h = h.value
        self._check(code)
        if tile is not None:
            self._check(x.pxs_batch_set_tile(self._h, int(tile[0]), int(tile[1])))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _lib().pxs_batch_destroy(h)
            self._h = None

    def _check(self, code):
        if code is None or code >= 0:
            return code
        msg = _lib().pxs_batch_last_error(self._h).decode() if self._h else "batch"
        if code == FDTD_E_INVALID:
            raise InvalidValue(msg)
        raise GpuError(msg)

    def run(self, steps: int) -> "Batch":
        """``steps`` steps of every simulation. The first run of a batch without a fixed tile
        shape (32x8, 32x16, 64x4, 64x8, 128x2, 128x4 or the 124x7 rows) times each shape on
        chunks of these steps and keeps the fastest, when it has at least 480 of them."""
        self._check(_lib().pxs_batch_run(self._h, int(steps)))
        return self

    @property
    def tile(self) -> Tuple[int, int]:
        """The tile shape in use, (0, 0) before the first run has chosen one."""
        w, h = C.c_int32(), C.c_int32()
        self._check(_lib().pxs_batch_tile(self._h, C.byref(w), C.byref(h)))
        return (w.value, h.value)

    @tile.setter
    def tile(self, shape: Tuple[int, int]):
        self._check(_lib().pxs_batch_set_tile(self._h, int(shape[0]), int(shape[1])))

    def launches(self) -> int:
        """Kernel launches the batch has made, graph replays included."""
        return int(_lib().pxs_batch_launches(self._h))
