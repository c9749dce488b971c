"""The device engine's C ABI (``include/photonoxide_fdtd.h``) from Python: the calls a caller
that builds its own tables makes (the reference's ``gpu::Resident`` seam, resident.rs:147-869).
:class:`photonoxide_b200.fdtd.Simulation` builds those tables itself; this module is for callers
that keep their own, and for timing the engine alone."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .fdtd import library
from .types import GpuError, InvalidValue

D, I32, I64, P = C.c_double, C.c_int32, C.c_int64, C.c_void_p
DP, I64P = C.POINTER(C.c_double), C.POINTER(C.c_int64)

_bound = False


def _bind():
    global _bound
    if _bound:
        return library()
    x = library()
    x.fdtd_last_error.argtypes = [P]
    x.fdtd_last_error.restype = C.c_char_p
    x.fdtd_upload_coeffs.argtypes = [P, DP, DP]
    x.fdtd_upload_fields.argtypes = [P, DP, DP, C.POINTER(DP)]
    x.fdtd_download_fields.argtypes = [P, DP, DP, C.POINTER(DP)]
    x.fdtd_run.argtypes = [P, I64, I64]
    x.fdtd_run_async.argtypes = [P, I64, I64]
    x.fdtd_synchronize.argtypes = [P]
    x.fdtd_read_probes.argtypes = [P, DP, I64, I64P]
    x.fdtd_read_dft.argtypes = [P, DP, I64]
    x.fdtd_stream.argtypes = [P]
    x.fdtd_stream.restype = P
    x.fdtd_launches.argtypes = [P]
    x.fdtd_launches.restype = I64
    x.fdtd_profile.argtypes = [P, I32]
    x.fdtd_profile_read.argtypes = [P, DP, I64P]
    _bound = True
    return x


class Engine:
    """A handle on one ``fdtd_ctx``."""

    def __init__(self, ctx: int):
        if not ctx:
            raise GpuError("no engine context: run the simulation once first")
        self.ctx = ctx
        self.lib = _bind()

    def check(self, code):
        if code < 0:
            msg = self.lib.fdtd_last_error(self.ctx).decode()
            raise (InvalidValue if code == -1 else GpuError)(msg)
        return code

    def stream(self) -> int:
        return self.lib.fdtd_stream(self.ctx)

    def upload_coeffs(self, ca, cb):
        ca_p = None if ca is None else np.ascontiguousarray(ca, np.float64).ctypes.data_as(DP)
        cb = np.ascontiguousarray(cb, np.float64)
        self.check(self.lib.fdtd_upload_coeffs(self.ctx, ca_p, cb.ctypes.data_as(DP)))

    def upload_fields(self, e, h):
        self.check(self.lib.fdtd_upload_fields(self.ctx, e.ctypes.data_as(DP),
                                               h.ctypes.data_as(DP), None))

    def download_fields(self, e, h):
        self.check(self.lib.fdtd_download_fields(self.ctx, e.ctypes.data_as(DP),
                                                 h.ctypes.data_as(DP), None))

    def run_async(self, steps: int, first: int):
        self.check(self.lib.fdtd_run_async(self.ctx, int(steps), int(first)))

    def run(self, steps: int, first: int):
        self.check(self.lib.fdtd_run(self.ctx, int(steps), int(first)))

    def synchronize(self):
        self.check(self.lib.fdtd_synchronize(self.ctx))

    def read_dft(self, sums: np.ndarray):
        self.check(self.lib.fdtd_read_dft(self.ctx, sums.ctypes.data_as(DP), sums.size // 2))

    def launches(self) -> int:
        return self.lib.fdtd_launches(self.ctx)

    def profile(self, on: bool):
        self.check(self.lib.fdtd_profile(self.ctx, int(on)))

    def profile_read(self):
        ms = C.c_double(0)
        n = C.c_int64(0)
        self.check(self.lib.fdtd_profile_read(self.ctx, C.byref(ms), C.byref(n)))
        return ms.value, n.value
