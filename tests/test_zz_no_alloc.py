"""The allocation-free upload, fdtd_upload_fields_static, against fdtd_upload_fields through the
C ABI: the same fields on the device, so the same run, on two calls in a row.

Some callers can't allocate device memory when they upload: a serving loop that has already
handed out its whole HBM budget, an application whose own CUDA allocator forbids others, code
that must leave a stream-ordered memory pool untouched. The static entry point stages through a
fixed device array instead; this file checks it gives exactly what the allocating one gives.
Collected last, so a run that stops at the first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from photonoxide_b200.fdtd import Simulation, library
from photonoxide_b200.types import Boundaries, Cpml, Grid3d, Pml, Periodic

pytestmark = pytest.mark.gpu

DP = C.POINTER(C.c_double)


def bind():
    lib = library()
    lib.fdtd_upload_fields.argtypes = [C.c_void_p, DP, DP, C.c_void_p]
    lib.fdtd_upload_fields_static.argtypes = [C.c_void_p, DP, DP]
    lib.fdtd_run.argtypes = [C.c_void_p, C.c_int64, C.c_int64]
    lib.fdtd_download_fields.argtypes = [C.c_void_p, DP, DP, C.c_void_p]
    lib.fdtd_last_error.argtypes = [C.c_void_p]
    lib.fdtd_last_error.restype = C.c_char_p
    return lib


def ptr(a):
    return a.ctypes.data_as(DP)


def pool_in_use():
    """Bytes the device's default memory pool (the one cudaMallocAsync draws on) has handed out,
    and the device's free memory: an upload that allocates moves one or the other."""
    from cuda.bindings import runtime as rt
    import torch
    dev = torch.cuda.current_device()
    err, pool = rt.cudaDeviceGetDefaultMemPool(dev)
    assert err == rt.cudaError_t.cudaSuccess
    err, used = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    assert err == rt.cudaError_t.cudaSuccess
    err, free, _total = rt.cudaMemGetInfo()
    assert err == rt.cudaError_t.cudaSuccess
    return int(used), int(free)


@pytest.mark.parametrize("precision", [32, 64])
def test_static_upload_matches_the_allocating_one_twice(precision):
    lib = bind()
    g = Grid3d.centred((44, 30, 20), 0.05)
    b = Boundaries(Pml(5, 4), Periodic(), Pml(3, 3), Cpml(kappa=2.0, alpha=0.1))
    sim = Simulation(g, np.full((3, g.cells()), 2.5), b, 0.8, precision=precision)
    sim.run(1)  # the engine exists from the first run
    ctx = sim.engine()
    assert ctx
    rng = np.random.default_rng(11)
    n = 3 * g.cells()
    for call in range(2):  # two calls in a row, different fields each time
        e = np.ascontiguousarray(rng.standard_normal(n))
        h = np.ascontiguousarray(rng.standard_normal(n))
        out = []
        for static in (False, True):
            if static:
                used0, free0 = pool_in_use()
                rc = lib.fdtd_upload_fields_static(ctx, ptr(e), ptr(h))
                # nothing allocated: the pool hands out no more, the device has no less free
                used1, free1 = pool_in_use()
                assert used1 == used0 and free1 >= free0, (call, used0, used1, free0, free1)
            else:
                rc = lib.fdtd_upload_fields(ctx, ptr(e), ptr(h), None)
            assert rc == 0, lib.fdtd_last_error(ctx)
            assert lib.fdtd_run(ctx, 7, 0) == 0, lib.fdtd_last_error(ctx)
            ed, hd = np.empty(n), np.empty(n)
            assert lib.fdtd_download_fields(ctx, ptr(ed), ptr(hd), None) == 0
            out.append((ed, hd))
        (ea, ha), (eb, hb) = out
        assert np.array_equal(ea, eb) and np.array_equal(ha, hb), call


def test_static_upload_refuses_a_grid_beyond_its_array():
    lib = bind()
    g = Grid3d(256, 128, 65, 0.05, 0.05, 0.05)  # 2 129 920 cells > 2^21
    sim = Simulation(g, np.ones((3, g.cells())), Boundaries.walls(), 0.5)
    sim.run(1)
    ctx = sim.engine()
    e = np.zeros(3 * g.cells())
    rc = lib.fdtd_upload_fields_static(ctx, ptr(e), ptr(e))
    assert rc == -1
    assert b"static staging array" in lib.fdtd_last_error(ctx)


def test_static_upload_takes_any_f64_grid():
    """Only an f32 context stages through the fixed array: an f64 context copies straight into
    its fields, so a grid beyond the array's 2^21 values is taken, with the allocating upload's
    result."""
    lib = bind()
    g = Grid3d(256, 128, 65, 0.05, 0.05, 0.05)  # 2 129 920 cells > 2^21
    sim = Simulation(g, np.full((3, g.cells()), 2.0), Boundaries.walls(), 0.5, precision=64)
    sim.run(1)
    ctx = sim.engine()
    rng = np.random.default_rng(3)
    n = 3 * g.cells()
    e, h = rng.standard_normal(n), rng.standard_normal(n)
    out = []
    for static in (False, True):
        rc = (lib.fdtd_upload_fields_static(ctx, ptr(e), ptr(h)) if static
              else lib.fdtd_upload_fields(ctx, ptr(e), ptr(h), None))
        assert rc == 0, lib.fdtd_last_error(ctx)
        assert lib.fdtd_run(ctx, 3, 0) == 0, lib.fdtd_last_error(ctx)
        ed = np.empty(n)
        assert lib.fdtd_download_fields(ctx, ptr(ed), None, None) == 0
        out.append(ed)
    assert np.array_equal(out[0], out[1])
