"""The serving loop (photonoxide_b200.serving): jobs admitted under a memory budget as others
finish, 2D TE jobs batched and 3D jobs on their own streams, each with the bits it has alone."""
import numpy as np
import pytest

from photonoxide_b200.serving import (CANCELLED, DONE, FAILED, JobSpec, Server, job_stream,
                                      make_job)
from photonoxide_b200.types import GpuError

pytestmark = pytest.mark.gpu


def small_stream(count, seed):
    return job_stream(count, rate=1000.0, seed=seed, cells=(4e3, 6e4), steps=(40, 300))


def results(sim):
    return ([sim.e(c) for c in range(3)] + [sim.h(c) for c in range(3)], sim.transforms(),
            sim.flux(0))


def test_each_job_has_its_bits_alone():
    specs = small_stream(14, 3)
    assert any(s.two_d for s in specs) and any(not s.two_d for s in specs)
    alone = []
    for sp in specs:
        s = make_job(sp)
        s.run(sp.steps)
        alone.append(results(s))
    # a budget that holds a few jobs at a time: the rest wait for memory, then join
    with Server(hbm_budget=200e6, max_active=6, chunk=64) as server:
        jobs = [server.submit(make_job(sp), sp.steps) for sp in specs]
        for j in jobs:
            assert j.wait() == DONE
        st = server.stats()
        assert st["bytes_admitted"] == 0
        assert st["cell_updates"] == sum(int(np.prod(sp.n)) * sp.steps for sp in specs)
        for j, (fields, sums, flux) in zip(jobs, alone):
            f2, s2, x2 = results(j.sim)
            for a, b in zip(fields, f2):
                assert np.array_equal(a, b)
            assert np.array_equal(sums, s2)
            assert np.array_equal(flux, x2)
            state, (sub, start, end) = j.poll()
            assert state == DONE and sub <= start <= end


def test_a_job_beyond_the_budget_fails_and_a_queued_job_cancels():
    sp = JobSpec(0.0, True, (200, 200, 1), 50, ((-0.2, -0.2, 0.2, 0.2),), 3)
    with Server(hbm_budget=10e6, max_active=1, chunk=1000) as server:
        big = server.submit(make_job(sp), 50)
        with pytest.raises(GpuError):
            big.wait()
    small = JobSpec(0.0, True, (64, 48, 1), 2000, ((-0.2, -0.2, 0.2, 0.2),), 1)
    with Server(hbm_budget=500e6, max_active=1, chunk=1000) as server:
        first = server.submit(make_job(small), 2000)
        second = server.submit(make_job(small), 2000)
        second.cancel()
        assert first.wait() == DONE
        assert second.poll()[0] == CANCELLED


def test_a_job_without_its_fields_keeps_its_transforms():
    sp = small_stream(1, 11)[0]
    alone = make_job(sp)
    alone.run(sp.steps)
    with Server(hbm_budget=500e6, max_active=2, chunk=64) as server:
        job = server.submit(make_job(sp), sp.steps, keep_fields=False)
        assert job.wait() == DONE
        assert np.array_equal(job.sim.transforms(), alone.transforms())
        assert np.array_equal(job.sim.flux(0), alone.flux(0))
        with pytest.raises(GpuError):
            job.sim.e(0)
        with pytest.raises(GpuError):
            job.sim.run(1)
