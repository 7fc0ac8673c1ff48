"""The request loop (gc_server_*). On CPU, in simulation mode (workers sleep
instead of using the GPU): admission by free worker and memory budget, a
fake free-memory provider, queue back-pressure, oversize rejection,
cancellation, bounded waits and latency statistics. On GPU: requests that
run concurrently give bitwise the same W tables as each request alone."""
from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from general_code_b200 import GCError, Lattice, generate_config, job_device_bytes
from general_code_b200 import _lib
from general_code_b200.batch import Job
from general_code_b200.server import Server

JOB = Job(dims=(8, 8, 8, 8), nc=3, ape_steps=2, r_max=2, t_max=2)


def bytes_of(job, precision="mixed"):
    return job_device_bytes(job.dims, job.nc, precision, job.r_max, job.t_max)


def test_slots_bound_concurrency_and_stats():
    with Server(slots=3, simulate_us=20000) as s:
        ids = [s.submit(JOB, None) for _ in range(12)]
        for i in ids:
            s.wait(i, timeout=30)
        st = s.stats()
    assert st["completed"] == 12 and st["failed"] == 0
    assert st["peak_inflight"] == 3
    assert st["p50_ms"] > 15 and st["p99_ms"] >= st["p50_ms"]


def test_memory_budget_bounds_concurrency():
    b = bytes_of(JOB)
    with Server(slots=8, simulate_us=20000, memory_budget=int(2.5 * b)) as s:
        ids = [s.submit(JOB, None) for _ in range(8)]
        for i in ids:
            s.wait(i, timeout=30)
        st = s.stats()
    assert st["peak_inflight"] == 2
    assert st["peak_bytes"] <= int(2.5 * b)


def test_free_memory_provider_gates_admission():
    b = bytes_of(JOB)
    calls = []

    def free():
        calls.append(1)
        return int(0.5 * b)   # never room for a second request

    with Server(slots=4, simulate_us=10000, memory_budget=100 * b, free_bytes=free) as s:
        ids = [s.submit(JOB, None) for _ in range(5)]
        for i in ids:
            s.wait(i, timeout=30)
        st = s.stats()
    assert st["peak_inflight"] == 1   # admitted one at a time (nothing else in flight)
    assert st["completed"] == 5
    assert calls


def test_oversize_request_rejected():
    with Server(slots=1, simulate_us=1000, memory_budget=bytes_of(JOB) // 2) as s:
        with pytest.raises(GCError) as e:
            s.submit(JOB, None)
        assert e.value.code == _lib.GC_ERR_NOMEM
        assert s.stats()["rejected"] == 1


def test_queue_capacity_back_pressure_and_cancel():
    with Server(slots=1, simulate_us=200000, queue_capacity=2) as s:
        a = s.submit(JOB, None)
        time.sleep(0.05)                 # a is running
        b = s.submit(JOB, None)
        c = s.submit(JOB, None)
        with pytest.raises(GCError) as e:
            s.submit(JOB, None)
        assert e.value.code == _lib.GC_ERR_BUSY
        s.cancel(c)
        with pytest.raises(GCError) as e:
            s.cancel(a)                  # already started
        assert e.value.code == _lib.GC_ERR_STATE
        with pytest.raises(GCError) as e:
            s.wait(a, timeout=0.01)      # bounded wait
        assert e.value.code == _lib.GC_ERR_TIMEOUT
        s.wait(a, timeout=30)
        s.wait(b, timeout=30)
        assert s.stats()["completed"] == 2


def test_destroy_cancels_pending_requests():
    s = Server(slots=1, simulate_us=100000)
    ids = [s.submit(JOB, None) for _ in range(4)]
    time.sleep(0.02)
    t0 = time.time()
    s.close()                            # waits for the running one only
    assert time.time() - t0 < 1.0


def _single(job, links, precision):
    with Lattice(job.dims, job.nc, precision) as lat:
        lat.upload(links)
        lat.hyp(*job.hyp_alpha, job.hyp_steps)
        lat.ape(job.ape_alpha, job.ape_steps)
        return lat.wilson_loop(job.r_min, job.r_max, job.t_min, job.t_max)


MIX = [Job(dims=(L, L, L, L), nc=nc, ape_steps=a, r_max=L // 2, t_max=L // 2)
       for L, nc, a in [(8, 3, 5), (4, 2, 3), (12, 3, 2), (6, 2, 7), (10, 3, 4), (8, 2, 9),
                        (4, 3, 1), (12, 2, 6), (6, 3, 3), (10, 2, 2), (8, 3, 8), (4, 2, 5)]]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_results_same_alone_and_in_the_mix(precision):
    inputs = [generate_config(j.dims, j.nc, 0.3 if j.nc == 2 else 0.25, 11, k)
              for k, j in enumerate(MIX)]
    alone = [_single(j, inputs[k], precision) for k, j in enumerate(MIX)]
    with Server(slots=4, precision=precision) as s:
        ids = [s.submit(j, inputs[k]) for k, j in enumerate(MIX)]
        got = [s.wait(i, timeout=120) for i in ids]
        st = s.stats()
    for k in range(len(MIX)):
        assert np.array_equal(got[k], alone[k]), k
    assert st["completed"] == len(MIX) and st["peak_inflight"] > 1


@pytest.mark.gpu
def test_server_request_matches_oracle(port):
    j = MIX[0]
    links = generate_config(j.dims, j.nc, 0.25, 4, 0)
    ref = links.copy()
    port.hyp(j.nc, j.dims, ref, *j.hyp_alpha, 1)
    port.ape(j.nc, j.dims, ref, j.ape_alpha, j.ape_steps)
    w_ref = port.wilson(j.nc, j.dims, ref, 1, j.r_max, 1, j.t_max)
    with Server(slots=2, precision="fp64") as s:
        w = s.wait(s.submit(j, links), timeout=120)
    np.testing.assert_allclose(w, w_ref, rtol=1e-12, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("reserve", [-1, 64 << 20, 0])
def test_pool_reserve_keeps_results_and_admission(reserve):
    """The server's stream-ordered pool reserved at creation (default),
    a small reserve the requests outgrow, or none: the same results, and a
    free-memory provider that reports only the device's free memory still
    admits requests (the pool's idle reserve counts as free)."""
    import torch
    inputs = [generate_config(j.dims, j.nc, 0.3 if j.nc == 2 else 0.25, 12, k)
              for k, j in enumerate(MIX[:6])]
    alone = [_single(j, inputs[k], "mixed") for k, j in enumerate(MIX[:6])]
    free = lambda: int(torch.cuda.mem_get_info()[0])
    with Server(slots=3, precision="mixed", reserve_bytes=reserve, free_bytes=free) as s:
        ids = [s.submit(j, inputs[k]) for k, j in enumerate(MIX[:6])]
        got = [s.wait(i, timeout=120) for i in ids]
        st = s.stats()
    for k in range(6):
        assert np.array_equal(got[k], alone[k]), k
    assert st["completed"] == 6
