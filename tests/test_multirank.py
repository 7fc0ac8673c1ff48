"""The N>1 path on CPU: two gloo ranks split a set of independent
configurations, each runs its share (here through the C oracle, the CPU
stand-in for the GPU job), and rank 0 collects every W table exactly once,
equal to the single-process results; timings reduce as a max over ranks."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from general_code_b200.multi import assign, my_jobs

JOBS = [(2, (4, 4, 4, 4)), (3, (3, 3, 3, 4)), (2, (6, 4, 4, 6)), (3, (4, 4, 4, 4)),
        (2, (4, 3, 5, 4)), (3, (4, 3, 3, 6)), (2, (8, 4, 4, 4))]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def run_job(k):
    from general_code_b200 import generate_config
    from oracle import py_oracle
    nc, dims = JOBS[k]
    port = py_oracle.port()
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 20261203, k)
    port.hyp(nc, dims, links, 1.0, 0.75, 0.6, 1)
    port.ape(nc, dims, links, 0.5, 2)
    return port.wilson(nc, dims, links, 1, 2, 1, 2)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from general_code_b200.multi import Ranks
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = Ranks()
        sites = [int(np.prod(d)) for _, d in JOBS]
        mine = my_jobs(sites, r.world, r.rank)
        res = {k: run_job(k) for k in mine}
        t = r.max(float(rank + 1))
        allres = r.gather(res)
        if rank == 0:
            merged = {}
            for part in allres:
                for k, v in part.items():
                    assert k not in merged
                    merged[k] = v
            q.put((sorted(merged), {k: merged[k].tolist() for k in merged}, t))
        r.barrier()
    finally:
        dist.destroy_process_group()


def test_assign_is_balanced_deterministic_and_complete():
    sites = [256, 108, 576, 256, 240, 216, 512]
    a = assign(sites, 2)
    assert sorted(a[0] + a[1]) == list(range(len(sites)))
    assert a == assign(sites, 2)
    loads = [sum(sites[i] for i in part) for part in a]
    assert max(loads) - min(loads) <= max(sites)
    assert assign(sites, 1) == [list(range(len(sites)))]
    assert [len(p) for p in assign([1, 1, 1], 5)] == [1, 1, 1, 0, 0]


def test_two_gloo_ranks_cover_every_configuration_once():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    keys, tables, tmax = q.get()
    assert keys == list(range(len(JOBS)))
    assert tmax == 2.0
    for k in keys:
        np.testing.assert_allclose(np.array(tables[k]), run_job(k), rtol=1e-13)
