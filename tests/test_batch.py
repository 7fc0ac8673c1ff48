"""Batches of uneven jobs (gc_batch_*): on CPU the job plan and argument
checks; on GPU every job of a batch equals the single-lattice path (bit for
bit with the default W block shapes), CUDA-graph replays repeat exactly, and
autotuned shapes stay within the FP64 tolerance."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import max_abs
from general_code_b200 import GCError, Lattice, generate_config
from general_code_b200 import _lib
from general_code_b200.batch import SIZES, Batch, Job, uneven_jobs

SMALL = [
    Job(dims=(8, 8, 8, 8), nc=2, ape_steps=3, r_max=4, t_max=4),
    Job(dims=(6, 6, 6, 8), nc=3, ape_steps=4, r_max=3, t_max=4),
    Job(dims=(4, 6, 4, 10), nc=2, ape_steps=0, r_max=2, t_max=5, r_min=2, t_min=2),
    Job(dims=(8, 8, 8, 8), nc=3, ape_steps=2, r_max=4, t_max=4, hyp_alpha=(1.0, 1.0, 0.5)),
    Job(dims=(4, 4, 4, 4), nc=3, ape_steps=1, r_max=0, t_max=0),
    Job(dims=(8, 8, 8, 16), nc=2, ape_steps=5, r_max=4, t_max=8, hyp_steps=0),
    Job(dims=(6, 4, 5, 6), nc=3, ape_steps=3, r_max=2, t_max=3, hyp_steps=2),
]
EPS = {2: 0.3, 3: 0.25}


def test_uneven_jobs_plan():
    jobs = uneven_jobs(64)
    assert len(jobs) == 64
    assert sum(j.nc == 2 for j in jobs) == 32
    assert all(j.dims in SIZES for j in jobs)
    assert all(5 <= j.ape_steps <= 30 for j in jobs)
    assert all(j.r_max == j.t_max == j.dims[0] // 2 for j in jobs)
    assert [(j.dims, j.nc, j.ape_steps) for j in jobs] == \
        [(j.dims, j.nc, j.ape_steps) for j in uneven_jobs(64)]


def test_batch_rejects_bad_jobs():
    bad = [Job(dims=(4, 4, 4, 4), nc=4, ape_steps=1, r_max=1, t_max=1)]
    with pytest.raises(GCError) as e:
        Batch(bad, "fp64")
    assert e.value.code == _lib.GC_ERR_ARG
    bad = [Job(dims=(4, 4, 4, 4), nc=3, ape_steps=1, r_max=2, t_max=2, r_min=3)]
    with pytest.raises(GCError) as e:
        Batch(bad, "fp64")
    assert e.value.code == _lib.GC_ERR_ARG


def single(job: Job, links: np.ndarray, precision: str):
    with Lattice(job.dims, job.nc, precision) as lat:
        lat.upload(links)
        if job.hyp_steps:
            lat.hyp(*job.hyp_alpha, job.hyp_steps)
        lat.ape(job.ape_alpha, job.ape_steps)
        w = lat.wilson_loop(job.r_min, job.r_max, job.t_min, job.t_max) if job.r_max else None
        return w, lat.download()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_lattice_path(precision):
    inputs = [generate_config(j.dims, j.nc, EPS[j.nc], 99, k) for k, j in enumerate(SMALL)]
    with Batch(SMALL, precision) as b:
        for k, a in enumerate(inputs):
            b.upload(k, a)
        b.run()            # eager run + graph capture
        first = [b.wilson(k) if j.r_max else None for k, j in enumerate(SMALL)]
        b.run()            # graph replay
        b.run()
        info = b.info()
        assert info["graph_nodes"] > 0
        for k, j in enumerate(SMALL):
            w_ref, links_ref = single(j, inputs[k], precision)
            assert max_abs(b.download(k), links_ref) == 0.0
            if j.r_max:
                assert np.array_equal(b.wilson(k), w_ref)
                assert np.array_equal(first[k], w_ref)


@pytest.mark.gpu
def test_batch_autotuned_shapes_within_tolerance():
    jobs = SMALL[:4]
    with Batch(jobs, "fp64") as b:
        b.generate(0.3, 0.25, 7, 0)
        b.autotune()
        b.run()
        b.run()
        for k, j in enumerate(jobs):
            rows, cols = b.shape(k)
            assert j.dims[3] % rows == 0 and rows * cols <= 256
            w_ref, _ = single(j, generate_config(j.dims, j.nc, EPS[j.nc], 7, k), "fp64")
            np.testing.assert_allclose(b.wilson(k), w_ref, rtol=1e-12, atol=1e-14)


@pytest.mark.gpu
def test_batch_job_matches_oracle(port):
    j = SMALL[1]
    links = generate_config(j.dims, j.nc, EPS[j.nc], 3, 0)
    ref = links.copy()
    port.hyp(j.nc, j.dims, ref, *j.hyp_alpha, 1)
    port.ape(j.nc, j.dims, ref, j.ape_alpha, j.ape_steps)
    w_ref = port.wilson(j.nc, j.dims, ref, j.r_min, j.r_max, j.t_min, j.t_max)
    with Batch([SMALL[0], j], "fp64") as b:
        b.upload(0, generate_config(SMALL[0].dims, 2, 0.3, 3, 1))
        b.upload(1, links)
        b.run()
        np.testing.assert_allclose(b.wilson(1), w_ref, rtol=1e-12, atol=1e-14)
        assert max_abs(b.download(1), ref) <= 1e-12


@pytest.mark.gpu
def test_uneven_batch_sample_runs():
    jobs = uneven_jobs(10, seed=5, ape_range=(2, 6))
    with Batch(jobs, "mixed") as b:
        b.generate(0.3, 0.25, 20261203, 0)
        b.run()
        b.run()
        for k in (0, len(jobs) - 1):
            j = jobs[k]
            w_ref, _ = single(j, generate_config(j.dims, j.nc, EPS[j.nc], 20261203, k), "mixed")
            assert np.array_equal(b.wilson(k), w_ref)
