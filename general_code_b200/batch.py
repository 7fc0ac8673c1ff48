"""Batches of independent smear-and-measure jobs (gc_batch_* in the C ABI).

A job is one configuration with its own lattice size, group, HYP/APE step
counts and W(R,T) ranges -- the loop of the reference's apps/smearing
(smearing.cpp:228-301) for one configuration. A Batch runs many of them
together: one launch per phase over all jobs, the schedule captured into a
CUDA graph on the first run and replayed afterwards.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

from ._lib import GcJob, check, dbl_ptr, lib
from .lattice import _LAYOUT, _PREC, link_size, volume


@dataclass
class Job:
    dims: Tuple[int, int, int, int]
    nc: int
    ape_steps: int
    r_max: int
    t_max: int
    hyp_steps: int = 1
    hyp_alpha: Tuple[float, float, float] = (1.0, 0.75, 0.6)
    ape_alpha: float = 0.5
    r_min: int = 1
    t_min: int = 1

    @property
    def sites(self) -> int:
        return volume(self.dims)

    def c_struct(self) -> GcJob:
        j = GcJob()
        j.dims[:] = [int(d) for d in self.dims]
        j.nc = self.nc
        j.hyp_steps = self.hyp_steps
        j.hyp_alpha[:] = [float(a) for a in self.hyp_alpha]
        j.ape_steps = self.ape_steps
        j.ape_alpha = float(self.ape_alpha)
        j.r_min, j.r_max = self.r_min, self.r_max
        j.time_min, j.time_max = self.t_min, self.t_max
        return j


class Batch:
    def __init__(self, jobs: Sequence[Job], precision: str = "mixed"):
        self.jobs = list(jobs)
        self.precision = precision
        arr = (GcJob * len(self.jobs))(*[j.c_struct() for j in self.jobs])
        self._h = ctypes.c_void_p()
        check(lib().gc_batch_create(arr, len(self.jobs), _PREC[precision], ctypes.byref(self._h)))

    def _check(self, rc: int) -> None:
        check(rc, None)

    def close(self) -> None:
        if self._h:
            lib().gc_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, job: int, links: np.ndarray, layout: str = "rowmajor") -> None:
        a = np.ascontiguousarray(links, dtype=np.float64)
        self._check(lib().gc_batch_upload(self._h, job, dbl_ptr(a), _LAYOUT[layout]))

    def generate(self, eps_su2: float, eps_su3: float, seed: int, first_index: int = 0) -> None:
        self._check(lib().gc_batch_generate(self._h, eps_su2, eps_su3, seed & 0xffffffff,
                                            first_index & 0xffffffff))

    def autotune(self) -> None:
        self._check(lib().gc_batch_autotune(self._h))

    def run(self, stream_ptr: int | None = None) -> None:
        self._check(lib().gc_batch_run(self._h, ctypes.c_void_p(stream_ptr or 0)))

    def synchronize(self) -> None:
        self._check(lib().gc_batch_synchronize(self._h))

    def wilson(self, job: int) -> np.ndarray:
        j = self.jobs[job]
        out = np.empty((j.t_max - j.t_min + 1, j.r_max - j.r_min + 1), dtype=np.float64)
        self._check(lib().gc_batch_wilson(self._h, job, dbl_ptr(out)))
        return out

    def download(self, job: int, layout: str = "rowmajor") -> np.ndarray:
        j = self.jobs[job]
        out = np.empty((4 * j.sites, link_size(j.nc)), dtype=np.float64)
        self._check(lib().gc_batch_download(self._h, job, dbl_ptr(out), _LAYOUT[layout]))
        return out

    def info(self) -> dict:
        b, n, l = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
        self._check(lib().gc_batch_info(self._h, ctypes.byref(b), ctypes.byref(n),
                                        ctypes.byref(l)))
        return {"device_bytes": b.value, "graph_nodes": n.value, "launches_per_run": l.value}

    def autotune_report(self) -> str:
        """The candidate block shapes the autotuner timed, with their times."""
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(lib().gc_batch_autotune_report(self._h, buf, len(buf)))
        return buf.value.decode()

    def shape(self, job: int) -> Tuple[int, int]:
        r, c = ctypes.c_int(), ctypes.c_int()
        self._check(lib().gc_batch_job_shape(self._h, job, ctypes.byref(r), ctypes.byref(c)))
        return r.value, c.value


SIZES = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 16), (16, 16, 16, 32),
         (24, 24, 24, 24), (24, 24, 24, 48)]


def uneven_jobs(n: int = 64, seed: int = 20261203, ape_range=(5, 30)) -> List[Job]:
    """The uneven batch: sizes uniform over SIZES, SU(2)/SU(3) 50/50 (exactly
    half each), APE steps uniform in ape_range, R,T up to L_s/2."""
    rng = np.random.default_rng(seed)
    groups = np.array([2] * (n // 2) + [3] * (n - n // 2))
    rng.shuffle(groups)
    jobs = []
    for k in range(n):
        dims = SIZES[int(rng.integers(len(SIZES)))]
        half = dims[0] // 2
        jobs.append(Job(dims=dims, nc=int(groups[k]),
                        ape_steps=int(rng.integers(ape_range[0], ape_range[1] + 1)),
                        r_max=half, t_max=half))
    return jobs
