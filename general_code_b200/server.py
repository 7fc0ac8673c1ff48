"""Serving smear-and-measure requests (gc_server_* in the C ABI).

Requests are admitted continuously: as workers and device memory free up,
queued requests start on their own CUDA streams and overlap on the GPU with
the requests already running. See include/gc_lattice.h for the policy.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Dict, Optional

import numpy as np

from ._lib import (FREE_BYTES_FN, GCError, ServerMetrics, ServerOpts, check, dbl_ptr, lib)
from .batch import Job
from .lattice import _LAYOUT, _PREC


class Server:
    def __init__(self, slots: int = 8, precision: str = "mixed", memory_budget: int = 0,
                 queue_capacity: int = 0, free_bytes: Optional[Callable[[], int]] = None,
                 simulate_us: int = 0, reserve_bytes: int = 0):
        self.precision = precision
        self._cb = FREE_BYTES_FN(lambda _ctx: int(free_bytes())) if free_bytes else FREE_BYTES_FN()
        opts = ServerOpts(slots=slots, precision=_PREC[precision], memory_budget=memory_budget,
                          queue_capacity=queue_capacity, free_bytes=self._cb,
                          free_bytes_ctx=None, simulate_us=simulate_us,
                          reserve_bytes=reserve_bytes)
        self._h = ctypes.c_void_p()
        check(lib().gc_server_create(ctypes.byref(opts), ctypes.byref(self._h)))
        self._keep: Dict[int, tuple] = {}  # host arrays and jobs of open requests

    def submit(self, job: Job, links: Optional[np.ndarray], layout: str = "rowmajor") -> int:
        cj = job.c_struct()
        ptr = None
        if links is not None:
            links = np.ascontiguousarray(links, dtype=np.float64)
            ptr = dbl_ptr(links)
        rid = ctypes.c_ulonglong()
        check(lib().gc_server_submit(self._h, ctypes.byref(cj), ptr, _LAYOUT[layout],
                                     ctypes.byref(rid)))
        self._keep[rid.value] = (links, job)
        return rid.value

    def wait(self, rid: int, timeout: float = 600.0) -> np.ndarray:
        _, job = self._keep[rid]
        nr = job.r_max - job.r_min + 1 if job.r_max else 0
        nt = job.t_max - job.t_min + 1 if job.t_max else 0
        out = np.zeros((nt, nr), dtype=np.float64)
        rc = lib().gc_server_wait(self._h, rid, dbl_ptr(out) if out.size else None,
                                  float(timeout))
        if rc != _TIMEOUT:
            self._keep.pop(rid, None)
        check(rc)
        return out

    def cancel(self, rid: int) -> None:
        check(lib().gc_server_cancel(self._h, rid))
        self._keep.pop(rid, None)

    def stats(self) -> dict:
        m = ServerMetrics()
        check(lib().gc_server_stats(self._h, ctypes.byref(m)))
        return {name: getattr(m, name) for name, _ in ServerMetrics._fields_}

    def close(self) -> None:
        if self._h:
            lib().gc_server_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_TIMEOUT = 7

__all__ = ["Server", "GCError"]
