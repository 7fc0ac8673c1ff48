"""ctypes binding of the C ABI in include/gc_lattice.h (libgc_b200.so).

The library is built in-tree (general_code_b200/build.py). Loading it does not
need a GPU; every entry point that touches the device returns
GC_ERR_NODEVICE on a machine without an sm_100 GPU, which the Python layer
raises as GCError. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(os.environ.get("GC_B200_LIB") or
                Path(__file__).resolve().parent / "libgc_b200.so")

GC_OK = 0
GC_ERR_ARG = 1
GC_ERR_CUDA = 2
GC_ERR_NOMEM = 3
GC_ERR_NODEVICE = 4
GC_ERR_IO = 5
GC_ERR_STATE = 6
GC_ERR_TIMEOUT = 7
GC_ERR_BUSY = 8

GC_PREC_FP64 = 0
GC_PREC_MIXED = 1
GC_LAYOUT_ROWMAJOR = 0
GC_WILSON_AUTO = 0
GC_WILSON_EXACT = 1
GC_WILSON_GAUGE = 2
GC_HYP_AUTO = 0
GC_HYP_LEVELS = 1
GC_HYP_SLICES = 2
GC_LAYOUT_EIGEN_COLMAJOR = 1

ERROR_NAMES = {
    GC_ERR_ARG: "GC_ERR_ARG", GC_ERR_CUDA: "GC_ERR_CUDA", GC_ERR_NOMEM: "GC_ERR_NOMEM",
    GC_ERR_NODEVICE: "GC_ERR_NODEVICE", GC_ERR_IO: "GC_ERR_IO", GC_ERR_STATE: "GC_ERR_STATE",
    GC_ERR_TIMEOUT: "GC_ERR_TIMEOUT", GC_ERR_BUSY: "GC_ERR_BUSY",
}

# Every symbol include/gc_lattice.h declares, with (restype, argtypes).
_c_int, _c_dbl, _c_uint = ctypes.c_int, ctypes.c_double, ctypes.c_uint
_p, _pint, _pdbl = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "gc_version": (_c_int, []),
    "gc_last_error": (ctypes.c_char_p, [_p]),
    "gc_lattice_create": (_c_int, [_pint, _c_int, _c_int, ctypes.POINTER(_p)]),
    "gc_lattice_destroy": (_c_int, [_p]),
    "gc_set_stream": (_c_int, [_p, _p]),
    "gc_synchronize": (_c_int, [_p]),
    "gc_upload": (_c_int, [_p, _pdbl, _c_int]),
    "gc_download": (_c_int, [_p, _pdbl, _c_int]),
    "gc_copy_links": (_c_int, [_p, _p]),
    "gc_upload_slices": (_c_int, [_p, _c_int, _c_int, _pdbl, _c_int]),
    "gc_slice_bytes": (ctypes.c_longlong, [_p, _c_int]),
    "gc_pack_slices": (_c_int, [_p, _c_int, _c_int, _p]),
    "gc_unpack_slices": (_c_int, [_p, _c_int, _c_int, _p]),
    "gc_copy_slices": (_c_int, [_p, _c_int, _p, _c_int, _c_int]),
    "gc_wilson_onaxis_tslab": (_c_int, [_p, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int,
                                        _pdbl]),
    "gc_ape": (_c_int, [_p, _c_dbl, _c_int]),
    "gc_hyp": (_c_int, [_p, _c_dbl, _c_dbl, _c_dbl, _c_int]),
    "gc_wilson_onaxis": (_c_int, [_p, _c_int, _c_int, _c_int, _c_int, _pdbl]),
    "gc_wilson_adjoint_onaxis": (_c_int, [_p, _c_int, _c_int, _c_int, _c_int, _pdbl]),
    "gc_set_wilson_method": (_c_int, [_p, _c_int]),
    "gc_set_hyp_method": (_c_int, [_p, _c_int]),
    "gc_wilson_method_used": (_c_int, [_p, _pint]),
    "gc_plaquette": (_c_int, [_p, _pdbl]),
    "gc_plaquette_space": (_c_int, [_p, _pdbl]),
    "gc_plaquette_time": (_c_int, [_p, _pdbl]),
    "gc_wilson_gevp_onaxis": (_c_int, [_p, _p, _c_int, _c_int, _c_int, _c_int, _pdbl]),
    "gc_wilson_gevp_adjoint_onaxis": (_c_int, [_p, _p, _c_int, _c_int, _c_int, _c_int, _pdbl]),
    "gc_polyakov_loop": (_c_int, [_p, _pdbl]),
    "gc_wilson_offaxis": (_c_int, [_p, _pint, _c_int, _c_dbl, _c_dbl, _c_int, _c_int, _c_int,
                                   _p, _c_int, _pint]),
    "gc_wilson_offaxis_result": (_c_int, [_p, _c_dbl, _c_dbl, _c_int, _c_int, _c_int, _p,
                                          _c_int, _pint]),
    "gc_ape_plane": (_c_int, [_p, _c_int, _c_int, _c_dbl, _c_int]),
    "gc_wilson_spatial_3d": (_c_int, [_p, _c_int, _c_int, _c_int, _c_int, _c_dbl, _c_int,
                                      _c_int, _c_int, _p, _c_int, _pint]),
    "gc_polyakov_correlator": (_c_int, [_p, _c_int, _c_int, _pdbl]),
    "gc_wilson_onaxis_noalloc": (_c_int, [_pint, _c_int, _c_int, ctypes.POINTER(_p), _c_int,
                                          _c_int, _c_int, _c_int, _p, _p]),
    "gc_read_config": (_c_int, [_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_longlong,
                                ctypes.c_char_p, _c_int]),
    "gc_write_config": (_c_int, [_p, ctypes.c_char_p]),
    "gc_probe_config": (_c_int, [_pint, _c_int, ctypes.c_char_p, ctypes.c_char_p,
                                 ctypes.c_longlong, ctypes.c_char_p,
                                 ctypes.POINTER(ctypes.c_longlong),
                                 ctypes.POINTER(ctypes.c_longlong)]),
    "gc_generate": (_c_int, [_p, _c_dbl, _c_uint, _c_uint, _c_int]),
    "gc_generate_host": (_c_int, [_pint, _c_int, _c_dbl, _c_uint, _c_uint, _c_int, _pdbl]),
    "gc_job_device_bytes": (ctypes.c_longlong, [_pint, _c_int, _c_int, _c_int, _c_int]),
    "gc_fma_peak": (_c_int, [_c_int, _pdbl]),
}

class GcJob(ctypes.Structure):
    """gc_job (include/gc_lattice.h)."""
    _fields_ = [("dims", ctypes.c_int * 4), ("nc", ctypes.c_int), ("hyp_steps", ctypes.c_int),
                ("hyp_alpha", ctypes.c_double * 3), ("ape_steps", ctypes.c_int),
                ("ape_alpha", ctypes.c_double), ("r_min", ctypes.c_int), ("r_max", ctypes.c_int),
                ("time_min", ctypes.c_int), ("time_max", ctypes.c_int)]


_pjob = ctypes.POINTER(GcJob)
SIGNATURES.update({
    "gc_batch_create": (_c_int, [_pjob, _c_int, _c_int, ctypes.POINTER(_p)]),
    "gc_batch_destroy": (_c_int, [_p]),
    "gc_batch_upload": (_c_int, [_p, _c_int, _pdbl, _c_int]),
    "gc_batch_generate": (_c_int, [_p, _c_dbl, _c_dbl, _c_uint, _c_uint]),
    "gc_batch_autotune": (_c_int, [_p]),
    "gc_batch_run": (_c_int, [_p, _p]),
    "gc_batch_synchronize": (_c_int, [_p]),
    "gc_batch_wilson": (_c_int, [_p, _c_int, _pdbl]),
    "gc_batch_download": (_c_int, [_p, _c_int, _pdbl, _c_int]),
    "gc_batch_info": (_c_int, [_p, ctypes.POINTER(ctypes.c_longlong), _pint, _pint]),
    "gc_batch_job_shape": (_c_int, [_p, _c_int, _pint, _pint]),
    "gc_batch_autotune_report": (_c_int, [_p, ctypes.c_char_p, _c_int]),
})

FREE_BYTES_FN = ctypes.CFUNCTYPE(ctypes.c_longlong, ctypes.c_void_p)


class ServerOpts(ctypes.Structure):
    """gc_server_opts (include/gc_lattice.h)."""
    _fields_ = [("slots", ctypes.c_int), ("precision", ctypes.c_int),
                ("memory_budget", ctypes.c_longlong), ("queue_capacity", ctypes.c_int),
                ("free_bytes", FREE_BYTES_FN), ("free_bytes_ctx", ctypes.c_void_p),
                ("simulate_us", ctypes.c_int), ("reserve_bytes", ctypes.c_longlong)]


class ServerMetrics(ctypes.Structure):
    """gc_server_metrics (include/gc_lattice.h)."""
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("rejected", ctypes.c_longlong), ("failed", ctypes.c_longlong),
                ("pending", ctypes.c_longlong), ("inflight", ctypes.c_int),
                ("peak_inflight", ctypes.c_int), ("peak_bytes", ctypes.c_longlong),
                ("budget", ctypes.c_longlong), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("sites_per_s", ctypes.c_double), ("queue_p50_ms", ctypes.c_double),
                ("queue_p99_ms", ctypes.c_double), ("run_p50_ms", ctypes.c_double),
                ("run_p99_ms", ctypes.c_double)]


SIGNATURES.update({
    "gc_lattice_create_on_stream": (_c_int, [_pint, _c_int, _c_int, _p, ctypes.POINTER(_p)]),
    "gc_server_create": (_c_int, [ctypes.POINTER(ServerOpts), ctypes.POINTER(_p)]),
    "gc_server_submit": (_c_int, [_p, _pjob, _pdbl, _c_int,
                                  ctypes.POINTER(ctypes.c_ulonglong)]),
    "gc_server_wait": (_c_int, [_p, ctypes.c_ulonglong, _pdbl, _c_dbl]),
    "gc_server_cancel": (_c_int, [_p, ctypes.c_ulonglong]),
    "gc_server_stats": (_c_int, [_p, ctypes.POINTER(ServerMetrics)]),
    "gc_server_destroy": (_c_int, [_p]),
})

_lib = None


class WilsonResult(ctypes.Structure):
    """gc_wilson_result (include/gc_lattice.h)."""
    _fields_ = [("wilson_loop", ctypes.c_double), ("time_size", ctypes.c_int),
                ("space_size", ctypes.c_double), ("statistics_size", ctypes.c_int)]


class WilsonSpatialResult(ctypes.Structure):
    """gc_wilson_spatial_result (include/gc_lattice.h)."""
    _fields_ = [("smearing", ctypes.c_int), ("time_size", ctypes.c_int),
                ("space_size", ctypes.c_int), ("wilson_loop", ctypes.c_double)]


class GCError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """Loads libgc_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m general_code_b200.build`")
        l = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(rc: int, handle=None) -> None:
    if rc != GC_OK:
        msg = lib().gc_last_error(handle)
        raise GCError(rc, msg.decode() if msg else "")


def dims_arg(dims) -> ctypes.Array:
    d = [int(v) for v in dims]
    if len(d) != 4:
        raise ValueError("dims must have 4 entries (Lx, Ly, Lz, Lt)")
    return (ctypes.c_int * 4)(*d)


def dbl_ptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_pdbl)
