"""The C ABI library on CPU: it loads, exports every declared symbol, validates
arguments before touching the device, reports a missing GPU as an error (no
CPU fallback), and its host-side generator is deterministic and produces
special-unitary links."""
from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT, max_abs, unitarity_error
from general_code_b200 import _lib, generate_config, job_device_bytes
from general_code_b200._lib import GCError, check, dims_arg, lib


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(gc_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    l = lib()
    syms = declared_symbols()
    assert "gc_wilson_onaxis" in syms and "gc_ape" in syms and "gc_hyp" in syms
    missing = [s for s in syms if not hasattr(l, s)]
    assert not missing, missing
    # the Python binding declares a signature for every one of them
    assert set(syms) <= set(_lib.SIGNATURES)


def test_version():
    assert lib().gc_version() >= 100


@pytest.mark.parametrize("dims,nc,prec", [((4, 4, 4, 4), 4, 0), ((4, 4, 4, 4), 3, 7),
                                          ((4, 1, 4, 4), 3, 0), ((0, 4, 4, 4), 2, 0)])
def test_create_rejects_bad_arguments(dims, nc, prec):
    h = ctypes.c_void_p()
    rc = lib().gc_lattice_create(dims_arg(dims), nc, prec, ctypes.byref(h))
    assert rc == _lib.GC_ERR_ARG
    assert not h.value
    assert lib().gc_last_error(None)


def test_null_handle_is_an_error_not_a_crash():
    out = (ctypes.c_double * 4)()
    assert lib().gc_ape(None, 0.5, 1) == _lib.GC_ERR_ARG
    assert lib().gc_plaquette(None, out) == _lib.GC_ERR_ARG
    assert lib().gc_wilson_onaxis(None, 1, 1, 1, 1, out) == _lib.GC_ERR_ARG
    assert lib().gc_lattice_destroy(None) == _lib.GC_OK


def test_slice_and_probe_entry_points_validate_arguments():
    """The t-slab slice entry points, the slab W and the FMA probe reject
    null handles and bad arguments before any device call."""
    l = lib()
    out = (ctypes.c_double * 4)()
    host = (ctypes.c_double * 4)()
    assert l.gc_upload_slices(None, 0, 1, host, 0) == _lib.GC_ERR_ARG
    assert l.gc_slice_bytes(None, 1) == -1
    assert l.gc_pack_slices(None, 0, 1, ctypes.c_void_p(16)) == _lib.GC_ERR_ARG
    assert l.gc_unpack_slices(None, 0, 1, ctypes.c_void_p(16)) == _lib.GC_ERR_ARG
    assert l.gc_copy_slices(None, 0, None, 0, 1) == _lib.GC_ERR_ARG
    assert l.gc_wilson_onaxis_tslab(None, 1, 1, 1, 1, 1, 0, out) == _lib.GC_ERR_ARG
    assert l.gc_fma_peak(7, out) == _lib.GC_ERR_ARG
    assert l.gc_fma_peak(0, None) == _lib.GC_ERR_ARG


def _has_gpu():
    h = ctypes.c_void_p()
    rc = lib().gc_lattice_create(dims_arg((2, 2, 2, 2)), 2, 0, ctypes.byref(h))
    if rc == _lib.GC_OK:
        lib().gc_lattice_destroy(h)
        return True
    return False


def test_no_gpu_is_reported_as_error():
    if _has_gpu():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = lib().gc_lattice_create(dims_arg((4, 4, 4, 4)), 3, 0, ctypes.byref(h))
    assert rc == _lib.GC_ERR_NODEVICE
    with pytest.raises(GCError):
        check(rc)


@pytest.mark.parametrize("nc,eps", [(2, 0.3), (3, 0.25)])
def test_generator_deterministic_and_special_unitary(nc, eps):
    dims = (4, 4, 6, 8)
    a = generate_config(dims, nc, eps, 20261203, 0)
    b = generate_config(dims, nc, eps, 20261203, 0)
    c = generate_config(dims, nc, eps, 20261203, 1)
    assert max_abs(a, b) == 0.0
    assert max_abs(a, c) > 0.1
    assert unitarity_error(nc, a) < 1e-13


@pytest.mark.parametrize("nc,eps", [(2, 0.3), (3, 0.25)])
def test_generator_amplitude(nc, eps):
    """Without the gauge transform, Re Tr U / N has the mean of exp(i eps ...)."""
    dims = (8, 8, 8, 8)
    a = generate_config(dims, nc, eps, 1, 0, gauge=False)
    if nc == 2:
        tr = a[:, 0]
        # E[cos(eps |a|)] for a ~ N(0, I_3)
        z = np.random.default_rng(0).standard_normal((400000, 3))
        expect = np.cos(eps * np.linalg.norm(z, axis=1)).mean()
    else:
        tr = (a[:, 0] + a[:, 8] + a[:, 16]) / 3
        expect = None
    if expect is not None:
        assert abs(tr.mean() - expect) < 5e-3
    assert 0.5 < tr.mean() < 1.0
    g = generate_config(dims, nc, eps, 1, 0, gauge=True)
    gtr = g[:, 0] if nc == 2 else (g[:, 0] + g[:, 8] + g[:, 16]) / 3
    assert abs(gtr.mean()) < 0.05  # a Haar gauge transform randomises link traces


def test_generator_rejects_bad_arguments():
    out = np.empty((4 * 16, 4))
    rc = lib().gc_generate_host(dims_arg((2, 2, 2, 2)), 5, 0.3, 1, 0, 1,
                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == _lib.GC_ERR_ARG


def test_job_device_bytes_scales_with_volume():
    small = job_device_bytes((8, 8, 8, 8), 3, "fp64", 4, 4)
    big = job_device_bytes((16, 16, 16, 16), 3, "fp64", 4, 4)
    mixed = job_device_bytes((16, 16, 16, 16), 3, "mixed", 4, 4)
    assert 14 < big / small < 17
    assert mixed < big
