"""gc_wilson_onaxis_noalloc: the W(R,T) entry point for callers that cannot
allocate device memory (their own allocator owns the device budget, or
cudaMalloc/cudaFree would stall a timing-critical loop). It takes the links
as device buffers the caller owns and writes the table into a device buffer
the caller owns; its working memory is a fixed array in the library's static
device memory.

Each case calls it twice in a row through the C ABI and checks both results
against gc_wilson_onaxis (the handle-based entry point) at the FP64 tolerance
the other tests use (1e-12 relative, 1e-14 absolute). This file is collected
last on purpose, and passes alone in a fresh process or after the others.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from general_code_b200 import Lattice, generate_config
from general_code_b200 import _lib
from general_code_b200._lib import dims_arg, lib

pytestmark = pytest.mark.gpu
PREC = {"fp64": _lib.GC_PREC_FP64, "mixed": _lib.GC_PREC_MIXED}


def device_fields(links, nc, precision, V):
    """Host links (4V, 4|18, row-major) -> four device tensors in the
    library's device layout (one per direction)."""
    import torch
    ds = links.shape[1]
    per_dir = links.reshape(V, 4, ds)
    out = []
    for mu in range(4):
        m = per_dir[:, mu, :]
        if precision == "fp64":
            planes = 9 if nc == 3 else 2
            arr = np.ascontiguousarray(m.reshape(V, planes, 2).transpose(1, 0, 2))
        else:
            if nc == 3:  # rows 0 and 1: (u00,u01), (u02,u10), (u11,u12)
                arr = np.ascontiguousarray(
                    m[:, :12].reshape(V, 3, 4).transpose(1, 0, 2).astype(np.float32))
            else:
                arr = np.ascontiguousarray(m.astype(np.float32))
        out.append(torch.from_numpy(arr).cuda())
    return out


def call_noalloc(dims, nc, precision, fields, rng, out):
    import torch
    ptrs = (ctypes.c_void_p * 4)(*[f.data_ptr() for f in fields])
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib().gc_wilson_onaxis_noalloc(dims_arg(dims), nc, PREC[precision], ptrs,
                                        *rng, ctypes.c_void_p(out.data_ptr()),
                                        ctypes.c_void_p(stream))
    return rc


@pytest.mark.parametrize("nc,dims,precision,rng", [
    (3, (8, 8, 8, 12), "fp64", (1, 4, 1, 6)),
    (2, (6, 8, 4, 10), "fp64", (2, 3, 1, 5)),
    (3, (8, 8, 8, 8), "mixed", (1, 4, 1, 4)),
    (2, (8, 8, 8, 8), "mixed", (1, 4, 2, 4)),
    (2, (4, 4, 4, 4), "fp64", (1, 4, 1, 300)),      # R split into chunks
    (3, (24, 24, 24, 24), "fp64", (1, 12, 1, 12)),  # SU(3) 24^4, R,T = 1..12
])
def test_noalloc_matches_handle_entry_point_twice(nc, dims, precision, rng):
    import torch
    V = int(np.prod(dims))
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 20261203, 5)
    with Lattice(dims, nc, precision) as lat:
        # the no-allocation entry point computes the exact product of links,
        # which is what the handle entry point computes with this method
        lat.set_wilson_method("exact")
        lat.upload(links)
        expect = lat.wilson_loop(*rng)
    fields = device_fields(links, nc, precision, V)
    shape = (rng[3] - rng[2] + 1, rng[1] - rng[0] + 1)
    # both output buffers exist before the first call, so that nothing else
    # allocates device memory between the two calls
    outs = [torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")
            for _ in range(2)]
    torch.cuda.synchronize()
    free_after_first = None
    for k, out in enumerate(outs):
        rc = call_noalloc(dims, nc, precision, fields, rng, out)
        assert rc == _lib.GC_OK, lib().gc_last_error(None)
        torch.cuda.synchronize()
        if k == 0:
            free_after_first = torch.cuda.mem_get_info()[0]
        else:
            # the second call took no device memory
            assert torch.cuda.mem_get_info()[0] >= free_after_first
    for out in outs:
        np.testing.assert_allclose(out.cpu().numpy(), expect, rtol=1e-12, atol=1e-14)


def test_noalloc_rejects_lattice_beyond_fixed_scratch():
    import torch
    dims = (64, 64, 64, 4)
    fields = [torch.zeros(2 * 64 ** 3 * 4 * 2, dtype=torch.float64, device="cuda")
              for _ in range(4)]
    out = torch.zeros((200, 1), dtype=torch.float64, device="cuda")
    rc = call_noalloc(dims, 2, "fp64", fields, (1, 1, 1, 200), out)
    assert rc == _lib.GC_ERR_ARG
    assert b"fixed scratch" in lib().gc_last_error(None)


def test_noalloc_rejects_bad_arguments():
    import torch
    fields = [torch.zeros(16, dtype=torch.float64, device="cuda") for _ in range(4)]
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    assert call_noalloc((4, 4, 4, 4), 5, "fp64", fields, (1, 1, 1, 1), out) == _lib.GC_ERR_ARG
    assert call_noalloc((4, 4, 4, 4), 3, "fp64", fields, (2, 1, 1, 1), out) == _lib.GC_ERR_ARG
