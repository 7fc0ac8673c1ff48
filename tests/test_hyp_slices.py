"""HYP smearing as a pipeline over time slices (hyp_slices_kernel) against
the level kernels (hyp_level{1,2,3}_kernel), on the GPU.

The pipeline runs the same site arithmetic with the decorated links in rings
of three time slices, so the smeared links must be the level kernels' bit for
bit: every form, SU(2) and SU(3), both HYP alpha sets of the reference's
tests, odd and unequal extents, Lt = 3 (the smallest ring), and two HYP steps.
The level kernels themselves are pinned to the reference by the golden
fixtures; the default method is checked against the oracle here as well.
"""
from __future__ import annotations

import numpy as np
import pytest

from general_code_b200 import Lattice, generate_config

pytestmark = pytest.mark.gpu

ALPHAS = [(1.0, 0.75, 0.6), (0.75, 0.6, 0.3)]


def _smeared(links, dims, nc, form, method, alphas, steps):
    with Lattice(dims, nc, form) as lat:
        lat.set_hyp_method(method)
        lat.upload(links)
        lat.hyp(*alphas, steps)
        return lat.download()


@pytest.mark.parametrize("form", ["fp64", "mixed"])
@pytest.mark.parametrize("nc,dims,alphas,steps", [
    (3, (8, 8, 8, 8), ALPHAS[0], 1),
    (2, (8, 8, 8, 8), ALPHAS[0], 1),
    (3, (5, 6, 7, 3), ALPHAS[1], 1),     # Lt = 3: every ring slot in use
    (2, (7, 5, 3, 4), ALPHAS[1], 2),
    (3, (6, 4, 5, 9), ALPHAS[0], 2),     # odd Lt, two steps
    (2, (4, 4, 4, 17), ALPHAS[0], 1),
    (3, (12, 12, 12, 16), ALPHAS[0], 1),
])
def test_slice_pipeline_equals_level_kernels(form, nc, dims, alphas, steps):
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 20261203, 5)
    a = _smeared(links, dims, nc, form, "levels", alphas, steps)
    b = _smeared(links, dims, nc, form, "slices", alphas, steps)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, links)


@pytest.mark.parametrize("nc", [2, 3])
def test_default_method_matches_oracle(port, nc):
    dims = (6, 5, 4, 7)
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 20261203, 9)
    ref = links.copy()
    port.hyp(nc, dims, ref, *ALPHAS[1], 1)
    got = _smeared(links, dims, nc, "fp64", "auto", ALPHAS[1], 1)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12)


def test_slices_need_three_time_slices():
    with Lattice((4, 4, 4, 2), 3, "fp64") as lat:
        with pytest.raises(RuntimeError):
            lat.set_hyp_method("slices")
        lat.set_hyp_method("auto")  # falls back to the level kernels
