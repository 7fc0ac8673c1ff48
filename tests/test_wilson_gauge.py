"""The two methods of the on-axis Wilson loops (GPU): the exact product of
links and the temporal-gauge form (gc_wilson_gauge.cu), which the library
uses for T <= Lt/2 once the device has checked that the temporal links are
unitary.

* Both methods against the reference's own W tables (golden fixtures) and
  against the C oracle on seeded lattices of odd, even and long time
  extents: FP64 within 1e-12 relative (1e-14 absolute floor); the mixed form
  within 1e-6 of FP64; the adjoint loops alike.
* The method actually run is the gauge form where it applies, and the exact
  product when T > Lt/2 or when a temporal link fails the unitarity check
  (links scaled by 1 + 1e-9 in FP64, 1 + 1e-5 in the mixed form), or when the
  caller asks for it.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_cases, load_golden
from general_code_b200 import Lattice, generate_config

pytestmark = pytest.mark.gpu
CASES = golden_cases()
W_RTOL, W_ATOL = 1e-12, 1e-14


def _both(lat, rng, adjoint=False):
    fn = lat.wilson_loop_adjoint if adjoint else lat.wilson_loop
    out = {}
    for method in ("auto", "exact"):
        lat.set_wilson_method(method)
        out[method] = fn(*rng)
        out[method + "_used"] = lat.wilson_method_used()
    lat.set_wilson_method("auto")
    return out


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_both_methods_match_reference_fixture(name, meta):
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    rng = (meta["r_min"], meta["r_max"], meta["time_min"], meta["time_max"])
    with Lattice(dims, nc, "fp64") as lat:
        lat.upload(g["links_ape"])
        w = _both(lat, rng)
        wa = _both(lat, rng, adjoint=True)
    assert w["auto_used"] == "gauge" and w["exact_used"] == "exact"
    for m in ("auto", "exact"):
        np.testing.assert_allclose(w[m], g["wilson"], rtol=W_RTOL, atol=W_ATOL)
        np.testing.assert_allclose(wa[m], g["wilson_adjoint"], rtol=W_RTOL, atol=W_ATOL)


@pytest.mark.parametrize("nc,dims,eps,n_ape,rng", [
    (3, (8, 8, 8, 8), 0.25, 3, (1, 4, 1, 4)),
    (2, (8, 8, 8, 8), 0.3, 3, (1, 4, 1, 4)),
    (3, (6, 5, 7, 9), 0.25, 2, (1, 3, 2, 4)),      # odd Lt: cut B at slice 4
    (2, (5, 7, 3, 11), 0.3, 2, (2, 4, 1, 5)),
    (3, (4, 4, 4, 48), 0.25, 2, (1, 2, 1, 24)),    # 48 start slices per column
    (2, (4, 3, 5, 40), 0.3, 2, (1, 2, 3, 20)),
    (3, (12, 12, 12, 12), 0.25, 4, (1, 6, 1, 6)),
    (2, (6, 6, 6, 96), 0.3, 1, (1, 3, 1, 12)),     # two start slices per thread
    # mixed SU(3) with 8 | Lt runs the one-column kernel (four starts per
    # thread): blocks of 32 columns over runs of sites, the last block part
    # full, R and T ranges not starting at 1
    (3, (5, 6, 7, 16), 0.25, 2, (2, 4, 3, 8)),
    (3, (3, 3, 3, 64), 0.25, 1, (1, 2, 1, 32)),    # 16 threads per column
    # SU(2) with 8 | Lt runs its one-column kernel (four starts per thread,
    # the T sweep in steps of five): fewer T values than one step, and a T
    # range that is not a multiple of five
    (2, (4, 5, 3, 32), 0.3, 2, (2, 3, 4, 7)),
    (2, (6, 5, 7, 48), 0.3, 1, (1, 3, 3, 24)),
    # long time extents: SU(2) beyond the one-column kernel's 32 threads per
    # column (the two-column kernel), SU(3) at 32 threads per column
    (2, (2, 3, 2, 192), 0.3, 1, (1, 1, 20, 24)),
    (3, (2, 2, 2, 128), 0.25, 1, (1, 2, 1, 4)),
])
def test_gauge_form_matches_oracle_seeded(port, nc, dims, eps, n_ape, rng):
    links = generate_config(dims, nc, eps, 20261203, 11)
    ref = links.copy()
    port.hyp(nc, dims, ref, 1.0, 0.75, 0.6, 1)
    port.ape(nc, dims, ref, 0.5, n_ape)
    w_ref = port.wilson(nc, dims, ref, *rng)
    wa_ref = port.wilson_adjoint(nc, dims, ref, *rng)
    res = {}
    for form in ("fp64", "mixed"):
        with Lattice(dims, nc, form) as lat:
            lat.upload(links)
            lat.hyp(1.0, 0.75, 0.6, 1)
            lat.ape(0.5, n_ape)
            res[form] = _both(lat, rng)
            res[form + "_adj"] = _both(lat, rng, adjoint=True)
    for key in ("fp64", "mixed"):
        assert res[key]["auto_used"] == "gauge"
    for m in ("auto", "exact"):
        np.testing.assert_allclose(res["fp64"][m], w_ref, rtol=W_RTOL, atol=W_ATOL)
        np.testing.assert_allclose(res["fp64_adj"][m], wa_ref, rtol=W_RTOL, atol=W_ATOL)
        assert np.max(np.abs(res["mixed"][m] - w_ref) / np.abs(w_ref)) <= 1e-6
        assert np.max(np.abs(res["mixed_adj"][m] - wa_ref)) <= 1e-6 * np.max(np.abs(wa_ref))


@pytest.mark.parametrize("form,scale", [("fp64", 1 + 1e-9), ("mixed", 1 + 1e-5)])
def test_non_unitary_temporal_links_take_the_exact_product(port, form, scale):
    """Temporal links that fail the unitarity check: the result is the exact
    product's (bit for bit), and in FP64 the reference's. (The mixed form
    keeps two rows of a link and rebuilds the third as for an SU(3) matrix, so
    its scaled links are not the reference's; only the method is checked.)"""
    nc, dims, rng = 3, (6, 6, 6, 8), (1, 3, 1, 4)
    links = generate_config(dims, nc, 0.25, 20261203, 3)
    links[3::4] *= scale  # every temporal link (index 4*site + 3)
    with Lattice(dims, nc, form) as lat:
        lat.upload(links)
        w = lat.wilson_loop(*rng)
        assert lat.wilson_method_used() == "exact"
        lat.set_wilson_method("exact")
        assert np.array_equal(lat.wilson_loop(*rng), w)
    if form == "fp64":
        np.testing.assert_allclose(w, port.wilson(nc, dims, links, *rng), rtol=W_RTOL,
                                   atol=W_ATOL)


def test_long_time_range_takes_the_exact_product():
    nc, dims = 2, (4, 4, 4, 8)
    links = generate_config(dims, nc, 0.3, 20261203, 3)
    with Lattice(dims, nc, "fp64") as lat:
        lat.upload(links)
        lat.wilson_loop(1, 2, 1, 4)
        assert lat.wilson_method_used() == "gauge"
        lat.wilson_loop(1, 2, 1, 5)
        assert lat.wilson_method_used() == "exact"


@pytest.mark.parametrize("nc,dims,n_ape,rt", [
    (3, (24, 24, 24, 24), 20, 12),
    (3, (8, 8, 8, 16), 3, 8),
    (2, (16, 16, 16, 16), 10, 8),
])
def test_mixed_gauge_form_keeps_the_exact_products_accuracy(nc, dims, n_ape, rt):
    """The mixed form's temporal links leave their last projection step with
    singular values a few 1e-10 below one; the gauge lines are built from the
    links made unitary in FP64, so the gauge form's W error against FP64 stays
    at the exact product's (measured 2-6e-9; with the stored links it grew
    linearly in R and T to 3.4e-8 at 24^4)."""
    links = generate_config(dims, nc, 0.25 if nc == 3 else 0.3, 20261203, 0)
    res = {}
    for form in ("fp64", "mixed"):
        with Lattice(dims, nc, form) as lat:
            lat.upload(links)
            lat.hyp(1.0, 0.75, 0.6, 1)
            lat.ape(0.5, n_ape)
            res[form] = _both(lat, (1, rt, 1, rt))
    ref = res["fp64"]["exact"]
    assert res["mixed"]["auto_used"] == "gauge"
    err = {m: float(np.max(np.abs(res["mixed"][m] - ref) / np.abs(ref))) for m in ("auto", "exact")}
    assert err["auto"] <= 1e-8, err
    assert err["auto"] <= 2 * err["exact"] + 2e-9, err
