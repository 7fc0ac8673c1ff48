"""The C restatement (oracle/gc_oracle.c) against the golden fixtures made by
the reference's own code, plus known-answer properties of the path.

Tolerances (FP64): links 1e-13 absolute (entries are O(1)); W(R,T) and the
plaquette 1e-12 relative. The restatement follows the reference's operation
order, so links agree bit for bit; the sums differ only in summation order.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_cases, load_golden, max_abs, unitarity_error
from general_code_b200 import generate_config, unit_config

CASES = golden_cases()


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_port_matches_reference_fixture(port, name, meta):
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    links = g["links0"].copy()
    assert abs(port.plaquette(nc, dims, links) - g["plaquettes"][0]) <= 1e-12 * abs(g["plaquettes"][0])
    port.hyp(nc, dims, links, *meta["hyp_alpha"], 1)
    assert max_abs(links, g["links_hyp"]) <= 1e-13
    port.ape(nc, dims, links, meta["ape_alpha"], meta["ape_steps"])
    assert max_abs(links, g["links_ape"]) <= 1e-13
    w = port.wilson(nc, dims, links, meta["r_min"], meta["r_max"], meta["time_min"], meta["time_max"])
    np.testing.assert_allclose(w, g["wilson"], rtol=1e-12, atol=0)
    wa = port.wilson_adjoint(nc, dims, links, meta["r_min"], meta["r_max"], meta["time_min"],
                             meta["time_max"])
    np.testing.assert_allclose(wa, g["wilson_adjoint"], rtol=1e-12, atol=1e-14)
    assert abs(port.plaquette(nc, dims, links) - g["plaquettes"][1]) <= 1e-12


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_reference_reproduces_fixture(name, meta):
    """When the reference was compiled here, it still produces the fixture."""
    from oracle import py_oracle
    if not py_oracle.ref_available("parity"):
        pytest.skip("reference not compiled in this checkout (oracle/_ref)")
    ref = py_oracle.ref("parity")
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    links = g["links0"].copy()
    ref.hyp(nc, dims, links, *meta["hyp_alpha"], 1)
    assert max_abs(links, g["links_hyp"]) == 0.0
    ref.ape(nc, dims, links, meta["ape_alpha"], meta["ape_steps"])
    assert max_abs(links, g["links_ape"]) == 0.0
    w = ref.wilson(nc, dims, links, meta["r_min"], meta["r_max"], meta["time_min"], meta["time_max"])
    np.testing.assert_allclose(w, g["wilson"], rtol=1e-13, atol=0)
    wa = ref.wilson_adjoint(nc, dims, links, meta["r_min"], meta["r_max"], meta["time_min"],
                            meta["time_max"])
    np.testing.assert_allclose(wa, g["wilson_adjoint"], rtol=1e-13, atol=0)


@pytest.mark.parametrize("nc", [2, 3])
def test_unit_configuration_known_answers(port, nc):
    dims = (4, 3, 4, 5)
    u = unit_config(dims, nc)
    assert port.plaquette(nc, dims, u) == pytest.approx(1.0, abs=1e-15)
    w = port.wilson(nc, dims, u, 1, 2, 1, 3)
    np.testing.assert_allclose(w, 1.0, atol=1e-15)
    v = u.copy()
    port.hyp(nc, dims, v, 1.0, 0.75, 0.6, 1)
    port.ape(nc, dims, v, 0.5, 2)
    assert max_abs(u, v) <= 1e-15  # unit links are a fixed point


@pytest.mark.parametrize("nc,eps", [(2, 0.3), (3, 0.25)])
def test_gauge_invariance_after_smearing(port, nc, eps):
    """W after HYP+APE is the same for a configuration and its gauge transform."""
    dims = (4, 4, 4, 6)
    a = generate_config(dims, nc, eps, 99, 0, gauge=False)
    b = generate_config(dims, nc, eps, 99, 0, gauge=True)
    assert max_abs(a, b) > 0.1
    for x in (a, b):
        port.hyp(nc, dims, x, 1.0, 0.75, 0.6, 1)
        port.ape(nc, dims, x, 0.5, 3)
    wa = port.wilson(nc, dims, a, 1, 2, 1, 3)
    wb = port.wilson(nc, dims, b, 1, 2, 1, 3)
    np.testing.assert_allclose(wa, wb, rtol=1e-11)
    assert port.plaquette(nc, dims, a) == pytest.approx(port.plaquette(nc, dims, b), rel=1e-12)


@pytest.mark.parametrize("nc,eps", [(2, 0.3), (3, 0.25)])
def test_smeared_links_are_special_unitary(port, nc, eps):
    dims = (4, 4, 4, 4)
    a = generate_config(dims, nc, eps, 3, 0)
    port.hyp(nc, dims, a, 1.0, 0.75, 0.6, 1)
    port.ape(nc, dims, a, 0.5, 2)
    assert unitarity_error(nc, a) < 1e-12


@pytest.mark.parametrize("nc", [2, 3])
def test_abelian_flux_closed_form(port, nc):
    from conftest import abelian_flux_config
    dims = (6, 5, 4, 8)
    links, wf, plaq = abelian_flux_config(dims, nc)
    assert port.plaquette(nc, dims, links) == pytest.approx(plaq, abs=1e-14)
    expect = np.array([[wf(r, t) for r in range(1, 4)] for t in range(1, 5)])
    np.testing.assert_allclose(port.wilson(nc, dims, links, 1, 3, 1, 4), expect, atol=1e-14)
    v = links.copy()
    port.ape(nc, dims, v, 0.5, 3)  # fixed point
    assert max_abs(v, links) <= 1e-14
    np.testing.assert_allclose(port.wilson(nc, dims, v, 1, 3, 1, 4), expect, atol=1e-14)
