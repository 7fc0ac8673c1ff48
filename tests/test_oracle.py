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


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_port_observables_match_reference_fixture(port, name, meta):
    """GEVP tables, time/space plaquettes, Polyakov loop and correlators."""
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    r0, r1, t0, t1 = meta["r_min"], meta["r_max"], meta["time_min"], meta["time_max"]
    for adjoint, key in ((False, "gevp"), (True, "gevp_adjoint")):
        w = port.wilson_gevp(nc, dims, g["links_ape"], g["links_hyp"], r0, r1, t0, t1, adjoint)
        np.testing.assert_allclose(w, g[key], rtol=1e-12, atol=1e-14)
    pt, ps = g["plaquettes_time_space"]
    assert port.plaquette_time(nc, dims, g["links_ape"]) == pytest.approx(pt, rel=1e-12)
    assert port.plaquette_space(nc, dims, g["links_ape"]) == pytest.approx(ps, rel=1e-12)
    assert port.polyakov_loop(nc, dims, g["links_hyp"]) == pytest.approx(
        float(g["polyakov_loop"][0]), rel=1e-12, abs=1e-14)
    d = meta["polyakov_d_max"]
    for singlet, key in ((True, "polyakov_singlet"), (False, "polyakov_color_average")):
        c = port.polyakov_correlator(nc, dims, g["links_hyp"], d, singlet)
        np.testing.assert_allclose(c, g[key], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_reference_reproduces_observable_fixture(name, meta):
    from oracle import py_oracle
    if not py_oracle.ref_available("parity"):
        pytest.skip("reference not compiled in this checkout (oracle/_ref)")
    ref = py_oracle.ref("parity")
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    r0, r1, t0, t1 = meta["r_min"], meta["r_max"], meta["time_min"], meta["time_max"]
    w = ref.wilson_gevp(nc, dims, g["links_ape"], g["links_hyp"], r0, r1, t0, t1, False)
    np.testing.assert_allclose(w, g["gevp"], rtol=1e-13, atol=0)
    assert ref.polyakov_loop(nc, dims, g["links_hyp"]) == float(g["polyakov_loop"][0])
    c = ref.polyakov_correlator(nc, dims, g["links_hyp"], meta["polyakov_d_max"], True)
    np.testing.assert_allclose(c, g["polyakov_singlet"], rtol=1e-13, atol=1e-16)


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_polyakov_distance_average_matches_reference(name, meta):
    """Host-side polyakov_average_directions against the reference's output."""
    from general_code_b200 import polyakov_average_directions
    g = load_golden(name)
    d = meta["polyakov_d_max"]
    for key in ("polyakov_singlet", "polyakov_color_average"):
        got = polyakov_average_directions(g[key], d)
        want = meta[f"{key}_by_distance"]
        assert [k for k in got] == pytest.approx([k for k, _ in want], abs=0)
        np.testing.assert_allclose(list(got.values()), [v for _, v in want], rtol=1e-15,
                                   atol=1e-17)


@pytest.mark.parametrize("nc", [2, 3])
def test_gevp_of_identical_configurations_is_the_wilson_table(port, nc):
    dims = (4, 4, 3, 6)
    a = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 21, 0)
    for adjoint in (False, True):
        w = port.wilson_gevp(nc, dims, a, a, 1, 2, 1, 3, adjoint)
        ref = (port.wilson_adjoint if adjoint else port.wilson)(nc, dims, a, 1, 2, 1, 3)
        np.testing.assert_allclose(w, ref, rtol=1e-13, atol=1e-15)


def visited_offsets(d):
    """Offsets the reference's correlators visit (polyakov_loops.h:100-113)."""
    out = []
    for dz in range(-d, d + 1):
        for dy in range(-d, d + 1):
            for dx in range(0 if (dy and dz) else -d, d + 1):
                if (dx * dx + dy * dy + dz * dz) ** 0.5 <= d:
                    out.append((dx, dy, dz))
    return out


@pytest.mark.parametrize("nc", [2, 3])
def test_polyakov_of_unit_and_abelian_configurations(port, nc):
    """Unit links: P = 1, loop 1, all visited correlator entries 1. The
    constant-flux configuration has unit time links, so the same holds."""
    from conftest import abelian_flux_config
    dims = (6, 5, 4, 8)
    for links in (unit_config(dims, nc), abelian_flux_config(dims, nc)[0]):
        assert port.polyakov_loop(nc, dims, links) == pytest.approx(1.0, abs=1e-14)
        for singlet in (True, False):
            c = port.polyakov_correlator(nc, dims, links, 2, singlet)
            assert set(np.round(c[c != 0], 12)) == {1.0}
            assert np.count_nonzero(c) == len(visited_offsets(2))


def _offaxis_fixture(meta, key):
    return {(int(t), float(s)): w for t, s, w in meta[key]}


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_port_offaxis_matches_reference_fixture(port, name, meta):
    """Merged off-axis loops (wilson_offaxis[_adjoint]_result) of the C
    restatement against the reference's values, 1e-12 relative."""
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    r0, r1, t0, t1 = meta["offaxis_range"]
    for adjoint, key in ((False, "offaxis"), (True, "offaxis_adjoint")):
        want = _offaxis_fixture(meta, key)
        if not want:
            continue
        got = port.wilson_offaxis_result(nc, dims, g["links_ape"], r0, r1, t0, t1, adjoint)
        assert set(got) == set(want)
        for k, v in want.items():
            assert got[k] == pytest.approx(v, rel=1e-12, abs=1e-14)


@pytest.mark.parametrize("nc", [2, 3])
def test_port_offaxis_entries_match_reference(nc):
    """Unmerged entries (order, sizes, orientation counts and values) of the
    C restatement against the reference compiled here, including directions
    with no zero component (whose identity reflection the reference counts
    twice) and multipliers above 1."""
    from oracle import py_oracle
    if not py_oracle.ref_available("parity"):
        pytest.skip("reference not compiled in this checkout (oracle/_ref)")
    port, ref = py_oracle.port(), py_oracle.ref("parity")
    dims = (4, 5, 4, 6)
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 17, 0)
    dirs = [[1, 0, 0], [1, 1, 0], [2, 1, 0], [1, 1, 1], [2, 1, 1]]
    for adjoint in ((False, True) if nc == 3 else (False,)):
        a = port.wilson_offaxis(nc, dims, links, dirs, 0.5, 3.5, 1, 3, adjoint)
        b = ref.wilson_offaxis(nc, dims, links, dirs, 0.5, 3.5, 1, 3, adjoint)
        assert [x[1:] for x in a] == [x[1:] for x in b]
        np.testing.assert_allclose([x[0] for x in a], [x[0] for x in b], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("nc", [2, 3])
def test_offaxis_of_unit_configuration_is_one(port, nc):
    dims = (4, 4, 4, 4)
    got = port.wilson_offaxis_result(nc, dims, unit_config(dims, nc), 1.0, 2.0, 1, 2)
    assert got and all(abs(v - 1.0) < 1e-14 for v in got.values())


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_port_spatial_loops_match_reference_fixture(port, name, meta):
    """smearing_APE_2d (bit for bit) and wilson_spatial_3d_indexed of the C
    restatement against the reference's values."""
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    a, b, alpha, steps = meta["ape_plane"]
    links = g["links_hyp"].copy()
    port.ape_plane(nc, dims, links, a, b, alpha, steps)
    assert max_abs(links, g["links_ape_plane"]) <= 1e-13
    got = port.wilson_spatial_3d(nc, dims, g["links_hyp"], *meta["spatial_args"])
    want = {(s, t, r): w for s, t, r, w in meta["spatial"]}
    assert set(got) == set(want)
    for k, v in want.items():
        assert got[k] == pytest.approx(v, rel=1e-12, abs=1e-14)


@pytest.mark.parametrize("nc", [2, 3])
def test_port_spatial_loops_match_reference_quirky_ranges(nc):
    """Ranges where the reference's space lines start with length time_min
    (r_min != time_min), a start above the step (only smearing 0 measured)
    and steps of 2."""
    from oracle import py_oracle
    if not py_oracle.ref_available("parity"):
        pytest.skip("reference not compiled in this checkout (oracle/_ref)")
    port, ref = py_oracle.port(), py_oracle.ref("parity")
    dims = (4, 5, 4, 6)
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 23, 0)
    for args in ((1, 2, 2, 3, 0.5, 0, 4, 2), (2, 3, 1, 2, 0.4, 2, 3, 1), (1, 3, 1, 3, 0.5, 1, 2, 1)):
        a = port.wilson_spatial_3d(nc, dims, links, *args)
        b = ref.wilson_spatial_3d(nc, dims, links, *args)
        assert set(a) == set(b)
        for k, v in b.items():
            assert a[k] == pytest.approx(v, rel=1e-12, abs=1e-14)


def test_fullsize_fixture_inputs_come_from_both_generators():
    """The large-lattice W tables (tests/golden/fullsize.json) were computed by
    the reference on the configurations the product's generator makes from
    the fixture's seed: both copies of the generator (the product library's
    and the checkers' oracle/libgen.so) reproduce the recorded input."""
    import hashlib
    import json
    from pathlib import Path

    from general_code_b200 import generate_config
    from oracle import py_oracle
    cases = json.loads((Path(__file__).resolve().parent / "golden" /
                        "fullsize.json").read_text())["cases"]
    assert "su3_32" in cases
    for name, c in cases.items():
        args = (tuple(c["dims"]), c["nc"], c["eps"], c["seed"], c["config_index"])
        a = generate_config(*args)
        assert hashlib.sha256(a.tobytes()).hexdigest() == c["input_sha256"], name
        b = py_oracle.generator().generate(*args)
        assert np.array_equal(a, b), name
        # the tables are the reference's W(R,T): O(1) positive, decreasing in T
        w = np.array(c["wilson"])
        assert w.shape == (c["time_max"] - c["time_min"] + 1, c["r_max"] - c["r_min"] + 1)
        assert np.all((w > 0) & (w < 1)) and np.all(np.diff(w, axis=0) < 0)
