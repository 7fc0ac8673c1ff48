"""GPU parity: the sm_100a kernels, called through the C ABI, against the
golden fixtures (made by the reference's own code) and against the C oracle on
seeded configurations.

FP64 tolerances: links 1e-12 absolute (entries are O(1)); W(R,T) and the
plaquette 1e-12 relative with a 1e-14 absolute floor (the GPU sums in a
different, fixed order than the reference's OpenMP reduction).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_cases, load_golden, max_abs, unitarity_error
from general_code_b200 import GCError, Lattice, generate_config, unit_config
from general_code_b200 import _lib

pytestmark = pytest.mark.gpu
CASES = golden_cases()
W_RTOL, W_ATOL = 1e-12, 1e-14
LINK_ATOL = 1e-12


def assert_w_close(w, ref):
    np.testing.assert_allclose(w, ref, rtol=W_RTOL, atol=W_ATOL)


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_fp64_matches_reference_fixture(name, meta):
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    with Lattice(dims, nc, "fp64") as lat:
        lat.upload(g["links0"])
        assert lat.plaquette() == pytest.approx(g["plaquettes"][0], rel=1e-12)
        lat.hyp(*meta["hyp_alpha"], 1)
        assert max_abs(lat.download(), g["links_hyp"]) <= LINK_ATOL
        lat.ape(meta["ape_alpha"], meta["ape_steps"])
        assert max_abs(lat.download(), g["links_ape"]) <= LINK_ATOL
        w = lat.wilson_loop(meta["r_min"], meta["r_max"], meta["time_min"], meta["time_max"])
        assert_w_close(w, g["wilson"])
        wa = lat.wilson_loop_adjoint(meta["r_min"], meta["r_max"], meta["time_min"],
                                     meta["time_max"])
        assert_w_close(wa, g["wilson_adjoint"])
        assert lat.plaquette() == pytest.approx(g["plaquettes"][1], rel=1e-12)


@pytest.mark.parametrize("nc,dims,eps,hyp,n_ape,rng", [
    (2, (8, 8, 8, 8), 0.3, (1.0, 0.75, 0.6), 10, (1, 4, 1, 4)),
    (3, (8, 8, 8, 12), 0.25, (1.0, 0.75, 0.6), 5, (1, 4, 1, 6)),
    (3, (6, 10, 4, 12), 0.25, (1.0, 1.0, 0.5), 3, (2, 3, 3, 6)),
    (2, (5, 7, 3, 9), 0.3, (0.8, 0.6, 0.4), 4, (1, 3, 1, 5)),
    # 7 warps x 25 (R,T) entries: an odd number of FP64 accumulators in the W
    # kernel's shared memory ahead of its 16-byte column arrays
    (3, (10, 10, 10, 10), 0.25, (1.0, 0.75, 0.6), 2, (1, 5, 1, 5)),
    # time extents above 32: one start slice per thread, 256-thread W blocks
    (3, (4, 4, 4, 48), 0.25, (1.0, 0.75, 0.6), 2, (1, 2, 1, 20)),
    (2, (4, 3, 5, 40), 0.3, (1.0, 0.75, 0.6), 2, (1, 2, 2, 17)),
])
def test_fp64_matches_oracle_seeded(port, nc, dims, eps, hyp, n_ape, rng):
    links = generate_config(dims, nc, eps, 20261203, 7)
    ref = links.copy()
    port.hyp(nc, dims, ref, *hyp, 1)
    port.ape(nc, dims, ref, 0.5, n_ape)
    w_ref = port.wilson(nc, dims, ref, *rng)
    with Lattice(dims, nc, "fp64") as lat:
        lat.upload(links)
        lat.hyp(*hyp, 1)
        lat.ape(0.5, n_ape)
        assert max_abs(lat.download(), ref) <= LINK_ATOL
        assert_w_close(lat.wilson_loop(*rng), w_ref)
        assert_w_close(lat.wilson_loop_adjoint(*rng), port.wilson_adjoint(nc, dims, ref, *rng))
        assert lat.plaquette() == pytest.approx(port.plaquette(nc, dims, ref), rel=1e-12)


@pytest.mark.parametrize("nc", [2, 3])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_unit_configuration(nc, precision):
    dims = (4, 6, 4, 8)
    with Lattice(dims, nc, precision) as lat:
        lat.upload(unit_config(dims, nc))
        lat.hyp(1.0, 0.75, 0.6, 1)
        lat.ape(0.5, 3)
        np.testing.assert_allclose(lat.wilson_loop(1, 2, 1, 4), 1.0, atol=1e-14)
        assert lat.plaquette() == pytest.approx(1.0, abs=1e-14)
        assert max_abs(lat.download(), unit_config(dims, nc)) <= 1e-15


@pytest.mark.parametrize("nc", [2, 3])
def test_long_time_range_uses_r_chunks(port, nc):
    """nT*nR above the per-block accumulator budget splits R into chunks; T
    beyond the extent wraps around the periodic lattice."""
    dims = (4, 4, 4, 4)
    links = generate_config(dims, nc, 0.2, 5, 0)
    w_ref = port.wilson(nc, dims, links, 1, 4, 1, 300)
    with Lattice(dims, nc, "fp64") as lat:
        lat.upload(links)
        assert_w_close(lat.wilson_loop(1, 4, 1, 300), w_ref)


@pytest.mark.parametrize("nc", [2, 3])
def test_eigen_layout_round_trip(nc):
    dims = (4, 4, 4, 6)
    links = generate_config(dims, nc, 0.3, 1, 0)
    with Lattice(dims, nc, "fp64") as lat:
        lat.upload(links)
        eig = lat.download(layout="eigen")
        back = lat.download()
        assert max_abs(back, links) == 0.0
        if nc == 3:
            m = links.reshape(-1, 3, 3, 2)
            assert max_abs(eig.reshape(-1, 3, 3, 2), np.transpose(m, (0, 2, 1, 3))) == 0.0
        lat.upload(eig, layout="eigen")
        assert max_abs(lat.download(), links) == 0.0


def test_state_and_argument_errors():
    with Lattice((4, 4, 4, 4), 3) as lat:
        with pytest.raises(GCError) as e:
            lat.wilson_loop(1, 2, 1, 2)
        assert e.value.code == _lib.GC_ERR_STATE
        lat.upload(unit_config((4, 4, 4, 4), 3))
        with pytest.raises(GCError) as e:
            lat.wilson_loop(2, 1, 1, 2)
        assert e.value.code == _lib.GC_ERR_ARG
        with pytest.raises(GCError) as e:
            lat.ape(0.5, -1)
        assert e.value.code == _lib.GC_ERR_ARG


@pytest.mark.parametrize("nc,eps", [(2, 0.3), (3, 0.25)])
def test_device_generator_matches_host(nc, eps):
    dims = (6, 4, 4, 8)
    host = generate_config(dims, nc, eps, 42, 3)
    with Lattice(dims, nc) as lat:
        lat.generate(eps, 42, 3)
        assert max_abs(lat.download(), host) == 0.0


@pytest.mark.parametrize("nc,eps", [(2, 0.3), (3, 0.25)])
def test_mixed_precision_error_budget(port, nc, eps):
    """Mixed form (FP32 links, FP64 final projection step and sums) against
    the FP64 oracle: links within 1e-5 and W within 1e-6 relative (the mixed
    form's bar) after HYP + 5 APE."""
    dims = (8, 8, 8, 8)
    links = generate_config(dims, nc, eps, 11, 0)
    ref = links.copy()
    port.hyp(nc, dims, ref, 1.0, 0.75, 0.6, 1)
    port.ape(nc, dims, ref, 0.5, 5)
    w_ref = port.wilson(nc, dims, ref, 1, 4, 1, 4)
    with Lattice(dims, nc, "mixed") as lat:
        lat.upload(links)
        lat.hyp(1.0, 0.75, 0.6, 1)
        lat.ape(0.5, 5)
        got = lat.download()
        assert max_abs(got, ref) < 1e-5
        assert unitarity_error(nc, got) < 1e-6
        w = lat.wilson_loop(1, 4, 1, 4)
    np.testing.assert_allclose(w, w_ref, rtol=1e-6)


@pytest.mark.parametrize("nc,eps", [(2, 0.3), (3, 0.25)])
def test_mixed_w_within_1e6_after_long_smearing(port, nc, eps):
    """Every W(R,T) of the mixed form within 1e-6 relative of the FP64 oracle
    after HYP + 20 APE steps on a 12^4 lattice, R, T up to 6."""
    dims = (12, 12, 12, 12)
    links = generate_config(dims, nc, eps, 20261203, 41)
    ref = links.copy()
    port.hyp(nc, dims, ref, 1.0, 0.75, 0.6, 1)
    port.ape(nc, dims, ref, 0.5, 20)
    w_ref = port.wilson(nc, dims, ref, 1, 6, 1, 6)
    with Lattice(dims, nc, "mixed") as lat:
        lat.upload(links)
        lat.hyp(1.0, 0.75, 0.6, 1)
        lat.ape(0.5, 20)
        w = lat.wilson_loop(1, 6, 1, 6)
    np.testing.assert_allclose(w, w_ref, rtol=1e-6, atol=0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_results_are_deterministic(precision):
    dims = (8, 8, 8, 8)
    out = []
    for _ in range(2):
        with Lattice(dims, 3, precision) as lat:
            lat.generate(0.25, 1, 0)
            lat.hyp(1.0, 0.75, 0.6, 1)
            lat.ape(0.5, 3)
            out.append((lat.wilson_loop(1, 4, 1, 4), lat.plaquette()))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]


@pytest.mark.parametrize("nc", [2, 3])
@pytest.mark.parametrize("precision,atol", [("fp64", 1e-14), ("mixed", 1e-6)])
def test_abelian_flux_closed_form(nc, precision, atol):
    """Closed-form W(R,T) and plaquette of a constant-flux diagonal
    configuration, before and after APE (for which it is a fixed point)."""
    from conftest import abelian_flux_config
    dims = (6, 5, 4, 8)
    links, wf, plaq = abelian_flux_config(dims, nc)
    expect = np.array([[wf(r, t) for r in range(1, 4)] for t in range(1, 5)])
    with Lattice(dims, nc, precision) as lat:
        lat.upload(links)
        assert lat.plaquette() == pytest.approx(plaq, abs=atol)
        np.testing.assert_allclose(lat.wilson_loop(1, 3, 1, 4), expect, atol=atol)
        lat.ape(0.5, 3)
        assert max_abs(lat.download(), links) <= (1e-14 if precision == "fp64" else 1e-6)
        np.testing.assert_allclose(lat.wilson_loop(1, 3, 1, 4), expect, atol=atol)


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_fp64_observables_match_reference_fixture(name, meta):
    """GEVP tables (two handles), time/space plaquettes, Polyakov loop and
    correlators against the reference's values."""
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    r0, r1, t0, t1 = meta["r_min"], meta["r_max"], meta["time_min"], meta["time_max"]
    with Lattice(dims, nc, "fp64") as a, Lattice(dims, nc, "fp64") as b:
        a.upload(g["links_ape"])
        b.upload(g["links_hyp"])
        assert_w_close(a.wilson_gevp(b, r0, r1, t0, t1), g["gevp"])
        assert_w_close(a.wilson_gevp(b, r0, r1, t0, t1, adjoint=True), g["gevp_adjoint"])
        pt, ps = g["plaquettes_time_space"]
        assert a.plaquette_time() == pytest.approx(pt, rel=1e-12)
        assert a.plaquette_space() == pytest.approx(ps, rel=1e-12)
        assert b.polyakov_loop() == pytest.approx(float(g["polyakov_loop"][0]), rel=1e-12,
                                                  abs=1e-14)
        d = meta["polyakov_d_max"]
        np.testing.assert_allclose(b.polyakov_correlator(d, True), g["polyakov_singlet"],
                                   rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(b.polyakov_correlator(d, False),
                                   g["polyakov_color_average"], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("nc,eps", [(2, 0.3), (3, 0.25)])
def test_observables_match_oracle_seeded(port, nc, eps):
    """Larger lattices (several W blocks, several Polyakov blocks) in both
    forms: FP64 within 1e-12, mixed within 1e-6 relative / 1e-7 absolute."""
    dims = (8, 6, 10, 12)
    a = generate_config(dims, nc, eps, 20261203, 31)
    b = generate_config(dims, nc, eps, 20261203, 32)
    want = {"gevp": port.wilson_gevp(nc, dims, a, b, 1, 4, 1, 6),
            "gevp_adj": port.wilson_gevp(nc, dims, a, b, 1, 4, 1, 6, True),
            "pt": port.plaquette_time(nc, dims, a), "ps": port.plaquette_space(nc, dims, a),
            "poly": port.polyakov_loop(nc, dims, a),
            "sing": port.polyakov_correlator(nc, dims, a, 3, True),
            "col": port.polyakov_correlator(nc, dims, a, 3, False)}
    for precision, rtol, atol in (("fp64", 1e-12, 1e-14), ("mixed", 1e-6, 1e-7)):
        with Lattice(dims, nc, precision) as la, Lattice(dims, nc, precision) as lb:
            la.upload(a)
            lb.upload(b)
            np.testing.assert_allclose(la.wilson_gevp(lb, 1, 4, 1, 6), want["gevp"], rtol=rtol,
                                       atol=atol)
            np.testing.assert_allclose(la.wilson_gevp(lb, 1, 4, 1, 6, True), want["gevp_adj"],
                                       rtol=rtol, atol=atol)
            assert la.plaquette_time() == pytest.approx(want["pt"], rel=rtol, abs=atol)
            assert la.plaquette_space() == pytest.approx(want["ps"], rel=rtol, abs=atol)
            assert la.plaquette() == pytest.approx(0.5 * (want["pt"] + want["ps"]), rel=rtol)
            assert la.polyakov_loop() == pytest.approx(want["poly"], rel=rtol, abs=atol)
            np.testing.assert_allclose(la.polyakov_correlator(3, True), want["sing"], rtol=rtol,
                                       atol=atol)
            np.testing.assert_allclose(la.polyakov_correlator(3, False), want["col"], rtol=rtol,
                                       atol=atol)


@pytest.mark.parametrize("nc", [2, 3])
def test_gevp_with_itself_and_argument_errors(nc):
    dims = (4, 4, 4, 6)
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 5, 0)
    with Lattice(dims, nc, "fp64") as a, Lattice((4, 4, 4, 8), nc, "fp64") as other, \
            Lattice(dims, nc, "mixed") as m:
        a.upload(links)
        other.upload(generate_config((4, 4, 4, 8), nc, 0.3, 5, 0))
        m.upload(links)
        # the same handle as both configurations gives the ordinary table
        np.testing.assert_allclose(a.wilson_gevp(a, 1, 2, 1, 3), a.wilson_loop(1, 2, 1, 3),
                                   rtol=1e-13, atol=1e-15)
        with pytest.raises(GCError):
            a.wilson_gevp(other, 1, 2, 1, 3)  # different sizes
        with pytest.raises(GCError):
            a.wilson_gevp(m, 1, 2, 1, 3)  # different precision
        with pytest.raises(GCError):
            a.polyakov_correlator(-1, True)


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_fp64_offaxis_matches_reference_fixture(name, meta):
    """Merged off-axis loops through the C ABI against the reference's values."""
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    r0, r1, t0, t1 = meta["offaxis_range"]
    with Lattice(dims, nc, "fp64") as lat:
        lat.upload(g["links_ape"])
        for adjoint, key in ((False, "offaxis"), (True, "offaxis_adjoint")):
            want = {(int(t), float(s)): w for t, s, w in meta[key]}
            if not want:
                continue
            got = lat.wilson_offaxis_result(r0, r1, t0, t1, adjoint)
            assert set(got) == set(want)
            for k, v in want.items():
                assert got[k] == pytest.approx(v, rel=W_RTOL, abs=W_ATOL)


@pytest.mark.parametrize("nc,eps,dims", [(2, 0.3, (7, 6, 8, 6)), (3, 0.25, (7, 6, 8, 6)),
                                         (3, 0.25, (4, 3, 5, 40))])
def test_offaxis_matches_oracle_seeded(port, nc, eps, dims):
    """Unmerged entries for several directions (multipliers up to 3, odd
    extents, negative displacements after reflection; Lt = 40: 40 threads
    per column in the fused kernel) in both forms: FP64 within 1e-12, mixed
    within 1e-6 relative."""
    links = generate_config(dims, nc, eps, 20261203, 51)
    dirs = [[1, 0, 0], [1, 1, 0], [2, 1, 0], [1, 1, 1], [2, 2, 1]]
    for adjoint in (False, True):
        want = port.wilson_offaxis(nc, dims, links, dirs, 0.9, 3.1, 1, 4, adjoint)
        for precision, rtol in (("fp64", 1e-12), ("mixed", 1e-6)):
            with Lattice(dims, nc, precision) as lat:
                lat.upload(links)
                got = lat.wilson_offaxis(dirs, 0.9, 3.1, 1, 4, adjoint)
            assert [x[1:] for x in got] == [x[1:] for x in want]
            np.testing.assert_allclose([x[0] for x in got], [x[0] for x in want], rtol=rtol,
                                       atol=1e-14 if precision == "fp64" else 1e-7)


def test_offaxis_argument_errors():
    dims = (4, 4, 4, 4)
    with Lattice(dims, 3, "fp64") as lat:
        lat.upload(generate_config(dims, 3, 0.25, 1, 0))
        with pytest.raises(GCError):
            lat.wilson_offaxis([[0, 1, 0]], 1.0, 2.0, 1, 2)  # a1 must be >= 1 and largest
        with pytest.raises(GCError):
            lat.wilson_offaxis([[1, 0, 0]], 1.0, 2.0, 0, 2)  # time_min >= 1
        with pytest.raises(GCError):
            lat.wilson_offaxis([[1, 0, 0]], 1.0, 400.0, 1, 2)  # a line over 256 links
        assert lat.wilson_offaxis([[3, 0, 0]], 1.0, 2.0, 1, 2) == []  # no length in range


@pytest.mark.parametrize("name,meta", CASES, ids=[c[0] for c in CASES])
def test_fp64_spatial_loops_match_reference_fixture(name, meta):
    """gc_ape_plane against the reference's smearing_APE_2d links, and the
    spatial loop table against wilson_spatial_3d_indexed."""
    g = load_golden(name)
    nc, dims = meta["nc"], meta["dims"]
    a, b, alpha, steps = meta["ape_plane"]
    with Lattice(dims, nc, "fp64") as lat:
        lat.upload(g["links_hyp"])
        got = lat.wilson_spatial_3d(*meta["spatial_args"])
        lat.ape_plane(a, b, alpha, steps)
        assert max_abs(lat.download(), g["links_ape_plane"]) <= LINK_ATOL
    want = {(s, t, r): w for s, t, r, w in meta["spatial"]}
    assert set(got) == set(want)
    for k, v in want.items():
        assert got[k] == pytest.approx(v, rel=W_RTOL, abs=W_ATOL)


@pytest.mark.parametrize("nc,eps", [(2, 0.3), (3, 0.25)])
def test_spatial_loops_match_oracle_seeded(port, nc, eps):
    """Larger, unequal lattice and the quirky ranges (r_min != time_min,
    measurement every second step) in both forms: FP64 within 1e-12, mixed
    within 1e-6 relative."""
    dims = (6, 8, 7, 5)
    links = generate_config(dims, nc, eps, 20261203, 61)
    for args in ((1, 3, 1, 3, 0.5, 1, 4, 1), (2, 4, 1, 2, 0.45, 0, 4, 2)):
        want = port.wilson_spatial_3d(nc, dims, links, *args)
        for precision, rtol, atol in (("fp64", 1e-12, 1e-14), ("mixed", 1e-6, 1e-7)):
            with Lattice(dims, nc, precision) as lat:
                lat.upload(links)
                got = lat.wilson_spatial_3d(*args)
            assert set(got) == set(want)
            for k, v in want.items():
                assert got[k] == pytest.approx(v, rel=rtol, abs=atol)


def test_fma_peak_is_plausible():
    """The measured FMA throughput behind the compute roofline: packed FP32
    near 148 SMs x 128 lanes x 2 flops x clock, FP64 about half of it."""
    from general_code_b200 import fma_peak
    f32, f64 = fma_peak("mixed"), fma_peak("fp64")
    assert 30.0 < f32 < 80.0, f32
    assert 15.0 < f64 < 40.0, f64
    assert 1.5 < f32 / f64 < 2.5


@pytest.mark.parametrize("dims", [(6, 6, 6, 48), (5, 4, 6, 36)])
def test_mixed_long_time_extent_within_1e6(dims):
    """W blocks with more than 32 threads per column (Lt = 48, 36) in the
    mixed form against the FP64 form."""
    links = generate_config(dims, 3, 0.25, 20261203, 11)
    out = {}
    for form in ("fp64", "mixed"):
        with Lattice(dims, 3, form) as lat:
            lat.upload(links)
            lat.hyp(1.0, 0.75, 0.6, 1)
            lat.ape(0.5, 4)
            out[form] = lat.wilson_loop(1, 3, 1, 16)
    assert np.max(np.abs(out["mixed"] - out["fp64"]) / np.abs(out["fp64"])) <= 1e-6
