"""Parity at the benchmark's full sizes (GPU).

* The SU(3) 24^4 job (HYP x1 + APE x20, W for R,T = 1..12) and the SU(2)
  16^4 job (HYP x1 + APE x10, R,T = 1..8) on the GPU against the reference's
  own CPU path on the same configuration (the oracle restatement when the
  reference library is not built): FP64 within 1e-12 relative, mixed within
  1e-6.
* SU(3) 32^4 (HYP x1 + APE x40, R,T = 1..16) and SU(2) 48^4 (HYP x1 + APE
  x10, R,T = 1..24), too slow for the CPU inside a test: against the W tables
  the reference's CPU path computed once on the same seeded configurations
  (tests/golden/fullsize.json, made by tests/golden/make_golden_fullsize.py
  from the reference compiled from its sources): FP64 within 1e-12 relative,
  mixed within 1e-6; the smeared links in SU(3) to FP32 precision.
* Gauge invariance at 24^4: the same configuration with and without a random
  gauge transformation gives the same smeared W(R,T) table.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import su3_matrices
from general_code_b200 import Lattice, generate_config
from oracle import py_oracle

pytestmark = pytest.mark.gpu
SEED = 20261203
HYP = (1.0, 0.75, 0.6)


def _job(lat, links, ape, rt):
    lat.upload(links)
    lat.hyp(*HYP, 1)
    lat.ape(0.5, ape)
    return lat.wilson_loop(1, rt, 1, rt)


def _cpu_job(nc, dims, links, ape, rt):
    """W table of the reference's CPU path (its library built from the
    reference sources), else the oracle restatement, on a copy of links."""
    a = links.copy()
    if py_oracle.ref_available("parity"):
        r = py_oracle.ref("parity")
        r.set_threads(os.cpu_count() or 1)
        w, _ = r.job(nc, dims, a, 1, *HYP, ape, 0.5, 1, rt, 1, rt)
        return w
    p = py_oracle.port()
    p.set_threads(os.cpu_count() or 1)
    p.hyp(nc, dims, a, *HYP, 1)
    p.ape(nc, dims, a, 0.5, ape)
    return p.wilson(nc, dims, a, 1, rt, 1, rt)


@pytest.mark.parametrize("nc,dims,eps,ape,rt", [
    (3, (24, 24, 24, 24), 0.25, 20, 12),
    (2, (16, 16, 16, 16), 0.3, 10, 8),
])
def test_full_size_job_matches_reference_cpu_path(nc, dims, eps, ape, rt):
    links = generate_config(dims, nc, eps, SEED, 0)
    want = _cpu_job(nc, dims, links, ape, rt)
    with Lattice(dims, nc, "fp64") as lat:
        w64 = _job(lat, links, ape, rt)
    with Lattice(dims, nc, "mixed") as lat:
        w32 = _job(lat, links, ape, rt)
    np.testing.assert_allclose(w64, want, rtol=1e-12, atol=1e-14)
    assert np.max(np.abs(w32 - want) / np.abs(want)) <= 1e-6


def _golden(name):
    import json
    from pathlib import Path
    p = Path(__file__).resolve().parent / "golden" / "fullsize.json"
    cases = json.loads(p.read_text())["cases"]
    if name not in cases:
        pytest.skip(f"no {name} table in tests/golden/fullsize.json")
    return cases[name]


def _sha(links):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(links).tobytes()).hexdigest()


@pytest.mark.parametrize("name", ["su3_32", "su2_48"])
def test_large_job_matches_reference_table(name):
    c = _golden(name)
    nc, dims = c["nc"], tuple(c["dims"])
    links = generate_config(dims, nc, c["eps"], c["seed"], c["config_index"])
    assert _sha(links) == c["input_sha256"], "the generator no longer gives the fixture's input"
    rng = (c["r_min"], c["r_max"], c["time_min"], c["time_max"])
    want = np.array(c["wilson"])
    res = {}
    for form in ("fp64", "mixed"):
        with Lattice(dims, nc, form) as lat:
            lat.upload(links)
            lat.hyp(*c["hyp_alpha"], c["hyp_steps"])
            lat.ape(c["ape_alpha"], c["ape_steps"])
            res[form] = lat.wilson_loop(*rng)
            if form == "fp64":
                res["plaq"] = lat.plaquette()
            elif nc == 3:
                m = su3_matrices(lat.download())
    np.testing.assert_allclose(res["fp64"], want, rtol=1e-12, atol=1e-14)
    assert res["plaq"] == pytest.approx(c["plaquette_out"], rel=1e-12)
    assert np.max(np.abs(res["mixed"] - want) / np.abs(want)) <= 1e-6
    if nc == 3:
        # every smeared link (APE'd spatial, HYP'd temporal) unitary with det 1
        # to FP32 precision
        uu = np.einsum("nij,nkj->nik", m, m.conj())
        assert np.max(np.abs(uu - np.eye(3))) <= 2e-6
        assert np.max(np.abs(np.linalg.det(m) - 1)) <= 2e-6


@pytest.mark.parametrize("form,rtol", [("fp64", 1e-11), ("mixed", 1e-6)])
def test_w_is_gauge_invariant_at_full_size(form, rtol):
    nc, dims, ape, rt = 3, (24, 24, 24, 24), 20, 12
    plain = generate_config(dims, nc, 0.25, SEED, 0, gauge=False)
    rotated = generate_config(dims, nc, 0.25, SEED, 0, gauge=True)
    assert np.max(np.abs(plain - rotated)) > 0.1  # the transformation is not trivial
    with Lattice(dims, nc, form) as lat:
        w0 = _job(lat, plain, ape, rt)
        w1 = _job(lat, rotated, ape, rt)
    np.testing.assert_allclose(w1, w0, rtol=rtol, atol=1e-14)


def test_offaxis_full_size_translation_and_mixed():
    """Off-axis loops on SU(3) 24^4 (r <= 6, T <= 6: 678 lines in three
    launches of the fused kernel): the same table for the configuration
    translated by (3, 0, 0, 5) (FP64, 1e-12), and the mixed form within 1e-6
    of FP64."""
    nc, dims = 3, (24, 24, 24, 24)
    links = generate_config(dims, nc, 0.25, SEED, 2)
    moved = np.roll(links.reshape(dims[3], dims[2], dims[1], dims[0], 4, 18), (5, 3),
                    axis=(0, 3)).reshape(links.shape)
    res = {}
    for key, form, x in (("a", "fp64", links), ("b", "fp64", moved), ("m", "mixed", links)):
        with Lattice(dims, nc, form) as lat:
            lat.upload(np.ascontiguousarray(x))
            res[key] = lat.wilson_offaxis_result(1.0, 6.0, 1, 6)
    assert res["a"].keys() == res["b"].keys() == res["m"].keys() and len(res["a"]) > 100
    for k, v in res["a"].items():
        assert res["b"][k] == pytest.approx(v, rel=1e-12, abs=1e-14)
        assert abs(res["m"][k] - v) <= 1e-6 * abs(v) + 1e-9
