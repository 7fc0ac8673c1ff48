"""Shared test setup.

Markers: `gpu` tests need an sm_100 GPU and call the CUDA kernels through the
C ABI; everything else runs on CPU. The product library and the C oracle are
built in-tree on first use if they are missing.
"""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


def _ensure_built():
    from general_code_b200 import build as gbuild
    gbuild.build()
    if not (ROOT / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "oracle"], check=True)


_ensure_built()


def golden_cases():
    meta = json.loads((GOLDEN / "index.json").read_text())
    return sorted(meta["cases"].items())


def load_golden(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


@pytest.fixture(scope="session")
def port():
    from oracle import py_oracle
    return py_oracle.port()


def max_abs(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))))


def su3_matrices(links):
    """(n, 18) row-major doubles -> (n, 3, 3) complex."""
    a = np.asarray(links).reshape(-1, 9, 2)
    return (a[..., 0] + 1j * a[..., 1]).reshape(-1, 3, 3)


def unitarity_error(nc, links):
    if nc == 2:
        return float(np.max(np.abs(np.sum(links ** 2, axis=1) - 1.0)))
    m = su3_matrices(links)
    eye = np.eye(3)
    u = np.max(np.abs(m @ np.conj(np.transpose(m, (0, 2, 1))) - eye))
    d = np.max(np.abs(np.linalg.det(m) - 1.0))
    return float(max(u, d))


def abelian_flux_config(dims, nc, k=(1, 2, 3)):
    """Diagonal (Abelian) configuration with constant flux through the (i, t)
    planes: U_t = 1 and U_i(x) = diag(e^{i phi}, e^{-i phi}[, 1]) with
    phi = b_i t, b_i = 2 pi k_i / Lt (periodic in t).

    Closed forms (the loop phase of an R x T rectangle in the (i, t) plane is
    R T b_i, spatial plaquettes are 1): W(R, T) = mean_i f(R T b_i) and the
    plaquette = (3 + sum_i f(b_i)) / 6, with f = cos for SU(2) and
    (2 cos + 1) / 3 for SU(3). Spatial staples equal the link, so an APE step
    leaves the configuration unchanged.
    Returns (links, W function of (R, T), plaquette).
    """
    lx, ly, lz, lt = dims
    b = [2 * np.pi * kk / lt for kk in k]
    v = lx * ly * lz * lt
    t = np.arange(v) // (lx * ly * lz)
    width = 4 if nc == 2 else 18
    links = np.zeros((v, 4, width))
    for mu in range(4):
        phi = b[mu] * t if mu < 3 else np.zeros(v)
        if nc == 2:
            links[:, mu, 0] = np.cos(phi)
            links[:, mu, 3] = np.sin(phi)
        else:
            links[:, mu, 0], links[:, mu, 1] = np.cos(phi), np.sin(phi)
            links[:, mu, 8], links[:, mu, 9] = np.cos(phi), -np.sin(phi)
            links[:, mu, 16] = 1.0
    f = np.cos if nc == 2 else (lambda a: (2 * np.cos(a) + 1) / 3)

    def w(r, tt):
        return float(np.mean([f(r * tt * bi) for bi in b]))

    plaq = float((3 + sum(f(bi) for bi in b)) / 6)
    return links.reshape(4 * v, width), w, plaq
