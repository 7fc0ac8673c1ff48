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
