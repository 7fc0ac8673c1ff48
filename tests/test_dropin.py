"""The C++ drop-in (include/gc_dropin.hpp) compiled against the reference's
own headers (oracle/_ref/dropin_check, built where the reference sources are
present): the app's unqualified calls bind to the GPU overloads, and on a GPU
they agree with the reference templates (FP64, 1e-12)."""
from __future__ import annotations

import subprocess

import pytest

from conftest import ROOT

BIN = ROOT / "oracle" / "_ref" / "dropin_check"


def _run(*args):
    if not BIN.exists():
        pytest.skip("drop-in check not built (needs the reference sources)")
    return subprocess.run([str(BIN), *map(str, args)], capture_output=True, text=True,
                          timeout=600)


def test_dropin_overloads_are_selected_without_gpu():
    from test_abi import _has_gpu
    if _has_gpu():
        pytest.skip("a GPU is present")
    r = _run(3, 4, 4, 1, 2, 2)
    # only the drop-in overloads can raise: the reference templates never throw
    assert r.returncode == 3, r.stdout + r.stderr
    assert "no CUDA device" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("nc,L,T,ape,rmax,tmax", [(2, 8, 8, 4, 4, 4), (3, 6, 8, 3, 3, 4)])
def test_dropin_matches_reference_templates(nc, L, T, ape, rmax, tmax):
    r = _run(nc, L, T, ape, rmax, tmax)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout
