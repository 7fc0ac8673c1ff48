"""Builds the product library general_code_b200/libgc_b200.so in-tree.

CUDA sources are compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); host C++ sources by g++. The CUDA
runtime is linked statically so the library loads without a CUDA toolkit on
the library path. Rebuilds only when a source or header is newer than the
library.

Usage: python -m general_code_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libgc_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo",
              "-Xcompiler", "-fPIC", "-Xptxas", "-O3", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fno-fast-math", "-pthread"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted(CSRC.glob("*.cpp"))
    return cu, cpp


def _deps():
    return list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]


def _stale(target: Path) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps() if p.is_file())


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... {cmd[-1]}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return r


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    if not force and not _stale(LIB):
        return LIB
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    cu, cpp = _sources()
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    for src in cu:
        obj = BUILD / (src.stem + ".o")
        _run([nvcc, *ARCH, *NVCC_FLAGS, *extra, "-I", INCLUDE, "-c", src, "-o", obj],
             verbose or ptxas_verbose)
        objs.append(obj)
    for src in cpp:
        obj = BUILD / (src.stem + ".o")
        _run(["g++", *CXX_FLAGS, "-I", INCLUDE, "-c", src, "-o", obj], verbose)
        objs.append(obj)
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs,
          "-Xcompiler", "-pthread"], verbose)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv,
          ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
