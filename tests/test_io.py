"""Configuration files: the reference's own reader accepts the test files
(CPU), gc_probe_config finds the link payload and rejects bad files (CPU),
and the device reader gc_read_config gives the same links as the reference's
reader (GPU, bit for bit; the optional conversion within 1e-15)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import max_abs
from general_code_b200 import GCError, Lattice, generate_config, probe_config
from general_code_b200 import _lib
from io_files import converted, write_ildg, write_lexicographical, write_qcdstag

DIMS = (4, 3, 5, 6)
V = int(np.prod(DIMS))


def make_file(tmp_path, nc, fmt, precision, header=b""):
    links = generate_config(DIMS, nc, 0.3 if nc == 2 else 0.25, 77, nc)
    p = tmp_path / f"conf_{nc}_{fmt}_{precision}"
    if fmt == "lexicographical":
        write_lexicographical(p, links, precision, header)
    elif fmt == "qcdstag":
        write_qcdstag(p, links, V, precision, header)
    else:
        write_ildg(p, links, DIMS, nc)
    if precision == "float":
        links = links.astype(np.float32).astype(np.float64)
    return p, links


CASES = [(nc, fmt, prec) for nc in (2, 3) for fmt, prec in
         [("lexicographical", "double"), ("lexicographical", "float"), ("qcdstag", "double"),
          ("qcdstag", "float"), ("ildg", "double")]]


def _ref():
    from oracle import py_oracle
    if not py_oracle.ref_available("parity"):
        return None
    return py_oracle.ref("parity")


@pytest.mark.parametrize("nc,fmt,prec", CASES)
def test_reference_reader_accepts_test_files(tmp_path, nc, fmt, prec):
    ref = _ref()
    if ref is None:
        pytest.skip("reference not compiled in this checkout")
    header = b"H" * 24 if fmt != "ildg" else b""
    p, links = make_file(tmp_path, nc, fmt, prec, header)
    got = ref.read(nc, DIMS, p, fmt, len(header), prec, 0)
    assert max_abs(got, links) == 0.0
    got = ref.read(nc, DIMS, p, fmt, len(header), prec, 1)
    assert max_abs(got, converted(links, nc)) <= 1e-15


@pytest.mark.parametrize("nc,fmt,prec", CASES)
def test_probe_finds_payload(tmp_path, nc, fmt, prec):
    header = b"H" * 40 if fmt != "ildg" else b""
    p, _ = make_file(tmp_path, nc, fmt, prec, header)
    off, ln = probe_config(DIMS, nc, p, fmt, len(header), prec)
    per = (4 if nc == 2 else 18) * (4 if prec == "float" else 8)
    assert ln == 4 * V * per
    if fmt == "ildg":
        raw = open(p, "rb").read()
        # the payload follows the 144-byte header of the ildg-binary-data record
        assert off == raw.index(b"ildg-binary-data") - 16 + 144
        assert off + ln == len(raw)
    else:
        assert off == len(header)


def test_probe_rejects_bad_files(tmp_path):
    p, _ = make_file(tmp_path, 3, "lexicographical", "double")
    with pytest.raises(GCError) as e:
        probe_config((4, 3, 5, 7), 3, p, "lexicographical")
    assert e.value.code == _lib.GC_ERR_IO
    with pytest.raises(GCError) as e:
        probe_config(DIMS, 3, tmp_path / "missing", "lexicographical")
    assert e.value.code == _lib.GC_ERR_IO
    with pytest.raises(GCError) as e:
        probe_config(DIMS, 3, p, "ildg")  # not a LIME file
    assert e.value.code == _lib.GC_ERR_IO
    q, _ = make_file(tmp_path, 3, "ildg", "double")
    raw = open(q, "rb").read()
    (tmp_path / "trunc").write_bytes(raw[:-100])
    with pytest.raises(GCError) as e:
        probe_config(DIMS, 3, tmp_path / "trunc", "ildg")
    assert e.value.code == _lib.GC_ERR_IO
    with pytest.raises(GCError) as e:
        probe_config(DIMS, 3, p, "binary")
    assert e.value.code == _lib.GC_ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("convert", [0, 1])
@pytest.mark.parametrize("nc,fmt,prec", CASES)
def test_device_reader_matches_reference_reader(tmp_path, nc, fmt, prec, convert):
    header = b"H" * 24 if fmt != "ildg" else b""
    p, links = make_file(tmp_path, nc, fmt, prec, header)
    ref = _ref()
    if ref is not None:
        expect = ref.read(nc, DIMS, p, fmt, len(header), prec, convert)
    else:
        expect = converted(links, nc) if convert else links
    with Lattice(DIMS, nc, "fp64") as lat:
        lat.read(p, fmt, len(header), prec, bool(convert))
        got = lat.download()
    if convert:
        assert max_abs(got, expect) <= 1e-15
    else:
        assert max_abs(got, expect) == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("nc", [2, 3])
def test_writer_matches_reference_writer_and_round_trips(tmp_path, nc):
    links = generate_config(DIMS, nc, 0.3, 5, 0)
    with Lattice(DIMS, nc, "fp64") as lat:
        lat.upload(links)
        lat.write(tmp_path / "ours")
    ref = _ref()
    if ref is not None:
        ref.write_lexicographical(nc, DIMS, links, tmp_path / "theirs")
        assert (tmp_path / "ours").read_bytes() == (tmp_path / "theirs").read_bytes()
    with Lattice(DIMS, nc, "fp64") as lat:
        lat.read(tmp_path / "ours", "lexicographical", 0, "double", False)
        assert max_abs(lat.download(), links) == 0.0


@pytest.mark.gpu
def test_device_reader_errors():
    with Lattice(DIMS, 3, "fp64") as lat:
        with pytest.raises(GCError) as e:
            lat.read("/nonexistent/conf", "lexicographical")
        assert e.value.code == _lib.GC_ERR_IO
