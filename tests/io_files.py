"""Writers of configuration files in the reference's reader formats, for the
I/O tests (the reference ships no configuration files).

  lexicographical : link index 4*site+mu, get_data element order
                    (FilePatternLexicographical, indexing.h:190-216)
  qcdstag         : (site + mu1*V) with mu1 = 0 for t, mu+1 otherwise; SU(2)
                    element order a0, a3, a2, a1 (indexing.h:218-323)
  ildg            : LIME container, record "ildg-binary-data", big-endian
                    doubles in the lexicographical pattern (data.h:144-173)
"""
from __future__ import annotations

import struct

import numpy as np

LIME_MAGIC = 0x456789AB


def _to_qcdstag(links: np.ndarray, V: int) -> np.ndarray:
    ds = links.shape[1]
    per = links.reshape(V, 4, ds)
    out = np.empty((4, V, ds), dtype=links.dtype)
    for mu in range(4):
        mu1 = 0 if mu == 3 else mu + 1
        m = per[:, mu, :]
        if ds == 4:
            m = m[:, [0, 3, 2, 1]]
        out[mu1] = m
    return out.reshape(-1)


def write_lexicographical(path, links, precision="double", header=b""):
    a = links.astype(np.float64 if precision == "double" else np.float32)
    with open(path, "wb") as f:
        f.write(header)
        f.write(a.tobytes())


def write_qcdstag(path, links, V, precision="double", header=b""):
    a = _to_qcdstag(links, V).astype(np.float64 if precision == "double" else np.float32)
    with open(path, "wb") as f:
        f.write(header)
        f.write(a.tobytes())


def _lime_record(rtype: str, payload: bytes, mb: bool, me: bool) -> bytes:
    flags = (0x80 if mb else 0) | (0x40 if me else 0)
    hdr = struct.pack(">IHBB", LIME_MAGIC, 1, flags, 0)
    hdr += struct.pack(">Q", len(payload))
    t = rtype.encode()
    hdr += t + b"\0" * (128 - len(t))
    pad = (-len(payload)) % 8
    return hdr + payload + b"\0" * pad


def write_ildg(path, links, dims, nc):
    fmt = ("<?xml version=\"1.0\" encoding=\"UTF-8\"?><ildgFormat><version>1.0</version>"
           f"<field>su{nc}gauge</field><precision>64</precision>"
           f"<lx>{dims[0]}</lx><ly>{dims[1]}</ly><lz>{dims[2]}</lz><lt>{dims[3]}</lt>"
           "</ildgFormat>").encode()
    data = links.astype(">f8").tobytes()
    with open(path, "wb") as f:
        f.write(_lime_record("ildg-format", fmt, True, False))
        f.write(_lime_record("ildg-binary-data", data, False, True))


def converted(links: np.ndarray, nc: int) -> np.ndarray:
    """MatrixConverter<MT,MT> (matrix.h:1104-1119): A * B^dag with B the
    diagonal phases (SU(3)) or (a0,0,0,a3)/|.| (SU(2))."""
    if nc == 2:
        a0, a1, a2, a3 = links.T
        n = np.sqrt(a0 * a0 + a3 * a3)
        b0, b3 = a0 / n, a3 / n
        # A ^ B for B = (b0, 0, 0, b3)  (quaternion A * B^dag)
        return np.stack([a0 * b0 + a3 * b3, b0 * a1 + a2 * b3,
                         b0 * a2 - a1 * b3, -a0 * b3 + b0 * a3], axis=1)
    m = links.reshape(-1, 9, 2)
    m = (m[..., 0] + 1j * m[..., 1]).reshape(-1, 3, 3)
    d = np.diagonal(m, axis1=1, axis2=2)
    ph = d / np.abs(d)
    r = m * np.conj(ph)[:, None, :]
    out = np.empty((m.shape[0], 9, 2))
    out[..., 0] = r.reshape(-1, 9).real
    out[..., 1] = r.reshape(-1, 9).imag
    return out.reshape(-1, 18)
