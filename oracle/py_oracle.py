"""ctypes access to the checkers. TEST INFRASTRUCTURE ONLY.

  port()            -> oracle/liboracle.so  (plain-C restatement, gc_oracle.c)
  ref("parity")     -> oracle/_ref/libref_parity.so (the reference's own code,
                       -O2, no fast-math), if it was built here
  ref("timed")      -> oracle/_ref/libref_timed.so (reference flags -Ofast)
  generator()       -> oracle/libgen.so (the seeded configuration generator,
                       built from its source for the checkers, so that they
                       make their input without loading the product library)

All take/return host link arrays of shape (4V, 4|18) in the row-major layout.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "liboracle.so"
GEN_LIB = HERE / "libgen.so"
REF_LIBS = {"parity": HERE / "_ref" / "libref_parity.so",
            "timed": HERE / "_ref" / "libref_timed.so"}

_pint = ctypes.POINTER(ctypes.c_int)
_pdbl = ctypes.POINTER(ctypes.c_double)
_c_int, _c_dbl = ctypes.c_int, ctypes.c_double


def _dims(d):
    return (ctypes.c_int * 4)(*[int(x) for x in d])


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_pdbl)


class _Checker:
    prefix = ""

    def __init__(self, path: Path):
        self.path = path
        self.lib = ctypes.CDLL(str(path))
        p = self.prefix
        sig = {
            f"{p}ape": (_c_int, [_c_int, _pint, _pdbl, _c_dbl, _c_int]),
            f"{p}hyp": (_c_int, [_c_int, _pint, _pdbl, _c_dbl, _c_dbl, _c_dbl, _c_int]),
            f"{p}wilson": (_c_int, [_c_int, _pint, _pdbl, _c_int, _c_int, _c_int, _c_int, _pdbl]),
            f"{p}wilson_adjoint": (_c_int, [_c_int, _pint, _pdbl, _c_int, _c_int, _c_int, _c_int,
                                            _pdbl]),
            f"{p}plaquette": (_c_dbl, [_c_int, _pint, _pdbl]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(self.lib, name)
            fn.restype, fn.argtypes = res, args

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def ape(self, nc, dims, links, alpha, steps=1):
        assert self._fn("ape")(nc, _dims(dims), _ptr(links), alpha, steps) == 0

    def hyp(self, nc, dims, links, a1, a2, a3, steps=1):
        assert self._fn("hyp")(nc, _dims(dims), _ptr(links), a1, a2, a3, steps) == 0

    def wilson(self, nc, dims, links, rmin, rmax, tmin, tmax):
        out = np.empty((tmax - tmin + 1, rmax - rmin + 1), dtype=np.float64)
        assert self._fn("wilson")(nc, _dims(dims), _ptr(links), rmin, rmax, tmin, tmax,
                                  _ptr(out)) == 0
        return out

    def wilson_adjoint(self, nc, dims, links, rmin, rmax, tmin, tmax):
        out = np.empty((tmax - tmin + 1, rmax - rmin + 1), dtype=np.float64)
        assert self._fn("wilson_adjoint")(nc, _dims(dims), _ptr(links), rmin, rmax, tmin,
                                          tmax, _ptr(out)) == 0
        return out

    def plaquette(self, nc, dims, links):
        return float(self._fn("plaquette")(nc, _dims(dims), _ptr(links)))

    def ape_plane(self, nc, dims, links, a, b, alpha, steps=1):
        """smearing_APE_2d on the direction fields a, b, in place."""
        fn = self._fn("ape_plane")
        fn.restype = _c_int
        fn.argtypes = [_c_int, _pint, _pdbl, _c_int, _c_int, _c_dbl, _c_int]
        assert fn(nc, _dims(dims), _ptr(links), a, b, alpha, steps) == 0

    def wilson_spatial_3d(self, nc, dims, links, rmin, rmax, tmin, tmax, alpha, sm_start,
                          sm_end, sm_step, capacity=100000):
        """wilson_spatial_3d_indexed: {(smearing, T, R): W}."""
        fn = self._fn("wilson_spatial_3d")
        fn.restype = _c_int
        fn.argtypes = [_c_int, _pint, _pdbl, _c_int, _c_int, _c_int, _c_int, _c_dbl, _c_int,
                       _c_int, _c_int, _pint, _pint, _pint, _pdbl, _c_int]
        s_, t_, r_ = (np.zeros(capacity, dtype=np.int32) for _ in range(3))
        w = np.zeros(capacity)
        n = fn(nc, _dims(dims), _ptr(links), rmin, rmax, tmin, tmax, alpha, sm_start, sm_end,
               sm_step, s_.ctypes.data_as(_pint), t_.ctypes.data_as(_pint),
               r_.ctypes.data_as(_pint), _ptr(w), capacity)
        assert 0 <= n <= capacity
        return {(int(s_[i]), int(t_[i]), int(r_[i])): float(w[i]) for i in range(n)}

    def _setup_observables(self):
        p = self.prefix
        sig = {
            f"{p}wilson_gevp": (_c_int, [_c_int, _pint, _pdbl, _pdbl, _c_int, _c_int, _c_int,
                                         _c_int, _c_int, _pdbl]),
            f"{p}polyakov_loop": (_c_dbl, [_c_int, _pint, _pdbl]),
            f"{p}polyakov_correlator": (_c_int, [_c_int, _pint, _pdbl, _c_int, _c_int, _pdbl]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(self.lib, name)
            fn.restype, fn.argtypes = res, args

    def wilson_gevp(self, nc, dims, links1, links2, rmin, rmax, tmin, tmax, adjoint=False):
        out = np.empty((tmax - tmin + 1, rmax - rmin + 1), dtype=np.float64)
        assert self._fn("wilson_gevp")(nc, _dims(dims), _ptr(links1), _ptr(links2), rmin, rmax,
                                       tmin, tmax, int(adjoint), _ptr(out)) == 0
        return out

    def polyakov_loop(self, nc, dims, links):
        return float(self._fn("polyakov_loop")(nc, _dims(dims), _ptr(links)))

    def polyakov_correlator(self, nc, dims, links, d_max, singlet):
        n = 2 * d_max + 1
        out = np.empty(n ** 3, dtype=np.float64)
        assert self._fn("polyakov_correlator")(nc, _dims(dims), _ptr(links), d_max,
                                               int(singlet), _ptr(out)) == 0
        return out


class WilsonResult(ctypes.Structure):
    """or_wilson_result / gc_wilson_result."""
    _fields_ = [("wilson_loop", ctypes.c_double), ("time_size", ctypes.c_int),
                ("space_size", ctypes.c_double), ("statistics_size", ctypes.c_int)]


def _as_dict(entries):
    """{(T, size): W} built in order, later entries replacing earlier ones."""
    out = {}
    for w, t, size, _ in entries:
        out[(t, size)] = w
    return out


class Port(_Checker):
    prefix = "or_"

    def __init__(self, path=PORT_LIB):
        super().__init__(path)
        self._setup_observables()
        for name in ("or_plaquette_time", "or_plaquette_space"):
            fn = getattr(self.lib, name)
            fn.restype, fn.argtypes = _c_dbl, [_c_int, _pint, _pdbl]
        self.lib.or_set_threads.argtypes = [_c_int]
        self.lib.or_proj_all.argtypes = [_c_int, ctypes.c_longlong, _pdbl]
        self.lib.or_proj_all.restype = _c_int

    def set_threads(self, n):
        self.lib.or_set_threads(int(n))

    def wilson_offaxis(self, nc, dims, links, directions, rmin, rmax, tmin, tmax,
                       adjoint=False, capacity=20000):
        """Unmerged off-axis entries [(W, T, size, statistics)] in order."""
        d = np.ascontiguousarray(directions, dtype=np.int32).reshape(-1, 3)
        fn = self.lib.or_wilson_offaxis
        fn.restype = _c_int
        fn.argtypes = [_c_int, _pint, _pdbl, _pint, _c_int, _c_dbl, _c_dbl, _c_int, _c_int,
                       _c_int, ctypes.POINTER(WilsonResult), _c_int]
        out = (WilsonResult * capacity)()
        n = fn(nc, _dims(dims), _ptr(links), d.ctypes.data_as(_pint), d.shape[0], rmin, rmax,
               tmin, tmax, int(adjoint), out, capacity)
        assert 0 <= n <= capacity
        return [(r.wilson_loop, r.time_size, r.space_size, r.statistics_size) for r in out[:n]]

    def wilson_offaxis_result(self, nc, dims, links, rmin, rmax, tmin, tmax, adjoint=False,
                              capacity=20000):
        """Merged off-axis loops {(T, size): W} (wilson_offaxis_result)."""
        fn = self.lib.or_wilson_offaxis_result
        fn.restype = _c_int
        fn.argtypes = [_c_int, _pint, _pdbl, _c_dbl, _c_dbl, _c_int, _c_int, _c_int,
                       ctypes.POINTER(WilsonResult), _c_int]
        out = (WilsonResult * capacity)()
        n = fn(nc, _dims(dims), _ptr(links), rmin, rmax, tmin, tmax, int(adjoint), out,
               capacity)
        assert 0 <= n <= capacity
        return _as_dict((r.wilson_loop, r.time_size, r.space_size, r.statistics_size)
                        for r in out[:n])

    def plaquette_time(self, nc, dims, links):
        return float(self.lib.or_plaquette_time(nc, _dims(dims), _ptr(links)))

    def plaquette_space(self, nc, dims, links):
        return float(self.lib.or_plaquette_space(nc, _dims(dims), _ptr(links)))

    def proj_all(self, nc, links):
        assert self.lib.or_proj_all(nc, links.shape[0], _ptr(links)) == 0


class Ref(_Checker):
    prefix = "ref_"

    def __init__(self, path):
        super().__init__(path)
        self._setup_observables()
        self.lib.ref_plaquette_part.restype = _c_dbl
        self.lib.ref_plaquette_part.argtypes = [_c_int, _pint, _pdbl, _c_int]
        self.lib.ref_polyakov_average_directions.restype = _c_int
        self.lib.ref_polyakov_average_directions.argtypes = [_pdbl, _c_int, _pdbl, _pdbl, _c_int]
        self.lib.ref_job.restype = _c_int
        self.lib.ref_job.argtypes = [_c_int, _pint, _pdbl, _c_int, _c_dbl, _c_dbl, _c_dbl,
                                     _c_int, _c_dbl, _c_int, _c_int, _c_int, _c_int, _pdbl,
                                     _pdbl]
        self.lib.ref_num_threads.restype = _c_int
        self.lib.ref_set_threads.argtypes = [_c_int]
        self.lib.ref_read.restype = _c_int
        self.lib.ref_read.argtypes = [_c_int, _pint, ctypes.c_char_p, ctypes.c_char_p, _c_int,
                                      ctypes.c_char_p, _c_int, _pdbl]
        self.lib.ref_write_lexicographical.restype = _c_int
        self.lib.ref_write_lexicographical.argtypes = [_c_int, _pint, _pdbl, ctypes.c_char_p]

    def num_threads(self):
        return int(self.lib.ref_num_threads())

    def _offaxis(self, nc, dims, links, mode, directions, rmin, rmax, tmin, tmax, adjoint,
                 capacity=20000):
        fn = self.lib.ref_wilson_offaxis
        fn.restype = _c_int
        fn.argtypes = [_c_int, _pint, _pdbl, _c_int, _pint, _c_int, _c_dbl, _c_dbl, _c_int,
                       _c_int, _c_int, _pdbl, _pint, _pdbl, _pint, _c_int]
        d = np.ascontiguousarray(directions if directions is not None else np.zeros((0, 3)),
                                 dtype=np.int32).reshape(-1, 3)
        w = np.zeros(capacity)
        t = np.zeros(capacity, dtype=np.int32)
        sz = np.zeros(capacity)
        st = np.zeros(capacity, dtype=np.int32)
        n = fn(nc, _dims(dims), _ptr(links), mode, d.ctypes.data_as(_pint), d.shape[0], rmin,
               rmax, tmin, tmax, int(adjoint), _ptr(w), t.ctypes.data_as(_pint), _ptr(sz),
               st.ctypes.data_as(_pint), capacity)
        assert 0 <= n <= capacity
        return [(float(w[i]), int(t[i]), float(sz[i]), int(st[i])) for i in range(n)]

    def wilson_offaxis(self, nc, dims, links, directions, rmin, rmax, tmin, tmax,
                       adjoint=False):
        """The reference's wilson_offaxis[_adjoint]: [(W, T, size, statistics)]."""
        return self._offaxis(nc, dims, links, 0, directions, rmin, rmax, tmin, tmax, adjoint)

    def wilson_offaxis_result(self, nc, dims, links, rmin, rmax, tmin, tmax, adjoint=False):
        """The reference's wilson_offaxis[_adjoint]_result: {(T, size): W}."""
        return _as_dict(self._offaxis(nc, dims, links, 1, None, rmin, rmax, tmin, tmax,
                                      adjoint))

    def plaquette_time(self, nc, dims, links):
        return float(self.lib.ref_plaquette_part(nc, _dims(dims), _ptr(links), 1))

    def plaquette_space(self, nc, dims, links):
        return float(self.lib.ref_plaquette_part(nc, _dims(dims), _ptr(links), 2))

    def polyakov_average_directions(self, table, d_max):
        """The reference's distance average: {distance: mean} (ascending)."""
        table = np.ascontiguousarray(table, dtype=np.float64)
        cap = table.size
        dist = np.empty(cap, dtype=np.float64)
        avg = np.empty(cap, dtype=np.float64)
        n = self.lib.ref_polyakov_average_directions(_ptr(table), d_max, _ptr(dist), _ptr(avg),
                                                     cap)
        return dict(zip(dist[:n].tolist(), avg[:n].tolist()))

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def job(self, nc, dims, links, hyp_steps, a1, a2, a3, ape_steps, alpha, rmin, rmax,
            tmin, tmax):
        """Runs HYP x hyp_steps, APE x ape_steps, W table; returns (W, times[3])."""
        out = np.zeros((max(tmax - tmin + 1, 1), max(rmax - rmin + 1, 1)), dtype=np.float64)
        times = np.zeros(3, dtype=np.float64)
        assert self.lib.ref_job(nc, _dims(dims), _ptr(links), hyp_steps, a1, a2, a3,
                                ape_steps, alpha, rmin, rmax, tmin, tmax, _ptr(out),
                                _ptr(times)) == 0
        return out, times

    def read(self, nc, dims, path, fmt, bytes_skip, precision, convert):
        n = 4
        for d in dims:
            n *= int(d)
        out = np.empty((n, 4 if nc == 2 else 18), dtype=np.float64)
        assert self.lib.ref_read(nc, _dims(dims), str(path).encode(), fmt.encode(),
                                 int(bytes_skip), precision.encode(), int(convert),
                                 _ptr(out)) == 0
        return out

    def write_lexicographical(self, nc, dims, links, path):
        assert self.lib.ref_write_lexicographical(nc, _dims(dims), _ptr(links),
                                                  str(path).encode()) == 0


class Generator:
    """Seeded synthetic configurations (the generator of gc_generate_host:
    Philox-4x32-10 keyed by (seed, config index), eps-scaled exp(iH) links and
    a Haar gauge transformation); host array (4V, 4|18), row-major."""

    def __init__(self, path: Path = GEN_LIB):
        self.lib = ctypes.CDLL(str(path))
        self.lib.og_generate_host.restype = _c_int
        self.lib.og_generate_host.argtypes = [_pint, _c_int, _c_dbl, ctypes.c_uint,
                                              ctypes.c_uint, _c_int, _pdbl]

    def generate(self, dims, nc, eps, seed, index=0, gauge=True, out=None):
        n = 4
        for d in dims:
            n *= int(d)
        if out is None:
            out = np.empty((n, 4 if nc == 2 else 18), dtype=np.float64)
        assert out.shape == (n, 4 if nc == 2 else 18)
        assert self.lib.og_generate_host(_dims(dims), nc, float(eps), int(seed) & 0xffffffff,
                                         int(index) & 0xffffffff, int(bool(gauge)),
                                         _ptr(out)) == 0
        return out


_port = None
_gen = None
_refs = {}


def generator() -> Generator:
    global _gen
    if _gen is None:
        if not GEN_LIB.exists():
            raise ImportError(f"{GEN_LIB} missing: run `make -C oracle gen`")
        _gen = Generator()
    return _gen


def port() -> Port:
    global _port
    if _port is None:
        if not PORT_LIB.exists():
            raise ImportError(f"{PORT_LIB} missing: run `make -C oracle oracle`")
        _port = Port()
    return _port


def ref_available(kind: str = "parity") -> bool:
    return REF_LIBS[kind].exists()


def ref(kind: str = "parity") -> Ref:
    if kind not in _refs:
        if not REF_LIBS[kind].exists():
            raise ImportError(f"{REF_LIBS[kind]} missing (built only where the reference "
                              "sources are present)")
        _refs[kind] = Ref(REF_LIBS[kind])
    return _refs[kind]
