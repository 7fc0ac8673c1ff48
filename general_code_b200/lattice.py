"""Python host API over the C ABI, mirroring the reference's C++ interface.

Reference interface (general_code, lib/cpu/include):
  Data::LatticeData<DataPattern, MatrixType>   data.h:78-237   -> LatticeData
  smearing_APE(conf, alpha)                    smearing.h:115  -> smearing_APE
  smearing_HYP(conf, alpha1, alpha2, alpha3)   smearing.h:480  -> smearing_HYP
  wilson_loop(conf, r_min, r_max, t_min, t_max) wilson_loops.h:1047 -> wilson_loop
  plaket(conf)                                 plaket.h:83     -> plaket

Like the reference, the LatticeData functions update the host links in place
(smearing) or return a dict keyed (T, R) (Wilson loops). Each call uploads the
links, runs the sm_100a kernels and downloads the result. `Lattice` is the
device-resident form: links stay in HBM between calls.
"""
from __future__ import annotations

import ctypes
import math
from typing import Dict, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import (GC_ERR_ARG, GC_LAYOUT_EIGEN_COLMAJOR, GC_LAYOUT_ROWMAJOR, GC_PREC_FP64,
                   GC_PREC_MIXED, GCError, WilsonResult, WilsonSpatialResult, check, dbl_ptr,
                   dims_arg, lib)

_PREC = {"fp64": GC_PREC_FP64, "mixed": GC_PREC_MIXED}
_LAYOUT = {"rowmajor": GC_LAYOUT_ROWMAJOR, "eigen": GC_LAYOUT_EIGEN_COLMAJOR}


def link_size(nc: int) -> int:
    """Doubles per link in the host layout: 4 (SU(2)) or 18 (SU(3))."""
    if nc == 2:
        return 4
    if nc == 3:
        return 18
    raise ValueError("nc must be 2 or 3")


def volume(dims: Sequence[int]) -> int:
    v = 1
    for d in dims:
        v *= int(d)
    return v


def generate_config(dims: Sequence[int], nc: int, eps: float, seed: int,
                    index: int = 0, gauge: bool = True, out: np.ndarray | None = None
                    ) -> np.ndarray:
    """Seeded synthetic configuration (host array, shape (4V, 4|18), row-major)."""
    n = 4 * volume(dims)
    if out is None:
        out = np.empty((n, link_size(nc)), dtype=np.float64)
    check(lib().gc_generate_host(dims_arg(dims), nc, float(eps), int(seed) & 0xffffffff,
                                 int(index) & 0xffffffff, int(bool(gauge)), dbl_ptr(out)))
    return out


# Kernels one call launches: gc_hyp per step, gc_ape per step, and
# gc_wilson_onaxis for the ranges the benchmark uses: the exact W kernel and
# its fixed-order reduction, or, where the temporal-gauge form applies, the
# gauge lines, the transformed links, both gated W kernels and the reduction.
HYP_LAUNCHES_PER_STEP = 3
APE_LAUNCHES_PER_STEP = 1
WILSON_LAUNCHES = {"exact": 2, "gauge": 5}


def launches_per_job(nc: int, ape_steps: int, hyp_steps: int = 1,
                     w_method: str = "gauge") -> int:
    """Our kernel launches in one smear-and-measure job (HYP, APE, W)."""
    return (hyp_steps * HYP_LAUNCHES_PER_STEP + ape_steps * APE_LAUNCHES_PER_STEP
            + WILSON_LAUNCHES[w_method])


def fma_peak(precision: str = "mixed") -> float:
    """Measured vector FMA throughput of the current device, TFLOP/s (packed
    FP32x2 for "mixed", FP64 for "fp64")."""
    out = ctypes.c_double()
    check(lib().gc_fma_peak(_PREC[precision], ctypes.byref(out)))
    return float(out.value)


def unit_config(dims: Sequence[int], nc: int) -> np.ndarray:
    n = 4 * volume(dims)
    a = np.zeros((n, link_size(nc)), dtype=np.float64)
    if nc == 2:
        a[:, 0] = 1.0
    else:
        a[:, 0] = a[:, 8] = a[:, 16] = 1.0
    return a


class Lattice:
    """A device-resident gauge configuration (one gc_lattice handle)."""

    def __init__(self, dims: Sequence[int], nc: int, precision: str = "fp64"):
        self.dims = tuple(int(d) for d in dims)
        self.nc = int(nc)
        self.precision = precision
        self._h = ctypes.c_void_p()
        check(lib().gc_lattice_create(dims_arg(self.dims), self.nc, _PREC[precision],
                                      ctypes.byref(self._h)))

    @property
    def handle(self):
        return self._h

    @property
    def V(self) -> int:
        return volume(self.dims)

    def _check(self, rc: int) -> None:
        check(rc, self._h)

    def close(self) -> None:
        if self._h:
            lib().gc_lattice_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None) -> None:
        self._check(lib().gc_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)))

    def synchronize(self) -> None:
        self._check(lib().gc_synchronize(self._h))

    def upload(self, links: np.ndarray, layout: str = "rowmajor") -> None:
        a = np.ascontiguousarray(links, dtype=np.float64)
        if a.size != 4 * self.V * link_size(self.nc):
            raise ValueError("link array has the wrong size for this lattice")
        self._check(lib().gc_upload(self._h, dbl_ptr(a), _LAYOUT[layout]))
        if a is not links:  # keep the temporary alive until the copy is done
            self.synchronize()

    def download(self, out: np.ndarray | None = None, layout: str = "rowmajor") -> np.ndarray:
        if out is None:
            out = np.empty((4 * self.V, link_size(self.nc)), dtype=np.float64)
        self._check(lib().gc_download(self._h, dbl_ptr(out), _LAYOUT[layout]))
        return out

    def read(self, path, conf_format: str = "lexicographical", bytes_skip: int = 0,
             file_precision: str = "double", convert: bool = False) -> None:
        """Reads a configuration file into the device links (gc_read_config)."""
        self._check(lib().gc_read_config(self._h, str(path).encode(), conf_format.encode(),
                                         int(bytes_skip), file_precision.encode(),
                                         int(bool(convert))))

    def write(self, path) -> None:
        """Writes the links as lexicographical doubles (gc_write_config)."""
        self._check(lib().gc_write_config(self._h, str(path).encode()))

    def copy_from(self, other: "Lattice") -> None:
        """Device-to-device copy of other's links (same shape and precision)."""
        self._check(lib().gc_copy_links(self._h, other.handle))

    # --- time slices (t-slab decomposition; see general_code_b200.tslab)
    def upload_slices(self, t0: int, links: np.ndarray, layout: str = "rowmajor") -> None:
        """Uploads host links of whole time slices (4 links per site, the
        reference's layout, t slowest) into the slices starting at t0."""
        a = np.ascontiguousarray(links, dtype=np.float64)
        per_slice = 4 * self.dims[0] * self.dims[1] * self.dims[2] * link_size(self.nc)
        if a.size % per_slice:
            raise ValueError("link array is not a whole number of time slices")
        self._check(lib().gc_upload_slices(self._h, int(t0), a.size // per_slice, dbl_ptr(a),
                                           _LAYOUT[layout]))
        if a is not links:
            self.synchronize()

    def slice_bytes(self, nt: int) -> int:
        """Bytes of nt packed time slices in this lattice's device form."""
        n = lib().gc_slice_bytes(self._h, int(nt))
        if n < 0:
            raise GCError(GC_ERR_ARG, "bad slice count")
        return int(n)

    def pack_slices(self, t0: int, nt: int, dev_ptr: int) -> None:
        """Packs the slices [t0, t0+nt) into the device buffer at dev_ptr."""
        self._check(lib().gc_pack_slices(self._h, int(t0), int(nt), ctypes.c_void_p(dev_ptr)))

    def unpack_slices(self, t0: int, nt: int, dev_ptr: int) -> None:
        """Fills the slices [t0, t0+nt) from the packed device buffer at dev_ptr."""
        self._check(lib().gc_unpack_slices(self._h, int(t0), int(nt),
                                           ctypes.c_void_p(dev_ptr)))

    def copy_slices_from(self, dst_t0: int, other: "Lattice", src_t0: int, nt: int) -> None:
        """Device copy of other's slices [src_t0, src_t0+nt) to [dst_t0, dst_t0+nt)."""
        self._check(lib().gc_copy_slices(self._h, int(dst_t0), other.handle, int(src_t0),
                                         int(nt)))

    def wilson_loop_tslab(self, t_starts: int, r_min: int, r_max: int, time_min: int,
                          time_max: int, adjoint: bool = False) -> np.ndarray:
        """W table averaged over the loops whose lower edge lies on the slices
        [0, t_starts) (a t-slab with its forward halo above); same layout as
        wilson_loop."""
        out = np.empty((time_max - time_min + 1, r_max - r_min + 1), dtype=np.float64)
        self._check(lib().gc_wilson_onaxis_tslab(self._h, int(t_starts), int(r_min), int(r_max),
                                                 int(time_min), int(time_max), int(bool(adjoint)),
                                                 dbl_ptr(out)))
        return out

    def generate(self, eps: float, seed: int, index: int = 0, gauge: bool = True) -> None:
        self._check(lib().gc_generate(self._h, float(eps), int(seed) & 0xffffffff,
                                      int(index) & 0xffffffff, int(bool(gauge))))

    def ape(self, alpha: float, steps: int = 1) -> None:
        self._check(lib().gc_ape(self._h, float(alpha), int(steps)))

    def hyp(self, alpha1: float, alpha2: float, alpha3: float, steps: int = 1) -> None:
        self._check(lib().gc_hyp(self._h, float(alpha1), float(alpha2), float(alpha3),
                                 int(steps)))

    def set_hyp_method(self, method: str) -> None:
        """"auto" (the library's choice: the level kernels), "levels" (one
        launch per decoration level) or "slices" (a pipeline over time slices
        with the decorated links in rings of three slices; Lt >= 3). The links
        are the same bit for bit."""
        m = {"auto": _lib.GC_HYP_AUTO, "levels": _lib.GC_HYP_LEVELS,
             "slices": _lib.GC_HYP_SLICES}[method]
        self._check(lib().gc_set_hyp_method(self._h, m))

    def wilson_loop(self, r_min: int, r_max: int, time_min: int, time_max: int) -> np.ndarray:
        """W table, shape (time_max-time_min+1, r_max-r_min+1): [T-t_min, R-r_min]."""
        out = np.empty((time_max - time_min + 1, r_max - r_min + 1), dtype=np.float64)
        self._check(lib().gc_wilson_onaxis(self._h, int(r_min), int(r_max), int(time_min),
                                           int(time_max), dbl_ptr(out)))
        return out

    def wilson_loop_adjoint(self, r_min: int, r_max: int, time_min: int,
                            time_max: int) -> np.ndarray:
        """Adjoint-representation W table (wilson_loops.h:1173-1200), same layout."""
        out = np.empty((time_max - time_min + 1, r_max - r_min + 1), dtype=np.float64)
        self._check(lib().gc_wilson_adjoint_onaxis(self._h, int(r_min), int(r_max),
                                                   int(time_min), int(time_max), dbl_ptr(out)))
        return out

    def set_wilson_method(self, method: str) -> None:
        """"auto" (the temporal-gauge form where it applies, after a device
        check of the temporal links' unitarity; else the exact product) or
        "exact" (always the exact product of links)."""
        m = {"auto": _lib.GC_WILSON_AUTO, "exact": _lib.GC_WILSON_EXACT}[method]
        self._check(lib().gc_set_wilson_method(self._h, m))

    def wilson_method_used(self) -> str:
        """Method of the last on-axis W call: "exact", "gauge" or "" (none yet)."""
        m = ctypes.c_int()
        self._check(lib().gc_wilson_method_used(self._h, ctypes.byref(m)))
        return {_lib.GC_WILSON_EXACT: "exact", _lib.GC_WILSON_GAUGE: "gauge"}.get(m.value, "")

    def plaquette(self) -> float:
        out = ctypes.c_double()
        self._check(lib().gc_plaquette(self._h, ctypes.byref(out)))
        return out.value

    def plaquette_time(self) -> float:
        """Average of the (mu, t) plaquettes (plaket.h:103-121)."""
        out = ctypes.c_double()
        self._check(lib().gc_plaquette_time(self._h, ctypes.byref(out)))
        return out.value

    def plaquette_space(self) -> float:
        """Average of the spatial plaquettes (plaket.h:123-141)."""
        out = ctypes.c_double()
        self._check(lib().gc_plaquette_space(self._h, ctypes.byref(out)))
        return out.value

    def wilson_gevp(self, other: "Lattice", r_min: int, r_max: int, time_min: int,
                    time_max: int, adjoint: bool = False) -> np.ndarray:
        """Two-configuration loops (wilson_gevp_indexed / wilson_gevp_adjoint_indexed,
        wilson_loops.h:1202-1266): time lines from self, space lines from self and
        other; same table layout as wilson_loop."""
        out = np.empty((time_max - time_min + 1, r_max - r_min + 1), dtype=np.float64)
        fn = lib().gc_wilson_gevp_adjoint_onaxis if adjoint else lib().gc_wilson_gevp_onaxis
        self._check(fn(self._h, other._h, int(r_min), int(r_max), int(time_min), int(time_max),
                       dbl_ptr(out)))
        return out

    def _offaxis(self, fn, *args):
        count = ctypes.c_int(0)
        cap = 4096
        while True:
            out = (WilsonResult * cap)()
            rc = fn(self._h, *args, ctypes.cast(out, ctypes.c_void_p), cap, ctypes.byref(count))
            if rc == GC_ERR_ARG and count.value > cap:
                cap = count.value
                continue
            self._check(rc)
            return [(r.wilson_loop, r.time_size, r.space_size, r.statistics_size)
                    for r in out[:count.value]]

    def wilson_offaxis(self, directions, r_min: float, r_max: float, time_min: int,
                       time_max: int, adjoint: bool = False):
        """Off-axis loops for the given directions (wilson_offaxis[_adjoint],
        wilson_loops.h:313-645): [(W, T, size, orientations)] in the
        reference's order, one per (direction, length multiple, T)."""
        d = np.ascontiguousarray(directions, dtype=np.int32).reshape(-1, 3)
        return self._offaxis(lib().gc_wilson_offaxis, d.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                             int(d.shape[0]), float(r_min), float(r_max), int(time_min),
                             int(time_max), 1 if adjoint else 0)

    def wilson_offaxis_result(self, r_min: float, r_max: float, time_min: int,
                              time_max: int, adjoint: bool = False) -> Dict[Tuple[int, float], float]:
        """Merged off-axis loops {(T, size): W} (wilson_offaxis[_adjoint]_result,
        wilson_loops.h:470-485, 648-663)."""
        entries = self._offaxis(lib().gc_wilson_offaxis_result, float(r_min), float(r_max),
                                int(time_min), int(time_max), 1 if adjoint else 0)
        out: Dict[Tuple[int, float], float] = {}
        for w, t, size, _ in entries:
            out[(t, size)] = w
        return out

    def ape_plane(self, a: int, b: int, alpha: float, steps: int = 1) -> None:
        """Two-dimensional APE steps of directions a and b in the (a, b) plane
        (smearing_APE_2d, smearing.h:223-277), in place."""
        self._check(lib().gc_ape_plane(self._h, int(a), int(b), float(alpha), int(steps)))

    def wilson_spatial_3d(self, r_min: int, r_max: int, time_min: int, time_max: int,
                          alpha: float, smearing_start: int, smearing_end: int,
                          smearing_step: int) -> Dict[Tuple[int, int, int], float]:
        """Spatial Wilson loops with two-dimensional APE smearing
        (wilson_spatial_3d_indexed, wilson_loops.h:1384-1428):
        {(smearing, T, R): W}."""
        count = ctypes.c_int(0)
        cap = 4096
        while True:
            out = (WilsonSpatialResult * cap)()
            rc = lib().gc_wilson_spatial_3d(self._h, int(r_min), int(r_max), int(time_min),
                                            int(time_max), float(alpha), int(smearing_start),
                                            int(smearing_end), int(smearing_step),
                                            ctypes.cast(out, ctypes.c_void_p), cap,
                                            ctypes.byref(count))
            if rc == GC_ERR_ARG and count.value > cap:
                cap = count.value
                continue
            self._check(rc)
            return {(r.smearing, r.time_size, r.space_size): r.wilson_loop
                    for r in out[:count.value]}

    def polyakov_loop(self) -> float:
        """Mean of Re Tr P / N over spatial sites (polyakov_loops.h:24-41)."""
        out = ctypes.c_double()
        self._check(lib().gc_polyakov_loop(self._h, ctypes.byref(out)))
        return out.value

    def polyakov_correlator(self, d_max: int, singlet: bool) -> np.ndarray:
        """(2 d_max + 1)^3 table of polyakov_loop_correlator_singlet (singlet) or
        _color_average (polyakov_loops.h:83-206), entry
        (Dz+d)(2d+1)^2 + (Dy+d)(2d+1) + Dx+d."""
        if int(d_max) < 0:
            raise GCError(GC_ERR_ARG, "D_max must be >= 0")
        n = 2 * int(d_max) + 1
        out = np.empty(n ** 3, dtype=np.float64)
        self._check(lib().gc_polyakov_correlator(self._h, int(d_max), 1 if singlet else 0,
                                                 dbl_ptr(out)))
        return out


class LatticeData:
    """Host-side configuration, like Data::LatticeData<DataPatternLexicographical, MT>.

    `array` has shape (4*V, 4) for SU(2) or (4*V, 18) for SU(3), link index
    4*site + mu, in the row-major layout of the reference's get_data().
    """

    def __init__(self, lat_dim: Sequence[int], nc: int, array: np.ndarray | None = None):
        self.lat_dim = tuple(int(d) for d in lat_dim)
        self.nc = int(nc)
        if array is None:
            array = unit_config(self.lat_dim, self.nc)
        self.array = np.ascontiguousarray(array, dtype=np.float64).reshape(
            4 * volume(self.lat_dim), link_size(self.nc))

    def _run(self, fn, precision: str = "fp64"):
        with Lattice(self.lat_dim, self.nc, precision) as lat:
            lat.upload(self.array)
            r = fn(lat)
            return lat, r


def smearing_APE(conf: LatticeData, alpha: float) -> None:
    """One APE step in place (smearing.h:115-161)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        lat.ape(alpha, 1)
        lat.download(conf.array)


def smearing_HYP(conf: LatticeData, alpha1: float, alpha2: float, alpha3: float) -> None:
    """One HYP step in place (smearing.h:480-516)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        lat.hyp(alpha1, alpha2, alpha3, 1)
        lat.download(conf.array)


def wilson_loop(conf: LatticeData, r_min: int, r_max: int, time_min: int,
                time_max: int) -> Dict[Tuple[int, int], float]:
    """On-axis W(R,T) as a dict keyed (T, R) (wilson_loops.h:1047-1074)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        w = lat.wilson_loop(r_min, r_max, time_min, time_max)
    return {(t, r): float(w[t - time_min, r - r_min])
            for t in range(time_min, time_max + 1) for r in range(r_min, r_max + 1)}


def plaket(conf: LatticeData) -> float:
    """Average plaquette (plaket.h:83-101)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return lat.plaquette()


def plaket_time(conf: LatticeData) -> float:
    """Average (mu, t) plaquette (plaket.h:103-121)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return lat.plaquette_time()


def plaket_space(conf: LatticeData) -> float:
    """Average spatial plaquette (plaket.h:123-141)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return lat.plaquette_space()


def _gevp(conf1: LatticeData, conf2: LatticeData, r_min, r_max, time_min, time_max, adjoint):
    if conf1.lat_dim != conf2.lat_dim or conf1.nc != conf2.nc:
        raise GCError(GC_ERR_ARG, "the two configurations differ in size or group")
    with Lattice(conf1.lat_dim, conf1.nc) as a, Lattice(conf2.lat_dim, conf2.nc) as b:
        a.upload(conf1.array)
        b.upload(conf2.array)
        w = a.wilson_gevp(b, r_min, r_max, time_min, time_max, adjoint)
    return {(t, r): float(w[t - time_min, r - r_min])
            for t in range(time_min, time_max + 1) for r in range(r_min, r_max + 1)}


def wilson_gevp_indexed(conf1: LatticeData, conf2: LatticeData, r_min: int, r_max: int,
                        time_min: int, time_max: int) -> Dict[Tuple[int, int], float]:
    """Two-configuration W(R,T) keyed (T, R) (wilson_loops.h:1202-1233)."""
    return _gevp(conf1, conf2, r_min, r_max, time_min, time_max, False)


def wilson_gevp_adjoint_indexed(conf1: LatticeData, conf2: LatticeData, r_min: int,
                                r_max: int, time_min: int,
                                time_max: int) -> Dict[Tuple[int, int], float]:
    """Adjoint two-configuration W(R,T) keyed (T, R) (wilson_loops.h:1235-1266)."""
    return _gevp(conf1, conf2, r_min, r_max, time_min, time_max, True)


def wilson_loop_adjoint(conf: LatticeData, r_min: int, r_max: int, time_min: int,
                        time_max: int) -> Dict[Tuple[int, int], float]:
    """Adjoint-representation W(R,T) keyed (T, R) (wilson_loops.h:1173-1200)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        w = lat.wilson_loop_adjoint(r_min, r_max, time_min, time_max)
    return {(t, r): float(w[t - time_min, r - r_min])
            for t in range(time_min, time_max + 1) for r in range(r_min, r_max + 1)}


def _wilson_result_list(entries):
    return [{"wilson_loop": w, "time_size": t, "space_size": size, "statistics_size": n}
            for w, t, size, n in entries]


def wilson_offaxis(conf: LatticeData, directions, r_min: float, r_max: float, time_min: int,
                   time_max: int):
    """Off-axis loops (wilson_loops.h:313-467) as a list of wilson_result dicts."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return _wilson_result_list(lat.wilson_offaxis(directions, r_min, r_max, time_min,
                                                      time_max))


def wilson_offaxis_adjoint(conf: LatticeData, directions, r_min: float, r_max: float,
                           time_min: int, time_max: int):
    """Adjoint off-axis loops (wilson_loops.h:487-645)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return _wilson_result_list(lat.wilson_offaxis(directions, r_min, r_max, time_min,
                                                      time_max, adjoint=True))


def wilson_offaxis_result(conf: LatticeData, r_min: float, r_max: float, time_min: int,
                          time_max: int) -> Dict[Tuple[int, float], float]:
    """Merged off-axis loops keyed (T, size) (wilson_loops.h:470-485)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return lat.wilson_offaxis_result(r_min, r_max, time_min, time_max)


def wilson_offaxis_adjoint_result(conf: LatticeData, r_min: float, r_max: float, time_min: int,
                                  time_max: int) -> Dict[Tuple[int, float], float]:
    """Merged adjoint off-axis loops keyed (T, size) (wilson_loops.h:648-663)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return lat.wilson_offaxis_result(r_min, r_max, time_min, time_max, adjoint=True)


def wilson_spatial_3d_indexed(conf: LatticeData, r_min: int, r_max: int, time_min: int,
                              time_max: int, alpha: float, smearing_start: int,
                              smearing_end: int,
                              smearing_step: int) -> Dict[Tuple[int, int, int], float]:
    """Spatial Wilson loops keyed (smearing, T, R) (wilson_loops.h:1384-1428)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return lat.wilson_spatial_3d(r_min, r_max, time_min, time_max, alpha, smearing_start,
                                     smearing_end, smearing_step)


def polyakov_loop(conf: LatticeData) -> float:
    """Polyakov loop (polyakov_loops.h:24-41)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return lat.polyakov_loop()


def polyakov_loop_correlator_singlet(conf: LatticeData, D_max: int) -> np.ndarray:
    """Singlet correlator table (polyakov_loops.h:147-206)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return lat.polyakov_correlator(D_max, True)


def polyakov_loop_correlator_color_average(conf: LatticeData, D_max: int) -> np.ndarray:
    """Color-averaged correlator table (polyakov_loops.h:83-145)."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.upload(conf.array)
        return lat.polyakov_correlator(D_max, False)


def polyakov_average_directions(correlators: np.ndarray, D_max: int) -> Dict[float, float]:
    """Average of a correlator table over offsets of equal length, origin
    excluded (the reference's polyakov_average_directions,
    lib/cpu/src/polyakov_loops.cpp:6-40): {distance: mean}, ascending."""
    n = 2 * int(D_max) + 1
    c = np.asarray(correlators, dtype=np.float64).reshape(n, n, n)  # [Dz][Dy][Dx]
    sums: Dict[float, float] = {}
    counts: Dict[float, int] = {}
    for dz in range(-D_max, D_max + 1):
        for dy in range(-D_max, D_max + 1):
            dx_min = 0 if (dy != 0 and dz != 0) else -D_max
            for dx in range(dx_min, D_max + 1):
                d = math.sqrt(dx * dx + dy * dy + dz * dz)
                if d <= D_max and not (dx == 0 and dy == 0 and dz == 0):
                    sums[d] = sums.get(d, 0.0) + float(c[dz + D_max, dy + D_max, dx + D_max])
                    counts[d] = counts.get(d, 0) + 1
    return {d: sums[d] / counts[d] for d in sorted(sums)}


def read_data_convert(conf: LatticeData, file_path, conf_format: str, bytes_skip: int,
                      file_precision: str, convert: bool) -> None:
    """Fills conf.array from a file (data.h:265-338), through the device reader."""
    with Lattice(conf.lat_dim, conf.nc) as lat:
        lat.read(file_path, conf_format, bytes_skip, file_precision, convert)
        lat.download(conf.array)


def probe_config(dims: Sequence[int], nc: int, path, conf_format: str, bytes_skip: int = 0,
                 file_precision: str = "double") -> Tuple[int, int]:
    """(offset, length) of a configuration file's link payload; raises GCError."""
    off, ln = ctypes.c_longlong(), ctypes.c_longlong()
    check(lib().gc_probe_config(dims_arg(dims), nc, str(path).encode(), conf_format.encode(),
                                int(bytes_skip), file_precision.encode(), ctypes.byref(off),
                                ctypes.byref(ln)))
    return off.value, ln.value


def job_device_bytes(dims: Sequence[int], nc: int, precision: str, r_max: int,
                     time_max: int) -> int:
    return int(lib().gc_job_device_bytes(dims_arg(dims), nc, _PREC[precision], r_max, time_max))


__all__ = ["Lattice", "LatticeData", "smearing_APE", "smearing_HYP", "wilson_loop", "plaket",
           "read_data_convert", "probe_config",
           "generate_config", "unit_config", "link_size", "volume", "job_device_bytes",
           "GCError"]
