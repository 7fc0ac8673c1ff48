"""Decomposition of one lattice into time slabs: smear and measure W(R,T) on
several GPUs, one rank per GPU, with one exchange of smeared slices.

The reference runs one lattice on the threads of one node; it has no domain
decomposition. Here rank r owns the time slices [start_r, start_r + n_r) of
the global lattice (balanced: the first Lt % world ranks own one more). What
a slice needs from the slices above it follows from the reference's
algorithms:

* APE (smearing.h:115-161) replaces the spatial links using spatial staples
  only: every time slice smears on its own.
* HYP (smearing.h:283-516, src/smearing.cpp:333-379) replaces the temporal
  links. The smeared U_4(x) reads the decorated links at x, x +- nu and
  x + 4 (level 3), the temporal decorated links read the level-1 links on
  their own slice and the spatial ones on the slice above, and the level-1
  links read raw links on their own slice and the one above: the smeared
  temporal links of slice t depend on the raw links of slices t and t + 1
  only. So `hyp_steps` forward raw slices make a slab's own slices exact.
* W(R,T) with its lower edge on slice t (wilson_loops.h:665-791) reads the
  smeared links of slices t .. t + T.

Each rank therefore (1) uploads its slices and `hyp_steps` forward raw
slices into a smearing lattice of n_r + hyp_steps slices, (2) runs HYP and
APE there (the temporal links of the top hyp_steps slices read slice 0 as
their neighbour above and are wrong; nothing uses them), (3) fills a
measuring lattice of n_r + T_max slices with its own smeared slices and the
T_max smeared slices above them, received from the ranks that own them in
one exchange (point-to-point sends of packed slices, NCCL on GPUs), and (4)
counts the loops that start on its own slices (gc_wilson_onaxis_tslab). One
all-reduce of W_r * n_r gives the global table times Lt.

The slab lattices are periodic in t like any lattice; the layout keeps every
counted loop inside a lattice's slices, so the wrap is never read by a
counted quantity. `emulate` runs the same plan for several slabs one after
another in one process on one GPU (slice copies in place of the exchange).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .lattice import Lattice, link_size, volume

__all__ = ["slab_bounds", "SlabPlan", "Run", "exchange_forward_halo", "TSlabJob",
           "smear_measure", "emulate"]


def slab_bounds(lt: int, world: int) -> List[Tuple[int, int]]:
    """(start, count) of every rank's slab: Lt slices over `world` ranks, the
    first Lt % world ranks one slice more."""
    if world < 1 or lt < world:
        raise ValueError(f"cannot split {lt} time slices over {world} ranks")
    base, extra = divmod(lt, world)
    out, start = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((start, n))
        start += n
    return out


@dataclass(frozen=True)
class Run:
    """Slices [src_t0, src_t0 + n) of `owner`'s smearing lattice go to the
    slices [dst_t0, dst_t0 + n) of the receiving rank's measuring lattice."""
    owner: int
    src_t0: int
    dst_t0: int
    n: int


@dataclass(frozen=True)
class SlabPlan:
    """The slab layout of one lattice over `world` ranks."""
    dims: Tuple[int, int, int, int]
    world: int
    t_max: int
    hyp_steps: int = 1

    def __post_init__(self):
        if self.t_max < 1:
            raise ValueError("time_max must be >= 1")
        if self.hyp_steps < 0:
            raise ValueError("hyp_steps must be >= 0")
        slab_bounds(self.dims[3], self.world)  # validates

    @property
    def bounds(self) -> List[Tuple[int, int]]:
        return slab_bounds(self.dims[3], self.world)

    def owner(self, t: int) -> int:
        """Rank owning global slice t (taken modulo Lt)."""
        t %= self.dims[3]
        for r, (s, n) in enumerate(self.bounds):
            if s <= t < s + n:
                return r
        raise AssertionError("unreachable")

    def smear_dims(self, rank: int) -> Tuple[int, int, int, int]:
        n = self.bounds[rank][1]
        return (*self.dims[:3], n + self.hyp_steps)

    def measure_dims(self, rank: int) -> Tuple[int, int, int, int]:
        n = self.bounds[rank][1]
        return (*self.dims[:3], n + self.t_max)

    def upload_runs(self, rank: int) -> List[Tuple[int, int, int]]:
        """(global first slice, local first slice, count) runs of raw slices
        that fill the smearing lattice (split where they wrap past Lt)."""
        lt = self.dims[3]
        start, n = self.bounds[rank]
        total = n + self.hyp_steps
        runs, local = [], 0
        while local < total:
            g = (start + local) % lt
            k = min(total - local, lt - g)
            runs.append((g, local, k))
            local += k
        return runs

    def forward_halo(self, rank: int) -> List[Run]:
        """Runs that fill the measuring lattice's slices [n_r, n_r + T_max):
        the smeared global slices end_r .. end_r + T_max - 1 (mod Lt), from
        their owners' smearing lattices (the receiving rank itself when the
        range wraps onto its own slab)."""
        lt = self.dims[3]
        bounds = self.bounds
        start, n = bounds[rank]
        runs: List[Run] = []
        j = 0
        while j < self.t_max:
            g = (start + n + j) % lt
            q = self.owner(g)
            qs, qn = bounds[q]
            k = min(self.t_max - j, qs + qn - g)
            runs.append(Run(q, g - qs, n + j, k))
            j += k
        return runs

    def sends(self, rank: int) -> Dict[int, List[Run]]:
        """For every other rank p, the runs p receives from `rank`, in p's
        order (the order both sides pack and unpack in)."""
        out: Dict[int, List[Run]] = {}
        for p in range(self.world):
            if p == rank:
                continue
            rs = [x for x in self.forward_halo(p) if x.owner == rank]
            if rs:
                out[p] = rs
        return out

    def receives(self, rank: int) -> Dict[int, List[Run]]:
        out: Dict[int, List[Run]] = {}
        for x in self.forward_halo(rank):
            if x.owner != rank:
                out.setdefault(x.owner, []).append(x)
        return out


def exchange_forward_halo(plan: SlabPlan, rank: int, source, dest, device, group=None) -> None:
    """Fills `dest`'s forward halo (plan.forward_halo(rank)).

    `source` (this rank's smearing lattice) and `dest` (its measuring
    lattice) expose slice_bytes(n), pack_slices(t0, n, ptr),
    unpack_slices(t0, n, ptr) and, on dest, copy_slices_from(dst_t0, source,
    src_t0, n): Lattice does; tests use host stand-ins. Buffers are uint8
    tensors on `device`; all sends and receives of a rank go out as one
    batch of point-to-point operations, so no rank waits on another's order.
    """
    import torch
    import torch.distributed as dist

    for x in plan.forward_halo(rank):
        if x.owner == rank:
            dest.copy_slices_from(x.dst_t0, source, x.src_t0, x.n)
    sends, recvs = plan.sends(rank), plan.receives(rank)
    ops, bufs = [], []
    for p, runs in sorted(sends.items()):
        buf = torch.empty(sum(source.slice_bytes(x.n) for x in runs), dtype=torch.uint8,
                          device=device)
        off = 0
        for x in runs:
            source.pack_slices(x.src_t0, x.n, buf.data_ptr() + off)
            off += source.slice_bytes(x.n)
        ops.append(dist.P2POp(dist.isend, buf, p, group=group))
        bufs.append(buf)
    if sends and hasattr(source, "synchronize"):
        source.synchronize()  # packed before the sends read the buffers
    incoming = []
    for q, runs in sorted(recvs.items()):
        buf = torch.empty(sum(dest.slice_bytes(x.n) for x in runs), dtype=torch.uint8,
                          device=device)
        ops.append(dist.P2POp(dist.irecv, buf, q, group=group))
        incoming.append((runs, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        if device is not None and torch.device(device).type == "cuda":
            torch.cuda.current_stream(device).synchronize()
    for runs, buf in incoming:
        off = 0
        for x in runs:
            dest.unpack_slices(x.dst_t0, x.n, buf.data_ptr() + off)
            off += dest.slice_bytes(x.n)
    if incoming and hasattr(dest, "synchronize"):
        dest.synchronize()  # the receive buffers are released on return


def _slices(host: np.ndarray, dims: Sequence[int], nc: int, g0: int, n: int) -> np.ndarray:
    per = 4 * dims[0] * dims[1] * dims[2]
    return host.reshape(-1, link_size(nc))[per * g0: per * (g0 + n)]


def _smear(plan: SlabPlan, rank: int, host: np.ndarray, nc: int, precision: str,
           hyp: Optional[Tuple[float, float, float]], ape_alpha: float, ape_steps: int,
           stream_ptr: Optional[int]) -> Lattice:
    lat = Lattice(plan.smear_dims(rank), nc, precision)
    if stream_ptr is not None:
        lat.set_stream(stream_ptr)
    for g0, l0, k in plan.upload_runs(rank):
        lat.upload_slices(l0, _slices(host, plan.dims, nc, g0, k))
    if hyp is not None and plan.hyp_steps:
        lat.hyp(*hyp, plan.hyp_steps)
    if ape_steps:
        lat.ape(ape_alpha, ape_steps)
    return lat


def _check_args(dims, nc, host, hyp, hyp_steps):
    dims = tuple(int(d) for d in dims)
    if len(dims) != 4:
        raise ValueError("dims must have four extents")
    if host.size != 4 * volume(dims) * link_size(nc):
        raise ValueError("link array has the wrong size for this lattice")
    return dims, (hyp_steps if hyp is not None else 0)


class TSlabJob:
    """One lattice's smear-and-measure job split into time slabs over the
    ranks of `group` (the default process group; a single process when
    torch.distributed is not initialised), with this rank's slab lattices
    kept between runs: `load` keeps the rank's raw slices resident, `run`
    smears and measures them (from the resident copy, or from a host array
    it uploads first) and returns the global W table on every rank. Every
    rank must call `run` the same number of times (each holds one batch of
    point-to-point operations and one all-reduce). The lattices, the
    exchange and the all-reduce run on the job's own CUDA stream
    (`self.stream`, a torch stream: record timing events there)."""

    def __init__(self, dims: Sequence[int], nc: int, *, precision: str = "mixed",
                 hyp: Optional[Tuple[float, float, float]] = (1.0, 1.0, 0.5),
                 hyp_steps: int = 1, ape_alpha: float = 0.5, ape_steps: int = 0,
                 r_min: int = 1, r_max: int = 1, time_min: int = 1, time_max: int = 1,
                 group=None):
        import torch
        import torch.distributed as dist

        self.dims = tuple(int(d) for d in dims)
        if len(self.dims) != 4:
            raise ValueError("dims must have four extents")
        self.nc, self.precision, self.group = nc, precision, group
        self.hyp, self.ape_alpha, self.ape_steps = hyp, ape_alpha, ape_steps
        self.ranges = (int(r_min), int(r_max), int(time_min), int(time_max))
        self.distributed = dist.is_available() and dist.is_initialized()
        self.world = dist.get_world_size(group) if self.distributed else 1
        self.rank = dist.get_rank(group) if self.distributed else 0
        self.plan = SlabPlan(self.dims, self.world, int(time_max),
                             hyp_steps if hyp is not None else 0)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream(self.device)
        stream = self.stream.cuda_stream
        self._lats = []
        try:
            for d in (self.plan.smear_dims(self.rank), self.plan.smear_dims(self.rank),
                      self.plan.measure_dims(self.rank)):
                lat = Lattice(d, nc, precision)
                self._lats.append(lat)
                lat.set_stream(stream)
        except Exception:
            self.close()
            raise
        self.pristine, self.smear, self.meas = self._lats
        self._loaded = False

    def _upload(self, lat: Lattice, host: np.ndarray) -> None:
        if host.size != 4 * volume(self.dims) * link_size(self.nc):
            raise ValueError("link array has the wrong size for this lattice")
        for g0, l0, k in self.plan.upload_runs(self.rank):
            lat.upload_slices(l0, _slices(host, self.dims, self.nc, g0, k))

    def load(self, host: np.ndarray) -> None:
        """Keeps this rank's raw slices (and the HYP halo above) resident."""
        self._upload(self.pristine, host)
        self._loaded = True

    def run(self, host: Optional[np.ndarray] = None) -> np.ndarray:
        """Smears and measures: from `host` (uploaded first) or the copy
        `load` keeps. Returns the global table [T - time_min, R - r_min]."""
        import torch
        import torch.distributed as dist

        if host is not None:
            self._upload(self.smear, host)
        elif self._loaded:
            self.smear.copy_from(self.pristine)
        else:
            raise RuntimeError("TSlabJob.run without links: call load() or pass host")
        plan, rank = self.plan, self.rank
        if self.hyp is not None and plan.hyp_steps:
            self.smear.hyp(*self.hyp, plan.hyp_steps)
        if self.ape_steps:
            self.smear.ape(self.ape_alpha, self.ape_steps)
        n = plan.bounds[rank][1]
        with torch.cuda.stream(self.stream):
            self.meas.copy_slices_from(0, self.smear, 0, n)
            if self.distributed and self.world > 1:
                exchange_forward_halo(plan, rank, self.smear, self.meas, self.device,
                                      self.group)
            else:
                for x in plan.forward_halo(rank):
                    self.meas.copy_slices_from(x.dst_t0, self.smear, x.src_t0, x.n)
            w = self.meas.wilson_loop_tslab(n, *self.ranges)
            if self.distributed and self.world > 1:
                t = torch.from_numpy(w * n).to(self.device)
                dist.all_reduce(t, group=self.group)
                return t.cpu().numpy() / self.dims[3]
        return w * n / self.dims[3]

    def close(self) -> None:
        for lat in getattr(self, "_lats", []):
            lat.close()
        self._lats = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def smear_measure(host: np.ndarray, dims: Sequence[int], nc: int, *, precision: str = "mixed",
                  hyp: Optional[Tuple[float, float, float]] = (1.0, 1.0, 0.5),
                  hyp_steps: int = 1, ape_alpha: float = 0.5, ape_steps: int = 0,
                  r_min: int = 1, r_max: int = 1, time_min: int = 1, time_max: int = 1,
                  group=None) -> np.ndarray:
    """HYP (hyp_steps steps, alphas `hyp`, None for none) then APE on one
    lattice split into time slabs over the ranks of `group` (the default
    process group; a single process when torch.distributed is not
    initialised), then on-axis W(R,T): returns the global table
    [T - time_min, R - r_min] on every rank. `host` is the global
    configuration in the reference's row-major layout; a rank reads only its
    slices and the hyp_steps above them. Every rank must call it (it holds
    one batch of point-to-point operations and one all-reduce)."""
    dims, _ = _check_args(dims, nc, host, hyp, hyp_steps)
    with TSlabJob(dims, nc, precision=precision, hyp=hyp, hyp_steps=hyp_steps,
                  ape_alpha=ape_alpha, ape_steps=ape_steps, r_min=r_min, r_max=r_max,
                  time_min=time_min, time_max=time_max, group=group) as job:
        return job.run(host)


def emulate(host: np.ndarray, dims: Sequence[int], nc: int, slabs: int, *,
            precision: str = "mixed", hyp: Optional[Tuple[float, float, float]] = (1.0, 1.0, 0.5),
            hyp_steps: int = 1, ape_alpha: float = 0.5, ape_steps: int = 0, r_min: int = 1,
            r_max: int = 1, time_min: int = 1, time_max: int = 1) -> np.ndarray:
    """The slab plan for `slabs` ranks run in this process on the current GPU:
    every slab's smearing and measuring lattice, the forward halos filled by
    slice copies between them, and the per-slab tables summed in rank order.
    Returns the global W table (same as smear_measure on `slabs` GPUs, up to
    the order of the final sum)."""
    dims, hsteps = _check_args(dims, nc, host, hyp, hyp_steps)
    plan = SlabPlan(dims, int(slabs), int(time_max), hsteps)
    smears = []
    try:
        for r in range(plan.world):
            smears.append(_smear(plan, r, host, nc, precision, hyp, ape_alpha, ape_steps, None))
        total = None
        for r in range(plan.world):
            n = plan.bounds[r][1]
            with Lattice(plan.measure_dims(r), nc, precision) as meas:
                meas.copy_slices_from(0, smears[r], 0, n)
                for x in plan.forward_halo(r):
                    meas.copy_slices_from(x.dst_t0, smears[x.owner], x.src_t0, x.n)
                w = meas.wilson_loop_tslab(n, r_min, r_max, time_min, time_max) * n
            total = w if total is None else total + w
        return total / dims[3]
    finally:
        for s in smears:
            s.close()
