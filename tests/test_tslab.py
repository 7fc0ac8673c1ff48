"""t-slab decomposition of one lattice.

CPU: the slab plan (bounds, upload runs, forward-halo runs), the halo depth
against the C oracle (HYP + APE on a slab's smearing lattice leave its own
slices bit-identical to the same slices smeared as one lattice), and the
exchange over gloo ranks with host stand-ins for the device lattices.
GPU: the slice entry points and the whole decomposition, emulated on one GPU,
against the same job run on one lattice.
"""
from __future__ import annotations

import ctypes
import os
import socket

import numpy as np
import pytest

from general_code_b200 import generate_config, link_size
from general_code_b200.tslab import Run, SlabPlan, exchange_forward_halo, slab_bounds


def _slices(a, dims, nc, g0, n):
    per = 4 * dims[0] * dims[1] * dims[2]
    return a.reshape(-1, link_size(nc))[per * g0: per * (g0 + n)]


def _global_rows(a, dims, nc, g0, n):
    """Slices g0 .. g0+n-1 (mod Lt) of a host array, in that order."""
    lt = dims[3]
    return np.concatenate([_slices(a, dims, nc, (g0 + j) % lt, 1) for j in range(n)])


# ----------------------------------------------------------------- the plan
def test_slab_bounds_balanced():
    assert slab_bounds(24, 8) == [(3 * r, 3) for r in range(8)]
    assert slab_bounds(10, 4) == [(0, 3), (3, 3), (6, 2), (8, 2)]
    assert slab_bounds(5, 1) == [(0, 5)]
    for lt, w in [(7, 0), (3, 4)]:
        with pytest.raises(ValueError):
            slab_bounds(lt, w)


@pytest.mark.parametrize("lt,world,t_max,hyp", [(24, 8, 12, 1), (10, 4, 3, 1), (8, 2, 7, 2),
                                                (6, 3, 6, 0), (9, 2, 13, 1), (5, 1, 4, 1)])
def test_plan_runs_cover_the_needed_slices(lt, world, t_max, hyp):
    plan = SlabPlan((2, 2, 2, lt), world, t_max, hyp)
    for r, (start, n) in enumerate(plan.bounds):
        # raw uploads: slices start .. start+n+hyp-1 (mod Lt), in order
        got = [(g0 + j) for g0, l0, k in plan.upload_runs(r) for j in range(k)]
        assert got == [(start + j) % lt for j in range(n + hyp)]
        assert [l0 for _, l0, _ in plan.upload_runs(r)] == sorted(
            {l0 for _, l0, _ in plan.upload_runs(r)})
        # forward halo: global slices end .. end+t_max-1 (mod Lt) at n .. n+t_max-1
        cover = {}
        for x in plan.forward_halo(r):
            qs, qn = plan.bounds[x.owner]
            assert 0 <= x.src_t0 and x.src_t0 + x.n <= qn  # only owned, smeared slices
            for j in range(x.n):
                cover[x.dst_t0 + j] = qs + x.src_t0 + j
        assert cover == {n + j: (start + n + j) % lt for j in range(t_max)}
    # sends and receives pair up
    for r in range(world):
        for p, runs in plan.sends(r).items():
            assert plan.receives(p)[r] == runs


def test_plan_wraps_onto_own_slab():
    plan = SlabPlan((2, 2, 2, 6), 2, 5, 1)  # rank 0 owns 0..2, needs 3..7 -> 3,4,5 and 0,1
    assert plan.forward_halo(0) == [Run(1, 0, 3, 3), Run(0, 0, 6, 2)]
    assert 0 not in plan.receives(0)


# ------------------------------------------------- halo depth, via the oracle
@pytest.mark.parametrize("nc,dims,world,hyp_steps,ape", [
    (3, (3, 3, 3, 8), 2, 1, 3),
    (3, (3, 4, 3, 7), 3, 1, 2),
    (2, (4, 4, 4, 8), 4, 2, 4),
    (2, (3, 3, 3, 5), 1, 1, 2),
])
def test_slab_smearing_is_exact(port, nc, dims, world, hyp_steps, ape):
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 20261203, 3)
    whole = links.copy()
    port.hyp(nc, dims, whole, 1.0, 0.75, 0.6, hyp_steps)
    port.ape(nc, dims, whole, 0.5, ape)
    plan = SlabPlan(dims, world, 1, hyp_steps)
    for r, (start, n) in enumerate(plan.bounds):
        sd = plan.smear_dims(r)
        slab = np.concatenate([_slices(links, dims, nc, g0, k)
                               for g0, _, k in plan.upload_runs(r)])
        port.hyp(nc, sd, slab, 1.0, 0.75, 0.6, hyp_steps)
        port.ape(nc, sd, slab, 0.5, ape)
        own = _slices(slab, sd, nc, 0, n)
        assert np.array_equal(own, _slices(whole, dims, nc, start, n)), f"rank {r}"


def test_one_halo_slice_fewer_is_not_exact(port):
    """The forward halo is needed: with hyp_steps raw slices fewer the top
    owned slice's temporal links differ (the depth is not larger than it
    must be, and not smaller)."""
    nc, dims = 3, (3, 3, 3, 6)
    links = generate_config(dims, nc, 0.25, 20261203, 4)
    whole = links.copy()
    port.hyp(nc, dims, whole, 1.0, 0.75, 0.6, 1)
    n = 3
    slab = _slices(links, dims, nc, 0, n).copy()  # no forward halo
    port.hyp(nc, (*dims[:3], n), slab, 1.0, 0.75, 0.6, 1)
    assert np.array_equal(_slices(slab, dims, nc, 0, n - 1), _slices(whole, dims, nc, 0, n - 1))
    assert not np.array_equal(_slices(slab, dims, nc, n - 1, 1),
                              _slices(whole, dims, nc, n - 1, 1))


# ----------------------------------------------- the exchange on gloo ranks
class HostSlices:
    """Host stand-in for a device lattice: the slices of a host link array."""

    def __init__(self, arr, dims, nc):
        self.arr, self.dims, self.nc = arr, dims, nc

    def _rows(self, t0, n):
        return _slices(self.arr, self.dims, self.nc, t0, n)

    def slice_bytes(self, n):
        return 4 * self.dims[0] * self.dims[1] * self.dims[2] * link_size(self.nc) * 8 * n

    def pack_slices(self, t0, n, ptr):
        src = np.ascontiguousarray(self._rows(t0, n))
        ctypes.memmove(ptr, src.ctypes.data, src.nbytes)

    def unpack_slices(self, t0, n, ptr):
        dst = self._rows(t0, n)
        ctypes.memmove(dst.ctypes.data, ptr, dst.nbytes)

    def copy_slices_from(self, dst_t0, other, src_t0, n):
        self._rows(dst_t0, n)[...] = other._rows(src_t0, n)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _exchange_worker(rank, world, port, nc, dims, t_max, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        links = generate_config(dims, nc, 0.25, 20261203, 9)
        plan = SlabPlan(dims, world, t_max, 1)
        start, n = plan.bounds[rank]
        # the smearing lattice's contents (here: raw slices; its HYP halo
        # rows are overwritten, so a halo row sent by mistake shows)
        sd = plan.smear_dims(rank)
        src = np.concatenate([_slices(links, dims, nc, g0, k)
                              for g0, _, k in plan.upload_runs(rank)])
        _slices(src, sd, nc, n, sd[3] - n)[...] = -1.0  # halo rows: never sent
        md = plan.measure_dims(rank)
        dst = np.full((4 * md[0] * md[1] * md[2] * md[3], link_size(nc)), np.nan)
        d = HostSlices(dst, md, nc)
        d.copy_slices_from(0, HostSlices(src, sd, nc), 0, n)
        exchange_forward_halo(plan, rank, HostSlices(src, sd, nc), d, "cpu")
        ok = np.array_equal(dst, _global_rows(links, dims, nc, start, n + t_max))
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dims,t_max", [(2, (2, 2, 3, 8), 5), (3, (2, 3, 2, 7), 6),
                                              (2, (2, 2, 2, 6), 5)])
def test_exchange_over_gloo_ranks(world, dims, t_max):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_worker, args=(r, world, port, 3, dims, t_max, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(res[r] for r in range(world)), res


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_upload_slices_pack_unpack_copy():
    from general_code_b200 import GCError, Lattice
    nc, dims = 3, (4, 3, 5, 6)
    links = generate_config(dims, nc, 0.25, 20261203, 5)
    for form in ("fp64", "mixed"):
        with Lattice(dims, nc, form) as a, Lattice(dims, nc, form) as b, \
                Lattice((*dims[:3], 4), nc, form) as c:
            a.upload(links)
            ref = a.download()
            for t0, n in [(0, 2), (2, 3), (5, 1)]:
                b.upload_slices(t0, _slices(links, dims, nc, t0, n))
            assert np.array_equal(b.download(), ref)
            import torch
            buf = torch.empty(a.slice_bytes(3), dtype=torch.uint8, device="cuda")
            a.pack_slices(3, 3, buf.data_ptr())
            a.synchronize()
            c.upload_slices(0, _slices(links, dims, nc, 0, 4))
            c.unpack_slices(1, 3, buf.data_ptr())
            c.synchronize()
            got = c.download()
            assert np.array_equal(_slices(got, dims, nc, 0, 1), _slices(ref, dims, nc, 0, 1))
            assert np.array_equal(_slices(got, dims, nc, 1, 3), _slices(ref, dims, nc, 3, 3))
            c.copy_slices_from(0, a, 5, 1)
            assert np.array_equal(_slices(c.download(), dims, nc, 0, 1),
                                  _slices(ref, dims, nc, 5, 1))
            with pytest.raises(GCError):
                c.copy_slices_from(2, a, 0, 3)  # past the end of c
            with pytest.raises(GCError):
                a.pack_slices(5, 2, buf.data_ptr())
            with pytest.raises(GCError):
                a.wilson_loop_tslab(0, 1, 1, 1, 1)
            with pytest.raises(GCError):
                a.wilson_loop_tslab(7, 1, 1, 1, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("nc", [2, 3])
def test_wilson_tslab_full_is_wilson_loop(nc):
    from general_code_b200 import Lattice
    dims = (6, 6, 6, 8)
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 20261203, 6)
    for form in ("fp64", "mixed"):
        with Lattice(dims, nc, form) as lat:
            # the exact product of links on both entries (the temporal-gauge
            # form of the t-slab entry: the next test)
            lat.set_wilson_method("exact")
            lat.upload(links)
            lat.ape(0.5, 2)
            w = lat.wilson_loop(1, 3, 1, 4)
            assert np.array_equal(lat.wilson_loop_tslab(8, 1, 3, 1, 4), w)
            wa = lat.wilson_loop_adjoint(1, 3, 1, 4)
            assert np.array_equal(lat.wilson_loop_tslab(8, 1, 3, 1, 4, adjoint=True), wa)
            # a partition of the start slices: the lattice translated so that
            # slices a .. a+k-1 come first, counted from k slices, adds up
            # (k-weighted) to the whole
            total = np.zeros_like(w)
            for a, k in [(0, 3), (3, 2), (5, 3)]:
                with Lattice(dims, nc, form) as moved:
                    moved.set_wilson_method("exact")
                    moved.upload(_global_rows(links, dims, nc, a, dims[3]))
                    moved.ape(0.5, 2)
                    total += moved.wilson_loop_tslab(k, 1, 3, 1, 4) * k
            np.testing.assert_allclose(total / dims[3], w, rtol=1e-12, atol=1e-15)


# A slab's W in the temporal gauge against the exact product of the whole
# lattice: FP64 to rounding, mixed within the mixed form's tolerance.
_SLAB_RTOL = {"fp64": 1e-12, "mixed": 1e-6}


@pytest.mark.gpu
@pytest.mark.parametrize("nc", [2, 3])
@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_wilson_tslab_partition_in_the_temporal_gauge(nc, form):
    """The t-slab entry's loops of the start slices [0, t_starts), in the
    temporal gauge with one cut at slice 0 (no counted loop passes the
    lattice's last slice): a partition of the start slices of translated
    lattices adds up to the whole lattice's table."""
    from general_code_b200 import Lattice
    dims = (6, 6, 6, 8)
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 20261203, 6)
    with Lattice(dims, nc, form) as lat:
        lat.upload(links)
        lat.ape(0.5, 2)
        w = lat.wilson_loop(1, 3, 1, 4)
        assert lat.wilson_method_used() == "gauge"
    total = np.zeros_like(w)
    for a, k in [(0, 3), (3, 2), (5, 3)]:
        with Lattice(dims, nc, form) as moved:
            moved.upload(_global_rows(links, dims, nc, a, dims[3]))
            moved.ape(0.5, 2)
            total += moved.wilson_loop_tslab(k, 1, 3, 1, 4) * k
            assert moved.wilson_method_used() == "gauge"
    np.testing.assert_allclose(total / dims[3], w, rtol=_SLAB_RTOL[form], atol=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("nc,dims,slabs,t_max,form", [
    (3, (6, 6, 6, 12), 2, 6, "fp64"),
    (3, (6, 6, 6, 12), 3, 6, "mixed"),
    (3, (5, 6, 4, 10), 4, 5, "mixed"),
    (2, (8, 8, 8, 8), 3, 4, "fp64"),
    (2, (8, 8, 8, 8), 5, 7, "mixed"),
    (3, (4, 4, 4, 6), 2, 5, "fp64"),  # forward halo wraps onto the own slab
])
def test_emulated_slabs_match_one_lattice(nc, dims, slabs, t_max, form):
    from general_code_b200 import Lattice
    from general_code_b200.tslab import emulate
    links = generate_config(dims, nc, 0.3 if nc == 2 else 0.25, 20261203, 8)
    hyp, ape = (1.0, 0.75, 0.6), 3
    with Lattice(dims, nc, form) as lat:
        lat.set_wilson_method("exact")  # the slabs' W is the exact product
        lat.upload(links)
        lat.hyp(*hyp, 1)
        lat.ape(0.5, ape)
        ref = lat.wilson_loop(1, 3, 1, t_max)
    w = emulate(links, dims, nc, slabs, precision=form, hyp=hyp, hyp_steps=1, ape_alpha=0.5,
                ape_steps=ape, r_min=1, r_max=3, time_min=1, time_max=t_max)
    # (the slabs take the temporal-gauge form: the exact product's table to
    # FP64 rounding, within the mixed form's 1e-6 of it in FP32)
    np.testing.assert_allclose(w, ref, rtol=_SLAB_RTOL[form], atol=1e-15)


@pytest.mark.gpu
def test_smear_measure_single_process_matches_fixture_job(port):
    """The distributed entry with one rank (no process group): the oracle's
    job on the same configuration."""
    from general_code_b200.tslab import smear_measure
    nc, dims = 3, (6, 6, 6, 8)
    links = generate_config(dims, nc, 0.25, 20261203, 10)
    ref = links.copy()
    port.hyp(nc, dims, ref, 1.0, 0.75, 0.6, 1)
    port.ape(nc, dims, ref, 0.5, 2)
    want = port.wilson(nc, dims, ref, 1, 3, 1, 4)
    w = smear_measure(links, dims, nc, precision="fp64", hyp=(1.0, 0.75, 0.6), ape_steps=2,
                      r_min=1, r_max=3, time_min=1, time_max=4)
    np.testing.assert_allclose(w, want, rtol=1e-12, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_tslab_job_reuses_its_lattices(form):
    """TSlabJob in one process: runs from the resident slices and from the
    host array agree bitwise, repeated runs are identical, and the table is
    the one-lattice job's within 1e-12."""
    from general_code_b200 import Lattice
    from general_code_b200.tslab import TSlabJob
    nc, dims = 3, (6, 6, 6, 10)
    links = generate_config(dims, nc, 0.25, 20261203, 12)
    with Lattice(dims, nc, form) as lat:
        lat.set_wilson_method("exact")  # the slabs' W is the exact product
        lat.upload(links)
        lat.hyp(1.0, 0.75, 0.6, 1)
        lat.ape(0.5, 3)
        ref = lat.wilson_loop(1, 3, 1, 5)
    with TSlabJob(dims, nc, precision=form, hyp=(1.0, 0.75, 0.6), ape_steps=3, r_min=1,
                  r_max=3, time_min=1, time_max=5) as job:
        with pytest.raises(RuntimeError):
            job.run()
        job.load(links)
        a = job.run()
        b = job.run()
        c = job.run(links)
    assert np.array_equal(a, b) and np.array_equal(a, c)
    np.testing.assert_allclose(a, ref, rtol=_SLAB_RTOL[form], atol=1e-15)
