#!/usr/bin/env python
"""Smear-and-measure throughput on B200.

One step = one smear-and-measure job on one synthetic configuration:
HYP x1 (alpha 1, 0.75, 0.6) + APE x n (alpha 0.5) + the on-axis W(R,T) table.
Default workload: SU(3) 32^4, 1 HYP + 40 APE, R,T = 1..16, the largest
single-GPU configuration of the metric. Metric: smeared+measured sites/s.

  value  : device-resident throughput. Each step restores the unsmeared links
           from a resident copy (device-to-device) and runs the job; inputs are
           in HBM when the timed region starts.
  e2e    : the same job through the public C ABI with HOST buffers: pinned
           host links -> gc_upload, gc_hyp, gc_ape, gc_wilson_onaxis -> host,
           for a stream of K configurations through two handles on two CUDA
           streams (job i+1's upload overlaps job i's smearing and
           measurement); every job's upload and result read lie inside the
           timed region. `e2e.serial_value` is the same with one handle, each
           job's upload, compute and result read one after the other.
Both forms are timed on the same configuration (--form both, the default):
the headline is the mixed form (FP32 links, FP64 sums); the FP64 form is
reported under "forms", with the largest relative difference of the two
W(R,T) tables (the mixed form's error against FP64).
Between timed steps the L2 cache is flushed by writing a 256 MiB buffer.
Timing: CUDA events on the stream the kernels run on, max over ranks.
Sections (default on, 1 GPU): "su2" times SU(2) 16^4 (HYP + APE x10, R,T <= 8)
and SU(2) 48^4 (HYP + APE x10, R,T <= 24, 680 MB of FP64 links) the same way,
with each kernel family's HBM and FP-pipe fractions; "batch", "serving" and
"observables" time the other forms and observables.

--gpus N (under torchrun): every rank runs the job on its own configuration
(config index = rank); no data-path collective; weak scaling.
--impl reference: the reference's own CPU implementation (oracle/_ref, compiled
from the reference sources) on the host cores, rank 0 only, on a bounded
sample of the same job (one phase per step: HYP, one APE step, the W table;
the job time is the phases' mean times with the APE step counted n times).
The input comes from oracle/libgen.so, so that arm loads no product library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # SU(3) 32^4, 1 HYP + 40 APE, W R,T=1..16 (the headline: the largest
    # single-GPU configuration)
    "su3_32": dict(nc=3, dims=(32, 32, 32, 32), eps=0.25, hyp=(1.0, 0.75, 0.6), ape=40,
                   alpha=0.5, r=(1, 16), t=(1, 16)),
    # SU(3) 24^4, 1 HYP + 20 APE, W R,T=1..12 (FP64 vs mixed comparison case)
    "su3_24": dict(nc=3, dims=(24, 24, 24, 24), eps=0.25, hyp=(1.0, 0.75, 0.6), ape=20,
                   alpha=0.5, r=(1, 12), t=(1, 12)),
    # SU(2) 16^4, 1 HYP + 10 APE, W R,T=1..8 (the reference's CPU-sized case)
    "su2_16": dict(nc=2, dims=(16, 16, 16, 16), eps=0.3, hyp=(1.0, 0.75, 0.6), ape=10,
                   alpha=0.5, r=(1, 8), t=(1, 8)),
    # SU(2) 48^4, 1 HYP + 10 APE, W R,T=1..24: SU(2) at a size where the
    # memory-bound kernels are HBM-bound rather than launch-bound
    "su2_48": dict(nc=2, dims=(48, 48, 48, 48), eps=0.3, hyp=(1.0, 0.75, 0.6), ape=10,
                   alpha=0.5, r=(1, 24), t=(1, 24)),
}
DEFAULT_WORKLOAD = "su3_32"
SEED = 20261203
L2_FLUSH_BYTES = 256 << 20
L2_NOTE = ("GPU arm: L2 flushed (256 MiB write) before every timed step; "
           "CPU arm: host caches, no flush")


def config_dict(name, wl, world):
    """The workload's description; the same dict in both arms."""
    return {"workload": name, "lattice": list(wl["dims"]), "group": f"SU({wl['nc']})",
            "hyp_steps": 1, "hyp_alpha": list(wl["hyp"]), "ape_steps": wl["ape"],
            "ape_alpha": wl["alpha"], "r_range": list(wl["r"]), "t_range": list(wl["t"]),
            "sites": int(np.prod(wl["dims"])), "l2": L2_NOTE,
            "parallelism": f"replicas x{world}"}


def link_bytes(nc, form):
    if nc == 3:
        return 144 if form == "fp64" else 48
    return 32 if form == "fp64" else 16


def algorithmic(wl, form, w_method="exact"):
    """Algorithmic bytes and FP flops per site for each kernel family. W's
    flops are those of the method that ran: the exact product (two products
    and a dot per (x, nu, R, T)) or the temporal-gauge form (per site: the
    gauge lines of two cuts, the six transformed links, per (nu, R) one
    product per cut for the space lines, per (nu, R, T) one dot)."""
    nc = wl["nc"]
    b = link_bytes(nc, form)
    mm = 198 if nc == 3 else 28          # one matrix product
    dot = 36 if nc == 3 else 8           # Re Tr(A B^dag)
    proj = 3000 if nc == 3 else 11       # one projection
    nr = wl["r"][1] - wl["r"][0] + 1
    nt = wl["t"][1] - wl["t"][0] + 1
    if w_method == "gauge":
        w_flops = 2 * mm + 3 * 2 * 2 * mm + 3 * (2 * wl["r"][1] * mm + nr * nt * dot)
    else:
        w_flops = 3 * nr * nt * (2 * mm + dot)
    return {
        "ape": {"bytes": 6 * b, "flops": 3 * (8 * mm + proj)},
        "hyp": {"bytes": 5 * b, "flops": 96 * mm + 16 * proj},
        # W needs the 4 link fields once (the lines stay on chip)
        "wilson": {"bytes": 4 * b, "flops": w_flops, "method": w_method},
    }


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Nominal vector-pipe peaks of one B200 (148 SMs at 1965 MHz): FP64 64 and
# FP32 128 fused multiply-adds per SM per clock. Not measured on this pool
# (the measured peaks cover HBM copy and bf16 GEMM only).
FP_PEAK_TFLOPS = {"fp64": 148 * 64 * 2 * 1.965e9 / 1e12, "fp32": 148 * 128 * 2 * 1.965e9 / 1e12}


def load_traffic():
    p = ROOT / "profiles" / "roofline_traffic.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


def reference_checker():
    """The reference's own CPU path (oracle/_ref/libref_timed.so: -Ofast
    -fopenmp, all host threads), else the C restatement. Returns (checker,
    kind, threads)."""
    from oracle import py_oracle
    threads = os.cpu_count() or 1
    if py_oracle.ref_available("timed"):
        chk = py_oracle.ref("timed")
        chk.set_threads(threads)
        return chk, "reference", chk.num_threads()
    chk = py_oracle.port()
    chk.set_threads(threads)
    return chk, "port", threads


PHASES = ("hyp", "ape", "wilson")


def cpu_sample(wl, workload, host_links, steps, warmup=0):
    """A bounded sample of the job on the host cores: step i runs one phase,
    PHASES[i % 3] (the HYP step on the input links, one APE step on the
    HYP-smeared links, the W(R,T) table on the HYP+APE-smeared links); the
    job time is mean(HYP) + n_APE * mean(APE) + mean(W). Returns (sites/s,
    detail)."""
    chk, kind, cores = reference_checker()
    nc, dims = wl["nc"], wl["dims"]
    V = int(np.prod(dims))
    r0, r1 = wl["r"]
    t0, t1 = wl["t"]
    # inputs of the three phases (untimed)
    hyp_in = host_links
    ape_in = host_links.copy()
    chk.hyp(nc, dims, ape_in, *wl["hyp"], 1)
    w_in = ape_in.copy()
    chk.ape(nc, dims, w_in, wl["alpha"], 1)
    times = {p: [] for p in PHASES}
    busy = 0.0
    for i in range(warmup + steps):
        phase = PHASES[i % 3]
        src = {"hyp": hyp_in, "ape": ape_in, "wilson": w_in}[phase]
        links = src.copy() if phase != "wilson" else src
        t = time.perf_counter()
        if phase == "hyp":
            chk.hyp(nc, dims, links, *wl["hyp"], 1)
        elif phase == "ape":
            chk.ape(nc, dims, links, wl["alpha"], 1)
        else:
            chk.wilson(nc, dims, links, r0, r1, t0, t1)
        dt = time.perf_counter() - t
        busy += dt
        if i >= warmup:
            times[phase].append(dt)
    for p in PHASES:  # every phase measured at least once
        if not times[p]:
            links = {"hyp": hyp_in, "ape": ape_in, "wilson": w_in}[p].copy()
            t = time.perf_counter()
            if p == "hyp":
                chk.hyp(nc, dims, links, *wl["hyp"], 1)
            elif p == "ape":
                chk.ape(nc, dims, links, wl["alpha"], 1)
            else:
                chk.wilson(nc, dims, links, r0, r1, t0, t1)
            dt = time.perf_counter() - t
            busy += dt
            times[p].append(dt)
    mean = {p: sum(v) / len(v) for p, v in times.items()}
    job_s = mean["hyp"] + wl["ape"] * mean["ape"] + mean["wilson"]
    sample = (f"{workload}, FP64: one phase per step in rotation (HYP x1; APE x1, counted "
              f"x{wl['ape']}; W R={r0}..{r1} T={t0}..{t1}), "
              f"{sum(len(v) for v in times.values())} timed phases, {busy:.1f} s of CPU "
              f"time; job = {job_s:.2f} s")
    return V / job_s, {"cores": cores, "kind": kind, "sample": sample, "job_seconds": job_s,
                       "phase_seconds": mean}


def batch_serial(jobs, form, first_index):
    """The batch's jobs one after another through the single-lattice API on
    one stream (input resident, restored by a device copy; HYP, APE, the W
    table read back): the sum of the jobs' CUDA-event times, and their W
    tables."""
    import torch
    from general_code_b200 import Lattice, generate_config
    s = torch.cuda.Stream()
    total, tables, per_job = 0.0, [], []
    for k, j in enumerate(jobs):
        links = generate_config(j.dims, j.nc, 0.3 if j.nc == 2 else 0.25, SEED, first_index + k)
        with Lattice(j.dims, j.nc, form) as pristine, Lattice(j.dims, j.nc, form) as lat:
            for x in (pristine, lat):
                x.set_stream(s.cuda_stream)
            pristine.upload(links)
            w = None
            for rep in range(2):  # the first run sets up the handle
                lat.copy_from(pristine)
                e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
                e0.record(s)
                lat.hyp(*j.hyp_alpha, j.hyp_steps)
                lat.ape(j.ape_alpha, j.ape_steps)
                w = lat.wilson_loop(j.r_min, j.r_max, j.t_min, j.t_max)
                e1.record(s)
                s.synchronize()
            total += e0.elapsed_time(e1)
            per_job.append(e0.elapsed_time(e1))
            tables.append(w)
    return total, tables, per_job


def bench_batch(steps: int):
    """64 configurations of uneven sizes ({8^4, 12^4, 16^4, 16^3x32, 24^4,
    24^3x48}, SU(2)/SU(3) 50/50, APE 5..30, R,T up to L_s/2) as one batch:
    autotuned W shapes, one CUDA graph launch per run. Times `steps` graph
    launches with CUDA events after the capture run, and the same jobs one
    after another through the single-lattice API (batch_serial)."""
    import torch
    from general_code_b200.batch import Batch, uneven_jobs
    out = {}
    jobs = uneven_jobs(64)
    sites = sum(j.sites for j in jobs)
    for form in ("mixed", "fp64"):
        with Batch(jobs, form) as b:
            b.generate(0.3, 0.25, SEED, 1000)
            b.autotune()
            b.run()
            b.synchronize()
            s = torch.cuda.Stream()
            ms = []
            for _ in range(steps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s)
                b.run(s.cuda_stream)
                e1.record(s)
                s.synchronize()
                ms.append(e0.elapsed_time(e1))
            info = b.info()
            w_batch = [b.wilson(k) for k in range(len(jobs))]
            report = b.autotune_report()
        serial_ms, w_serial, per_job = batch_serial(jobs, form, 1000)
        # where the serial time goes: per lattice shape (jobs, ms)
        by_shape = {}
        for j, t in zip(jobs, per_job):
            key = f"SU({j.nc}) " + "x".join(map(str, j.dims))
            n, ms_ = by_shape.get(key, (0, 0.0))
            by_shape[key] = (n + 1, ms_ + t)
        worst = max(float(np.max(np.abs(a - c) / np.abs(c))) for a, c in zip(w_batch, w_serial))
        batch_ms = sum(ms) / len(ms)
        out[form] = {"sites_per_s": sites / (batch_ms * 1e-3),
                     "ms_per_batch": batch_ms, "graph_nodes": info["graph_nodes"],
                     "kernel_launches_per_batch": info["launches_per_run"],
                     "device_bytes": info["device_bytes"],
                     "serial_ms": serial_ms, "batch_over_serial": batch_ms / serial_ms,
                     "serial_sites_per_s": sites / (serial_ms * 1e-3),
                     "max_rel_diff_W_vs_serial": worst,
                     "serial_ms_by_shape": {k: {"jobs": n, "ms": round(t, 3)}
                                            for k, (n, t) in sorted(by_shape.items())},
                     "autotune_report": report.splitlines()}
    return {"workload": "64 uneven configurations, one CUDA graph per run", "jobs": 64,
            "sites": sites, "total_ape_steps": sum(j.ape_steps for j in jobs),
            "value": out["mixed"]["sites_per_s"], "unit": "sites/s", "forms": out}


def bench_serving(duration_s: float, rate: float = 200.0, slots: int = 8):
    """Poisson stream of smear-and-measure requests: V log-uniform in
    [8^4, 32^4], L = round(V^(1/4)), SU(2)/SU(3) 50/50, APE 5..40, R,T up to
    L/2, mixed precision, admission by free device memory. Reports the
    submit-to-result latency percentiles and the completed sites/s, and the
    largest W error of a sample of requests against the FP64 form run alone."""
    from general_code_b200 import Lattice, generate_config
    from general_code_b200.batch import Job
    from general_code_b200.server import Server
    rng = np.random.default_rng(SEED + 5)
    n = max(1, int(duration_s * rate))
    gaps = rng.exponential(1.0 / rate, n)
    reqs = []
    for _ in range(n):
        v = float(np.exp(rng.uniform(np.log(8 ** 4), np.log(32 ** 4))))
        L = int(min(32, max(8, round(v ** 0.25))))
        nc = int(rng.choice([2, 3]))
        reqs.append(Job(dims=(L, L, L, L), nc=nc, ape_steps=int(rng.integers(5, 41)),
                        r_max=L // 2, t_max=L // 2))
    import torch
    pool, pinned = {}, []
    for j in reqs:
        key = (j.dims[0], j.nc)
        if key not in pool:
            # pinned host memory: the request's upload is an asynchronous DMA
            t = torch.empty((4 * j.sites, 4 if j.nc == 2 else 18), dtype=torch.float64,
                            pin_memory=True)
            pinned.append(t)
            pool[key] = generate_config(j.dims, j.nc, 0.3 if j.nc == 2 else 0.25, SEED,
                                        len(pool), out=t.numpy())
    results = {}
    with Server(slots=slots, precision="mixed") as srv:
        ids = []

        def collect():
            for k, rid in enumerate(ids_ready()):
                results[k] = srv.wait(rid, timeout=600)

        import queue
        import threading
        q = queue.Queue()

        def ids_ready():
            while True:
                item = q.get()
                if item is None:
                    return
                yield item

        t = threading.Thread(target=collect)
        t.start()
        t0 = time.perf_counter()
        next_t = t0
        for k, j in enumerate(reqs):
            next_t += gaps[k]
            dt = next_t - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            rid = srv.submit(j, pool[(j.dims[0], j.nc)])
            ids.append(rid)
            q.put(rid)
        q.put(None)
        t.join()
        wall = time.perf_counter() - t0
        st = srv.stats()
    # accuracy of the served (mixed) results against FP64 alone, on a sample
    sample = sorted(set(int(i) for i in rng.choice(n, min(8, n), replace=False)))
    err = 0.0
    for k in sample:
        j = reqs[k]
        with Lattice(j.dims, j.nc, "fp64") as lat:
            lat.upload(pool[(j.dims[0], j.nc)])
            lat.hyp(*j.hyp_alpha, 1)
            lat.ape(j.ape_alpha, j.ape_steps)
            w = lat.wilson_loop(1, j.r_max, 1, j.t_max)
        err = max(err, float(np.max(np.abs(results[k] - w) / np.abs(w))))
    return {"workload": f"Poisson {rate:g} req/s for {duration_s:g} s, L^4 with L 8..32",
            "requests": n, "completed": st["completed"], "offered_rate": rate,
            "wall_s": wall, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "mean_ms": st["mean_ms"], "queue_p50_ms": st["queue_p50_ms"],
            "queue_p99_ms": st["queue_p99_ms"], "run_p50_ms": st["run_p50_ms"],
            "run_p99_ms": st["run_p99_ms"], "value": st["sites_per_s"], "unit": "sites/s",
            "slots": slots, "peak_inflight": st["peak_inflight"],
            "peak_device_bytes": st["peak_bytes"], "mixed_vs_fp64_max_rel_err_W": err,
            "checked_requests": len(sample)}


OBS_DIMS_GPU, OBS_DIMS_CPU = (24, 24, 24, 24), (12, 12, 12, 12)


def _observable_calls(rt=6):
    """(name, GPU call on a Lattice (second lattice for GEVP), reference CPU
    call on (nc, dims, links, links2)) for each observable of the widened
    rows, all with the same ranges (R, T <= 6, D_max = 6) so that per-site
    rates compare."""
    return [
        ("wilson_loop_adjoint R,T<=6",
         lambda a, b: a.wilson_loop_adjoint(1, rt, 1, rt),
         lambda r, nc, d, x, y: r.wilson_adjoint(nc, d, x.copy(), 1, rt, 1, rt)),
        ("wilson_gevp R,T<=6",
         lambda a, b: a.wilson_gevp(b, 1, rt, 1, rt),
         lambda r, nc, d, x, y: r.wilson_gevp(nc, d, x, y, 1, rt, 1, rt)),
        ("polyakov_loop",
         lambda a, b: a.polyakov_loop(),
         lambda r, nc, d, x, y: r.polyakov_loop(nc, d, x)),
        ("polyakov_correlator singlet D<=6",
         lambda a, b: a.polyakov_correlator(rt, True),
         lambda r, nc, d, x, y: r.polyakov_correlator(nc, d, x, rt, True)),
        ("plaket_time",
         lambda a, b: a.plaquette_time(),
         lambda r, nc, d, x, y: r.plaquette_time(nc, d, x)),
        ("wilson_offaxis_result r<=6, T<=6",
         lambda a, b: a.wilson_offaxis_result(1.0, float(rt), 1, rt),
         lambda r, nc, d, x, y: r.wilson_offaxis_result(nc, d, x, 1.0, float(rt), 1, rt)),
        ("smearing_APE_2d x10",
         lambda a, b: a.ape_plane(0, 1, 0.5, 10),
         lambda r, nc, d, x, y: r.ape_plane(nc, d, x.copy(), 0, 1, 0.5, 10)),
        ("wilson_spatial_3d R,T<=6, APE2d 1..10/3",
         lambda a, b: a.wilson_spatial_3d(1, rt, 1, rt, 0.5, 1, 10, 3),
         lambda r, nc, d, x, y: r.wilson_spatial_3d(nc, d, x.copy(), 1, rt, 1, rt, 0.5, 1, 10,
                                                    3)),
    ]


def cpu_reference_observables():
    """The reference's own CPU implementation of each observable (oracle/_ref,
    the reference's flags, all host threads) on a bounded sample: SU(3) 12^4.
    Returns {name: sites/s} and the thread count, or None without the
    library."""
    sys.path.insert(0, str(ROOT))
    from oracle import py_oracle
    if not py_oracle.ref_available("timed"):
        return None, 0
    from general_code_b200 import generate_config
    ref = py_oracle.ref("timed")
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    d = OBS_DIMS_CPU
    x = generate_config(d, 3, 0.25, SEED, 0)
    y = generate_config(d, 3, 0.25, SEED, 1)
    V = int(np.prod(d))
    out = {}
    for name, _, cpu in _observable_calls():
        t0 = time.perf_counter()
        cpu(ref, 3, d, x, y)
        out[name] = V / (time.perf_counter() - t0)
    return out, cores


def bench_observables(steps: int):
    """The observables beside the on-axis loops, on the GPU: SU(3) 24^4 in both
    forms, each call timed with CUDA events on the lattice's stream (mean of
    `steps` calls after one untimed), next to the reference's CPU path on a
    bounded SU(3) 12^4 sample with the same ranges. Also the configuration
    reader on a 24^4 lexicographical file and the t-slab decomposition
    emulated on one GPU (all slabs one after another) against one lattice."""
    import tempfile

    import torch
    from general_code_b200 import Lattice, generate_config
    from general_code_b200.tslab import emulate
    d = OBS_DIMS_GPU
    V = int(np.prod(d))
    x = generate_config(d, 3, 0.25, SEED, 0)
    y = generate_config(d, 3, 0.25, SEED, 1)
    cpu, cores = cpu_reference_observables()
    res = {}
    for form in ("mixed", "fp64"):
        s = torch.cuda.Stream()
        with Lattice(d, 3, form) as a, Lattice(d, 3, form) as b:
            for lat in (a, b):
                lat.set_stream(s.cuda_stream)
            a.upload(x)
            b.upload(y)
            for name, gpu, _ in _observable_calls():
                gpu(a, b)
                a.upload(x)
                ms = []
                for _ in range(max(1, steps)):
                    e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
                    e0.record(s)
                    gpu(a, b)
                    e1.record(s)
                    s.synchronize()
                    ms.append(e0.elapsed_time(e1))
                    a.upload(x)  # the smearing calls change the links
                m = sum(ms) / len(ms)
                r = res.setdefault(name, {})
                r[f"{form}_ms"] = m
                r[f"{form}_sites_per_s"] = V / (m * 1e-3)
    for name in res:
        if cpu:
            res[name]["reference_cpu_sites_per_s"] = cpu[name]
            res[name]["fp64_vs_reference"] = res[name]["fp64_sites_per_s"] / cpu[name]
    # configuration reader: 24^4 SU(3) lexicographical doubles, file -> device
    rd = {}
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "conf.lex")
        with Lattice(d, 3, "fp64") as a:
            a.upload(x)
            a.write(path)
            nbytes = os.path.getsize(path)
            for form in ("fp64", "mixed"):
                with Lattice(d, 3, form) as c:
                    c.read(path)
                    c.synchronize()
                    t0 = time.perf_counter()
                    for _ in range(max(1, steps)):
                        c.read(path)
                        c.synchronize()
                    dt = (time.perf_counter() - t0) / max(1, steps)
                rd[form] = {"ms": dt * 1e3, "file_GB_per_s": nbytes / dt / 1e9}
        if cpu is not None:
            from oracle import py_oracle
            ref = py_oracle.ref("timed")
            t0 = time.perf_counter()
            ref.read(3, d, path, "lexicographical", 0, "double", False)
            dt = time.perf_counter() - t0
            rd["reference_cpu"] = {"ms": dt * 1e3, "file_GB_per_s": nbytes / dt / 1e9}
    rd["file_bytes"] = nbytes
    # t-slab decomposition emulated on one GPU: the headline job as 1 and 2 slabs
    job = dict(precision="mixed", hyp=(1.0, 0.75, 0.6), hyp_steps=1, ape_alpha=0.5,
               ape_steps=20, r_min=1, r_max=12, time_min=1, time_max=12)
    ts = {}
    for k in (1, 2):
        emulate(x, d, 3, k, **job)
        t0 = time.perf_counter()
        emulate(x, d, 3, k, **job)
        ts[f"slabs_{k}_ms"] = (time.perf_counter() - t0) * 1e3
    return {"workload": "SU(3) 24^4 on the GPU (both forms), the reference's CPU path on "
                        "SU(3) 12^4 with the same ranges",
            "reference_cpu_threads": cores, "unit": "sites/s", "observables": res,
            "reader_lexicographical_double": rd,
            "tslab_emulated_one_gpu": dict(ts, note="wall time incl. lattice allocation; "
                                                    "slabs run one after another on one GPU")}


def bench_dropin():
    """The apps/smearing job as the reference's app runs it (HYP, APE x20, the
    W table, SU(3) 24^4 FP64; smearing.cpp:228-301), through the C++ drop-in
    overloads (every call uploads and downloads the whole configuration) and
    through the reference's templates on the host cores: both timed by
    oracle/_ref/dropin_check --time, the reference compiled with the drop-in
    header."""
    exe = ROOT / "oracle" / "_ref" / "dropin_check"
    if not exe.exists():
        return {"unavailable": "oracle/_ref/dropin_check not built (needs the reference sources)"}
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    p = subprocess.run([str(exe), "--time", "3", "24", "24", "20", "12", "12"],
                       capture_output=True, text=True, timeout=900, env=env)
    if p.returncode != 0:
        return {"error": (p.stdout + p.stderr)[-500:], "rc": p.returncode}
    d = json.loads(p.stdout.strip().splitlines()[-1])
    V = 24 ** 4
    gpu = sum(d["dropin_s"].values())
    ref = sum(d["reference_s"].values())
    copy_bytes = 2 * d["config_bytes"] * d["calls"]
    return {"workload": "SU(3) 24^4 FP64, HYP + APE x20 + W R,T<=12, the app's call sequence",
            "dropin_s": d["dropin_s"], "reference_s": d["reference_s"],
            "dropin_sites_per_s": V / gpu, "reference_sites_per_s": V / ref,
            "speedup": ref / gpu, "host_device_bytes": copy_bytes,
            "calls": d["calls"], "w_max_rel_diff": d["w_max_rel_diff"],
            "reference_threads": os.cpu_count()}


def run_tslab(args, wl, rank, world, dist):
    """One lattice (the workload's) split into time slabs over the ranks:
    strong scaling. Each step smears and measures from the rank's resident raw
    slices (value) or from the pinned host configuration (e2e), with the
    forward-halo exchange and the all-reduce of the W table inside; CUDA
    events on the current stream, max over ranks. The mixed form."""
    import torch
    from general_code_b200 import generate_config, link_size
    from general_code_b200.lattice import HYP_LAUNCHES_PER_STEP, WILSON_LAUNCHES
    from general_code_b200.tslab import TSlabJob

    nc, dims = wl["nc"], wl["dims"]
    V = int(np.prod(dims))
    host_t = torch.empty((4 * V, link_size(nc)), dtype=torch.float64, pin_memory=True)
    host = host_t.numpy()
    generate_config(dims, nc, wl["eps"], SEED, 0, out=host)  # the same lattice on every rank
    flush_buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    form = "fp64" if args.form == "fp64" else "mixed"

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(job, steps, from_host):
        ms, w = 0.0, None
        for _ in range(steps):
            with torch.cuda.stream(job.stream):
                flush_buf.fill_(1.0)
            e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
            e0.record(job.stream)
            w = job.run(host if from_host else None)
            e1.record(job.stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        return ms, w

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    with TSlabJob(dims, nc, precision=form, hyp=wl["hyp"], hyp_steps=1, ape_alpha=wl["alpha"],
                  ape_steps=wl["ape"], r_min=wl["r"][0], r_max=wl["r"][1],
                  time_min=wl["t"][0], time_max=wl["t"][1]) as job:
        job.load(host)
        timed(job, args.warmup, False)
        barrier()
        ms, w = timed(job, args.steps, False)
        barrier()
        timed(job, args.warmup, True)
        barrier()
        ms_e2e, w_e2e = timed(job, args.steps, True)
        barrier()
        slab = job.plan.bounds[rank][1]
        runs = job.plan.upload_runs(rank)
        w_method = job.meas.wilson_method_used() or "exact"
    h2d = sum(k for _, _, k in runs) * 4 * (V // dims[3]) * link_size(nc) * 8
    assert np.array_equal(w, w_e2e), "resident and end-to-end runs disagree"
    ms, ms_e2e = max_over_ranks(ms), max_over_ranks(ms_e2e)
    if rank == 0:
        print(json.dumps({
            "metric": "smeared+measured sites/s", "value": V * args.steps / (ms * 1e-3),
            "unit": "sites/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if form == "fp64" else "f32/f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "form": form, "lattice": list(dims),
                       "decomposition": f"{world} time slabs (rank 0: {slab} slices)",
                       "l2": "flushed (256 MiB write) before every timed step",
                       "parallelism": f"tslab x{world}"},
            "e2e": {"value": V * args.steps / (ms_e2e * 1e-3), "unit": "sites/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(w.nbytes)},
            # per step: HYP 3 + APE n + W kernels (of the method the slab took);
            # e2e adds a layout conversion per uploaded run of slices
            "gpu_launches": args.steps * (2 * (HYP_LAUNCHES_PER_STEP + wl["ape"]
                                               + WILSON_LAUNCHES[w_method]) + len(runs)),
            "w_method": w_method,
            "roofline": None,
            "note": "the headline run (--decomp replicas) carries the roofline and CPU baseline"}),
            flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_reference(args, wl, rank):
    if rank != 0:
        return 0
    from oracle import py_oracle
    host = py_oracle.generator().generate(wl["dims"], wl["nc"], wl["eps"], SEED, 0)
    value, info = cpu_sample(wl, args.workload, host, steps=args.steps, warmup=args.warmup)
    line = {
        "impl": "reference", "metric": "smeared+measured sites/s", "value": value,
        "unit": "sites/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * info["job_seconds"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "form": "fp64 (the reference's only form)",
        "config": config_dict(args.workload, wl, args.gpus),
        "cpu_baseline": {"value": value, "unit": "sites/s", "cores": info["cores"],
                         "kind": info["kind"], "sample": info["sample"]},
        "phase_seconds": info["phase_seconds"],
        "e2e": {"value": value, "unit": "sites/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


class Runner:
    """Times smear-and-measure jobs on this rank's GPU."""

    def __init__(self, rank, world, dist):
        import torch
        self.torch = torch
        self.rank, self.world, self.dist = rank, world, dist
        self.stream = torch.cuda.Stream()
        self.flush_buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def flush(self, stream=None):
        with self.torch.cuda.stream(stream or self.stream):
            self.flush_buf.fill_(1.0)

    def ev(self, stream=None):
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(stream or self.stream)
        return e

    def barrier(self):
        self.torch.cuda.synchronize()
        if self.dist is not None:
            self.dist.barrier()
        self.torch.cuda.synchronize()

    def max_over_ranks(self, x):
        if self.dist is None:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device="cuda")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def measure(self, wl, host, form, steps, warmup):
        """One form of the job: device-resident steps, serial end-to-end steps,
        then pipelined end-to-end steps (two handles)."""
        torch = self.torch
        from general_code_b200 import Lattice
        nc, dims = wl["nc"], wl["dims"]
        r0, r1 = wl["r"]
        t0, t1 = wl["t"]
        stream = self.stream
        pristine = Lattice(dims, nc, form)
        work = Lattice(dims, nc, form)
        for lat in (pristine, work):
            lat.set_stream(stream.cuda_stream)
        pristine.upload(host)
        pristine.synchronize()

        def device_step(record):
            self.flush()
            e0 = self.ev()
            work.copy_from(pristine)  # the step's input: the unsmeared links
            ec = self.ev()
            work.hyp(*wl["hyp"], 1)
            e1 = self.ev()
            work.ape(wl["alpha"], wl["ape"])
            e2 = self.ev()
            w = work.wilson_loop(r0, r1, t0, t1)
            e3 = self.ev()
            stream.synchronize()
            if record is not None:
                record.append((e0.elapsed_time(e3), ec.elapsed_time(e1), e1.elapsed_time(e2),
                               e2.elapsed_time(e3), e0.elapsed_time(ec)))
            return w

        stream2 = torch.cuda.Stream()
        work2 = Lattice(dims, nc, form)
        work2.set_stream(stream2.cuda_stream)
        pair = ((work, stream), (work2, stream2))

        def e2e_pipelined(k, record):
            # two handles: job i+1's upload (pinned host -> device, on the
            # other handle's stream) is issued before job i's result is read,
            # so the copy engine overlaps job i's kernels; the other handle is
            # idle then (its previous job's result has been read)
            e0 = self.ev()
            stream2.wait_event(e0)
            pair[0][0].upload(host)
            w = None
            for i in range(k):
                lat, s = pair[i % 2]
                self.flush(s)
                lat.hyp(*wl["hyp"], 1)
                lat.ape(wl["alpha"], wl["ape"])
                if i + 1 < k:
                    pair[(i + 1) % 2][0].upload(host)
                w = lat.wilson_loop(r0, r1, t0, t1)
            last = pair[(k - 1) % 2][1]
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record(last)
            last.synchronize()
            if record is not None:
                record.append(e0.elapsed_time(e1))
            return w

        def e2e_step(record):
            self.flush()
            e0 = self.ev()
            work.upload(host)
            work.hyp(*wl["hyp"], 1)
            work.ape(wl["alpha"], wl["ape"])
            w = work.wilson_loop(r0, r1, t0, t1)
            e1 = self.ev()
            stream.synchronize()
            if record is not None:
                record.append(e0.elapsed_time(e1))
            return w

        for _ in range(warmup):
            device_step(None)
        self.barrier()
        rec = []
        for _ in range(steps):
            w = device_step(rec)
        self.barrier()
        for _ in range(warmup):
            e2e_step(None)
        self.barrier()
        rec_e2e = []
        for _ in range(steps):
            w_e2e = e2e_step(rec_e2e)
        self.barrier()
        assert np.array_equal(w, w_e2e), "device and end-to-end runs disagree"
        e2e_pipelined(max(2, warmup), None)
        self.barrier()
        rec_pipe = []
        w_pipe = e2e_pipelined(steps, rec_pipe)
        self.barrier()
        assert np.array_equal(w, w_pipe), "device and pipelined end-to-end runs disagree"
        w_method = work.wilson_method_used()  # (after the timed runs: it synchronises)
        pristine.close()
        work.close()
        work2.close()
        from general_code_b200 import launches_per_job
        per_job = launches_per_job(nc, wl["ape"], w_method=w_method or "exact")
        return {"w": w, "w_method": w_method,
                "total_ms": self.max_over_ranks(sum(r[0] for r in rec)),
                "total_e2e_ms": self.max_over_ranks(sum(rec_pipe)),
                "total_serial_ms": self.max_over_ranks(sum(rec_e2e)),
                "restore_ms": sum(r[4] for r in rec) / steps,
                "hyp_ms": sum(r[1] for r in rec) / steps,
                "ape_ms": sum(r[2] for r in rec) / steps,
                "w_ms": sum(r[3] for r in rec) / steps,
                # our kernels per timed step in the device-resident, serial and
                # pipelined end-to-end runs; the two end-to-end runs add one
                # layout conversion per upload
                "launches": steps * per_job * 3 + 2 * steps}


def summarize(wl, name, form, r, steps, world, peak, peak_kind, fp_peak, traffic):
    """Throughput, phase times and per-kernel-family rooflines of one form."""
    V = int(np.prod(wl["dims"]))
    alg = algorithmic(wl, form, r["w_method"])
    per_launch = {"hyp": r["hyp_ms"], "ape": r["ape_ms"] / wl["ape"], "wilson": r["w_ms"]}
    totals = {"hyp": r["hyp_ms"], "ape": r["ape_ms"], "wilson": r["w_ms"]}
    pipe = "fp64" if form == "fp64" else "fp32"
    kernels = {}
    for k, ms in per_launch.items():
        gbs = alg[k]["bytes"] * V / (ms * 1e-3) / 1e9
        tf = alg[k]["flops"] * V / (ms * 1e-3) / 1e12
        tr = traffic.get(f"{k}:{name}:{form}")
        kernels[k] = {"ms_per_launch": ms, "share_of_step": totals[k] / sum(totals.values()),
                      "alg_bytes_per_launch": alg[k]["bytes"] * V,
                      "hbm_gbs": gbs, "hbm_frac": gbs / peak,
                      "traffic_per_launch": (tr["dram_bytes_per_site"] * V if tr else None),
                      "fp_flops_per_launch": alg[k]["flops"] * V, "fp_tflops": tf,
                      "fp_pipe": pipe, "fp_frac": tf / fp_peak[pipe]}
        if k == "wilson":
            kernels[k]["method"] = alg[k]["method"]
    dom = max(totals, key=totals.get)
    kd = kernels[dom]
    return {
        "value": world * V * steps / (r["total_ms"] * 1e-3),
        "e2e_value": world * V * steps / (r["total_e2e_ms"] * 1e-3),
        "e2e_serial": world * V * steps / (r["total_serial_ms"] * 1e-3),
        "ms_per_step": r["total_ms"] / steps,
        "phases_ms": {"restore": r["restore_ms"], "hyp": r["hyp_ms"], "ape_total": r["ape_ms"],
                      "ape_per_step": r["ape_ms"] / wl["ape"], "wilson": r["w_ms"]},
        "kernels": kernels,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": kd["hbm_gbs"], "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": kd["hbm_frac"],
                     "traffic": kd["traffic_per_launch"],
                     "alg_bytes_per_launch": kd["alg_bytes_per_launch"],
                     # the SU(3) kernels are bound by the vector FP pipes, not
                     # HBM: algorithmic FLOPs over the pipe the form computes
                     # in, against that pipe's FMA throughput measured in this run
                     "compute": {"pipe": pipe, "achieved_tflops": kd["fp_tflops"],
                                 "peak_tflops": fp_peak[pipe],
                                 "peak_kind": "measured in-run (gc_fma_peak)",
                                 "frac": kd["fp_frac"]}},
    }


def run_workload(runner, name, wl, forms, steps, warmup, peak, peak_kind, fp_peak, traffic):
    """Both forms of one workload; returns (per-form summaries, results)."""
    import torch
    from general_code_b200 import generate_config, link_size
    V = int(np.prod(wl["dims"]))
    host_t = torch.empty((4 * V, link_size(wl["nc"])), dtype=torch.float64, pin_memory=True)
    host = host_t.numpy()
    generate_config(wl["dims"], wl["nc"], wl["eps"], SEED, runner.rank, out=host)
    results = {f: runner.measure(wl, host, f, steps, warmup) for f in forms}
    sums = {f: summarize(wl, name, f, results[f], steps, runner.world, peak, peak_kind,
                         fp_peak, traffic) for f in forms}
    return sums, results, host


def form_errors(results):
    wm, wd = results["mixed"]["w"], results["fp64"]["w"]
    rel = np.abs(wm - wd) / np.abs(wd)
    return {"max_rel_err_W": float(np.max(rel)), "tolerance": 1e-6,
            # per W(R,T): rows T = t_min.., columns R = r_min..
            "rel_err_W": [[float(f"{v:.3g}") for v in row] for row in rel]}


def bench_su2(runner, steps, warmup, peak, peak_kind, fp_peak, traffic, cpu=True):
    """SU(2) 16^4 (the reference's CPU-sized case) and SU(2) 48^4, both forms,
    device-resident and end to end, with per-kernel HBM and FP fractions and
    the reference's CPU path on a bounded sample."""
    out = {}
    for name in ("su2_16", "su2_48"):
        wl = WORKLOADS[name]
        sums, results, host = run_workload(runner, name, wl, ["mixed", "fp64"], steps, warmup,
                                           peak, peak_kind, fp_peak, traffic)
        sec = {"config": config_dict(name, wl, 1),
               "value": sums["mixed"]["value"], "unit": "sites/s",
               "forms": {f: {"value": v["value"], "e2e": v["e2e_value"],
                             "e2e_serial": v["e2e_serial"], "ms_per_step": v["ms_per_step"],
                             "phases_ms": v["phases_ms"], "kernels": v["kernels"]}
                         for f, v in sums.items()},
               "mixed_vs_fp64_max_rel_err_W": form_errors(results)["max_rel_err_W"],
               "h2d_bytes_per_step": int(host.nbytes)}
        if cpu:
            v, info = cpu_sample(wl, name, host, steps=3)
            sec["cpu_baseline"] = {"value": v, "unit": "sites/s", "cores": info["cores"],
                                   "kind": info["kind"], "sample": info["sample"]}
        out[name] = sec
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["both", "fp64", "mixed"], default="both")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sections", default="su2,batch,serving,observables,dropin",
                    help="extra single-GPU measurements: su2, batch, serving, observables, "
                         "dropin (comma list, or none)")
    ap.add_argument("--serving-seconds", type=float, default=10.0)
    ap.add_argument("--decomp", choices=["replicas", "tslab"], default="replicas",
                    help="replicas: one configuration per rank (weak scaling); tslab: one "
                         "lattice split into time slabs over the ranks (strong scaling)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    wl = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, wl, rank)

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))

    if args.decomp == "tslab":
        return run_tslab(args, wl, rank, world, dist)

    from general_code_b200 import fma_peak
    nc, dims = wl["nc"], wl["dims"]
    runner = Runner(rank, world, dist)
    peak, peak_kind = load_peaks()
    traffic = load_traffic()
    fp_peak = {"fp32": fma_peak("mixed"), "fp64": fma_peak("fp64")}
    forms = ["mixed", "fp64"] if args.form == "both" else [args.form]
    sampler = ClockSampler(local_rank)
    sampler.start()
    sums, results, host = run_workload(runner, args.workload, wl, forms, args.steps,
                                       args.warmup, peak, peak_kind, fp_peak, traffic)
    clocks = sampler.stop()

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    head = forms[0]
    hs = sums[head]
    line = {
        "metric": "smeared+measured sites/s", "value": hs["value"], "unit": "sites/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": hs["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32/f64",
        "data": "synthetic", "form": head,
        "config": config_dict(args.workload, wl, world),
        "phases_ms": hs["phases_ms"],
        "roofline": hs["roofline"],
        "kernels": hs["kernels"],
        "e2e": {"value": hs["e2e_value"], "unit": "sites/s",
                "h2d_bytes_per_step": int(host.nbytes),
                "d2h_bytes_per_step": int(results[head]["w"].nbytes),
                "mode": "two handles on two streams: job i+1's upload overlaps job i",
                "serial_value": hs["e2e_serial"]},
        "gpu_launches": sum(results[f]["launches"] for f in forms),
        "clocks": clocks,
        "fp_peak_tflops_measured": fp_peak,
    }
    if len(forms) > 1:
        line["mixed_vs_fp64"] = form_errors(results)
        line["forms"] = {f: {"value": sums[f]["value"], "e2e": sums[f]["e2e_value"],
                             "e2e_serial": sums[f]["e2e_serial"],
                             "ms_per_step": sums[f]["ms_per_step"],
                             "phases_ms": sums[f]["phases_ms"],
                             "roofline": sums[f]["roofline"],
                             "kernels": sums[f]["kernels"]} for f in forms}
    sections = [x for x in args.sections.split(",") if x and x != "none"]
    if world == 1 and "su2" in sections:
        line["su2"] = bench_su2(runner, min(args.steps, 10), args.warmup, peak, peak_kind,
                                fp_peak, traffic, cpu=not args.no_cpu_baseline)
    if world == 1 and "batch" in sections:
        line["batch"] = bench_batch(args.steps)
    if world == 1 and "serving" in sections:
        line["serving"] = bench_serving(args.serving_seconds)
    if world == 1 and "observables" in sections:
        line["observables"] = bench_observables(min(args.steps, 5))
    if world == 1 and "dropin" in sections:
        line["dropin"] = bench_dropin()
    if world == 1 and not args.no_cpu_baseline:
        v, info = cpu_sample(wl, args.workload, host, steps=3)
        line["cpu_baseline"] = {"value": v, "unit": "sites/s", "cores": info["cores"],
                                "kind": info["kind"], "sample": info["sample"]}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0

if __name__ == "__main__":
    sys.exit(main())
