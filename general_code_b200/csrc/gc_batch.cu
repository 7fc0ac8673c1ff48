// Batches of independent smear-and-measure jobs of uneven sizes.
//
// A batch is planned once (gc_batch_create): every job gets its device fields
// (its input, two working link sets, the HYP decorated links), its W partial
// sums and result table, all in a few large allocations. The schedule of a
// run is static:
//   restore inputs -> HYP (per-job step counts, in rounds) -> APE rounds
//   (round k covers the jobs with more than k steps) -> W -> reductions ->
//   one copy of all W tables to pinned host memory,
// with SU(2) and SU(3) jobs as two classes on two streams that run
// concurrently. Each smearing phase is ONE launch over all jobs of a class:
// blocks find their job in a per-launch job table (tables built on the host
// at plan time and kept in device memory). The W phase runs each job's loops
// in the temporal gauge where that applies (T <= Lt/2, the job has HYP
// scratch to hold the transformed links): the job's unitarity check, gauge
// lines and transformed links, then both W kernels gated on the check (the
// exact product computes only when the check failed) and the reduction, the
// jobs spread over kWStreams side streams per class so that the small jobs'
// launches overlap; other jobs share multi-job exact W launches. The first
// gc_batch_run captures the whole schedule into a CUDA graph; every run after
// that is one graph launch.
//
// gc_batch_autotune times the candidate W block shapes (threads per column
// x columns per block) for each distinct (time extent, group, R/T range) in
// the batch on this GPU and keeps the fastest; results are bitwise
// independent of the shape only up to the summation order, so the chosen
// shape is fixed for the life of the batch.
#include "../../include/gc_lattice.h"
#include "gc_internal.cuh"
#include "gc_kernels.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace gc {
int record_error(int code, const std::string &msg);
const std::string &last_launch_error();
int generate_host(const int dims[4], int nc, double eps, unsigned seed, unsigned cfg,
                  int gauge, double *out);
} // namespace gc

namespace {

using namespace gc;

#define GC_DISPATCH_NC(NC, PREC, FN, ...)                                      \
  ((NC) == 3 ? ((PREC) == GC_PREC_FP64 ? FN<StoreF64SU3, double>(__VA_ARGS__)  \
                                       : FN<StoreF32SU3, float>(__VA_ARGS__))  \
             : ((PREC) == GC_PREC_FP64 ? FN<StoreF64SU2, double>(__VA_ARGS__)  \
                                       : FN<StoreF32SU2, float>(__VA_ARGS__)))

constexpr int kBlock = 128; // smearing kernels' block size
constexpr int kWStreams = 8; // side streams of each class's per-job W launches

size_t link_bytes(int nc, int prec) {
  if (nc == 3)
    return prec == GC_PREC_FP64 ? 144 : 48;
  return prec == GC_PREC_FP64 ? 32 : 16;
}
size_t align256(size_t b) { return (b + 255) / 256 * 256; }

struct CopyJob {
  const uint4 *src;
  uint4 *dst;
  long long n16; // 16-byte units
  int block_start;
};

__global__ void copy_batch_kernel(const CopyJob *__restrict__ jobs, int njobs) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].block_start <= (int)blockIdx.x)
      lo = mid;
    else
      hi = mid - 1;
  }
  const CopyJob &j = jobs[lo];
  const long long base = (long long)(blockIdx.x - j.block_start) * blockDim.x * 4;
  for (int k = 0; k < 4; k++) {
    const long long i = base + k * blockDim.x + threadIdx.x;
    if (i < j.n16)
      j.dst[i] = j.src[i];
  }
}

struct JobState {
  gc_job desc;
  Geom g;
  size_t field_bytes;
  size_t hyp_bytes; // one HYP decorated-link field
  void *input[4];  // the job's configuration (kept between runs)
  void *setA[4], *setB[4];
  void *hyp[15];
  double *partials = nullptr;
  double *out_dev = nullptr;
  int nr = 0, nt = 0;
  int rows = 0, cols = 0; // W block shape
  int w_blocks = 0;
  bool gauge = false;     // W in the temporal gauge (per-job launches)
  int gunits = 0;         // its block shape (column units; 0 = default)
  Fields4 wU{};           // the job's links when its W runs
  int *flag = nullptr;    // the job's unitarity flag (device)
  void *GA = nullptr, *GB = nullptr; // gauge lines (in the HYP scratch)
  Fields4 UA{}, UB{};     // transformed spatial links (in the HYP scratch)
  bool has_input = false;
};

// One launch of the schedule.
struct Launch {
  enum Kind { COPY, HYP, APE, W, REDUCE, WAUTO } kind;
  int cls;            // 0: SU(2), 1: SU(3)
  size_t table_off;   // byte offset of the job table in the descriptor arena
  int njobs;
  int blocks[3];
  size_t smem;
};

} // namespace

struct gc_batch {
  int prec = 0;
  std::vector<JobState> jobs;
  void *arena = nullptr;       // job fields
  double *partials = nullptr;  // all W partials
  double *outs = nullptr;      // all W tables (device)
  double *outs_host = nullptr; // pinned mirror
  size_t outs_count = 0;
  double *staging = nullptr;   // host-layout upload buffer (largest job)
  size_t staging_bytes = 0;
  unsigned char *desc = nullptr; // job tables
  size_t desc_bytes = 0;
  std::vector<unsigned char> desc_host;
  std::vector<Launch> launches;
  bool planned = false;        // tables + launches built
  cudaStream_t main = nullptr, side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaStream_t wstream[2][kWStreams] = {}; // per class: per-job W launches
  cudaEvent_t wfork[2] = {}, wjoin[2][kWStreams] = {};
  int *status = nullptr;       // device: [0] a multi-job W launch could not run a job
  int *status_host = nullptr;  // pinned mirror, copied with the results
  int *flags = nullptr;        // device: one unitarity flag per job
  cudaEvent_t done = nullptr;  // recorded after each run's result copy
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_nodes = 0;
  long long device_bytes = 0;
  std::string tune_report; // gc_batch_autotune's measurements
  std::string err;
  std::mutex mu;
};

namespace {

int bfail(gc_batch *b, int code, const std::string &msg) {
  if (b)
    b->err = msg;
  return record_error(code, msg);
}

int cfail(gc_batch *b, const char *what, cudaError_t e) {
  return bfail(b, e == cudaErrorMemoryAllocation ? GC_ERR_NOMEM : GC_ERR_CUDA,
               std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T> size_t push_table(std::vector<unsigned char> &arena, const std::vector<T> &v) {
  size_t off = align256(arena.size());
  arena.resize(off + v.size() * sizeof(T));
  std::memcpy(arena.data() + off, v.data(), v.size() * sizeof(T));
  return off;
}

// Default W block shape of a job (the plan the single-lattice path uses).
void default_shape(JobState &j, int ct_bytes) {
  WilsonPlan p = wilson_plan(j.g, j.nr, j.nt, j.desc.nc, ct_bytes);
  j.rows = p.rows;
  j.cols = p.cols_per_block;
  j.w_blocks = p.blocks;
}

// Builds the job tables and the launch list for the current shapes.
int build_schedule(gc_batch *b) {
  std::vector<unsigned char> &arena = b->desc_host;
  arena.clear();
  b->launches.clear();
  const int prec = b->prec;
  for (int cls = 0; cls < 2; cls++) {
    const int nc = cls == 0 ? 2 : 3;
    std::vector<int> ids;
    for (int i = 0; i < (int)b->jobs.size(); i++)
      if (b->jobs[i].desc.nc == nc)
        ids.push_back(i);
    if (ids.empty())
      continue;
    // current link pointers of every job as the schedule advances
    std::map<int, Fields4> cur, alt;
    for (int i : ids) {
      Fields4 a, bb;
      for (int d = 0; d < 4; d++) {
        a.f[d] = b->jobs[i].setA[d];
        bb.f[d] = b->jobs[i].setB[d];
      }
      cur[i] = a;
      alt[i] = bb;
    }
    // restore the inputs into set A
    {
      std::vector<CopyJob> t;
      int blocks = 0;
      for (int i : ids)
        for (int d = 0; d < 4; d++) {
          CopyJob c;
          c.src = (const uint4 *)b->jobs[i].input[d];
          c.dst = (uint4 *)b->jobs[i].setA[d];
          c.n16 = (long long)(link_bytes(nc, prec) * b->jobs[i].g.V) / 16;
          c.block_start = blocks;
          blocks += (int)((c.n16 + 4 * 256 - 1) / (4 * 256));
          t.push_back(c);
        }
      Launch L{Launch::COPY, cls, push_table(arena, t), (int)t.size(), {blocks, 0, 0}, 0};
      b->launches.push_back(L);
    }
    // HYP rounds
    int max_hyp = 0;
    for (int i : ids)
      max_hyp = std::max(max_hyp, b->jobs[i].desc.hyp_steps);
    for (int k = 0; k < max_hyp; k++) {
      std::vector<HypJob> t;
      int b1 = 0, b2 = 0, b3 = 0;
      for (int i : ids) {
        const JobState &j = b->jobs[i];
        if (j.desc.hyp_steps <= k)
          continue;
        HypJob h;
        h.g = j.g;
        h.U = cur[i];
        for (int f = 0; f < 9; f++)
          h.l1.f[f] = j.hyp[f];
        for (int f = 0; f < 6; f++)
          h.l2.f[f] = j.hyp[9 + f];
        h.out_t = alt[i].f[3];
        h.a1 = j.desc.hyp_alpha[0];
        h.a2 = j.desc.hyp_alpha[1];
        h.a3 = j.desc.hyp_alpha[2];
        const int nb = (j.g.V + kBlock - 1) / kBlock;
        h.start1 = b1;
        h.start2 = b2;
        h.start3 = b3;
        b1 += 9 * nb;
        b2 += 6 * nb;
        b3 += nb;
        t.push_back(h);
        std::swap(cur[i].f[3], alt[i].f[3]);
      }
      if (!t.empty()) {
        Launch L{Launch::HYP, cls, push_table(arena, t), (int)t.size(), {b1, b2, b3}, 0};
        b->launches.push_back(L);
      }
    }
    // APE rounds
    int max_ape = 0;
    for (int i : ids)
      max_ape = std::max(max_ape, b->jobs[i].desc.ape_steps);
    for (int k = 0; k < max_ape; k++) {
      std::vector<ApeJob> t;
      int blocks = 0;
      for (int i : ids) {
        const JobState &j = b->jobs[i];
        if (j.desc.ape_steps <= k)
          continue;
        ApeJob a;
        a.g = j.g;
        a.in = cur[i];
        a.out = cur[i];
        for (int d = 0; d < 3; d++)
          a.out.f[d] = alt[i].f[d];
        a.alpha = j.desc.ape_alpha;
        a.block_start = blocks;
        // (one thread per site and link for SU(3), per site for SU(2): see
        // ape_items in gc_smear.cu)
        blocks += (nc == 2 ? 1 : 3) * ((j.g.V + kBlock - 1) / kBlock);
        t.push_back(a);
        for (int d = 0; d < 3; d++)
          std::swap(cur[i].f[d], alt[i].f[d]);
      }
      if (!t.empty()) {
        Launch L{Launch::APE, cls, push_table(arena, t), (int)t.size(), {blocks, 0, 0}, 0};
        b->launches.push_back(L);
      }
    }
    // W and the reductions. Jobs are launched in occupancy classes (threads
    // per block, blocks that fit on an SM by shared memory): a launch runs at
    // the widest shape and largest shared memory of its jobs, and one launch
    // over all jobs would hold every block to the occupancy of the largest
    // one (a 24^3x48 job's ~93 KB per block halves the resident blocks of
    // every other job's W). A block's work depends only on its own job's
    // shape, so the results do not depend on the grouping.
    {
      const int ct = prec == GC_PREC_FP64 ? 8 : 4;
      std::map<std::pair<int, int>, std::vector<int>> classes; // (threads, blocks/SM) -> jobs
      // per-job temporal-gauge W, largest lattices first
      std::vector<int> gids;
      for (int i : ids)
        if (b->jobs[i].gauge) {
          b->jobs[i].wU = cur[i];
          gids.push_back(i);
        }
      std::stable_sort(gids.begin(), gids.end(),
                       [&](int x, int y) { return b->jobs[x].g.V > b->jobs[y].g.V; });
      for (int i : gids) {
        Launch L{Launch::WAUTO, cls, 0, i, {0, 0, 0}, 0};
        b->launches.push_back(L);
      }
      for (int i : ids) {
        JobState &j = b->jobs[i];
        if (j.nr <= 0 || j.gauge)
          continue;
        WJob w;
        w.g = j.g;
        w.rmin = j.desc.r_min;
        w.rmax = j.desc.r_max;
        w.tmin = j.desc.time_min;
        w.tmax = j.desc.time_max;
        w.cols = j.cols;
        w.rows = j.rows;
        const int th = wilson_threads(j.cols, j.rows, wilson_lanes(nc, ct));
        const size_t sm = wilson_job_smem(w, nc, ct, th);
        const int per_sm = (int)std::max<size_t>(1, (227u * 1024u) / std::max<size_t>(sm, 1));
        classes[{th, std::min(per_sm, 2048 / th)}].push_back(i);
      }
      std::vector<RJob> r;
      int entries = 0;
      for (const auto &kv : classes) {
        std::vector<WJob> t;
        int blocks = 0, threads = 32;
        size_t smem = 0;
        for (int i : kv.second) {
          JobState &j = b->jobs[i];
          WJob w;
          w.g = j.g;
          w.U = cur[i];
          w.rmin = j.desc.r_min;
          w.rmax = j.desc.r_max;
          w.tmin = j.desc.time_min;
          w.tmax = j.desc.time_max;
          w.cols = j.cols;
          w.rows = j.rows;
          w.partials = j.partials;
          w.status = b->status;
          w.block_start = blocks;
          w.blocks = j.w_blocks;
          blocks += j.w_blocks;
          threads = std::max(threads, wilson_threads(j.cols, j.rows, wilson_lanes(nc, ct)));
          t.push_back(w);
          RJob q;
          q.partials = j.partials;
          q.nblocks = j.w_blocks;
          q.nr = j.nr;
          q.nt = j.nt;
          q.scale = wilson_scale(j.g.V, j.desc.nc, false);
          q.out = j.out_dev;
          q.entry_start = entries;
          entries += j.nr * j.nt;
          r.push_back(q);
        }
        for (const WJob &w : t)
          smem = std::max(smem, wilson_job_smem(w, nc, ct, threads));
        // blocks[1]: threads per block (the widest job shape of the launch)
        Launch L{Launch::W, cls, push_table(arena, t), (int)t.size(), {blocks, threads, 0}, smem};
        b->launches.push_back(L);
      }
      if (!r.empty()) {
        Launch R{Launch::REDUCE, cls, push_table(arena, r), (int)r.size(), {entries, 0, 0}, 0};
        b->launches.push_back(R);
      }
    }
  }
  // upload the tables
  if (arena.size() > b->desc_bytes) {
    if (b->desc)
      cudaFree(b->desc);
    b->desc = nullptr;
    cudaError_t e = cudaMalloc(&b->desc, arena.size());
    if (e != cudaSuccess)
      return cfail(b, "cudaMalloc(batch job tables)", e);
    b->desc_bytes = arena.size();
  }
  cudaError_t e = cudaMemcpy(b->desc, arena.data(), arena.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess)
    return cfail(b, "cudaMemcpy(batch job tables)", e);
  b->planned = true;
  return GC_OK;
}

// The per-job gauge-form W launches of a class, spread over the class's
// side streams (forked from and joined back into s).
template <class Store, class CT>
int enqueue_wauto(gc_batch *b, int cls, const std::vector<int> &jobs, cudaStream_t s) {
  if (jobs.empty())
    return GC_OK;
  cudaEventRecord(b->wfork[cls], s);
  const int ns = std::min<int>(kWStreams, (int)jobs.size());
  for (int k = 0; k < ns; k++)
    cudaStreamWaitEvent(b->wstream[cls][k], b->wfork[cls], 0);
  for (size_t m = 0; m < jobs.size(); m++) {
    JobState &j = b->jobs[jobs[m]];
    cudaStream_t ws = b->wstream[cls][m % ns];
    int rc = launch_wilson_gauge_prep<Store, CT>(j.g, j.wU, j.GA, j.GB, j.UA, j.UB, j.flag, ws);
    if (rc)
      return rc;
    rc = launch_wilson_auto<Store, CT>(j.g, j.wU, j.UA, j.UB, j.desc.r_min, j.desc.r_max,
                                       j.desc.time_min, j.desc.time_max, false, j.flag,
                                       j.partials, j.out_dev, ws, j.gunits);
    if (rc)
      return rc;
  }
  for (int k = 0; k < ns; k++) {
    cudaEventRecord(b->wjoin[cls][k], b->wstream[cls][k]);
    cudaStreamWaitEvent(s, b->wjoin[cls][k], 0);
  }
  return GC_OK;
}

template <class Store, class CT>
int enqueue_class(gc_batch *b, int cls, cudaStream_t s) {
  std::vector<int> wauto;
  for (const Launch &L : b->launches)
    if (L.cls == cls && L.kind == Launch::WAUTO)
      wauto.push_back(L.njobs);
  bool wauto_done = false;
  for (const Launch &L : b->launches) {
    if (L.cls != cls)
      continue;
    const unsigned char *tab = b->desc + L.table_off;
    int rc = GC_OK;
    switch (L.kind) {
    case Launch::WAUTO:
      if (!wauto_done)
        rc = enqueue_wauto<Store, CT>(b, cls, wauto, s);
      wauto_done = true;
      break;
    case Launch::COPY:
      copy_batch_kernel<<<L.blocks[0], 256, 0, s>>>((const CopyJob *)tab, L.njobs);
      rc = launch_check("copy_batch_kernel");
      break;
    case Launch::HYP:
      rc = launch_hyp_batch<Store, CT>((const HypJob *)tab, L.njobs, L.blocks, s);
      break;
    case Launch::APE:
      rc = launch_ape_batch<Store, CT>((const ApeJob *)tab, L.njobs, L.blocks[0], s);
      break;
    case Launch::W:
      rc = launch_wilson_batch<Store, CT>((const WJob *)tab, L.njobs, L.blocks[0], L.blocks[1],
                                          L.smem, s);
      break;
    case Launch::REDUCE:
      rc = launch_reduce_batch((const RJob *)tab, L.njobs, L.blocks[0], s);
      break;
    }
    if (rc)
      return rc;
  }
  return GC_OK;
}

int enqueue_class_any(gc_batch *b, int cls, cudaStream_t s) {
  if (cls == 0)
    return b->prec == GC_PREC_FP64 ? enqueue_class<StoreF64SU2, double>(b, 0, s)
                                   : enqueue_class<StoreF32SU2, float>(b, 0, s);
  return b->prec == GC_PREC_FP64 ? enqueue_class<StoreF64SU3, double>(b, 1, s)
                                 : enqueue_class<StoreF32SU3, float>(b, 1, s);
}

// The whole run on `s`: SU(3) jobs on s, SU(2) jobs on the side stream,
// joined before the result copy.
int enqueue_run(gc_batch *b, cudaStream_t s) {
  cudaMemsetAsync(b->status, 0, sizeof(int), s);
  cudaEventRecord(b->fork, s);
  cudaStreamWaitEvent(b->side, b->fork, 0);
  int rc = enqueue_class_any(b, 1, s);
  if (rc)
    return bfail(b, rc, last_launch_error());
  rc = enqueue_class_any(b, 0, b->side);
  if (rc)
    return bfail(b, rc, last_launch_error());
  cudaEventRecord(b->join, b->side);
  cudaStreamWaitEvent(s, b->join, 0);
  cudaError_t e = cudaMemcpyAsync(b->outs_host, b->outs, b->outs_count * sizeof(double),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->status_host, b->status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess)
    return cfail(b, "cudaMemcpyAsync(batch results)", e);
  return GC_OK;
}

void free_graph(gc_batch *b) {
  if (b->exec)
    cudaGraphExecDestroy(b->exec);
  if (b->graph)
    cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graph_nodes = 0;
}

template <class Store, class CT>
int time_shape(JobState &j, int rows, int cols, double *scratch, cudaStream_t s,
               float *ms) {
  const int ct = sizeof(CT);
  WilsonPlan p = wilson_plan_shape(j.g, j.nr, j.nt, j.desc.nc, ct, rows, cols);
  if (!p.fits)
    return GC_ERR_ARG;
  Fields4 U;
  for (int d = 0; d < 4; d++)
    U.f[d] = j.input[d];
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = launch_wilson_plan<Store, CT>(j.g, U, j.desc.r_min, j.desc.r_max, j.desc.time_min,
                                         j.desc.time_max, p, scratch, nullptr, s);
  float best = 1e30f;
  for (int rep = 0; rep < 3 && rc == GC_OK; rep++) {
    cudaEventRecord(e0, s);
    rc = launch_wilson_plan<Store, CT>(j.g, U, j.desc.r_min, j.desc.r_max, j.desc.time_min,
                                       j.desc.time_max, p, scratch, nullptr, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    best = std::min(best, t);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = best;
  return rc;
}

int tune_job(gc_batch *b, JobState &j, double *scratch, cudaStream_t s, int *rows_out,
             int *cols_out) {
  const int Lt = j.g.L[3];
  float best = 1e30f;
  int br = j.rows, bc = j.cols;
  for (int rows = 1; rows <= 64 && rows <= Lt; rows++) {
    if (Lt % rows || rows < std::min(4, Lt))
      continue;
    for (int threads : {128, 256}) {
      const int cols = wilson_lanes(j.desc.nc, b->prec == GC_PREC_FP64 ? 8 : 4) * (threads / rows);
      if (cols < 1)
        continue;
      float ms = 0;
      int rc;
      if (j.desc.nc == 3)
        rc = b->prec == GC_PREC_FP64 ? time_shape<StoreF64SU3, double>(j, rows, cols, scratch, s, &ms)
                                     : time_shape<StoreF32SU3, float>(j, rows, cols, scratch, s, &ms);
      else
        rc = b->prec == GC_PREC_FP64 ? time_shape<StoreF64SU2, double>(j, rows, cols, scratch, s, &ms)
                                     : time_shape<StoreF32SU2, float>(j, rows, cols, scratch, s, &ms);
      if (rc == GC_ERR_ARG) {
        cudaGetLastError();
        continue;
      }
      if (rc)
        return rc;
      char line[192];
      std::snprintf(line, sizeof line, "SU(%d) %dx%dx%dx%d R<=%d T<=%d exact-W rows=%d cols=%d "
                    "%.4f ms\n", j.desc.nc, j.g.L[0], j.g.L[1], j.g.L[2], j.g.L[3],
                    j.desc.r_max, j.desc.time_max, rows, cols, ms);
      b->tune_report += line;
      if (ms < best) {
        best = ms;
        br = rows;
        bc = cols;
      }
    }
  }
  *rows_out = br;
  *cols_out = bc;
  return GC_OK;
}

// W partial sums of a job: its multi-job exact launch's blocks, or for the
// gauge form whichever of the two gated kernels has more blocks.
size_t partials_doubles(const JobState &j) {
  if (j.gauge)
    return wilson_auto_partials_count(j.g, j.nr, j.nt, j.desc.nc, j.gunits);
  return (size_t)j.w_blocks * j.nr * j.nt;
}

int alloc_partials(gc_batch *b) {
  if (b->partials)
    cudaFree(b->partials);
  b->partials = nullptr;
  size_t total = 0;
  for (JobState &j : b->jobs)
    total += align256(partials_doubles(j) * sizeof(double));
  if (total == 0)
    return GC_OK;
  cudaError_t e = cudaMalloc(&b->partials, total);
  if (e != cudaSuccess)
    return cfail(b, "cudaMalloc(batch partials)", e);
  size_t off = 0;
  for (JobState &j : b->jobs) {
    j.partials = (double *)((char *)b->partials + off);
    off += align256(partials_doubles(j) * sizeof(double));
  }
  return GC_OK;
}

int check_job(const gc_job &d, std::string &why) {
  if (d.nc != 2 && d.nc != 3) {
    why = "nc must be 2 or 3";
    return GC_ERR_ARG;
  }
  long long V = 1;
  for (int k = 0; k < 4; k++) {
    if (d.dims[k] < 2) {
      why = "every extent must be >= 2";
      return GC_ERR_ARG;
    }
    V *= d.dims[k];
  }
  if (V >= (1LL << 30)) {
    why = "lattice too large";
    return GC_ERR_ARG;
  }
  if (d.hyp_steps < 0 || d.ape_steps < 0) {
    why = "step counts must be >= 0";
    return GC_ERR_ARG;
  }
  const bool w = !(d.r_max == 0 && d.time_max == 0);
  if (w && (d.r_min < 1 || d.time_min < 1 || d.r_max < d.r_min || d.time_max < d.time_min)) {
    why = "need 1 <= r_min <= r_max and 1 <= time_min <= time_max (or r_max = time_max = 0)";
    return GC_ERR_ARG;
  }
  if (w && (d.r_max - d.r_min + 1) * (d.time_max - d.time_min + 1) > kWilsonMaxEntries) {
    why = "at most 1024 (R,T) entries per job";
    return GC_ERR_ARG;
  }
  return GC_OK;
}

} // namespace

extern "C" {

int gc_batch_create(const gc_job *jobs, int njobs, int precision, gc_batch **out) {
  if (!jobs || !out || njobs <= 0)
    return record_error(GC_ERR_ARG, "gc_batch_create: need at least one job");
  *out = nullptr;
  if (precision != GC_PREC_FP64 && precision != GC_PREC_MIXED)
    return record_error(GC_ERR_ARG, "gc_batch_create: unknown precision");
  for (int i = 0; i < njobs; i++) {
    std::string why;
    int rc = check_job(jobs[i], why);
    if (rc)
      return record_error(rc, "gc_batch_create: job " + std::to_string(i) + ": " + why);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return record_error(GC_ERR_NODEVICE, "no CUDA device available");
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10)
    return record_error(GC_ERR_NODEVICE, "device is not sm_100 (built for sm_100a only)");

  gc_batch *b = new gc_batch();
  b->prec = precision;
  b->jobs.resize(njobs);
  size_t total = 0, staging = 0, outs = 0;
  for (int i = 0; i < njobs; i++) {
    JobState &j = b->jobs[i];
    j.desc = jobs[i];
    for (int d = 0; d < 4; d++)
      j.g.L[d] = jobs[i].dims[d];
    j.g.stride[0] = 1;
    j.g.stride[1] = j.g.L[0];
    j.g.stride[2] = j.g.L[0] * j.g.L[1];
    j.g.stride[3] = j.g.L[0] * j.g.L[1] * j.g.L[2];
    j.g.V = j.g.stride[3] * j.g.L[3];
    j.g.Vs = j.g.stride[3];
    j.field_bytes = align256(link_bytes(j.desc.nc, precision) * (size_t)j.g.V);
    const bool w = !(j.desc.r_max == 0 && j.desc.time_max == 0);
    j.nr = w ? j.desc.r_max - j.desc.r_min + 1 : 0;
    j.nt = w ? j.desc.time_max - j.desc.time_min + 1 : 0;
    j.hyp_bytes = align256(inter_link_bytes(j.desc.nc, precision) * (size_t)j.g.V);
    // the HYP decorated-link scratch also holds the gauge-form W's lines and
    // transformed links, so a job that measures W has it without HYP steps
    total += 12 * j.field_bytes + (j.desc.hyp_steps > 0 || w ? 15 * j.hyp_bytes : 0);
    staging = std::max(staging, (size_t)(j.desc.nc == 3 ? 18 : 4) * 8 * 4 * (size_t)j.g.V);
    outs += (size_t)j.nr * j.nt;
    if (w)
      default_shape(j, precision == GC_PREC_FP64 ? 8 : 4);
  }
  cudaError_t e = cudaMalloc(&b->arena, total);
  if (e != cudaSuccess) {
    delete b;
    return record_error(e == cudaErrorMemoryAllocation ? GC_ERR_NOMEM : GC_ERR_CUDA,
                        std::string("cudaMalloc(batch fields, ") + std::to_string(total) +
                            " bytes): " + cudaGetErrorString(e));
  }
  size_t off = 0;
  for (JobState &j : b->jobs) {
    char *base = (char *)b->arena + off;
    for (int d = 0; d < 4; d++) {
      j.input[d] = base + d * j.field_bytes;
      j.setA[d] = base + (4 + d) * j.field_bytes;
      j.setB[d] = base + (8 + d) * j.field_bytes;
    }
    const int nh = j.desc.hyp_steps > 0 || j.nr > 0 ? 15 : 0;
    for (int f = 0; f < 15; f++)
      j.hyp[f] = nh ? base + 12 * j.field_bytes + f * j.hyp_bytes : nullptr;
    off += 12 * j.field_bytes + nh * j.hyp_bytes;
  }
  b->outs_count = std::max<size_t>(outs, 1);
  bool ok = cudaMalloc(&b->outs, b->outs_count * sizeof(double)) == cudaSuccess &&
            cudaMallocHost(&b->outs_host, b->outs_count * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&b->staging, staging) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess;
  for (int c = 0; c < 2 && ok; c++) {
    ok = cudaEventCreateWithFlags(&b->wfork[c], cudaEventDisableTiming) == cudaSuccess;
    for (int k = 0; k < kWStreams && ok; k++)
      ok = cudaStreamCreateWithFlags(&b->wstream[c][k], cudaStreamNonBlocking) == cudaSuccess &&
           cudaEventCreateWithFlags(&b->wjoin[c][k], cudaEventDisableTiming) == cudaSuccess;
  }
  if (ok)
    ok = cudaMalloc(&b->flags, 256 * ((njobs + 63) / 64)) == cudaSuccess &&
         cudaMalloc(&b->status, 256) == cudaSuccess &&
         cudaMallocHost(&b->status_host, sizeof(int)) == cudaSuccess;
  if (ok)
    *b->status_host = 0;
  b->staging_bytes = staging;
  size_t o = 0;
  const int ct_bytes = precision == GC_PREC_FP64 ? 8 : 4;
  for (int i = 0; i < njobs; i++) {
    JobState &j = b->jobs[i];
    j.out_dev = b->outs + o;
    o += (size_t)j.nr * j.nt;
    // the temporal-gauge W: its lines and transformed links go into the HYP
    // decorated-link scratch (a job without HYP steps has none)
    const size_t lb = wilson_gauge_line_bytes(j.g, j.desc.nc);
    j.gauge = ok && j.nr > 0 &&
              wilson_gauge_applies(j.g, j.desc.time_max, j.nt, j.desc.nc, ct_bytes) &&
              2 * lb + 6 * j.field_bytes <= 15 * j.hyp_bytes;
    if (j.gauge) {
      char *base = (char *)j.hyp[0];
      j.GA = base;
      j.GB = base + lb;
      for (int d = 0; d < 3; d++) {
        j.UA.f[d] = base + 2 * lb + d * j.field_bytes;
        j.UB.f[d] = base + 2 * lb + (3 + d) * j.field_bytes;
      }
      j.flag = b->flags + i;
    }
  }
  if (ok)
    ok = alloc_partials(b) == GC_OK;
  if (!ok) {
    gc_batch_destroy(b);
    return record_error(GC_ERR_NOMEM, "gc_batch_create: allocation failed");
  }
  b->device_bytes = (long long)(total + staging + b->outs_count * 8);
  for (JobState &j : b->jobs)
    b->device_bytes += (long long)j.w_blocks * j.nr * j.nt * 8;
  *out = b;
  return GC_OK;
}

int gc_batch_destroy(gc_batch *b) {
  if (!b)
    return GC_OK;
  if (b->main)
    cudaStreamSynchronize(b->main);
  if (b->side)
    cudaStreamSynchronize(b->side);
  free_graph(b);
  cudaFree(b->arena);
  cudaFree(b->partials);
  cudaFree(b->outs);
  cudaFree(b->staging);
  cudaFree(b->desc);
  cudaFree(b->flags);
  cudaFree(b->status);
  if (b->status_host)
    cudaFreeHost(b->status_host);
  for (int c = 0; c < 2; c++) {
    for (int k = 0; k < kWStreams; k++) {
      if (b->wstream[c][k]) {
        cudaStreamSynchronize(b->wstream[c][k]);
        cudaStreamDestroy(b->wstream[c][k]);
      }
      if (b->wjoin[c][k])
        cudaEventDestroy(b->wjoin[c][k]);
    }
    if (b->wfork[c])
      cudaEventDestroy(b->wfork[c]);
  }
  if (b->outs_host)
    cudaFreeHost(b->outs_host);
  if (b->fork)
    cudaEventDestroy(b->fork);
  if (b->join)
    cudaEventDestroy(b->join);
  if (b->done)
    cudaEventDestroy(b->done);
  if (b->main)
    cudaStreamDestroy(b->main);
  if (b->side)
    cudaStreamDestroy(b->side);
  delete b;
  return GC_OK;
}

int gc_batch_upload(gc_batch *b, int job, const double *host, int layout) {
  if (!b || !host || job < 0 || job >= (int)b->jobs.size())
    return bfail(b, GC_ERR_ARG, "gc_batch_upload: bad argument");
  std::lock_guard<std::mutex> lk(b->mu);
  JobState &j = b->jobs[job];
  const size_t bytes = (size_t)(j.desc.nc == 3 ? 18 : 4) * 8 * 4 * (size_t)j.g.V;
  cudaError_t e = cudaMemcpyAsync(b->staging, host, bytes, cudaMemcpyHostToDevice, b->main);
  if (e != cudaSuccess)
    return cfail(b, "cudaMemcpyAsync(batch upload)", e);
  Fields4 U;
  for (int d = 0; d < 4; d++)
    U.f[d] = j.input[d];
  int rc = launch_aos_to_soa(j.g, j.desc.nc, b->prec, layout, b->staging, U, b->main);
  if (rc)
    return bfail(b, rc, last_launch_error());
  e = cudaStreamSynchronize(b->main);
  if (e != cudaSuccess)
    return cfail(b, "batch upload", e);
  j.has_input = true;
  return GC_OK;
}

int gc_batch_generate(gc_batch *b, double eps_su2, double eps_su3, unsigned int seed,
                      unsigned int first_index) {
  if (!b)
    return record_error(GC_ERR_ARG, "null batch");
  size_t maxn = 0;
  for (JobState &j : b->jobs)
    maxn = std::max(maxn, (size_t)(j.desc.nc == 3 ? 18 : 4) * 4 * (size_t)j.g.V);
  double *buf = nullptr;
  cudaError_t e = cudaMallocHost(&buf, maxn * sizeof(double));
  if (e != cudaSuccess)
    return cfail(b, "cudaMallocHost(batch generator)", e);
  int rc = GC_OK;
  for (int i = 0; i < (int)b->jobs.size() && rc == GC_OK; i++) {
    JobState &j = b->jobs[i];
    rc = generate_host(j.g.L, j.desc.nc, j.desc.nc == 3 ? eps_su3 : eps_su2, seed,
                       first_index + (unsigned)i, 1, buf);
    if (rc == GC_OK)
      rc = gc_batch_upload(b, i, buf, GC_LAYOUT_ROWMAJOR);
  }
  cudaFreeHost(buf);
  return rc;
}

int gc_batch_autotune(gc_batch *b) {
  if (!b)
    return record_error(GC_ERR_ARG, "null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  for (JobState &j : b->jobs)
    if (!j.has_input)
      return bfail(b, GC_ERR_STATE, "gc_batch_autotune: every job needs its links first");
  // scratch partials large enough for the narrowest candidate (1 column)
  size_t need = 0;
  for (JobState &j : b->jobs)
    need = std::max(need, (size_t)j.g.Vs * 3 * j.nr * j.nt);
  double *scratch = nullptr;
  cudaError_t e = cudaMalloc(&scratch, std::max<size_t>(need, 1) * sizeof(double));
  if (e != cudaSuccess)
    return cfail(b, "cudaMalloc(autotune scratch)", e);
  b->tune_report.clear();
  // one tuning per distinct (Lt, nc, nr, nt, Vs)
  std::map<std::tuple<int, int, int, int, int>, std::pair<int, int>> cache;
  std::map<std::tuple<int, int, int, int, int>, int> gcache;
  int rc = GC_OK;
  for (JobState &j : b->jobs) {
    if (j.nr <= 0)
      continue;
    if (j.gauge) {
      // the gauge-form W kernel's columns per block, timed on the job's input
      auto key = std::make_tuple(j.g.L[3], j.desc.nc, j.nr, j.nt, j.g.Vs);
      auto it = gcache.find(key);
      if (it != gcache.end()) {
        j.gunits = it->second;
        continue;
      }
      Fields4 U;
      for (int d = 0; d < 4; d++)
        U.f[d] = j.input[d];
      rc = GC_DISPATCH_NC(j.desc.nc, b->prec, launch_wilson_gauge_prep, j.g, U, j.GA, j.GB,
                          j.UA, j.UB, j.flag, b->main);
      if (rc)
        break;
      float best = 1e30f;
      int bu = 0;
      const WilsonPlan dp = wilson_gauge_plan(j.g, j.nt, j.desc.nc,
                                              b->prec == GC_PREC_FP64 ? 8 : 4);
      char cls[96];
      std::snprintf(cls, sizeof cls, "SU(%d) %dx%dx%dx%d R<=%d T<=%d", j.desc.nc, j.g.L[0],
                    j.g.L[1], j.g.L[2], j.g.L[3], j.desc.r_max, j.desc.time_max);
      std::string lines;
      for (int units = 1; units * dp.rows <= 256; units *= 2) {
        float ms = 0;
        rc = GC_DISPATCH_NC(j.desc.nc, b->prec, time_wilson_gauge, j.g, j.UA, j.UB,
                            j.desc.r_min, j.desc.r_max, j.desc.time_min, j.desc.time_max,
                            units, scratch, b->main, &ms);
        if (rc == GC_ERR_ARG) {
          cudaGetLastError();
          rc = GC_OK;
          continue;
        }
        if (rc)
          break;
        char line[192];
        std::snprintf(line, sizeof line, "%s gauge-W rows=%d units=%d %.4f ms\n", cls, dp.rows,
                      units, ms);
        lines += line;
        if (ms < best) {
          best = ms;
          bu = units;
        }
      }
      if (rc)
        break;
      b->tune_report += lines;
      char line[192];
      std::snprintf(line, sizeof line, "%s gauge-W chosen units=%d\n", cls, bu);
      b->tune_report += line;
      j.gunits = bu;
      gcache[key] = bu;
      continue;
    }
    auto key = std::make_tuple(j.g.L[3], j.desc.nc, j.nr, j.nt, j.g.Vs);
    auto it = cache.find(key);
    int rows, cols;
    if (it != cache.end()) {
      rows = it->second.first;
      cols = it->second.second;
    } else {
      rc = tune_job(b, j, scratch, b->main, &rows, &cols);
      if (rc)
        break;
      cache[key] = {rows, cols};
    }
    j.rows = rows;
    j.cols = cols;
    j.w_blocks = ((j.g.Vs + cols - 1) / cols) * 3;
  }
  cudaFree(scratch);
  if (rc)
    return bfail(b, rc, last_launch_error());
  rc = alloc_partials(b);
  if (rc)
    return rc;
  free_graph(b);
  b->planned = false;
  return GC_OK;
}

int gc_batch_run(gc_batch *b, void *stream) {
  if (!b)
    return record_error(GC_ERR_ARG, "null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  for (JobState &j : b->jobs)
    if (!j.has_input)
      return bfail(b, GC_ERR_STATE, "gc_batch_run: every job needs its links first");
  cudaStream_t s = stream ? (cudaStream_t)stream : b->main;
  if (!b->planned) {
    int rc = build_schedule(b);
    if (rc)
      return rc;
    // first run: eager (sets kernel attributes, validates), then capture
    rc = enqueue_run(b, s);
    if (rc)
      return rc;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
      return cfail(b, "batch run", e);
    cudaStream_t cap = b->main;
    e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess)
      return cfail(b, "cudaStreamBeginCapture", e);
    rc = enqueue_run(b, cap);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(cap, &g);
    if (rc || e != cudaSuccess) {
      if (g)
        cudaGraphDestroy(g);
      return rc ? rc : cfail(b, "cudaStreamEndCapture", e);
    }
    b->graph = g;
    size_t n = 0;
    cudaGraphGetNodes(g, nullptr, &n);
    b->graph_nodes = (int)n;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess)
      return cfail(b, "cudaGraphInstantiate", e);
    cudaEventRecord(b->done, s); // the eager run already produced the results
    return GC_OK;
  }
  cudaError_t e = cudaGraphLaunch(b->exec, s);
  if (e != cudaSuccess)
    return cfail(b, "cudaGraphLaunch", e);
  cudaEventRecord(b->done, s);
  return GC_OK;
}

int gc_batch_synchronize(gc_batch *b) {
  if (!b)
    return record_error(GC_ERR_ARG, "null batch");
  cudaError_t e = cudaEventSynchronize(b->done);
  if (e != cudaSuccess)
    return cfail(b, "batch synchronize", e);
  if (*b->status_host)
    return bfail(b, GC_ERR_STATE, "batch run: a multi-job W launch had fewer threads per "
                                  "block than a job's shape needs; its results are invalid");
  return GC_OK;
}

int gc_batch_wilson(gc_batch *b, int job, double *out) {
  if (!b || !out || job < 0 || job >= (int)b->jobs.size())
    return bfail(b, GC_ERR_ARG, "gc_batch_wilson: bad argument");
  cudaError_t e = cudaEventSynchronize(b->done);
  if (e != cudaSuccess)
    return cfail(b, "gc_batch_wilson", e);
  if (*b->status_host)
    return bfail(b, GC_ERR_STATE, "gc_batch_wilson: a multi-job W launch had fewer threads "
                                  "per block than a job's shape needs");
  const JobState &j = b->jobs[job];
  const size_t off = (size_t)(j.out_dev - b->outs);
  std::memcpy(out, b->outs_host + off, (size_t)j.nr * j.nt * sizeof(double));
  return GC_OK;
}

int gc_batch_download(gc_batch *b, int job, double *host, int layout) {
  if (!b || !host || job < 0 || job >= (int)b->jobs.size())
    return bfail(b, GC_ERR_ARG, "gc_batch_download: bad argument");
  if (!b->planned)
    return bfail(b, GC_ERR_STATE, "gc_batch_download: run the batch first");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaEventSynchronize(b->done);
  const JobState &j = b->jobs[job];
  // the final link set of this job: follow the swaps of its steps
  Fields4 cur, alt;
  for (int d = 0; d < 4; d++) {
    cur.f[d] = j.setA[d];
    alt.f[d] = j.setB[d];
  }
  for (int k = 0; k < j.desc.hyp_steps; k++)
    std::swap(cur.f[3], alt.f[3]);
  for (int k = 0; k < j.desc.ape_steps; k++)
    for (int d = 0; d < 3; d++)
      std::swap(cur.f[d], alt.f[d]);
  int rc = launch_soa_to_aos(j.g, j.desc.nc, b->prec, layout, cur, b->staging, b->main);
  if (rc)
    return bfail(b, rc, last_launch_error());
  const size_t bytes = (size_t)(j.desc.nc == 3 ? 18 : 4) * 8 * 4 * (size_t)j.g.V;
  cudaError_t e = cudaMemcpyAsync(host, b->staging, bytes, cudaMemcpyDeviceToHost, b->main);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(b->main);
  if (e != cudaSuccess)
    return cfail(b, "batch download", e);
  return GC_OK;
}

int gc_batch_info(const gc_batch *b, long long *device_bytes, int *graph_nodes,
                  int *launches) {
  if (!b)
    return record_error(GC_ERR_ARG, "null batch");
  if (device_bytes)
    *device_bytes = b->device_bytes;
  if (graph_nodes)
    *graph_nodes = b->graph_nodes;
  if (launches) {
    int n = 0;
    // HYP: three levels; per-job gauge W: lines, transform, the two gated
    // W kernels, the reduction
    for (const Launch &L : b->launches)
      n += (L.kind == Launch::HYP) ? 3 : (L.kind == Launch::WAUTO) ? 5 : 1;
    *launches = n;
  }
  return GC_OK;
}

int gc_batch_autotune_report(const gc_batch *b, char *buf, int len) {
  if (!b || !buf || len <= 0)
    return record_error(GC_ERR_ARG, "gc_batch_autotune_report: bad argument");
  const size_t n = std::min(b->tune_report.size(), (size_t)len - 1);
  std::memcpy(buf, b->tune_report.data(), n);
  buf[n] = 0;
  return GC_OK;
}

int gc_batch_job_shape(const gc_batch *b, int job, int *rows, int *cols) {
  if (!b || job < 0 || job >= (int)b->jobs.size())
    return record_error(GC_ERR_ARG, "gc_batch_job_shape: bad argument");
  if (rows)
    *rows = b->jobs[job].rows;
  if (cols)
    *cols = b->jobs[job].cols;
  return GC_OK;
}

} // extern "C"
