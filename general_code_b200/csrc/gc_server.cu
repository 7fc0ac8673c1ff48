// A request loop for smear-and-measure jobs with continuous admission.
//
// Requests (one configuration each: a gc_job plus its host links) enter a
// FIFO queue. `slots` worker threads, each with its own CUDA stream, take
// the head of the queue as soon as (a) a worker is free and (b) the head's
// device memory (gc_job_device_bytes) fits in what is left of the memory
// budget and in the free device memory reported by the free-memory provider.
// A request then runs on its worker's stream with stream-ordered memory
// (gc_lattice_create_on_stream): upload, HYP, APE, W, result to host, free.
// Requests that arrive while others are on the GPU are admitted as workers
// and memory free up, and their kernels overlap with the others' on the
// device. Every request runs the same kernels with the same launch shapes
// as it would alone, and all reductions have a fixed order, so its result is
// bitwise the same alone and in the mix.
//
// Waits are bounded (gc_server_wait takes a timeout); destroying a server
// cancels requests that have not started and waits for running ones.
#include "../../include/gc_lattice.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

namespace gc {
int record_error(int code, const std::string &msg);
}

namespace {

using Clock = std::chrono::steady_clock;

double now_s() {
  return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

enum State { PENDING, RUNNING, DONE, FAILED, CANCELLED };

struct Request {
  gc_job job;
  const double *links = nullptr;
  int layout = 0;
  long long bytes = 0;
  long long sites = 0;
  State state = PENDING;
  int rc = GC_OK;
  std::string err;
  std::vector<double> w;
  double t_submit = 0, t_start = 0, t_done = 0;
};

long long default_free_bytes(void *) {
  size_t free_b = 0, total = 0;
  if (cudaMemGetInfo(&free_b, &total) != cudaSuccess)
    return 0;
  return (long long)free_b;
}

} // namespace

struct gc_server {
  gc_server_opts opts{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<unsigned long long> pending;
  std::unordered_map<unsigned long long, Request> reqs;
  std::vector<std::thread> workers;
  std::vector<cudaStream_t> streams;
  unsigned long long next_id = 1;
  long long budget = 0, in_use = 0, peak_bytes = 0;
  int inflight = 0, peak_inflight = 0;
  bool stop = false;
  int device = 0;
  // statistics
  long long submitted = 0, completed = 0, rejected = 0, failed = 0;
  long long sites_done = 0;
  double t_first = 0, t_last = 0;
  std::vector<double> latencies_ms, queue_ms, run_ms;
};

namespace {

// Bytes the requests' pool holds but no request uses: free for the next
// request although the device's free memory does not count them.
long long pool_slack(const gc_server *s) {
  if (s->opts.simulate_us > 0)
    return 0;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, s->device) != cudaSuccess)
    return 0;
  unsigned long long reserved = 0, used = 0;
  if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) !=
          cudaSuccess ||
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess)
    return 0;
  return reserved > used ? (long long)(reserved - used) : 0;
}

int run_request(gc_server *s, cudaStream_t st, Request &r) {
  if (s->opts.simulate_us > 0) {
    std::this_thread::sleep_for(std::chrono::microseconds(s->opts.simulate_us));
    const int nr = r.job.r_max ? r.job.r_max - r.job.r_min + 1 : 0;
    const int nt = r.job.time_max ? r.job.time_max - r.job.time_min + 1 : 0;
    r.w.assign((size_t)nr * nt, 0.0);
    return GC_OK;
  }
  gc_lattice *h = nullptr;
  int rc = gc_lattice_create_on_stream(r.job.dims, r.job.nc, s->opts.precision, st, &h);
  if (rc) {
    r.err = gc_last_error(nullptr);
    return rc;
  }
  rc = gc_upload(h, r.links, r.layout);
  if (!rc && r.job.hyp_steps > 0)
    rc = gc_hyp(h, r.job.hyp_alpha[0], r.job.hyp_alpha[1], r.job.hyp_alpha[2], r.job.hyp_steps);
  if (!rc && r.job.ape_steps > 0)
    rc = gc_ape(h, r.job.ape_alpha, r.job.ape_steps);
  if (!rc && r.job.r_max > 0) {
    const int nr = r.job.r_max - r.job.r_min + 1, nt = r.job.time_max - r.job.time_min + 1;
    r.w.assign((size_t)nr * nt, 0.0);
    rc = gc_wilson_onaxis(h, r.job.r_min, r.job.r_max, r.job.time_min, r.job.time_max,
                          r.w.data());
  }
  if (rc)
    r.err = gc_last_error(h);
  gc_lattice_destroy(h);
  return rc;
}

void worker(gc_server *s, int slot) {
  if (s->opts.simulate_us <= 0)
    cudaSetDevice(s->device);
  cudaStream_t st = s->streams.empty() ? nullptr : s->streams[slot];
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    // admit the head of the queue when it fits
    unsigned long long id = 0;
    for (;;) {
      if (s->stop)
        return;
      if (!s->pending.empty()) {
        Request &head = s->reqs[s->pending.front()];
        // The budget bounds what admitted requests hold together. A
        // free-memory provider, when given, also has to report room for the
        // head (memory held by running requests is already out of what it
        // reports); with nothing in flight the head is admitted on the
        // budget alone, so the queue cannot stall.
        bool fits = s->in_use + head.bytes <= s->budget;
        if (fits && s->opts.free_bytes && s->inflight > 0)
          fits = head.bytes <= s->opts.free_bytes(s->opts.free_bytes_ctx) + pool_slack(s);
        if (fits) {
          id = s->pending.front();
          s->pending.pop_front();
          break;
        }
      }
      s->cv_work.wait(lk);
    }
    Request &r = s->reqs[id];
    r.state = RUNNING;
    r.t_start = now_s();
    s->in_use += r.bytes;
    s->inflight++;
    s->peak_bytes = std::max(s->peak_bytes, s->in_use);
    s->peak_inflight = std::max(s->peak_inflight, s->inflight);
    lk.unlock();
    const int rc = run_request(s, st, r);
    lk.lock();
    r.rc = rc;
    r.t_done = now_s();
    r.state = rc ? FAILED : DONE;
    s->in_use -= r.bytes;
    s->inflight--;
    if (rc) {
      s->failed++;
    } else {
      s->completed++;
      s->sites_done += r.sites;
      s->latencies_ms.push_back(1e3 * (r.t_done - r.t_submit));
      s->queue_ms.push_back(1e3 * (r.t_start - r.t_submit));
      s->run_ms.push_back(1e3 * (r.t_done - r.t_start));
      s->t_last = std::max(s->t_last, r.t_done);
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

double percentile(std::vector<double> v, double q) {
  if (v.empty())
    return 0;
  size_t k = (size_t)(q * (v.size() - 1) + 0.5);
  std::nth_element(v.begin(), v.begin() + k, v.end());
  return v[k];
}

} // namespace

extern "C" {

int gc_server_create(const gc_server_opts *opts, gc_server **out) {
  if (!opts || !out)
    return gc::record_error(GC_ERR_ARG, "gc_server_create: null argument");
  *out = nullptr;
  if (opts->slots < 1 || opts->slots > 256)
    return gc::record_error(GC_ERR_ARG, "gc_server_create: slots must be 1..256");
  if (opts->precision != GC_PREC_FP64 && opts->precision != GC_PREC_MIXED)
    return gc::record_error(GC_ERR_ARG, "gc_server_create: unknown precision");
  gc_server *s = new gc_server();
  s->opts = *opts;
  if (opts->simulate_us <= 0) {
    int n = 0, major = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      delete s;
      return gc::record_error(GC_ERR_NODEVICE, "no CUDA device available");
    }
    cudaGetDevice(&s->device);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, s->device);
    if (major != 10) {
      delete s;
      return gc::record_error(GC_ERR_NODEVICE, "device is not sm_100");
    }
    // keep freed stream-ordered memory in the pool for the next request
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
      unsigned long long thr = ~0ULL;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    s->streams.resize(opts->slots);
    for (auto &st : s->streams)
      cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  }
  const long long avail = opts->free_bytes ? opts->free_bytes(opts->free_bytes_ctx)
                          : opts->simulate_us > 0 ? (1LL << 40)
                                                  : default_free_bytes(nullptr);
  s->budget = opts->memory_budget > 0 ? opts->memory_budget : (long long)(0.9 * (double)avail);
  if (opts->simulate_us <= 0 && !s->streams.empty()) {
    // Grow the pool once, now: a pool that grows while requests run maps new
    // device memory, and the mapping holds up every stream on the device
    // (measured: all requests in flight stalled together for ~250 ms, most
    // after another program had freed tens of GB). Freed back at once, the
    // reserve stays in the pool (release threshold above) and requests
    // suballocate from it.
    const long long reserve =
        opts->reserve_bytes == 0 ? std::min(s->budget, 16LL << 30) : opts->reserve_bytes;
    if (reserve > 0) {
      void *p = nullptr;
      if (cudaMallocAsync(&p, (size_t)reserve, s->streams[0]) == cudaSuccess) {
        cudaFreeAsync(p, s->streams[0]);
        cudaStreamSynchronize(s->streams[0]);
      } else {
        cudaGetLastError(); // no reserve: requests grow the pool as before
      }
    }
  }
  for (int i = 0; i < opts->slots; i++)
    s->workers.emplace_back(worker, s, i);
  *out = s;
  return GC_OK;
}

int gc_server_submit(gc_server *s, const gc_job *job, const double *host_links, int layout,
                     unsigned long long *id) {
  if (!s || !job || !id || (!host_links && s->opts.simulate_us <= 0))
    return gc::record_error(GC_ERR_ARG, "gc_server_submit: null argument");
  if (job->nc != 2 && job->nc != 3)
    return gc::record_error(GC_ERR_ARG, "gc_server_submit: nc must be 2 or 3");
  long long V = 1;
  for (int d = 0; d < 4; d++) {
    if (job->dims[d] < 2)
      return gc::record_error(GC_ERR_ARG, "gc_server_submit: every extent must be >= 2");
    V *= job->dims[d];
  }
  if (job->r_max > 0 && (job->r_min < 1 || job->time_min < 1 || job->r_max < job->r_min ||
                         job->time_max < job->time_min))
    return gc::record_error(GC_ERR_ARG, "gc_server_submit: bad W ranges");
  const long long bytes =
      gc_job_device_bytes(job->dims, job->nc, s->opts.precision, job->r_max, job->time_max);
  std::lock_guard<std::mutex> lk(s->mu);
  if (bytes > s->budget) {
    s->rejected++;
    return gc::record_error(GC_ERR_NOMEM, "gc_server_submit: the job needs " +
                                              std::to_string(bytes) +
                                              " device bytes, the budget is " +
                                              std::to_string(s->budget));
  }
  if (s->opts.queue_capacity > 0 && (int)s->pending.size() >= s->opts.queue_capacity) {
    s->rejected++;
    return gc::record_error(GC_ERR_BUSY, "gc_server_submit: queue full");
  }
  const unsigned long long rid = s->next_id++;
  Request &r = s->reqs[rid];
  r.job = *job;
  r.links = host_links;
  r.layout = layout;
  r.bytes = bytes;
  r.sites = V;
  r.t_submit = now_s();
  if (s->submitted == 0)
    s->t_first = r.t_submit;
  s->submitted++;
  s->pending.push_back(rid);
  *id = rid;
  s->cv_work.notify_all();
  return GC_OK;
}

int gc_server_wait(gc_server *s, unsigned long long id, double *out_w, double timeout_s) {
  if (!s)
    return gc::record_error(GC_ERR_ARG, "gc_server_wait: null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end())
    return gc::record_error(GC_ERR_ARG, "gc_server_wait: unknown request id");
  const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                           std::chrono::duration<double>(timeout_s));
  while (it->second.state == PENDING || it->second.state == RUNNING) {
    if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
        (it->second.state == PENDING || it->second.state == RUNNING))
      return gc::record_error(GC_ERR_TIMEOUT, "gc_server_wait: timed out");
    it = s->reqs.find(id);
  }
  Request &r = it->second;
  int rc = r.rc;
  if (r.state == CANCELLED)
    rc = gc::record_error(GC_ERR_STATE, "gc_server_wait: request was cancelled");
  else if (r.state == FAILED)
    rc = gc::record_error(r.rc, "request failed: " + r.err);
  else if (out_w && !r.w.empty())
    std::memcpy(out_w, r.w.data(), r.w.size() * sizeof(double));
  s->reqs.erase(it);
  return rc;
}

int gc_server_cancel(gc_server *s, unsigned long long id) {
  if (!s)
    return gc::record_error(GC_ERR_ARG, "gc_server_cancel: null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end())
    return gc::record_error(GC_ERR_ARG, "gc_server_cancel: unknown request id");
  if (it->second.state != PENDING)
    return gc::record_error(GC_ERR_STATE, "gc_server_cancel: request already started");
  s->pending.erase(std::find(s->pending.begin(), s->pending.end(), id));
  it->second.state = CANCELLED;
  s->cv_done.notify_all();
  s->cv_work.notify_all();
  return GC_OK;
}

int gc_server_stats(gc_server *s, gc_server_metrics *st) {
  if (!s || !st)
    return gc::record_error(GC_ERR_ARG, "gc_server_stats: null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(st, 0, sizeof(*st));
  st->submitted = s->submitted;
  st->completed = s->completed;
  st->rejected = s->rejected;
  st->failed = s->failed;
  st->pending = (long long)s->pending.size();
  st->inflight = s->inflight;
  st->peak_inflight = s->peak_inflight;
  st->peak_bytes = s->peak_bytes;
  st->budget = s->budget;
  st->p50_ms = percentile(s->latencies_ms, 0.50);
  st->p99_ms = percentile(s->latencies_ms, 0.99);
  double sum = 0;
  for (double v : s->latencies_ms)
    sum += v;
  st->mean_ms = s->latencies_ms.empty() ? 0 : sum / s->latencies_ms.size();
  st->queue_p50_ms = percentile(s->queue_ms, 0.50);
  st->queue_p99_ms = percentile(s->queue_ms, 0.99);
  st->run_p50_ms = percentile(s->run_ms, 0.50);
  st->run_p99_ms = percentile(s->run_ms, 0.99);
  const double span = s->t_last - s->t_first;
  st->sites_per_s = span > 0 ? (double)s->sites_done / span : 0;
  return GC_OK;
}

int gc_server_destroy(gc_server *s) {
  if (!s)
    return GC_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (unsigned long long id : s->pending)
      s->reqs[id].state = CANCELLED;
    s->pending.clear();
    s->stop = true;
    s->cv_work.notify_all();
    s->cv_done.notify_all();
  }
  for (auto &t : s->workers)
    t.join();
  for (auto &st : s->streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  delete s;
  return GC_OK;
}

} // extern "C"
