// C ABI (include/gc_lattice.h): device-resident lattice handles, uploads and
// downloads in the reference's host layouts, and dispatch to the kernels by
// group (SU(2)/SU(3)) and precision (FP64 / mixed).
#include "../../include/gc_lattice.h"
#include "gc_internal.cuh"
#include "gc_kernels.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <tuple>
#include <mutex>
#include <string>
#include <vector>

namespace gc {
int generate_host(const int dims[4], int nc, double eps, unsigned seed,
                  unsigned cfg, int gauge, double *out);
int probe_config(const int dims[4], int nc, const char *path, const char *format,
                 long long bytes_skip, const char *precision, long long *offset,
                 long long *length, std::string &err);
int launch_file_to_soa(const Geom &g, int nc, int prec, const char *format,
                       const char *precision, int convert, const unsigned char *data,
                       const Fields4 &U, cudaStream_t s);

namespace {
thread_local std::string g_launch_error;
std::mutex g_global_err_mu;
std::string g_global_err;
} // namespace

int launch_check(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    return GC_OK;
  g_launch_error = std::string(what) + ": " + cudaGetErrorString(e);
  return GC_ERR_CUDA;
}

int plan_error(const char *what) {
  g_launch_error = what;
  return GC_ERR_ARG;
}

// For entry points without a handle defined in other files: records the
// message returned by gc_last_error(NULL); returns code.
int record_error(int code, const std::string &msg) {
  std::lock_guard<std::mutex> lk(g_global_err_mu);
  g_global_err = msg;
  return code;
}

const std::string &last_launch_error() { return g_launch_error; }

} // namespace gc

struct gc_lattice {
  gc::Geom g{};
  int nc = 0, prec = 0;
  size_t field_bytes = 0;   // one direction's field
  void *links = nullptr;    // 8 fields: two sets of 4 directions
  gc::Fields4 cur{}, alt{}; // current / spare buffer of each direction
  void *hyp = nullptr;      // 15 decorated-link fields (allocated on first HYP)
  double *staging = nullptr; // host-layout staging buffer (device)
  double *partials = nullptr;
  size_t partials_cap = 0;  // doubles
  double *dev_out = nullptr;
  size_t dev_out_cap = 0;   // doubles
  void *aux = nullptr;      // Polyakov lines and offset tables
  size_t aux_cap = 0;       // bytes
  unsigned char *io_buf[2] = {nullptr, nullptr}; // pinned file chunks (reader, writer)
  cudaEvent_t io_ev[2] = {nullptr, nullptr};     // last copy out of / into each chunk
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  bool stream_ordered = false; // device memory from cudaMallocAsync on `stream`
  bool has_links = false;
  int *flag_dev = nullptr;    // device word: temporal links failed the unitarity check
  int wilson_method = GC_WILSON_AUTO;
  int hyp_method = GC_HYP_AUTO;
  int wilson_used = 0;        // GC_WILSON_EXACT or GC_WILSON_GAUGE, last W call
  std::string err;
  std::mutex mu;
};

namespace {

using namespace gc;

int fail(gc_lattice *h, int code, const std::string &msg) {
  if (h)
    h->err = msg;
  else {
    std::lock_guard<std::mutex> lk(g_global_err_mu);
    g_global_err = msg;
  }
  return code;
}

int cuda_fail(gc_lattice *h, const char *what, cudaError_t e) {
  return fail(h, e == cudaErrorMemoryAllocation ? GC_ERR_NOMEM : GC_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

int launch_fail(gc_lattice *h, int rc) {
  if (rc == GC_OK)
    return GC_OK;
  return fail(h, rc, g_launch_error);
}

// Device allocations of a handle: ordinary, or stream-ordered on the handle's
// stream (no device-wide synchronisation when freed).
cudaError_t dev_alloc(gc_lattice *h, void **p, size_t n) {
  if (h->stream_ordered)
    return cudaMallocAsync(p, n, h->stream);
  return cudaMalloc(p, n);
}
void dev_free(gc_lattice *h, void *p) {
  if (!p)
    return;
  if (h->stream_ordered)
    cudaFreeAsync(p, h->stream);
  else
    cudaFree(p);
}

size_t bytes_per_link(int nc, int prec) {
  if (nc == 3)
    return prec == GC_PREC_FP64 ? 144 : 48;
  return prec == GC_PREC_FP64 ? 32 : 16;
}

// (an attribute query, not cudaGetDeviceProperties, which is slow and is
// otherwise paid by every handle a request loop creates)
int check_device(gc_lattice *h) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(h, GC_ERR_NODEVICE, "no CUDA device available");
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (e != cudaSuccess)
    return cuda_fail(h, "cudaDeviceGetAttribute", e);
  if (major != 10) {
    char name[256] = "?";
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) == cudaSuccess)
      std::snprintf(name, sizeof name, "%s", p.name);
    return fail(h, GC_ERR_NODEVICE,
                "device " + std::string(name) +
                    " is not sm_100 (this library is built for sm_100a only)");
  }
  return GC_OK;
}

int ensure_staging(gc_lattice *h) {
  if (h->staging)
    return GC_OK;
  const size_t per = (h->nc == 3 ? 18 : 4) * sizeof(double);
  cudaError_t e = dev_alloc(h, (void **)&h->staging, per * 4 * (size_t)h->g.V);
  if (e != cudaSuccess) {
    h->staging = nullptr;
    return cuda_fail(h, "cudaMalloc(staging)", e);
  }
  return GC_OK;
}

int ensure_partials(gc_lattice *h, size_t n) {
  if (h->partials_cap >= n)
    return GC_OK;
  dev_free(h, h->partials);
  h->partials = nullptr;
  h->partials_cap = 0;
  cudaError_t e = dev_alloc(h, (void **)&h->partials, n * sizeof(double));
  if (e != cudaSuccess) {
    h->partials = nullptr;
    return cuda_fail(h, "cudaMalloc(partials)", e);
  }
  h->partials_cap = n;
  return GC_OK;
}

int ensure_dev_out(gc_lattice *h, size_t n) {
  if (h->dev_out_cap >= n)
    return GC_OK;
  dev_free(h, h->dev_out);
  h->dev_out = nullptr;
  h->dev_out_cap = 0;
  cudaError_t e = dev_alloc(h, (void **)&h->dev_out, n * sizeof(double));
  if (e != cudaSuccess) {
    h->dev_out = nullptr;
    return cuda_fail(h, "cudaMalloc(result)", e);
  }
  h->dev_out_cap = n;
  return GC_OK;
}

int ensure_aux(gc_lattice *h, size_t bytes) {
  if (h->aux_cap >= bytes)
    return GC_OK;
  dev_free(h, h->aux);
  h->aux = nullptr;
  h->aux_cap = 0;
  cudaError_t e = dev_alloc(h, &h->aux, bytes);
  if (e != cudaSuccess) {
    h->aux = nullptr;
    return cuda_fail(h, "cudaMalloc(Polyakov scratch)", e);
  }
  h->aux_cap = bytes;
  return GC_OK;
}

// Two pinned host chunks for configuration files: the reader fills one from
// the file while the other is copied to the device, the writer writes one to
// the file while the next is copied from the device (no pinning of a whole
// configuration per call, which costs more than reading it).
constexpr size_t kIoChunk = 16u << 20;

int ensure_io(gc_lattice *h) {
  for (int i = 0; i < 2; i++) {
    if (h->io_buf[i])
      continue;
    cudaError_t e = cudaMallocHost(reinterpret_cast<void **>(&h->io_buf[i]), kIoChunk);
    if (e == cudaSuccess)
      e = cudaEventCreateWithFlags(&h->io_ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess)
      return cuda_fail(h, "cudaMallocHost(file chunks)", e);
  }
  return GC_OK;
}

// One HYP decorated-link field (256-byte aligned).
size_t hyp_field_bytes(const gc_lattice *h) {
  return ((inter_link_bytes(h->nc, h->prec) * (size_t)h->g.V + 255) / 256) * 256;
}

int ensure_hyp(gc_lattice *h) {
  if (h->hyp)
    return GC_OK;
  cudaError_t e = dev_alloc(h, &h->hyp, 15 * hyp_field_bytes(h));
  if (e != cudaSuccess) {
    h->hyp = nullptr;
    return cuda_fail(h, "cudaMalloc(HYP decorated links)", e);
  }
  return GC_OK;
}

#define GC_DISPATCH(h, FN, ...)                                                \
  ((h)->nc == 3 ? ((h)->prec == GC_PREC_FP64                                   \
                       ? FN<StoreF64SU3, double>(__VA_ARGS__)                  \
                       : FN<StoreF32SU3, float>(__VA_ARGS__))                  \
                : ((h)->prec == GC_PREC_FP64                                   \
                       ? FN<StoreF64SU2, double>(__VA_ARGS__)                  \
                       : FN<StoreF32SU2, float>(__VA_ARGS__)))

int check_ready(gc_lattice *h) {
  if (!h)
    return fail(nullptr, GC_ERR_ARG, "null handle");
  if (!h->has_links)
    return fail(h, GC_ERR_STATE, "no links on the device yet (upload or generate first)");
  return GC_OK;
}

} // namespace

extern "C" {

int gc_version(void) { return 100; }

const char *gc_last_error(const gc_lattice *h) {
  if (h)
    return h->err.c_str();
  std::lock_guard<std::mutex> lk(g_global_err_mu);
  static thread_local std::string copy;
  copy = g_global_err;
  return copy.c_str();
}

static int create_impl(const int dims[4], int nc, int precision, cudaStream_t ordered,
                       gc_lattice **out);

int gc_lattice_create(const int dims[4], int nc, int precision,
                      gc_lattice **out) {
  return create_impl(dims, nc, precision, nullptr, out);
}

int gc_lattice_create_on_stream(const int dims[4], int nc, int precision,
                                void *cuda_stream, gc_lattice **out) {
  if (!cuda_stream)
    return fail(nullptr, GC_ERR_ARG, "gc_lattice_create_on_stream: null stream");
  return create_impl(dims, nc, precision, (cudaStream_t)cuda_stream, out);
}

static int create_impl(const int dims[4], int nc, int precision, cudaStream_t ordered,
                       gc_lattice **out) {
  if (!out || !dims)
    return fail(nullptr, GC_ERR_ARG, "null argument");
  *out = nullptr;
  if (nc != 2 && nc != 3)
    return fail(nullptr, GC_ERR_ARG, "nc must be 2 or 3");
  if (precision != GC_PREC_FP64 && precision != GC_PREC_MIXED)
    return fail(nullptr, GC_ERR_ARG, "precision must be GC_PREC_FP64 or GC_PREC_MIXED");
  long long V = 1;
  for (int d = 0; d < 4; d++) {
    if (dims[d] < 2)
      return fail(nullptr, GC_ERR_ARG, "every lattice extent must be >= 2");
    V *= dims[d];
  }
  if (V * 4 * 18 >= (1LL << 31) * 8)
    return fail(nullptr, GC_ERR_ARG, "lattice too large (4*V*18 must fit in 2^34)");
  if (V >= (1LL << 30))
    return fail(nullptr, GC_ERR_ARG, "lattice too large (V must be < 2^30)");
  int rc = check_device(nullptr);
  if (rc)
    return rc;
  gc_lattice *h = new gc_lattice();
  h->nc = nc;
  h->prec = precision;
  for (int d = 0; d < 4; d++)
    h->g.L[d] = dims[d];
  h->g.stride[0] = 1;
  h->g.stride[1] = dims[0];
  h->g.stride[2] = dims[0] * dims[1];
  h->g.stride[3] = dims[0] * dims[1] * dims[2];
  h->g.V = (int)V;
  h->g.Vs = dims[0] * dims[1] * dims[2];
  // 256-byte aligned fields
  h->field_bytes = ((bytes_per_link(nc, precision) * (size_t)V + 255) / 256) * 256;
  cudaError_t e;
  if (ordered) {
    h->stream_ordered = true;
    h->stream = ordered;
  } else {
    e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete h;
      return cuda_fail(nullptr, "cudaStreamCreate", e);
    }
    h->stream = h->own_stream;
  }
  e = dev_alloc(h, &h->links, 8 * h->field_bytes);
  if (e != cudaSuccess) {
    if (h->own_stream)
      cudaStreamDestroy(h->own_stream);
    delete h;
    return cuda_fail(nullptr, "cudaMalloc(links)", e);
  }
  for (int d = 0; d < 4; d++) {
    h->cur.f[d] = (char *)h->links + d * h->field_bytes;
    h->alt.f[d] = (char *)h->links + (4 + d) * h->field_bytes;
  }
  *out = h;
  return GC_OK;
}

int gc_lattice_destroy(gc_lattice *h) {
  if (!h)
    return GC_OK;
  {
    std::lock_guard<std::mutex> lk(h->mu);
    // stream-ordered memory is released in the stream's order, without waiting
    if (!h->stream_ordered)
      cudaStreamSynchronize(h->stream);
    dev_free(h, h->links);
    dev_free(h, h->hyp);
    dev_free(h, h->staging);
    dev_free(h, h->partials);
    dev_free(h, h->dev_out);
    dev_free(h, h->aux);
    dev_free(h, h->flag_dev);
    for (int i = 0; i < 2; i++) {
      if (h->io_ev[i])
        cudaEventSynchronize(h->io_ev[i]);
      if (h->io_buf[i])
        cudaFreeHost(h->io_buf[i]);
      if (h->io_ev[i])
        cudaEventDestroy(h->io_ev[i]);
    }
    if (h->own_stream)
      cudaStreamDestroy(h->own_stream);
  }
  delete h;
  return GC_OK;
}

int gc_set_stream(gc_lattice *h, void *stream) {
  if (!h)
    return fail(nullptr, GC_ERR_ARG, "null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  if (h->stream_ordered)
    return fail(h, GC_ERR_STATE,
                "a handle made by gc_lattice_create_on_stream stays on its stream");
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return GC_OK;
}

int gc_synchronize(gc_lattice *h) {
  if (!h)
    return fail(nullptr, GC_ERR_ARG, "null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "cudaStreamSynchronize", e);
  return GC_OK;
}

int gc_upload(gc_lattice *h, const double *host, int layout) {
  if (!h || !host)
    return fail(h, GC_ERR_ARG, "null argument");
  if (layout != GC_LAYOUT_ROWMAJOR && layout != GC_LAYOUT_EIGEN_COLMAJOR)
    return fail(h, GC_ERR_ARG, "unknown layout");
  std::lock_guard<std::mutex> lk(h->mu);
  int rc = ensure_staging(h);
  if (rc)
    return rc;
  const size_t bytes = (h->nc == 3 ? 18 : 4) * sizeof(double) * 4 * (size_t)h->g.V;
  cudaError_t e = cudaMemcpyAsync(h->staging, host, bytes, cudaMemcpyHostToDevice, h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "cudaMemcpyAsync(upload)", e);
  rc = launch_aos_to_soa(h->g, h->nc, h->prec, layout, h->staging, h->cur, h->stream);
  if (rc)
    return launch_fail(h, rc);
  h->has_links = true;
  return GC_OK;
}

int gc_download(gc_lattice *h, double *host, int layout) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  if (!host)
    return fail(h, GC_ERR_ARG, "null argument");
  if (layout != GC_LAYOUT_ROWMAJOR && layout != GC_LAYOUT_EIGEN_COLMAJOR)
    return fail(h, GC_ERR_ARG, "unknown layout");
  std::lock_guard<std::mutex> lk(h->mu);
  rc = ensure_staging(h);
  if (rc)
    return rc;
  rc = launch_soa_to_aos(h->g, h->nc, h->prec, layout, h->cur, h->staging, h->stream);
  if (rc)
    return launch_fail(h, rc);
  const size_t bytes = (h->nc == 3 ? 18 : 4) * sizeof(double) * 4 * (size_t)h->g.V;
  cudaError_t e = cudaMemcpyAsync(host, h->staging, bytes, cudaMemcpyDeviceToHost, h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "cudaMemcpyAsync(download)", e);
  e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "download synchronize", e);
  return GC_OK;
}

int gc_copy_links(gc_lattice *dst, gc_lattice *src) {
  if (!dst || !src)
    return fail(dst, GC_ERR_ARG, "null handle");
  if (dst == src)
    return GC_OK;
  int rc = check_ready(src);
  if (rc)
    return fail(dst, rc, std::string("source: ") + src->err);
  bool same = dst->nc == src->nc && dst->prec == src->prec;
  for (int d = 0; d < 4; d++)
    same = same && dst->g.L[d] == src->g.L[d];
  if (!same)
    return fail(dst, GC_ERR_ARG, "gc_copy_links: handles differ in shape, group or precision");
  std::scoped_lock lk(dst->mu, src->mu);
  if (src->stream != dst->stream) {
    cudaEvent_t ev;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess)
      return cuda_fail(dst, "cudaEventCreate", e);
    cudaEventRecord(ev, src->stream);
    cudaStreamWaitEvent(dst->stream, ev, 0);
    cudaEventDestroy(ev);
  }
  const size_t bytes = bytes_per_link(dst->nc, dst->prec) * (size_t)dst->g.V;
  for (int d = 0; d < 4; d++) {
    cudaError_t e = cudaMemcpyAsync(dst->cur.f[d], src->cur.f[d], bytes,
                                    cudaMemcpyDeviceToDevice, dst->stream);
    if (e != cudaSuccess)
      return cuda_fail(dst, "cudaMemcpyAsync(copy links)", e);
  }
  dst->has_links = true;
  return GC_OK;
}

// ---------------------------------------------------------------- t-slices
// A run of time slices [t0, t0 + nt) is, in every plane of every direction's
// field, one contiguous range of nt * Vs 16-byte elements (t varies slowest
// over the sites): a slice copy is one 2-D copy per direction, with the
// plane stride as the pitch.

static size_t slice_planes(const gc_lattice *h) { return bytes_per_link(h->nc, h->prec) / 16; }

static int check_slices(gc_lattice *h, int t0, int nt) {
  if (!h)
    return fail(nullptr, GC_ERR_ARG, "null handle");
  if (t0 < 0 || nt < 0 || t0 + nt > h->g.L[3])
    return fail(h, GC_ERR_ARG, "time slices outside the lattice");
  return GC_OK;
}

// Copies nt slices of every direction between two SoA field sets; dst_t0 /
// src_t0 are the first slices, dst_pitch / src_pitch the plane strides in
// bytes (a packed buffer has pitch nt * Vs * 16).
static cudaError_t copy_slice_planes(const gc_lattice *h, void *const dst[4], size_t dst_pitch,
                                     int dst_t0, const void *const src[4], size_t src_pitch,
                                     int src_t0, int nt, cudaMemcpyKind kind, cudaStream_t s) {
  const size_t vs = (size_t)h->g.Vs;
  const size_t width = (size_t)nt * vs * 16;
  for (int d = 0; d < 4 && width; d++) {
    cudaError_t e = cudaMemcpy2DAsync(
        static_cast<unsigned char *>(dst[d]) + (size_t)dst_t0 * vs * 16, dst_pitch,
        static_cast<const unsigned char *>(src[d]) + (size_t)src_t0 * vs * 16, src_pitch,
        width, slice_planes(h), kind, s);
    if (e != cudaSuccess)
      return e;
  }
  return cudaSuccess;
}

long long gc_slice_bytes(const gc_lattice *h, int nt) {
  if (!h || nt < 0)
    return -1;
  return 4LL * (long long)bytes_per_link(h->nc, h->prec) * h->g.Vs * nt;
}

int gc_upload_slices(gc_lattice *h, int t0, int nt, const double *host, int layout) {
  int rc = check_slices(h, t0, nt);
  if (rc)
    return rc;
  if (!host)
    return fail(h, GC_ERR_ARG, "null argument");
  if (layout != GC_LAYOUT_ROWMAJOR && layout != GC_LAYOUT_EIGEN_COLMAJOR)
    return fail(h, GC_ERR_ARG, "unknown layout");
  std::lock_guard<std::mutex> lk(h->mu);
  rc = ensure_staging(h);
  if (rc)
    return rc;
  const size_t sites = (size_t)nt * h->g.Vs;
  const size_t bytes = (h->nc == 3 ? 18 : 4) * sizeof(double) * 4 * sites;
  if (bytes) {
    cudaError_t e = cudaMemcpyAsync(h->staging, host, bytes, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess)
      return cuda_fail(h, "cudaMemcpyAsync(upload slices)", e);
  }
  rc = launch_aos_to_soa(h->g, h->nc, h->prec, layout, h->staging, h->cur, h->stream,
                         t0 * h->g.Vs, (int)sites);
  if (rc)
    return launch_fail(h, rc);
  h->has_links = true;
  return GC_OK;
}

int gc_pack_slices(gc_lattice *h, int t0, int nt, void *dev_buf) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  rc = check_slices(h, t0, nt);
  if (rc)
    return rc;
  if (!dev_buf)
    return fail(h, GC_ERR_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(h->mu);
  const size_t per_dir = slice_planes(h) * (size_t)nt * h->g.Vs * 16;
  void *dst[4];
  for (int d = 0; d < 4; d++)
    dst[d] = static_cast<unsigned char *>(dev_buf) + d * per_dir;
  cudaError_t e = copy_slice_planes(h, dst, (size_t)nt * h->g.Vs * 16, 0, h->cur.f,
                                    16 * (size_t)h->g.V, t0, nt, cudaMemcpyDeviceToDevice,
                                    h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "cudaMemcpy2DAsync(pack slices)", e);
  return GC_OK;
}

int gc_unpack_slices(gc_lattice *h, int t0, int nt, const void *dev_buf) {
  int rc = check_slices(h, t0, nt);
  if (rc)
    return rc;
  if (!dev_buf)
    return fail(h, GC_ERR_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(h->mu);
  const size_t per_dir = slice_planes(h) * (size_t)nt * h->g.Vs * 16;
  const void *src[4];
  for (int d = 0; d < 4; d++)
    src[d] = static_cast<const unsigned char *>(dev_buf) + d * per_dir;
  cudaError_t e = copy_slice_planes(h, h->cur.f, 16 * (size_t)h->g.V, t0, src,
                                    (size_t)nt * h->g.Vs * 16, 0, nt,
                                    cudaMemcpyDeviceToDevice, h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "cudaMemcpy2DAsync(unpack slices)", e);
  h->has_links = true;
  return GC_OK;
}

int gc_copy_slices(gc_lattice *dst, int dst_t0, gc_lattice *src, int src_t0, int nt) {
  if (!dst || !src)
    return fail(dst, GC_ERR_ARG, "null handle");
  int rc = check_ready(src);
  if (rc)
    return fail(dst, rc, std::string("source: ") + src->err);
  bool same = dst->nc == src->nc && dst->prec == src->prec;
  for (int d = 0; d < 3; d++)
    same = same && dst->g.L[d] == src->g.L[d];
  if (!same)
    return fail(dst, GC_ERR_ARG,
                "gc_copy_slices: handles differ in spatial extents, group or precision");
  rc = check_slices(dst, dst_t0, nt);
  if (rc)
    return rc;
  if (src_t0 < 0 || src_t0 + nt > src->g.L[3])
    return fail(dst, GC_ERR_ARG, "source time slices outside the lattice");
  if (dst == src) {
    if (nt && dst_t0 != src_t0 && std::abs(dst_t0 - src_t0) < nt)
      return fail(dst, GC_ERR_ARG, "overlapping slice ranges in one lattice");
  }
  std::unique_lock<std::mutex> lk1, lk2;
  if (dst != src) {
    gc_lattice *a = std::less<gc_lattice *>()(dst, src) ? dst : src;
    gc_lattice *b = a == dst ? src : dst;
    lk1 = std::unique_lock<std::mutex>(a->mu);
    lk2 = std::unique_lock<std::mutex>(b->mu);
  } else {
    lk1 = std::unique_lock<std::mutex>(dst->mu);
  }
  if (src->stream != dst->stream) {
    cudaEvent_t ev;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess)
      return cuda_fail(dst, "cudaEventCreate", e);
    cudaEventRecord(ev, src->stream);
    cudaStreamWaitEvent(dst->stream, ev, 0);
    cudaEventDestroy(ev);
  }
  cudaError_t e = copy_slice_planes(dst, dst->cur.f, 16 * (size_t)dst->g.V, dst_t0, src->cur.f,
                                    16 * (size_t)src->g.V, src_t0, nt,
                                    cudaMemcpyDeviceToDevice, dst->stream);
  if (e != cudaSuccess)
    return cuda_fail(dst, "cudaMemcpy2DAsync(copy slices)", e);
  dst->has_links = true;
  return GC_OK;
}

int gc_ape(gc_lattice *h, double alpha, int steps) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  if (steps < 0)
    return fail(h, GC_ERR_ARG, "steps must be >= 0");
  std::lock_guard<std::mutex> lk(h->mu);
  for (int s = 0; s < steps; s++) {
    Fields4 out = h->cur;
    for (int d = 0; d < 3; d++)
      out.f[d] = h->alt.f[d];
    rc = GC_DISPATCH(h, launch_ape, h->g, h->cur, out, alpha, h->stream);
    if (rc)
      return launch_fail(h, rc);
    for (int d = 0; d < 3; d++)
      std::swap(h->cur.f[d], h->alt.f[d]);
  }
  return GC_OK;
}

int gc_hyp(gc_lattice *h, double a1, double a2, double a3, int steps) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  if (steps < 0)
    return fail(h, GC_ERR_ARG, "steps must be >= 0");
  std::lock_guard<std::mutex> lk(h->mu);
  if (steps == 0)
    return GC_OK;
  rc = ensure_hyp(h);
  if (rc)
    return rc;
  HypL1 l1;
  HypL2 l2;
  const size_t hb = hyp_field_bytes(h);
  for (int i = 0; i < 9; i++)
    l1.f[i] = (char *)h->hyp + i * hb;
  for (int i = 0; i < 6; i++)
    l2.f[i] = (char *)h->hyp + (9 + i) * hb;
  // the level kernels unless the slice pipeline is asked for: it moves less
  // DRAM but takes 1.2-1.45x the time of the (issue-bound) level kernels at
  // 24^4-48^4 and 3x on small lattices (Lt + 3 short launches)
  const bool slices = h->hyp_method == GC_HYP_SLICES;
  for (int s = 0; s < steps; s++) {
    rc = slices ? GC_DISPATCH(h, launch_hyp_slices, h->g, h->cur, l1, l2, h->alt.f[3], a1, a2,
                              a3, h->stream)
                : GC_DISPATCH(h, launch_hyp, h->g, h->cur, l1, l2, h->alt.f[3], a1, a2, a3,
                              h->stream);
    if (rc)
      return launch_fail(h, rc);
    std::swap(h->cur.f[3], h->alt.f[3]);
  }
  return GC_OK;
}

// Prepares the temporal-gauge form of W: the gauge time lines of both cuts
// and the transformed spatial links, in the HYP decorated-link scratch (which
// holds them: per site at most 2 x 144 + 6 x 144 bytes against 15 x 144 for
// FP64 SU(3)), and the device's unitarity check of the temporal links into
// h->flag_dev. *use is cleared when the scratch cannot hold them.
static int gauge_prepare(gc_lattice *h, Fields4 *UA, Fields4 *UB, bool *use) {
  int rc = ensure_hyp(h);
  if (rc)
    return rc;
  if (!h->flag_dev) {
    cudaError_t e = dev_alloc(h, (void **)&h->flag_dev, 256);
    if (e != cudaSuccess) {
      h->flag_dev = nullptr;
      return cuda_fail(h, "cudaMalloc(flag)", e);
    }
  }
  const size_t lb = wilson_gauge_line_bytes(h->g, h->nc);
  if (2 * lb + 6 * h->field_bytes > 15 * hyp_field_bytes(h)) {
    *use = false;
    return GC_OK;
  }
  char *base = (char *)h->hyp;
  void *GA = base, *GB = base + lb;
  for (int d = 0; d < 3; d++) {
    UA->f[d] = base + 2 * lb + d * h->field_bytes;
    UB->f[d] = base + 2 * lb + (3 + d) * h->field_bytes;
  }
  UA->f[3] = UB->f[3] = nullptr;
  rc = GC_DISPATCH(h, launch_wilson_gauge_prep, h->g, h->cur, GA, GB, *UA, *UB, h->flag_dev,
                   h->stream);
  if (rc)
    return launch_fail(h, rc);
  return GC_OK;
}

// W(R,T) of h, or with `second` the GEVP loops of the pair (h, second):
// h's time lines, space lines of both (wilson_gevp_indexed).
static int wilson_impl(gc_lattice *h, int rmin, int rmax, int tmin, int tmax,
                       double *out, bool adjoint, gc_lattice *second = nullptr,
                       int tstarts = 0) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  if (!out)
    return fail(h, GC_ERR_ARG, "null output");
  if (rmin < 1 || tmin < 1 || rmax < rmin || tmax < tmin)
    return fail(h, GC_ERR_ARG, "need 1 <= r_min <= r_max and 1 <= time_min <= time_max");
  if (second && second != h) {
    rc = check_ready(second);
    if (rc)
      return fail(h, rc, std::string("second configuration: ") + gc_last_error(second));
    for (int d = 0; d < 4; d++)
      if (second->g.L[d] != h->g.L[d])
        return fail(h, GC_ERR_ARG, "the two configurations have different lattice sizes");
    if (second->nc != h->nc || second->prec != h->prec)
      return fail(h, GC_ERR_ARG, "the two configurations differ in group or precision");
  }
  // both handles locked (in a fixed order, so two calls on the same pair in
  // opposite roles cannot deadlock)
  std::unique_lock<std::mutex> lk1, lk2;
  if (second && second != h) {
    gc_lattice *a = std::less<gc_lattice *>()(h, second) ? h : second;
    gc_lattice *b = a == h ? second : h;
    lk1 = std::unique_lock<std::mutex>(a->mu);
    lk2 = std::unique_lock<std::mutex>(b->mu);
    // h's stream waits for the work queued on the second handle
    cudaEvent_t ev;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess)
      return cuda_fail(h, "cudaEventCreate(second configuration)", e);
    e = cudaEventRecord(ev, second->stream);
    if (e == cudaSuccess)
      e = cudaStreamWaitEvent(h->stream, ev, 0);
    cudaEventDestroy(ev);
    if (e != cudaSuccess)
      return cuda_fail(h, "ordering after the second configuration", e);
  } else {
    lk1 = std::unique_lock<std::mutex>(h->mu);
  }
  const gc::Fields4 *u2 = second ? &second->cur : nullptr;
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  // The per-warp accumulators live in shared memory; split R into chunks so
  // that a block's accumulators stay small.
  const int max_entries = 1024;
  if (nt > max_entries)
    return fail(h, GC_ERR_ARG, "time range too large (at most 1024 values of T)");
  const int rchunk = std::max(1, max_entries / nt);
  rc = ensure_dev_out(h, (size_t)nr * nt + (size_t)rchunk * nt);
  if (rc)
    return rc;
  rc = ensure_partials(h, wilson_partials_count(h->g, std::min(rchunk, nr), nt, h->nc,
                                                second ? 4 : 3));
  if (rc)
    return rc;
  double *chunk_out = h->dev_out + (size_t)nr * nt;
  // The temporal-gauge form (gc_wilson_gauge.cu) for one configuration's
  // on-axis or adjoint loops with T <= Lt/2, or, for the t-slab entry's start
  // slices [0, t_starts), with T <= Lt - t_starts (one cut at slice 0: no
  // counted loop passes the slab lattice's last slice); it runs only where
  // the device finds the temporal links unitary to the form's tolerance, and
  // the exact recursion otherwise.
  const int ct_bytes = h->prec == GC_PREC_FP64 ? 8 : 4;
  bool gauge = h->wilson_method == GC_WILSON_AUTO && !second &&
               wilson_gauge_applies(h->g, tmax, nt, h->nc, ct_bytes, tstarts);
  Fields4 UA{}, UB{};
  if (gauge) {
    rc = gauge_prepare(h, &UA, &UB, &gauge);
    if (rc)
      return rc;
  }
  if (gauge) {
    rc = ensure_partials(h, wilson_auto_partials_count(h->g, std::min(rchunk, nr), nt, h->nc));
    if (rc)
      return rc;
  }
  // (the method the device chose is read back only when asked for)
  h->wilson_used = gauge ? -1 : GC_WILSON_EXACT;
  for (int r0 = rmin; r0 <= rmax; r0 += rchunk) {
    const int r1 = std::min(rmax, r0 + rchunk - 1);
    const int ncr = r1 - r0 + 1;
    if (gauge)
      rc = GC_DISPATCH(h, launch_wilson_auto, h->g, h->cur, UA, UB, r0, r1, tmin, tmax,
                       adjoint, h->flag_dev, h->partials, chunk_out, h->stream, 0, tstarts);
    else
      rc = GC_DISPATCH(h, launch_wilson, h->g, h->cur, r0, r1, tmin, tmax,
                       h->partials, chunk_out, h->stream, adjoint, u2, tstarts);
    if (rc)
      return launch_fail(h, rc);
    // chunk_out[(T-tmin)*ncr + (R-r0)] -> dev_out[(T-tmin)*nr + (R-rmin)]
    cudaError_t e = cudaMemcpy2DAsync(h->dev_out + (r0 - rmin), nr * sizeof(double),
                                      chunk_out, ncr * sizeof(double),
                                      ncr * sizeof(double), nt,
                                      cudaMemcpyDeviceToDevice, h->stream);
    if (e != cudaSuccess)
      return cuda_fail(h, "cudaMemcpy2DAsync(wilson chunk)", e);
  }
  cudaError_t e = cudaMemcpyAsync(out, h->dev_out, (size_t)nr * nt * sizeof(double),
                                  cudaMemcpyDeviceToHost, h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "cudaMemcpyAsync(wilson result)", e);
  e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "wilson synchronize", e);
  return GC_OK;
}

int gc_wilson_onaxis(gc_lattice *h, int rmin, int rmax, int tmin, int tmax,
                     double *out) {
  return wilson_impl(h, rmin, rmax, tmin, tmax, out, false);
}

int gc_wilson_adjoint_onaxis(gc_lattice *h, int rmin, int rmax, int tmin, int tmax,
                             double *out) {
  return wilson_impl(h, rmin, rmax, tmin, tmax, out, true);
}

int gc_wilson_onaxis_tslab(gc_lattice *h, int t_starts, int rmin, int rmax, int tmin,
                           int tmax, int adjoint, double *out) {
  if (h && (t_starts < 1 || t_starts > h->g.L[3]))
    return fail(h, GC_ERR_ARG, "t_starts must be in [1, Lt]");
  return wilson_impl(h, rmin, rmax, tmin, tmax, out, adjoint != 0, nullptr, t_starts);
}

int gc_set_hyp_method(gc_lattice *h, int method) {
  if (!h)
    return fail(nullptr, GC_ERR_ARG, "null handle");
  if (method != GC_HYP_AUTO && method != GC_HYP_LEVELS && method != GC_HYP_SLICES)
    return fail(h, GC_ERR_ARG, "method must be GC_HYP_AUTO, GC_HYP_LEVELS or GC_HYP_SLICES");
  if (method == GC_HYP_SLICES && h->g.L[3] < 3)
    return fail(h, GC_ERR_ARG, "GC_HYP_SLICES needs Lt >= 3");
  std::lock_guard<std::mutex> lk(h->mu);
  h->hyp_method = method;
  return GC_OK;
}

int gc_set_wilson_method(gc_lattice *h, int method) {
  if (!h)
    return fail(nullptr, GC_ERR_ARG, "null handle");
  if (method != GC_WILSON_AUTO && method != GC_WILSON_EXACT)
    return fail(h, GC_ERR_ARG, "method must be GC_WILSON_AUTO or GC_WILSON_EXACT");
  std::lock_guard<std::mutex> lk(h->mu);
  h->wilson_method = method;
  return GC_OK;
}

int gc_wilson_method_used(gc_lattice *h, int *method) {
  if (!h || !method)
    return fail(h, GC_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(h->mu);
  if (h->wilson_used == -1) { // chosen on the device: read the flag
    int flag = 1;
    cudaError_t e = cudaMemcpyAsync(&flag, h->flag_dev, sizeof(int), cudaMemcpyDeviceToHost,
                                    h->stream);
    if (e == cudaSuccess)
      e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess)
      return cuda_fail(h, "gc_wilson_method_used", e);
    h->wilson_used = flag ? GC_WILSON_EXACT : GC_WILSON_GAUGE;
  }
  *method = h->wilson_used;
  return GC_OK;
}

int gc_wilson_gevp_onaxis(gc_lattice *h1, gc_lattice *h2, int rmin, int rmax, int tmin,
                          int tmax, double *out) {
  if (!h2)
    return fail(h1, GC_ERR_ARG, "null second configuration");
  return wilson_impl(h1, rmin, rmax, tmin, tmax, out, false, h2);
}

int gc_wilson_gevp_adjoint_onaxis(gc_lattice *h1, gc_lattice *h2, int rmin, int rmax,
                                  int tmin, int tmax, double *out) {
  if (!h2)
    return fail(h1, GC_ERR_ARG, "null second configuration");
  return wilson_impl(h1, rmin, rmax, tmin, tmax, out, true, h2);
}

// Both plaquette averages: out2[0] spatial planes, out2[1] (mu, t) planes.
static int plaquettes(gc_lattice *h, double out2[2]) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  std::lock_guard<std::mutex> lk(h->mu);
  rc = ensure_dev_out(h, 2);
  if (rc)
    return rc;
  rc = ensure_partials(h, plaquette_partials_count(h->g));
  if (rc)
    return rc;
  rc = GC_DISPATCH(h, launch_plaquette, h->g, h->cur, h->partials, h->dev_out, h->stream);
  if (rc)
    return launch_fail(h, rc);
  cudaError_t e = cudaMemcpyAsync(out2, h->dev_out, 2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "cudaMemcpyAsync(plaquette)", e);
  e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "plaquette synchronize", e);
  return GC_OK;
}

int gc_plaquette(gc_lattice *h, double *out) {
  if (!out)
    return fail(h, GC_ERR_ARG, "null output");
  double v[2];
  int rc = plaquettes(h, v);
  if (rc)
    return rc;
  *out = 0.5 * (v[0] + v[1]);
  return GC_OK;
}

int gc_plaquette_space(gc_lattice *h, double *out) {
  if (!out)
    return fail(h, GC_ERR_ARG, "null output");
  double v[2];
  int rc = plaquettes(h, v);
  if (rc)
    return rc;
  *out = v[0];
  return GC_OK;
}

int gc_plaquette_time(gc_lattice *h, double *out) {
  if (!out)
    return fail(h, GC_ERR_ARG, "null output");
  double v[2];
  int rc = plaquettes(h, v);
  if (rc)
    return rc;
  *out = v[1];
  return GC_OK;
}

// Off-axis loops: one space-line field and one loop launch per line of the
// plan, all loop averages copied back once, then averaged per (direction,
// multiplier, T) in the plan's order (a left-to-right sum from 0, as
// std::accumulate).
static int offaxis_impl(gc_lattice *h, const std::vector<std::array<int, 3>> &dirs,
                        double r_min, double r_max, int tmin, int tmax, bool adjoint,
                        std::vector<gc_wilson_result> &res) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  if (tmin < 1 || tmax < tmin)
    return fail(h, GC_ERR_ARG, "need 1 <= time_min <= time_max");
  const int nt = tmax - tmin + 1;
  if (nt > kWilsonMaxEntries)
    return fail(h, GC_ERR_ARG, "time range too large (at most 1024 values of T)");
  for (const auto &d : dirs)
    if (d[0] < 1 || d[1] < 0 || d[2] < 0 || d[0] < d[1] || d[1] < d[2])
      return fail(h, GC_ERR_ARG, "directions need a1 >= a2 >= a3 >= 0 and a1 >= 1");
  const OffaxisPlan plan = offaxis_plan(dirs, r_min, r_max);
  for (const auto &line : plan.lines)
    if ((int)line.pattern.size() > kOffaxisMaxSteps)
      return fail(h, GC_ERR_ARG, "off-axis line longer than 256 links (reduce r_max)");
  res.clear();
  if (plan.lines.empty())
    return GC_OK;
  std::lock_guard<std::mutex> lk(h->mu);
  // the lines as a device table (steps and end displacement as residues)
  std::vector<OffaxisLineDesc> table(plan.lines.size());
  for (size_t i = 0; i < table.size(); i++) {
    const OffaxisLine &line = plan.lines[i];
    OffaxisLineDesc &d = table[i];
    std::memset(&d, 0, sizeof d);
    d.n = (int)line.pattern.size();
    for (int k = 0; k < 3; k++)
      d.d[k] = ((line.disp[k] % h->g.L[k]) + h->g.L[k]) % h->g.L[k];
    for (int q = 0; q < d.n; q++)
      d.s[q] = (signed char)line.pattern[q];
  }
  rc = ensure_aux(h, table.size() * sizeof(OffaxisLineDesc));
  if (rc)
    return rc;
  // (from pageable memory: returns once the table is staged, so `table` may go)
  cudaError_t ce = cudaMemcpyAsync(h->aux, table.data(), table.size() * sizeof(OffaxisLineDesc),
                                   cudaMemcpyHostToDevice, h->stream);
  if (ce != cudaSuccess)
    return cuda_fail(h, "cudaMemcpyAsync(off-axis lines)", ce);
  // Lines go in chunks whose partials, [block][line][T], stay within 32 MB,
  // one fused launch and one reduction per chunk.
  const int blocks = offaxis_fused_blocks(h->g, h->nc, h->prec == GC_PREC_FP64 ? 8 : 4);
  const size_t per_line = (size_t)blocks * nt;
  const size_t chunk =
      std::max<size_t>(1, std::min(plan.lines.size(), ((size_t)4 << 20) / per_line));
  rc = ensure_partials(h, per_line * chunk);
  if (rc)
    return rc;
  rc = ensure_dev_out(h, plan.lines.size() * (size_t)nt);
  if (rc)
    return rc;
  const OffaxisLineDesc *dev_lines = static_cast<const OffaxisLineDesc *>(h->aux);
  for (size_t c0 = 0; c0 < plan.lines.size(); c0 += chunk) {
    const int n = (int)std::min(chunk, plan.lines.size() - c0);
    int b = 0;
    rc = GC_DISPATCH(h, launch_offaxis_fused, h->g, h->cur, dev_lines + c0, n, tmin, tmax,
                     adjoint, h->partials, &b, h->stream);
    if (!rc)
      rc = launch_reduce_rows(h->partials, b, n * nt, line_loop_scale(h->g, h->nc, adjoint),
                              h->dev_out + c0 * nt, h->stream);
    if (rc)
      return launch_fail(h, rc);
  }
  std::vector<double> vals(plan.lines.size() * (size_t)nt);
  cudaError_t e = cudaMemcpyAsync(vals.data(), h->dev_out, vals.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "off-axis results", e);
  for (const auto &grp : plan.groups)
    for (int T = tmin; T <= tmax; T++) {
      double sum = 0.0;
      for (int li : grp.lines)
        sum += vals[(size_t)li * nt + (T - tmin)];
      gc_wilson_result r;
      r.statistics_size = (int)grp.lines.size();
      r.wilson_loop = sum / r.statistics_size;
      r.time_size = T;
      r.space_size = grp.length * grp.multiplier;
      res.push_back(r);
    }
  return GC_OK;
}

static int offaxis_out(gc_lattice *h, const std::vector<gc_wilson_result> &res,
                       gc_wilson_result *out, int capacity, int *count) {
  *count = (int)res.size();
  if ((int)res.size() > capacity)
    return fail(h, GC_ERR_ARG, "output capacity too small (*count holds the size needed)");
  if (!res.empty())
    std::memcpy(out, res.data(), res.size() * sizeof(gc_wilson_result));
  return GC_OK;
}

int gc_wilson_offaxis(gc_lattice *h, const int *directions, int ndirections, double r_min,
                      double r_max, int time_min, int time_max, int adjoint,
                      gc_wilson_result *out, int capacity, int *count) {
  if (!count || (capacity > 0 && !out) || ndirections < 0 || (ndirections > 0 && !directions))
    return fail(h, GC_ERR_ARG, "null or negative argument");
  std::vector<std::array<int, 3>> dirs(ndirections);
  for (int i = 0; i < ndirections; i++)
    dirs[i] = {directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]};
  std::vector<gc_wilson_result> res;
  int rc = offaxis_impl(h, dirs, r_min, r_max, time_min, time_max, adjoint != 0, res);
  if (rc)
    return rc;
  return offaxis_out(h, res, out, capacity, count);
}

int gc_wilson_offaxis_result(gc_lattice *h, double r_min, double r_max, int time_min,
                             int time_max, int adjoint, gc_wilson_result *out, int capacity,
                             int *count) {
  if (!count || (capacity > 0 && !out))
    return fail(h, GC_ERR_ARG, "null argument");
  std::vector<gc_wilson_result> res;
  int rc = offaxis_impl(h, offaxis_directions(4), r_min - 0.1, r_max + 0.1, time_min, time_max,
                        adjoint != 0, res);
  if (rc)
    return rc;
  offaxis_reduce(res);
  return offaxis_out(h, res, out, capacity, count);
}

int gc_ape_plane(gc_lattice *h, int a, int b, double alpha, int steps) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  if (a < 0 || a > 3 || b < 0 || b > 3 || a == b || steps < 0)
    return fail(h, GC_ERR_ARG, "need two different directions 0..3 and steps >= 0");
  std::lock_guard<std::mutex> lk(h->mu);
  for (int i = 0; i < steps; i++) {
    rc = GC_DISPATCH(h, launch_ape_plane, h->g, h->cur.f[a], h->cur.f[b], h->alt.f[a],
                     h->alt.f[b], a, b, alpha, h->stream);
    if (rc)
      return launch_fail(h, rc);
    std::swap(h->cur.f[a], h->alt.f[a]);
    std::swap(h->cur.f[b], h->alt.f[b]);
  }
  return GC_OK;
}

int gc_wilson_spatial_3d(gc_lattice *h, int r_min, int r_max, int time_min, int time_max,
                         double alpha, int smearing_start, int smearing_end, int smearing_step,
                         gc_wilson_spatial_result *out, int capacity, int *count) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  if (!count || (capacity > 0 && !out))
    return fail(h, GC_ERR_ARG, "null argument");
  if (r_min < 1 || r_max < r_min || time_min < 1 || time_max < time_min)
    return fail(h, GC_ERR_ARG, "need 1 <= r_min <= r_max and 1 <= time_min <= time_max");
  if (smearing_step < 1 || smearing_end < 0)
    return fail(h, GC_ERR_ARG, "need smearing_step >= 1 and smearing_end >= 0");
  const int nt = time_max - time_min + 1, nr = r_max - r_min + 1;
  if (nt > kWilsonMaxEntries)
    return fail(h, GC_ERR_ARG, "time range too large (at most 1024 values of T)");
  // smearing steps measured (wilson_loops.h:1410-1419)
  std::vector<int> measured{0};
  for (int sm = 1; sm <= smearing_end; sm++)
    if ((sm - smearing_start) % smearing_step == 0 && smearing_step >= smearing_start)
      measured.push_back(sm);
  const int nm = (int)measured.size();
  std::lock_guard<std::mutex> lk(h->mu);
  const size_t fb = h->field_bytes;
  const size_t lb = ((inter_link_bytes(h->nc, h->prec) * (size_t)h->g.V + 255) / 256) * 256;
  rc = ensure_aux(h, 4 * fb + 2 * lb);
  if (rc)
    return rc;
  // the 2 nr lines of one (plane, measurement) share a partials buffer,
  // [block][(r, axis)][T], and one reduction launch when it stays within 32 MB
  const size_t per_line = (size_t)offaxis_partials_count(h->g, nt);
  const bool shared_reduce = per_line * 2 * nr <= ((size_t)4 << 20);
  rc = ensure_partials(h, shared_reduce ? per_line * 2 * nr : per_line);
  if (rc)
    return rc;
  // values[plane][measurement][r][axis][T]
  const size_t per_plane = (size_t)nm * nr * 2 * nt;
  rc = ensure_dev_out(h, 3 * per_plane);
  if (rc)
    return rc;
  char *base = (char *)h->aux;
  void *F[2] = {base, base + fb}, *G[2] = {base + 2 * fb, base + 3 * fb};
  void *S[2] = {base + 4 * fb, base + 4 * fb + lb};
  const int planes[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int p = 0; p < 3; p++) {
    const int ax[2] = {planes[p][0], planes[p][1]};
    const int mu = 3 - ax[0] - ax[1];
    for (int k = 0; k < 2; k++) {
      cudaError_t e = cudaMemcpyAsync(F[k], h->cur.f[ax[k]], fb, cudaMemcpyDeviceToDevice,
                                      h->stream);
      if (e != cudaSuccess)
        return cuda_fail(h, "copy of a direction field", e);
    }
    int mi = 0, sm = 0;
    for (;;) {
      if (mi < nm && measured[mi] == sm) {
        for (int k = 0; k < 2; k++) {
          // line of the reference's initial length (see the declaration)
          rc = GC_DISPATCH(h, launch_line_extend, h->g, F[k], S[k], ax[k], time_min,
                           time_min - 1, true, h->stream);
          if (rc)
            return launch_fail(h, rc);
        }
        double *plane_out = h->dev_out + p * per_plane + (size_t)mi * nr * 2 * nt;
        for (int r = r_min; r <= r_max; r++) {
          for (int k = 0; k < 2; k++) {
            int disp[4] = {0, 0, 0, 0};
            disp[ax[k]] = r;
            const size_t q = (size_t)(r - r_min) * 2 + k;
            rc = shared_reduce
                     ? GC_DISPATCH(h, launch_line_loops, h->g, h->cur.f[mu], mu, S[k], disp,
                                   time_min, time_max, false, h->partials + q * nt,
                                   (double *)nullptr, h->stream, 2 * nr * nt)
                     : GC_DISPATCH(h, launch_line_loops, h->g, h->cur.f[mu], mu, S[k], disp,
                                   time_min, time_max, false, h->partials,
                                   plane_out + q * nt, h->stream, 0);
            if (rc)
              return launch_fail(h, rc);
          }
          for (int k = 0; k < 2; k++) {
            rc = GC_DISPATCH(h, launch_line_extend, h->g, F[k], S[k], ax[k], r, 1, false,
                             h->stream);
            if (rc)
              return launch_fail(h, rc);
          }
        }
        if (shared_reduce) {
          rc = launch_reduce_rows(h->partials, (int)(per_line / nt), 2 * nr * nt,
                                  line_loop_scale(h->g, h->nc, false), plane_out, h->stream);
          if (rc)
            return launch_fail(h, rc);
        }
        mi++;
      }
      if (sm == smearing_end)
        break;
      rc = GC_DISPATCH(h, launch_ape_plane, h->g, F[0], F[1], G[0], G[1], ax[0], ax[1], alpha,
                       h->stream);
      if (rc)
        return launch_fail(h, rc);
      std::swap(F[0], G[0]);
      std::swap(F[1], G[1]);
      sm++;
    }
  }
  std::vector<double> vals(3 * per_plane);
  cudaError_t e = cudaMemcpyAsync(vals.data(), h->dev_out, vals.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "spatial loop results", e);
  // sums per (smearing, T, R) in the reference's order: planes, then r, t,
  // the nu axis before the eta axis; then / 6
  std::map<std::tuple<int, int, int>, double> acc;
  for (int p = 0; p < 3; p++)
    for (int mi2 = 0; mi2 < nm; mi2++)
      for (int r = r_min; r <= r_max; r++)
        for (int t = time_min; t <= time_max; t++)
          for (int k = 0; k < 2; k++)
            acc[std::make_tuple(measured[mi2], t, r)] +=
                vals[p * per_plane + (((size_t)mi2 * nr + (r - r_min)) * 2 + k) * nt +
                     (t - time_min)];
  *count = (int)acc.size();
  if (*count > capacity)
    return fail(h, GC_ERR_ARG, "output capacity too small (*count holds the size needed)");
  int i = 0;
  for (const auto &kv : acc) {
    out[i].smearing = std::get<0>(kv.first);
    out[i].time_size = std::get<1>(kv.first);
    out[i].space_size = std::get<2>(kv.first);
    out[i].wilson_loop = kv.second / 6;
    i++;
  }
  return GC_OK;
}

// Offsets (Dx, Dy, Dz) that polyakov_loop_correlator_{singlet,color_average}
// visit (polyakov_loops.h:100-113, 163-176): Dz, Dy in [-D, D]; Dx from 0 when
// Dy and Dz are both non-zero, else from -D; |D| <= D_max. w = the entry's
// place in the (2 D_max + 1)^3 table.
static std::vector<int4> correlator_offsets(int D) {
  std::vector<int4> v;
  const int n = 2 * D + 1;
  for (int dz = -D; dz <= D; dz++)
    for (int dy = -D; dy <= D; dy++) {
      const int dx_min = (dy != 0 && dz != 0) ? 0 : -D;
      for (int dx = dx_min; dx <= D; dx++)
        if (std::sqrt((double)(dx * dx + dy * dy + dz * dz)) <= D)
          v.push_back(make_int4(dx, dy, dz, (dz + D) * n * n + (dy + D) * n + dx + D));
    }
  return v;
}

// Polyakov lines into h->aux (FP64 planes); optionally the loop average.
static int polyakov_lines(gc_lattice *h, size_t extra_bytes, double *loop_dev) {
  const size_t lines_bytes = (size_t)(h->nc == 3 ? 9 : 2) * h->g.Vs * sizeof(double2);
  int rc = ensure_aux(h, ((lines_bytes + 255) / 256) * 256 + extra_bytes);
  if (rc)
    return rc;
  rc = ensure_partials(h, (h->g.Vs + 255) / 256);
  if (rc)
    return rc;
  rc = GC_DISPATCH(h, launch_polyakov_lines, h->g, h->cur, (double2 *)h->aux, h->partials,
                   loop_dev, h->stream);
  return rc ? launch_fail(h, rc) : GC_OK;
}

int gc_polyakov_loop(gc_lattice *h, double *out) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  if (!out)
    return fail(h, GC_ERR_ARG, "null output");
  std::lock_guard<std::mutex> lk(h->mu);
  rc = ensure_dev_out(h, 1);
  if (rc)
    return rc;
  rc = polyakov_lines(h, 0, h->dev_out);
  if (rc)
    return rc;
  cudaError_t e = cudaMemcpyAsync(out, h->dev_out, sizeof(double), cudaMemcpyDeviceToHost,
                                  h->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(h->stream);
  return e == cudaSuccess ? GC_OK : cuda_fail(h, "Polyakov loop result", e);
}

int gc_polyakov_correlator(gc_lattice *h, int d_max, int kind, double *out) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  if (!out)
    return fail(h, GC_ERR_ARG, "null output");
  if (d_max < 0)
    return fail(h, GC_ERR_ARG, "D_max must be >= 0");
  if (kind != GC_POLYAKOV_COLOR_AVERAGE && kind != GC_POLYAKOV_SINGLET)
    return fail(h, GC_ERR_ARG, "unknown correlator kind");
  const size_t n = (size_t)(2 * d_max + 1) * (2 * d_max + 1) * (2 * d_max + 1);
  if (n > (size_t)1 << 24)
    return fail(h, GC_ERR_ARG, "D_max too large");
  std::lock_guard<std::mutex> lk(h->mu);
  const std::vector<int4> offs = correlator_offsets(d_max);
  rc = ensure_dev_out(h, n);
  if (rc)
    return rc;
  rc = polyakov_lines(h, offs.size() * sizeof(int4), nullptr);
  if (rc)
    return rc;
  const size_t lines_bytes = (size_t)(h->nc == 3 ? 9 : 2) * h->g.Vs * sizeof(double2);
  int4 *dev_offs = (int4 *)((char *)h->aux + ((lines_bytes + 255) / 256) * 256);
  cudaError_t e = cudaMemcpyAsync(dev_offs, offs.data(), offs.size() * sizeof(int4),
                                  cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(h->dev_out, 0, n * sizeof(double), h->stream);
  if (e != cudaSuccess)
    return cuda_fail(h, "Polyakov correlator setup", e);
  rc = launch_polyakov_correlator(h->g, h->nc, (const double2 *)h->aux, dev_offs,
                                  (int)offs.size(), kind == GC_POLYAKOV_SINGLET, h->dev_out,
                                  h->stream);
  if (rc)
    return launch_fail(h, rc);
  e = cudaMemcpyAsync(out, h->dev_out, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(h->stream);
  return e == cudaSuccess ? GC_OK : cuda_fail(h, "Polyakov correlator result", e);
}

int gc_read_config(gc_lattice *h, const char *path, const char *format,
                   long long bytes_skip, const char *precision, int convert) {
  if (!h || !path || !format)
    return fail(h, GC_ERR_ARG, "null argument");
  long long offset = 0, length = 0;
  std::string err;
  int rc = gc::probe_config(h->g.L, h->nc, path, format, bytes_skip, precision, &offset,
                            &length, err);
  if (rc)
    return fail(h, rc, err);
  std::lock_guard<std::mutex> lk(h->mu);
  rc = ensure_staging(h);
  if (!rc)
    rc = ensure_io(h);
  if (rc)
    return rc;
  // chunk k of the file goes through pinned buffer k % 2: its read waits only
  // for the copy of chunk k - 2 out of the same buffer
  FILE *f = std::fopen(path, "rb");
  bool ok = f && std::fseek(f, (long)offset, SEEK_SET) == 0;
  cudaError_t e = cudaSuccess;
  unsigned char *dst = reinterpret_cast<unsigned char *>(h->staging);
  for (size_t done = 0, k = 0; ok && e == cudaSuccess && done < (size_t)length; k ^= 1) {
    const size_t n = std::min(kIoChunk, (size_t)length - done);
    e = cudaEventSynchronize(h->io_ev[k]);
    if (e != cudaSuccess)
      break;
    ok = std::fread(h->io_buf[k], 1, n, f) == n;
    if (!ok)
      break;
    e = cudaMemcpyAsync(dst + done, h->io_buf[k], n, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
      e = cudaEventRecord(h->io_ev[k], h->stream);
    done += n;
  }
  if (f)
    std::fclose(f);
  if (e == cudaSuccess && ok) {
    rc = gc::launch_file_to_soa(h->g, h->nc, h->prec, format, precision, convert != 0,
                                reinterpret_cast<const unsigned char *>(h->staging), h->cur,
                                h->stream);
    e = cudaStreamSynchronize(h->stream);
  } else {
    cudaStreamSynchronize(h->stream); // the chunks in flight finish before a retry reuses them
  }
  if (!ok)
    return fail(h, GC_ERR_IO, std::string("read failed: ") + path);
  if (rc)
    return launch_fail(h, rc);
  if (e != cudaSuccess)
    return cuda_fail(h, "read_config", e);
  h->has_links = true;
  return GC_OK;
}

int gc_write_config(gc_lattice *h, const char *path) {
  int rc = check_ready(h);
  if (rc)
    return rc;
  if (!path)
    return fail(h, GC_ERR_ARG, "null path");
  const size_t bytes = (size_t)(h->nc == 3 ? 18 : 4) * 4 * (size_t)h->g.V * sizeof(double);
  std::lock_guard<std::mutex> lk(h->mu);
  rc = ensure_staging(h);
  if (!rc)
    rc = ensure_io(h);
  if (rc)
    return rc;
  rc = launch_soa_to_aos(h->g, h->nc, h->prec, GC_LAYOUT_ROWMAJOR, h->cur, h->staging,
                         h->stream);
  if (rc)
    return launch_fail(h, rc);
  // chunk k is copied into buffer k % 2 while chunk k - 1 is written out
  const unsigned char *src = reinterpret_cast<const unsigned char *>(h->staging);
  const size_t nchunks = (bytes + kIoChunk - 1) / kIoChunk;
  auto issue = [&](size_t k) {
    const size_t off = k * kIoChunk, n = std::min(kIoChunk, bytes - off);
    cudaError_t e = cudaMemcpyAsync(h->io_buf[k & 1], src + off, n, cudaMemcpyDeviceToHost,
                                    h->stream);
    return e == cudaSuccess ? cudaEventRecord(h->io_ev[k & 1], h->stream) : e;
  };
  FILE *f = std::fopen(path, "wb");
  bool ok = f != nullptr;
  cudaError_t e = ok && nchunks ? issue(0) : cudaSuccess;
  for (size_t k = 0; ok && e == cudaSuccess && k < nchunks; k++) {
    if (k + 1 < nchunks)
      e = issue(k + 1);
    if (e == cudaSuccess)
      e = cudaEventSynchronize(h->io_ev[k & 1]);
    if (e != cudaSuccess)
      break;
    const size_t n = std::min(kIoChunk, bytes - k * kIoChunk);
    ok = std::fwrite(h->io_buf[k & 1], 1, n, f) == n;
  }
  cudaStreamSynchronize(h->stream);
  if (f)
    ok = (std::fclose(f) == 0) && ok;
  if (e != cudaSuccess)
    return cuda_fail(h, "write_config", e);
  if (!ok)
    return fail(h, GC_ERR_IO, std::string("write failed: ") + path);
  return GC_OK;
}

int gc_generate_host(const int dims[4], int nc, double eps, unsigned int seed,
                     unsigned int config_index, int gauge, double *host) {
  if (!dims || !host)
    return fail(nullptr, GC_ERR_ARG, "null argument");
  if (nc != 2 && nc != 3)
    return fail(nullptr, GC_ERR_ARG, "nc must be 2 or 3");
  for (int d = 0; d < 4; d++)
    if (dims[d] < 2)
      return fail(nullptr, GC_ERR_ARG, "every lattice extent must be >= 2");
  return gc::generate_host(dims, nc, eps, seed, config_index, gauge, host);
}

int gc_generate(gc_lattice *h, double eps, unsigned int seed,
                unsigned int config_index, int gauge) {
  if (!h)
    return fail(nullptr, GC_ERR_ARG, "null handle");
  const size_t n = (size_t)(h->nc == 3 ? 18 : 4) * 4 * (size_t)h->g.V;
  double *buf = nullptr;
  cudaError_t e = cudaMallocHost(&buf, n * sizeof(double));
  if (e != cudaSuccess)
    return cuda_fail(h, "cudaMallocHost(generator)", e);
  int rc = gc::generate_host(h->g.L, h->nc, eps, seed, config_index, gauge, buf);
  if (rc == GC_OK) {
    rc = gc_upload(h, buf, GC_LAYOUT_ROWMAJOR);
    if (rc == GC_OK)
      rc = gc_synchronize(h);
  }
  cudaFreeHost(buf);
  return rc;
}

long long gc_job_device_bytes(const int dims[4], int nc, int precision,
                              int rmax, int tmax) {
  if (!dims || (nc != 2 && nc != 3))
    return -1;
  long long V = 1;
  for (int d = 0; d < 4; d++)
    V *= dims[d];
  const long long field = ((long long)bytes_per_link(nc, precision) * V + 255) / 256 * 256;
  const long long staging = (long long)(nc == 3 ? 18 : 4) * 8 * 4 * V;
  Geom g{};
  for (int d = 0; d < 4; d++)
    g.L[d] = dims[d];
  g.V = (int)V;
  g.Vs = dims[0] * dims[1] * dims[2];
  const int nr = std::max(1, rmax), nt = std::max(1, tmax);
  const long long partials =
      (long long)wilson_auto_partials_count(g, std::min(nr, std::max(1, 1024 / nt)), nt, nc) *
      8;
  const long long hfield =
      ((long long)inter_link_bytes(nc, precision) * V + 255) / 256 * 256;
  return 8 * field + 15 * hfield + staging + partials + 64LL * 1024;
}

} // extern "C"
