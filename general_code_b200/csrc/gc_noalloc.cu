// W(R,T) for callers that cannot allocate device memory.
//
// Some programs cannot let a library call cudaMalloc: an application whose
// own allocator owns the whole device-memory budget and must account for
// every byte, or a timing-critical loop in which cudaMalloc / cudaFree would
// synchronise the device and stall every stream. gc_wilson_onaxis_noalloc
// serves them. The caller passes the link fields (device memory it owns, in
// this library's device layout) and a device buffer for the result; the
// working memory the Wilson-loop kernel needs — one partial sum per (block,
// R, T) and a per-chunk result table — is the fixed array below, which the
// CUDA runtime places in the library's static device memory when the
// library's module is loaded. No cudaMalloc, cudaFree, cudaMallocHost or
// allocating library routine is called on this path.
//
// Size: 16 MiB (2,097,152 doubles) per GPU, held until the process exits.
// The array belongs to the library's device module, and the CUDA runtime
// loads modules lazily: the 16 MiB are taken on a device when the module is
// loaded there, which is the first call of this entry point on that device
// (its cudaGetSymbolAddress), unless another entry point of the library ran
// on that device before. A caller whose allocator claims the device budget
// should therefore make one call before the allocator takes its share; if the
// device has no room left then, the call fails with GC_ERR_NOMEM. One value
// of R needs blocks*nT + nT doubles, where blocks = 3 * ceil(Lx*Ly*Lz /
// columns_per_block); larger R ranges are done in chunks of R. A lattice for
// which even one R does not fit is rejected with GC_ERR_ARG (SU(3) 24^4 with T
// up to 12 needs 49,800 doubles per R).
//
// Set-up: every call looks up the array's device address with
// cudaGetSymbolAddress while the caller's device is current (the host-side
// name of a __device__ array is not a device address), so the address stays
// right after cudaDeviceReset re-creates the context. The first call for each
// group and precision on a device also raises the W kernel's shared-memory
// limit (cudaFuncSetAttribute): make that first call outside stream capture.
//
// Sharing: all calls in the process use the same array and it keeps the last
// call's contents. Every element a call reads was written earlier in the same
// call, so nothing has to start at zero. Two calls whose work overlaps on the
// GPU (different streams, or different host threads) race on the array and
// give wrong results: serialise them.
#include "../../include/gc_lattice.h"
#include "gc_internal.cuh"
#include "gc_kernels.h"

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>

namespace gc {
int record_error(int code, const std::string &msg);
const std::string &last_launch_error();
} // namespace gc

namespace {

constexpr size_t kNoAllocScratchDoubles = (size_t(16) << 20) / sizeof(double);
constexpr int kMaxDevices = 64;

} // namespace

static __device__ __align__(256) double g_wilson_scratch[kNoAllocScratchDoubles];

namespace {

std::mutex g_setup_mu;
bool g_checked[kMaxDevices] = {};

// Device address of g_wilson_scratch on the current device. The address is
// looked up on every call (a host-side table lookup once the module is
// loaded), so a context re-created by cudaDeviceReset gets its own address.
int scratch_for_current_device(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return gc::record_error(GC_ERR_NODEVICE,
                            std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return gc::record_error(GC_ERR_NODEVICE, "device ordinal out of range");
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_checked[dev]) {
      int major = 0;
      e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
      if (e != cudaSuccess)
        return gc::record_error(GC_ERR_NODEVICE,
                                std::string("no CUDA device: ") + cudaGetErrorString(e));
      if (major != 10)
        return gc::record_error(GC_ERR_NODEVICE,
                                "device is not sm_100 (this library is built for sm_100a only)");
      g_checked[dev] = true;
    }
  }
  void *p = nullptr;
  e = cudaGetSymbolAddress(&p, g_wilson_scratch);
  if (e == cudaErrorMemoryAllocation)
    return gc::record_error(GC_ERR_NOMEM,
                            "gc_wilson_onaxis_noalloc: loading the library's device module "
                            "needs 16 MiB of free device memory for the fixed scratch array; "
                            "make the first call before the device memory is claimed");
  if (e != cudaSuccess || p == nullptr)
    return gc::record_error(GC_ERR_CUDA,
                            std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  *out = static_cast<double *>(p);
  return GC_OK;
}

} // namespace

extern "C" int gc_wilson_onaxis_noalloc(const int dims[4], int nc, int precision,
                                        const void *const fields[4], int rmin,
                                        int rmax, int tmin, int tmax,
                                        double *out_dev, void *cuda_stream) {
  using namespace gc;
  if (!dims || !fields || !out_dev)
    return record_error(GC_ERR_ARG, "gc_wilson_onaxis_noalloc: null argument");
  if (nc != 2 && nc != 3)
    return record_error(GC_ERR_ARG, "gc_wilson_onaxis_noalloc: nc must be 2 or 3");
  if (precision != GC_PREC_FP64 && precision != GC_PREC_MIXED)
    return record_error(GC_ERR_ARG, "gc_wilson_onaxis_noalloc: unknown precision");
  long long V = 1;
  for (int d = 0; d < 4; d++) {
    if (dims[d] < 2)
      return record_error(GC_ERR_ARG, "gc_wilson_onaxis_noalloc: every extent must be >= 2");
    V *= dims[d];
  }
  if (V >= (1LL << 30))
    return record_error(GC_ERR_ARG, "gc_wilson_onaxis_noalloc: lattice too large");
  for (int d = 0; d < 4; d++)
    if (!fields[d])
      return record_error(GC_ERR_ARG, "gc_wilson_onaxis_noalloc: null link field");
  if (rmin < 1 || tmin < 1 || rmax < rmin || tmax < tmin)
    return record_error(GC_ERR_ARG,
                        "gc_wilson_onaxis_noalloc: need 1 <= r_min <= r_max and "
                        "1 <= time_min <= time_max");
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  if (nt > 1024)
    return record_error(GC_ERR_ARG,
                        "gc_wilson_onaxis_noalloc: at most 1024 values of T");

  Geom g{};
  for (int d = 0; d < 4; d++)
    g.L[d] = dims[d];
  g.stride[0] = 1;
  g.stride[1] = dims[0];
  g.stride[2] = dims[0] * dims[1];
  g.stride[3] = dims[0] * dims[1] * dims[2];
  g.V = (int)V;
  g.Vs = dims[0] * dims[1] * dims[2];

  const size_t blocks = (size_t)wilson_max_blocks(g, nc);
  const size_t per_r = blocks * nt + nt;
  const size_t fit = kNoAllocScratchDoubles / per_r;
  if (fit < 1) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "gc_wilson_onaxis_noalloc: one value of R needs %zu doubles of "
                  "scratch; the fixed scratch holds %zu (16 MiB)",
                  per_r, kNoAllocScratchDoubles);
    return record_error(GC_ERR_ARG, msg);
  }
  const int ncr = (int)std::min<size_t>({(size_t)nr, (size_t)(1024 / nt), fit});

  double *scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc)
    return rc;
  double *partials = scratch;
  double *chunk_out = scratch + blocks * ncr * nt;

  Fields4 U;
  for (int d = 0; d < 4; d++)
    U.f[d] = const_cast<void *>(fields[d]);
  cudaStream_t s = (cudaStream_t)cuda_stream;
  for (int r0 = rmin; r0 <= rmax; r0 += ncr) {
    const int r1 = std::min(rmax, r0 + ncr - 1);
    const int nc_r = r1 - r0 + 1;
    if (nc == 3)
      rc = precision == GC_PREC_FP64
               ? launch_wilson<StoreF64SU3, double>(g, U, r0, r1, tmin, tmax, partials, chunk_out, s)
               : launch_wilson<StoreF32SU3, float>(g, U, r0, r1, tmin, tmax, partials, chunk_out, s);
    else
      rc = precision == GC_PREC_FP64
               ? launch_wilson<StoreF64SU2, double>(g, U, r0, r1, tmin, tmax, partials, chunk_out, s)
               : launch_wilson<StoreF32SU2, float>(g, U, r0, r1, tmin, tmax, partials, chunk_out, s);
    if (rc)
      return record_error(rc, last_launch_error());
    cudaError_t e = cudaMemcpy2DAsync(out_dev + (r0 - rmin), nr * sizeof(double), chunk_out,
                                      nc_r * sizeof(double), nc_r * sizeof(double), nt,
                                      cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess)
      return record_error(GC_ERR_CUDA, std::string("cudaMemcpy2DAsync: ") +
                                           cudaGetErrorString(e));
  }
  return GC_OK;
}
