// Vector FMA throughput of the device, measured: the denominator of the
// compute roofline of kernels bound by the FP32 or FP64 pipe (the smearing
// and Wilson-loop kernels), in the same run as the kernels it is compared
// with. Each thread runs 8 independent fused multiply-add chains (packed
// FP32x2 for FP32, the form the mixed kernels use; scalar FP64), enough to
// cover the pipe latency at full occupancy.
#include "../../include/gc_lattice.h"
#include "gc_internal.cuh"
#include "gc_kernels.h"

#include <cuda_runtime.h>
#include <string>

namespace gc {
int record_error(int code, const std::string &msg);
}

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) fma_chains_f32(float *out, float m, float c) {
  float2 a[kChains];
#pragma unroll
  for (int i = 0; i < kChains; i++)
    a[i] = make_float2(threadIdx.x * 1e-3f + i, blockIdx.x * 1e-3f - i);
  const float2 mm = make_float2(m, m), cc = make_float2(c, c);
#pragma unroll 1
  for (int it = 0; it < kIters; it++) {
#pragma unroll
    for (int i = 0; i < kChains; i++)
      a[i] = __ffma2_rn(a[i], mm, cc);
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < kChains; i++)
    s += a[i].x + a[i].y;
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) fma_chains_f64(double *out, double m, double c) {
  double a[kChains];
#pragma unroll
  for (int i = 0; i < kChains; i++)
    a[i] = threadIdx.x * 1e-3 + blockIdx.x * 1e-6 + i;
#pragma unroll 1
  for (int it = 0; it < kIters; it++) {
#pragma unroll
    for (int i = 0; i < kChains; i++)
      a[i] = fma(a[i], m, c);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kChains; i++)
    s += a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

} // namespace

extern "C" int gc_fma_peak(int precision, double *tflops) {
  if (!tflops || (precision != GC_PREC_FP64 && precision != GC_PREC_MIXED))
    return gc::record_error(GC_ERR_ARG, "gc_fma_peak: bad argument");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || !sms)
    return gc::record_error(GC_ERR_NODEVICE, "gc_fma_peak: no device");
  const int blocks = sms * 8; // 2048 threads per SM
  void *out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * kThreads * sizeof(double)) != cudaSuccess)
    return gc::record_error(GC_ERR_NOMEM, "gc_fma_peak: cudaMalloc");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // (m, c) keep the chains bounded: a -> 0.5 a + 0.25 converges to 0.5
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) { // the first launch warms up
    cudaEventRecord(e0);
    if (precision == GC_PREC_MIXED)
      fma_chains_f32<<<blocks, kThreads>>>(static_cast<float *>(out), 0.5f, 0.25f);
    else
      fma_chains_f64<<<blocks, kThreads>>>(static_cast<double *>(out), 0.5, 0.25);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best)
      best = ms;
  }
  const cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess)
    return gc::record_error(GC_ERR_CUDA, std::string("gc_fma_peak: ") + cudaGetErrorString(e));
  const double lanes = precision == GC_PREC_MIXED ? 2.0 : 1.0;
  const double flops = 2.0 * lanes * kChains * kIters * (double)blocks * kThreads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return GC_OK;
}
