// Two FP32 lanes packed in one register pair, with the sm_100 packed FP32x2
// arithmetic (one FMUL2/FFMA2 instruction computes both lanes). A thread that
// carries two independent matrices (two lattice sites) as SU3<f2> issues half
// as many arithmetic instructions as two SU3<float> computations, with the
// same per-lane rounding (each lane is an FP32 round-to-nearest multiply or
// fused multiply-add, exactly as the scalar operation).
//
// f2 provides what the algebra templates in gc_algebra.cuh use for the
// matrix products: construction from a scalar, *, unary -, and fma().
#pragma once

#include "gc_algebra.cuh"
#include <cuda_runtime.h>

namespace gc {

struct f2 {
  float2 v;
  f2() = default;
  __device__ __forceinline__ explicit f2(float x) : v(make_float2(x, x)) {}
  __device__ __forceinline__ f2(float2 a) : v(a) {}
};

__device__ __forceinline__ f2 operator*(f2 a, f2 b) { return f2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ f2 operator-(f2 a) {
  return f2(__fmul2_rn(a.v, make_float2(-1.0f, -1.0f)));
}
// (the scalar overloads stay visible to the algebra templates in namespace gc)
using ::fma;
__device__ __forceinline__ f2 fma(f2 a, f2 b, f2 c) {
  return f2(__ffma2_rn(a.v, b.v, c.v));
}

// Two SU(3) matrices -> one SU3<f2> (lane 0 = a, lane 1 = b) and back.
__device__ __forceinline__ SU3<f2> zip(const SU3<float> &a, const SU3<float> &b) {
  SU3<f2> z;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      z.e[i][j].re = f2(make_float2(a.e[i][j].re, b.e[i][j].re));
      z.e[i][j].im = f2(make_float2(a.e[i][j].im, b.e[i][j].im));
    }
  return z;
}

} // namespace gc
