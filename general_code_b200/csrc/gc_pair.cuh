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
__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return f2(__fadd2_rn(a.v, b.v)); }
// a - b with one rounding, as fma(b, -1, a)
__device__ __forceinline__ f2 operator-(f2 a, f2 b) {
  return f2(__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v));
}

// Products of lane-packed SU(3) matrices. Each complex sum of products is
// split into its added and its subtracted products, accumulated as two fused
// chains and subtracted once: a packed instruction has no per-operand sign,
// so this takes one subtraction per element where the generic templates
// would negate an operand for every product term.
//   mul    C = A B     : re = sum A.re B.re - sum A.im B.im,
//                        im = sum (A.re B.im + A.im B.re)
//   mul_ad C = A B^dag : re = sum (A.re B.re + A.im B.im),
//                        im = sum A.im B.re - sum A.re B.im
//   mul_da C = A^dag B : re = sum (A.re B.re + A.im B.im),
//                        im = sum A.re B.im - sum A.im B.re
__device__ __forceinline__ SU3<f2> mul(const SU3<f2> &A, const SU3<f2> &B) {
  SU3<f2> C;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      f2 p = A.e[i][0].re * B.e[0][j].re;
      f2 q = A.e[i][0].im * B.e[0][j].im;
      f2 im = A.e[i][0].re * B.e[0][j].im;
      im = fma(A.e[i][0].im, B.e[0][j].re, im);
#pragma unroll
      for (int k = 1; k < 3; k++) {
        p = fma(A.e[i][k].re, B.e[k][j].re, p);
        q = fma(A.e[i][k].im, B.e[k][j].im, q);
        im = fma(A.e[i][k].re, B.e[k][j].im, im);
        im = fma(A.e[i][k].im, B.e[k][j].re, im);
      }
      C.e[i][j] = {p - q, im};
    }
  return C;
}
__device__ __forceinline__ SU3<f2> mul_ad(const SU3<f2> &A, const SU3<f2> &B) {
  SU3<f2> C;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      f2 re = A.e[i][0].re * B.e[j][0].re;
      re = fma(A.e[i][0].im, B.e[j][0].im, re);
      f2 p = A.e[i][0].im * B.e[j][0].re;
      f2 q = A.e[i][0].re * B.e[j][0].im;
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = fma(A.e[i][k].re, B.e[j][k].re, re);
        re = fma(A.e[i][k].im, B.e[j][k].im, re);
        p = fma(A.e[i][k].im, B.e[j][k].re, p);
        q = fma(A.e[i][k].re, B.e[j][k].im, q);
      }
      C.e[i][j] = {re, p - q};
    }
  return C;
}
__device__ __forceinline__ SU3<f2> mul_da(const SU3<f2> &A, const SU3<f2> &B) {
  SU3<f2> C;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      f2 re = A.e[0][i].re * B.e[0][j].re;
      re = fma(A.e[0][i].im, B.e[0][j].im, re);
      f2 p = A.e[0][i].re * B.e[0][j].im;
      f2 q = A.e[0][i].im * B.e[0][j].re;
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = fma(A.e[k][i].re, B.e[k][j].re, re);
        re = fma(A.e[k][i].im, B.e[k][j].im, re);
        p = fma(A.e[k][i].re, B.e[k][j].im, p);
        q = fma(A.e[k][i].im, B.e[k][j].re, q);
      }
      C.e[i][j] = {re, p - q};
    }
  return C;
}

// Rows 0 and 1 of two 12-real FP32 links (lane 0 = p0, lane 1 = p1: float4
// pointers to the first of the link's three planes, plane stride V), third
// row rebuilt as conj(row0 x row1) in packed arithmetic.
__device__ __forceinline__ SU3<f2> load_pair_f32su3(const float4 *p0, const float4 *p1,
                                                    size_t V) {
  const float4 a0 = __ldg(p0), b0 = __ldg(p0 + V), c0 = __ldg(p0 + 2 * V);
  const float4 a1 = __ldg(p1), b1 = __ldg(p1 + V), c1 = __ldg(p1 + 2 * V);
  SU3<f2> u;
  u.e[0][0] = {f2(make_float2(a0.x, a1.x)), f2(make_float2(a0.y, a1.y))};
  u.e[0][1] = {f2(make_float2(a0.z, a1.z)), f2(make_float2(a0.w, a1.w))};
  u.e[0][2] = {f2(make_float2(b0.x, b1.x)), f2(make_float2(b0.y, b1.y))};
  u.e[1][0] = {f2(make_float2(b0.z, b1.z)), f2(make_float2(b0.w, b1.w))};
  u.e[1][1] = {f2(make_float2(c0.x, c1.x)), f2(make_float2(c0.y, c1.y))};
  u.e[1][2] = {f2(make_float2(c0.z, c1.z)), f2(make_float2(c0.w, c1.w))};
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const int a = (j + 1) % 3, b = (j + 2) % 3;
    // conj(u0a u1b - u0b u1a)
    const cx<f2> x = u.e[0][a], y = u.e[1][b], z = u.e[0][b], w = u.e[1][a];
    const f2 pre = fma(x.im, y.im, z.re * w.re);  // x.im y.im + z.re w.re
    const f2 qre = fma(z.im, w.im, x.re * y.re);  // z.im w.im + x.re y.re
    const f2 pim = fma(z.im, w.re, z.re * w.im);  // im of z w
    const f2 qim = fma(x.im, y.re, x.re * y.im);  // im of x y
    u.e[2][j] = {qre - pre, pim - qim};
  }
  return u;
}

// Two 18-real FP32 matrices (9 planes of float2, element (k/3, k%3); lane 0
// at p0, lane 1 at p1, plane stride V) as one lane-packed matrix.
__device__ __forceinline__ SU3<f2> load_pair_f32full(const float2 *p0, const float2 *p1,
                                                     size_t V) {
  SU3<f2> u;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const float2 a = __ldg(p0 + k * V), b = __ldg(p1 + k * V);
    u.e[k / 3][k % 3] = {f2(make_float2(a.x, b.x)), f2(make_float2(a.y, b.y))};
  }
  return u;
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
