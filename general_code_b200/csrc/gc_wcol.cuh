// Shared pieces of the on-axis Wilson-loop kernels (gc_wilson.cu: the exact
// T-walk recursion; gc_wilson_gauge.cu: the temporal-gauge form): the layout
// of matrices kept in shared memory, the per-loop trace values, warp sums and
// lane-packed link loads.
#pragma once

#include "gc_internal.cuh"
#include "gc_kernels.h"
#include "gc_pair.cuh"

namespace gc {

namespace {

// ------------------------------------------------------ shared column storage
// A block keeps three sets of matrices in shared memory (space lines, own
// time links, neighbour time links), one slot per (t, column unit), slot
// index t * cs + u. SU(3) slots are contiguous 144-byte records, read and
// written as 16-byte vectors at immediate offsets from one address per slot:
//   SU3<double>: element k at double2 [9 i + k]  = (re, im)
//   SU3<f2>    : element k at float4  [9 i + k]  = (re lane0, re lane1,
//                                                   im lane0, im lane1)
// Consecutive threads hold consecutive slots (a 144-byte = 36-word stride),
// so each quarter-warp phase of a 16-byte access covers all 32 banks once.
// SU(2) slots (16 or 32 bytes) stay element-major planes of 2-vectors,
// element pair k of slot i at [k * nslots + i].
template <class M> struct ColSet;
template <> struct ColSet<SU3<double>> {
  static constexpr int kBytes = 144;
  __device__ __forceinline__ static void store(unsigned char *set, int, int i,
                                               const SU3<double> &m) {
    double2 *p = reinterpret_cast<double2 *>(set) + 9 * i;
#pragma unroll
    for (int k = 0; k < 9; k++)
      p[k] = make_double2(m.e[k / 3][k % 3].re, m.e[k / 3][k % 3].im);
  }
  __device__ __forceinline__ static SU3<double> load(const unsigned char *set, int, int i) {
    const double2 *p = reinterpret_cast<const double2 *>(set) + 9 * i;
    SU3<double> m;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const double2 v = p[k];
      m.e[k / 3][k % 3] = {v.x, v.y};
    }
    return m;
  }
};
template <> struct ColSet<SU3<f2>> {
  static constexpr int kBytes = 144;
  __device__ __forceinline__ static void store(unsigned char *set, int, int i,
                                               const SU3<f2> &m) {
    float4 *p = reinterpret_cast<float4 *>(set) + 9 * i;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const float2 re = m.e[k / 3][k % 3].re.v, im = m.e[k / 3][k % 3].im.v;
      p[k] = make_float4(re.x, re.y, im.x, im.y);
    }
  }
  __device__ __forceinline__ static SU3<f2> load(const unsigned char *set, int, int i) {
    const float4 *p = reinterpret_cast<const float4 *>(set) + 9 * i;
    SU3<f2> m;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const float4 v = p[k];
      m.e[k / 3][k % 3].re = f2(make_float2(v.x, v.y));
      m.e[k / 3][k % 3].im = f2(make_float2(v.z, v.w));
    }
    return m;
  }
};
template <class T> struct V2;
template <> struct V2<double> {
  using type = double2;
};
template <> struct V2<float> {
  using type = float2;
};
template <class T> struct ColSet<SU2<T>> {
  using VT = typename V2<T>::type;
  static constexpr int kBytes = 2 * sizeof(VT);
  __device__ __forceinline__ static void store(unsigned char *set, int nslots, int i,
                                               const SU2<T> &m) {
    VT *p = reinterpret_cast<VT *>(set);
    p[i] = {m.a0, m.a1};
    p[nslots + i] = {m.a2, m.a3};
  }
  __device__ __forceinline__ static SU2<T> load(const unsigned char *set, int nslots, int i) {
    const VT *p = reinterpret_cast<const VT *>(set);
    const VT a = p[i], b = p[nslots + i];
    return {a.x, a.y, b.x, b.y};
  }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ------------------------------------------------------------ loop values
// The per-loop quantity from the loop's trace Tr[S K^dag], summed over the
// thread's active lanes in FP64: the fundamental Re Tr W (multiply_conj_tr,
// matrix.h:54-56, 260-262; the 1/N normalisation is applied once to the
// final sums) or, with ADJ, the adjoint character |Tr W|^2 - 1
// (multiply_conj_tr_adjoint / tr_adjoint, matrix.h:62-65, 264-270; SU(2):
// 4 (a.b)^2 - 1).
template <bool ADJ, class T>
__device__ __forceinline__ double loop_value(const SU3<T> &a, const SU3<T> &b, bool) {
  if (!ADJ) {
    T s = a.e[0][0].re * b.e[0][0].re;
    s = GC_FMA(a.e[0][0].im, b.e[0][0].im, s);
#pragma unroll
    for (int k = 1; k < 9; k++) {
      s = GC_FMA(a.e[k / 3][k % 3].re, b.e[k / 3][k % 3].re, s);
      s = GC_FMA(a.e[k / 3][k % 3].im, b.e[k / 3][k % 3].im, s);
    }
    return double(s);
  }
  T re = a.e[0][0].re * b.e[0][0].re;
  T im = a.e[0][0].im * b.e[0][0].re;
  re = GC_FMA(a.e[0][0].im, b.e[0][0].im, re);
  im = GC_FMA(-a.e[0][0].re, b.e[0][0].im, im);
#pragma unroll
  for (int k = 1; k < 9; k++) {
    re = GC_FMA(a.e[k / 3][k % 3].re, b.e[k / 3][k % 3].re, re);
    re = GC_FMA(a.e[k / 3][k % 3].im, b.e[k / 3][k % 3].im, re);
    im = GC_FMA(a.e[k / 3][k % 3].im, b.e[k / 3][k % 3].re, im);
    im = GC_FMA(-a.e[k / 3][k % 3].re, b.e[k / 3][k % 3].im, im);
  }
  const double r = double(re), i = double(im);
  return fma(r, r, fma(i, i, -1.0));
}
template <bool ADJ, class T>
__device__ __forceinline__ double loop_value(const SU2<T> &a, const SU2<T> &b, bool) {
  T s = a.a0 * b.a0;
  s = GC_FMA(a.a1, b.a1, s);
  s = GC_FMA(a.a2, b.a2, s);
  s = GC_FMA(a.a3, b.a3, s);
  const double d = double(s);
  return ADJ ? 4.0 * d * d - 1.0 : d;
}
// Two lanes (lane 1 counted only when active).
template <bool ADJ>
__device__ __forceinline__ double loop_value(const SU3<f2> &a, const SU3<f2> &b, bool lane1) {
  if (!ADJ) {
    f2 s = a.e[0][0].re * b.e[0][0].re;
    s = fma(a.e[0][0].im, b.e[0][0].im, s);
#pragma unroll
    for (int k = 1; k < 9; k++) {
      s = fma(a.e[k / 3][k % 3].re, b.e[k / 3][k % 3].re, s);
      s = fma(a.e[k / 3][k % 3].im, b.e[k / 3][k % 3].im, s);
    }
    const double v0 = double(s.v.x);
    return lane1 ? v0 + double(s.v.y) : v0;
  }
  f2 re = a.e[0][0].re * b.e[0][0].re;
  f2 im = a.e[0][0].im * b.e[0][0].re;
  re = fma(a.e[0][0].im, b.e[0][0].im, re);
  im = fma(-a.e[0][0].re, b.e[0][0].im, im);
#pragma unroll
  for (int k = 1; k < 9; k++) {
    re = fma(a.e[k / 3][k % 3].re, b.e[k / 3][k % 3].re, re);
    re = fma(a.e[k / 3][k % 3].im, b.e[k / 3][k % 3].im, re);
    im = fma(a.e[k / 3][k % 3].im, b.e[k / 3][k % 3].re, im);
    im = fma(-a.e[k / 3][k % 3].re, b.e[k / 3][k % 3].im, im);
  }
  const double r0 = double(re.v.x), i0 = double(im.v.x);
  const double v0 = fma(r0, r0, fma(i0, i0, -1.0));
  if (!lane1)
    return v0;
  const double r1 = double(re.v.y), i1 = double(im.v.y);
  return v0 + fma(r1, r1, fma(i1, i1, -1.0));
}

// Matrix of `lanes` adjacent sites from a link field (lane 1 = site s1).
template <class Store, class CT, int LANES> struct LaneLoad {
  using M = typename Store::template M<CT>;
  __device__ __forceinline__ static M load(const void *f, size_t V, int s0, int) {
    return Store::template load<CT>(f, V, s0);
  }
};
template <> struct LaneLoad<StoreF32SU3, float, 2> {
  using M = SU3<f2>;
  __device__ __forceinline__ static M load(const void *f, size_t V, int s0, int s1) {
    return zip(StoreF32SU3::load<float>(f, V, s0), StoreF32SU3::load<float>(f, V, s1));
  }
};


} // namespace

} // namespace gc
