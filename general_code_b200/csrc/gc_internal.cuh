// Internal device-side types: lattice geometry, structure-of-arrays link
// storage, and the launch helpers shared by the kernels.
//
// Device layout (one "field" = one link direction, or one decorated-link
// field of HYP, or one line field): component planes, each V sites long, so
// that consecutive threads (consecutive sites) read consecutive 16-byte
// vectors.
//   FP64 SU(3): 9 planes of double2, plane k = element (k/3, k%3)   144 B/link
//   FP64 SU(2): 2 planes of double2: (a0,a1), (a2,a3)               32 B/link
//   FP32 SU(3): 3 planes of float4: (u00,u01), (u02,u10), (u11,u12); the
//               third row is rebuilt in registers as conj(row0 x row1)
//                                                                   48 B/link
//   FP32 SU(2): 1 plane of float4: (a0,a1,a2,a3)                   16 B/link
#pragma once

#include "gc_algebra.cuh"
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gc {

struct Geom {
  int L[4];      // Lx, Ly, Lz, Lt
  int stride[4]; // 1, Lx, Lx*Ly, Lx*Ly*Lz
  int V;         // sites
  int Vs;        // spatial sites (Lx*Ly*Lz)
};

__host__ __device__ inline void site_coords(const Geom &g, int site, int x[4]) {
  x[0] = site % g.L[0];
  int r = site / g.L[0];
  x[1] = r % g.L[1];
  r /= g.L[1];
  x[2] = r % g.L[2];
  x[3] = r / g.L[2];
}

// a[d] for a direction d known only at run time, as selects (a dynamically
// indexed array would be placed in local memory).
__host__ __device__ __forceinline__ int sel4(const int a[4], int d) {
  return d == 0 ? a[0] : d == 1 ? a[1] : d == 2 ? a[2] : a[3];
}

// Offset of a one-step move in direction mu (+1 or -1) from coordinate xm.
__host__ __device__ inline int step_off(const Geom &g, int xm, int mu, int dir) {
  const int L = sel4(g.L, mu), st = sel4(g.stride, mu);
  if (dir > 0)
    return (xm == L - 1) ? -(L - 1) * st : st;
  return (xm == 0) ? (L - 1) * st : -st;
}

// Offset of an n-step forward move (n >= 0, any size) from coordinate xm.
__host__ __device__ inline int fwd_off(const Geom &g, int xm, int mu, int n) {
  int xn = (xm + n) % sel4(g.L, mu);
  return (xn - xm) * sel4(g.stride, mu);
}

// ------------------------------------------------------------- storage
struct StoreF64SU3 {
  static constexpr int NC = 3;
  static constexpr int kBytes = 144;
  template <class CT> using M = SU3<CT>;
  template <class CT>
  __device__ __forceinline__ static SU3<CT> load(const void *f, size_t V,
                                                 int site) {
    const double2 *p = reinterpret_cast<const double2 *>(f) + site;
    SU3<CT> u;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      double2 v = __ldg(p + k * V);
      u.e[k / 3][k % 3] = {CT(v.x), CT(v.y)};
    }
    return u;
  }
  template <class CT>
  __device__ __forceinline__ static void store(void *f, size_t V, int site,
                                               const SU3<CT> &u) {
    double2 *p = reinterpret_cast<double2 *>(f) + site;
#pragma unroll
    for (int k = 0; k < 9; k++)
      p[k * V] = make_double2(double(u.e[k / 3][k % 3].re),
                              double(u.e[k / 3][k % 3].im));
  }
};

struct StoreF64SU2 {
  static constexpr int NC = 2;
  static constexpr int kBytes = 32;
  template <class CT> using M = SU2<CT>;
  template <class CT>
  __device__ __forceinline__ static SU2<CT> load(const void *f, size_t V,
                                                 int site) {
    const double2 *p = reinterpret_cast<const double2 *>(f) + site;
    double2 a = __ldg(p), b = __ldg(p + V);
    return {CT(a.x), CT(a.y), CT(b.x), CT(b.y)};
  }
  template <class CT>
  __device__ __forceinline__ static void store(void *f, size_t V, int site,
                                               const SU2<CT> &u) {
    double2 *p = reinterpret_cast<double2 *>(f) + site;
    p[0] = make_double2(double(u.a0), double(u.a1));
    p[V] = make_double2(double(u.a2), double(u.a3));
  }
};

struct StoreF32SU3 {
  static constexpr int NC = 3;
  static constexpr int kBytes = 48;
  template <class CT> using M = SU3<CT>;
  template <class CT>
  __device__ __forceinline__ static SU3<CT> load(const void *f, size_t V,
                                                 int site) {
    const float4 *p = reinterpret_cast<const float4 *>(f) + site;
    float4 a = __ldg(p), b = __ldg(p + V), c = __ldg(p + 2 * V);
    SU3<CT> u;
    u.e[0][0] = {CT(a.x), CT(a.y)};
    u.e[0][1] = {CT(a.z), CT(a.w)};
    u.e[0][2] = {CT(b.x), CT(b.y)};
    u.e[1][0] = {CT(b.z), CT(b.w)};
    u.e[1][1] = {CT(c.x), CT(c.y)};
    u.e[1][2] = {CT(c.z), CT(c.w)};
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const int a1 = (j + 1) % 3, b1 = (j + 2) % 3;
      cx<CT> t = csub(cmul(u.e[0][a1], u.e[1][b1]), cmul(u.e[0][b1], u.e[1][a1]));
      u.e[2][j] = {t.re, -t.im};
    }
    return u;
  }
  template <class CT>
  __device__ __forceinline__ static void store(void *f, size_t V, int site,
                                               const SU3<CT> &u) {
    float4 *p = reinterpret_cast<float4 *>(f) + site;
    p[0] = make_float4(float(u.e[0][0].re), float(u.e[0][0].im),
                       float(u.e[0][1].re), float(u.e[0][1].im));
    p[V] = make_float4(float(u.e[0][2].re), float(u.e[0][2].im),
                       float(u.e[1][0].re), float(u.e[1][0].im));
    p[2 * V] = make_float4(float(u.e[1][1].re), float(u.e[1][1].im),
                           float(u.e[1][2].re), float(u.e[1][2].im));
  }
};

// FP32 SU(3) with all 18 reals: 9 planes of float2 (element (k/3, k%3)).
// Used for fields that may hold matrices that are not in SU(3) -- HYP's
// decorated links, whose projection (six Newton-Schulz steps, as in the
// reference) need not converge -- where rebuilding the third row would
// change the matrix.
struct StoreF32SU3Full {
  static constexpr int NC = 3;
  static constexpr int kBytes = 72;
  template <class CT> using M = SU3<CT>;
  template <class CT>
  __device__ __forceinline__ static SU3<CT> load(const void *f, size_t V,
                                                 int site) {
    const float2 *p = reinterpret_cast<const float2 *>(f) + site;
    SU3<CT> u;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      float2 v = __ldg(p + k * V);
      u.e[k / 3][k % 3] = {CT(v.x), CT(v.y)};
    }
    return u;
  }
  template <class CT>
  __device__ __forceinline__ static void store(void *f, size_t V, int site,
                                               const SU3<CT> &u) {
    float2 *p = reinterpret_cast<float2 *>(f) + site;
#pragma unroll
    for (int k = 0; k < 9; k++)
      p[k * V] = make_float2(float(u.e[k / 3][k % 3].re), float(u.e[k / 3][k % 3].im));
  }
};

struct StoreF32SU2 {
  static constexpr int NC = 2;
  static constexpr int kBytes = 16;
  template <class CT> using M = SU2<CT>;
  template <class CT>
  __device__ __forceinline__ static SU2<CT> load(const void *f, size_t V,
                                                 int site) {
    float4 a = __ldg(reinterpret_cast<const float4 *>(f) + site);
    return {CT(a.x), CT(a.y), CT(a.z), CT(a.w)};
  }
  template <class CT>
  __device__ __forceinline__ static void store(void *f, size_t V, int site,
                                               const SU2<CT> &u) {
    reinterpret_cast<float4 *>(f)[site] =
        make_float4(float(u.a0), float(u.a1), float(u.a2), float(u.a3));
  }
};

// Storage of HYP's decorated-link fields for a link storage type: the same,
// except that 12-real SU(3) becomes the full 18-real form.
template <class Store> struct InterStore {
  using type = Store;
};
template <> struct InterStore<StoreF32SU3> {
  using type = StoreF32SU3Full;
};
// Bytes per link of HYP's decorated-link fields.
inline size_t inter_link_bytes(int nc, int prec) {
  if (nc == 3)
    return prec == 0 ? 144 : 72;
  return prec == 0 ? 32 : 16;
}

// Conversion between compute types (identity when equal).
template <class TO, class FROM>
__host__ __device__ __forceinline__ SU3<TO> convert(const SU3<FROM> &a, SU3<TO> *) {
  SU3<TO> b;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      b.e[i][j] = {TO(a.e[i][j].re), TO(a.e[i][j].im)};
  return b;
}
template <class TO, class FROM>
__host__ __device__ __forceinline__ SU2<TO> convert(const SU2<FROM> &a, SU2<TO> *) {
  return {TO(a.a0), TO(a.a1), TO(a.a2), TO(a.a3)};
}

// Set of per-direction field pointers passed to kernels by value.
struct Fields4 {
  void *f[4];
};

// Launch-status helper used by all host launchers.
int launch_check(const char *what);
// Records a launch-planning error (returned by the launcher as GC_ERR_ARG).
int plan_error(const char *what);

} // namespace gc
