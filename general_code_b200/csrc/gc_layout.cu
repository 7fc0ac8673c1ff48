// Conversion between the reference's host link layout (array of structures,
// link index 4*site+mu; data.h:78-112, indexing.h:111-123) and the device
// structure-of-arrays fields. The host array is copied verbatim into a device
// staging buffer first; one thread then converts one link. The host-to-device
// direction takes a window of sites [site0, site0 + nsites): the staging
// buffer holds just those sites' links (a run of time slices of a larger
// lattice, whose sites are contiguous because t varies slowest).
#include "gc_internal.cuh"
#include "gc_kernels.h"

namespace gc {

namespace {

// Offset (in doubles) of element (i,j) inside one SU(3) link of the host array.
__device__ __forceinline__ int su3_off(int layout, int i, int j) {
  return layout == 0 ? (3 * i + j) * 2 : (i + 3 * j) * 2;
}

template <class Store>
__global__ void aos_to_soa_su3(Geom g, int layout, const double *__restrict__ in,
                               Fields4 U, int site0, int nsites) {
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= 4LL * nsites)
    return;
  const int site = site0 + (int)(l >> 2), mu = (int)(l & 3);
  const double *p = in + l * 18;
  SU3<double> m;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const int o = su3_off(layout, i, j);
      m.e[i][j] = {p[o], p[o + 1]};
    }
  Store::template store<double>(U.f[mu], g.V, site, m);
}

template <class Store>
__global__ void soa_to_aos_su3(Geom g, int layout, Fields4 U,
                               double *__restrict__ out) {
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= 4LL * g.V)
    return;
  const int site = (int)(l >> 2), mu = (int)(l & 3);
  SU3<double> m = Store::template load<double>(U.f[mu], g.V, site);
  double *p = out + l * 18;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const int o = su3_off(layout, i, j);
      p[o] = m.e[i][j].re;
      p[o + 1] = m.e[i][j].im;
    }
}

template <class Store>
__global__ void aos_to_soa_su2(Geom g, const double *__restrict__ in, Fields4 U, int site0,
                               int nsites) {
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= 4LL * nsites)
    return;
  const int site = site0 + (int)(l >> 2), mu = (int)(l & 3);
  const double2 a = reinterpret_cast<const double2 *>(in)[2 * l];
  const double2 b = reinterpret_cast<const double2 *>(in)[2 * l + 1];
  Store::template store<double>(U.f[mu], g.V, site,
                                SU2<double>{a.x, a.y, b.x, b.y});
}

template <class Store>
__global__ void soa_to_aos_su2(Geom g, Fields4 U, double *__restrict__ out) {
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= 4LL * g.V)
    return;
  const int site = (int)(l >> 2), mu = (int)(l & 3);
  SU2<double> a = Store::template load<double>(U.f[mu], g.V, site);
  reinterpret_cast<double2 *>(out)[2 * l] = make_double2(a.a0, a.a1);
  reinterpret_cast<double2 *>(out)[2 * l + 1] = make_double2(a.a2, a.a3);
}

} // namespace

int launch_aos_to_soa(const Geom &g, int nc, int prec, int layout,
                      const double *staging, const Fields4 &U, cudaStream_t s, int site0,
                      int nsites) {
  if (nsites < 0)
    nsites = g.V - site0;
  if (site0 < 0 || nsites < 0 || site0 + nsites > g.V)
    return plan_error("aos_to_soa: site window outside the lattice");
  if (nsites == 0)
    return GC_OK;
  const long long n = 4LL * nsites;
  const int blk = 256;
  const unsigned grid = (unsigned)((n + blk - 1) / blk);
  if (nc == 3) {
    if (prec == 0)
      aos_to_soa_su3<StoreF64SU3><<<grid, blk, 0, s>>>(g, layout, staging, U, site0, nsites);
    else
      aos_to_soa_su3<StoreF32SU3><<<grid, blk, 0, s>>>(g, layout, staging, U, site0, nsites);
  } else {
    if (prec == 0)
      aos_to_soa_su2<StoreF64SU2><<<grid, blk, 0, s>>>(g, staging, U, site0, nsites);
    else
      aos_to_soa_su2<StoreF32SU2><<<grid, blk, 0, s>>>(g, staging, U, site0, nsites);
  }
  return launch_check("aos_to_soa");
}

int launch_soa_to_aos(const Geom &g, int nc, int prec, int layout,
                      const Fields4 &U, double *staging, cudaStream_t s) {
  const long long n = 4LL * g.V;
  const int blk = 256;
  const unsigned grid = (unsigned)((n + blk - 1) / blk);
  if (nc == 3) {
    if (prec == 0)
      soa_to_aos_su3<StoreF64SU3><<<grid, blk, 0, s>>>(g, layout, U, staging);
    else
      soa_to_aos_su3<StoreF32SU3><<<grid, blk, 0, s>>>(g, layout, U, staging);
  } else {
    if (prec == 0)
      soa_to_aos_su2<StoreF64SU2><<<grid, blk, 0, s>>>(g, U, staging);
    else
      soa_to_aos_su2<StoreF32SU2><<<grid, blk, 0, s>>>(g, U, staging);
  }
  return launch_check("soa_to_aos");
}

} // namespace gc
