// Polyakov loops and their correlators (sm_100a).
//
// Reference (lib/cpu/include/polyakov_loops.h):
//   get_polyakov_loop            :10-22  P(s) = U_t(s,0) U_t(s,1) ... U_t(s,Lt-1)
//   polyakov_loop                :24-41  mean over spatial sites of tr_real P
//   polyakov_loop_correlator_color_average  :83-145
//       C(D) = (1/Vs) sum_s Re[ tr P(s) conj(tr P(s+D)) ],  tr = Tr / N
//   polyakov_loop_correlator_singlet        :147-206
//       C(D) = (1/Vs) sum_s Re Tr[ P(s) P(s+D)^dag ] / N
// for the offsets D = (Dx,Dy,Dz) with |D| <= D_max that the reference visits
// (Dx >= 0 when Dy and Dz are both non-zero), stored at
// (Dz+D_max)(2D_max+1)^2 + (Dy+D_max)(2D_max+1) + Dx+D_max; other entries 0.
//
// polyakov_lines_kernel: thread per spatial site, the Lt time links of the
// site's column read in order (coalesced across threads), the product kept
// in the compute type and stored in FP64 as element planes
// (SU(3): 9 double2 planes, SU(2): 2 double2 planes, Vs entries each), with
// fixed-order block sums of Re Tr P for the loop itself.
// polyakov_correlator_kernel: one block per offset, each thread summing its
// sites in a fixed order, then a fixed-order block tree: deterministic.
#include "gc_internal.cuh"
#include "gc_kernels.h"

namespace gc {

namespace {

// FP64 element planes of the Polyakov lines (SU(3): 9 planes, SU(2): 2).
__device__ __forceinline__ void line_store(double2 *lines, int Vs, int s, const SU3<double> &m) {
#pragma unroll
  for (int k = 0; k < 9; k++)
    lines[(size_t)k * Vs + s] = make_double2(m.e[k / 3][k % 3].re, m.e[k / 3][k % 3].im);
}
__device__ __forceinline__ void line_store(double2 *lines, int Vs, int s, const SU2<double> &m) {
  lines[s] = make_double2(m.a0, m.a1);
  lines[(size_t)Vs + s] = make_double2(m.a2, m.a3);
}
__device__ __forceinline__ void line_load(const double2 *lines, int Vs, int s, SU3<double> &m) {
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const double2 v = __ldg(lines + (size_t)k * Vs + s);
    m.e[k / 3][k % 3] = {v.x, v.y};
  }
}
__device__ __forceinline__ void line_load(const double2 *lines, int Vs, int s, SU2<double> &m) {
  const double2 a = __ldg(lines + s), b = __ldg(lines + (size_t)Vs + s);
  m = {a.x, a.y, b.x, b.y};
}

// tr P = Tr P / N: SU(3) complex, SU(2) the real a0 (the quaternion trace).
__device__ __forceinline__ double2 norm_trace(const SU3<double> &m) {
  return make_double2((m.e[0][0].re + m.e[1][1].re + m.e[2][2].re) / 3.0,
                      (m.e[0][0].im + m.e[1][1].im + m.e[2][2].im) / 3.0);
}
__device__ __forceinline__ double2 norm_trace(const SU2<double> &m) {
  return make_double2(m.a0, 0.0);
}

template <class T> __device__ __forceinline__ SU3<double> to_double(const SU3<T> &a) {
  return convert(a, (SU3<double> *)nullptr);
}
template <class T> __device__ __forceinline__ SU2<double> to_double(const SU2<T> &a) {
  return convert(a, (SU2<double> *)nullptr);
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  return sh[0];
}

template <class Store, class CT>
__global__ void __launch_bounds__(256)
    polyakov_lines_kernel(const __grid_constant__ Geom g, const void *Ut, double2 *lines,
                          double *partials) {
  using M = typename Store::template M<CT>;
  using MD = typename Store::template M<double>;
  __shared__ double sh[256];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  double tr = 0.0;
  if (s < g.Vs) {
    const size_t V = g.V;
    M A = Store::template load<CT>(Ut, V, s);
#pragma unroll 1
    for (int t = 1; t < g.L[3]; t++)
      A = mul(A, Store::template load<CT>(Ut, V, s + t * g.Vs));
    const MD P = to_double(A);
    line_store(lines, g.Vs, s, P);
    tr = norm_trace(P).x;
  }
  const double b = block_sum(tr, sh);
  if (threadIdx.x == 0)
    partials[blockIdx.x] = b;
}

// offsets[i] = (Dx, Dy, Dz, place) of the i-th visited offset.
template <class MD, bool SINGLET>
__global__ void __launch_bounds__(256)
    polyakov_correlator_kernel(const __grid_constant__ Geom g, const double2 *lines,
                               const int4 *offsets, double scale, double *out) {
  __shared__ double sh[256];
  const int4 off = offsets[blockIdx.x];
  const int Lx = g.L[0], Ly = g.L[1], Lz = g.L[2];
  // shifts as non-negative residues
  const int dx = ((off.x % Lx) + Lx) % Lx, dy = ((off.y % Ly) + Ly) % Ly,
            dz = ((off.z % Lz) + Lz) % Lz;
  double acc = 0.0;
#pragma unroll 1
  for (int s = threadIdx.x; s < g.Vs; s += blockDim.x) {
    const int x = s % Lx, y = (s / Lx) % Ly, z = s / (Lx * Ly);
    int x2 = x + dx, y2 = y + dy, z2 = z + dz;
    x2 -= (x2 >= Lx) ? Lx : 0;
    y2 -= (y2 >= Ly) ? Ly : 0;
    z2 -= (z2 >= Lz) ? Lz : 0;
    const int s2 = x2 + Lx * (y2 + Ly * z2);
    MD a, b;
    line_load(lines, g.Vs, s, a);
    line_load(lines, g.Vs, s2, b);
    if (SINGLET) {
      // multiply_conj_tr: Re Tr(a b^dag) / N
      acc += conj_tr(a, b);
    } else {
      const double2 p = norm_trace(a), q = norm_trace(b);
      acc += fma(p.y, q.y, p.x * q.x); // Re(p conj(q))
    }
  }
  const double sum = block_sum(acc, sh);
  if (threadIdx.x == 0)
    out[off.w] = sum * scale;
}

} // namespace

template <class Store, class CT>
int launch_polyakov_lines(const Geom &g, const Fields4 &U, double2 *lines, double *partials,
                          double *out_dev, cudaStream_t s) {
  const int nb = (g.Vs + 255) / 256;
  polyakov_lines_kernel<Store, CT><<<nb, 256, 0, s>>>(g, U.f[3], lines, partials);
  int rc = launch_check("polyakov_lines_kernel");
  if (rc)
    return rc;
  if (!out_dev)
    return GC_OK;
  return launch_reduce_sum(partials, nb, 1.0 / (double)g.Vs, out_dev, s);
}

int launch_polyakov_correlator(const Geom &g, int nc, const double2 *lines, const int4 *offsets,
                               int noffsets, bool singlet, double *out_dev, cudaStream_t s) {
  if (noffsets <= 0)
    return GC_OK;
  const double scale = 1.0 / (double)g.Vs;
  if (nc == 3) {
    if (singlet)
      polyakov_correlator_kernel<SU3<double>, true>
          <<<noffsets, 256, 0, s>>>(g, lines, offsets, scale, out_dev);
    else
      polyakov_correlator_kernel<SU3<double>, false>
          <<<noffsets, 256, 0, s>>>(g, lines, offsets, scale, out_dev);
  } else {
    if (singlet)
      polyakov_correlator_kernel<SU2<double>, true>
          <<<noffsets, 256, 0, s>>>(g, lines, offsets, scale, out_dev);
    else
      polyakov_correlator_kernel<SU2<double>, false>
          <<<noffsets, 256, 0, s>>>(g, lines, offsets, scale, out_dev);
  }
  return launch_check("polyakov_correlator_kernel");
}

#define GC_INSTANTIATE_P(STORE, CT)                                                      \
  template int launch_polyakov_lines<STORE, CT>(const Geom &, const Fields4 &, double2 *, \
                                                double *, double *, cudaStream_t);

GC_INSTANTIATE_P(StoreF64SU3, double)
GC_INSTANTIATE_P(StoreF64SU2, double)
GC_INSTANTIATE_P(StoreF32SU3, float)
GC_INSTANTIATE_P(StoreF32SU2, float)

} // namespace gc
