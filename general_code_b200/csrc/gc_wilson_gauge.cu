// On-axis Wilson loops W(R,T) in the temporal gauge (sm_100a).
//
// Reference: wilson_loop (wilson_loops.h:1047-1074) averages, over x and the
// spatial directions nu, the loop
//     Re Tr[S(x,R) L(x+R nu,T) S(x+T t,R)^dag L(x,T)^dag] / N
// with time lines L(x,T) = U_t(x) U_t(x+t) ... U_t(x+(T-1)t) and space lines
// S(x,R) = U_nu(x) ... U_nu(x+(R-1)nu).
//
// The loop is gauge invariant. With G_c(s,t) the time line of spatial site s
// from a cut slice c up to slice t (G_c(s,c) = 1, G_c(s,t+1) = G_c(s,t)
// U_t(s,t) walking forward from c), a time line that does not pass the cut
// is L(s;t0,T) = G_c(s,t0)^dag G_c(s,t0+T) when the temporal links are
// unitary, and the loop becomes
//     Re Tr[S'(x,R) S'(x+T t,R)^dag] / N,
//     S'(s,t,R) = G_c(s,t) S(s,t,R) G_c(s+R nu,t)^dag
//               = U'_nu(s,t) ... U'_nu(s+(R-1)nu,t),
//     U'_nu(s,t) = G_c(s,t) U_nu(s,t) G_c(s+nu,t)^dag.
// Two cuts cover every loop with T <= h = floor(Lt/2): cut A at slice 0 for
// loops starting on slices t0 < h (they end at t0+T <= 2h-1 <= Lt-1), cut B
// at slice h for loops starting on t0 >= h (t0-h+T <= Lt-1). A loop then
// costs one 9-element trace instead of two matrix products (the T walk of
// the exact recursion in gc_wilson.cu), and each space line one product per
// R and cut.
//
// The identity needs unitary temporal links. The lines kernel measures the
// largest unitarity defect max |U_t U_t^dag - 1| of the lattice's temporal
// links and raises a flag above the form's tolerance (FP64: 1e-14, a few
// roundings; mixed: 1e-6, FP32 rounding of the 12-real links is 2.6e-7).
// Both W kernels are launched and read the flag on the device: the exact
// product (gc_wilson.cu) computes when it is raised, this form when it is
// not, and the reduction sums the partials of the one that ran; no host
// synchronisation, so the sequence can be captured in a graph. With defect
// d per link a
// loop differs from the reference's product of links by at most about
// 2 T d (the two time lines), well inside the parity tolerances at these d.
//
// Kernels:
//   gauge_lines_kernel      thread per (spatial site, cut): G_A(s,t) and the
//                           defect, or G_B(s,t), for all t (FP64, stored as
//                           FP64 fields)
//   gauge_transform_kernel  thread per (site, spatial nu): U'_nu for both
//                           cuts, computed in FP64, stored in the lattice's
//                           link format
//   wilson_gauge_kernel     block = `cols` columns (s, nu) over all t: the
//                           transformed space lines of both cuts in shared
//                           memory, extended by one link per R; a thread per
//                           (column unit, 1, 2 or 4 start slices) adds the
//                           traces of its loops for every T into a per-thread
//                           slot; a
//                           fixed-order sum over the block's threads gives
//                           one partial per (block, R, T), and the fixed-order
//                           tree over blocks of gc_wilson.cu finishes
//   wilson_gauge_reg_kernel the mixed SU(3) fundamental loops (8 | Lt), and
//   wilson_gauge_q_kernel   the SU(2) fundamental loops (8 | Lt): one column
//                           per thread, the space lines of its 4 start slices
//                           kept in registers
#include "gc_internal.cuh"
#include "gc_kernels.h"
#include "gc_pair.cuh"
#include "gc_rows01.cuh"
#include "gc_wcol.cuh"

#include <algorithm>
#include <type_traits>

namespace gc {

namespace {

template <int NC> struct F64Store;
template <> struct F64Store<3> {
  using type = StoreF64SU3;
};
template <> struct F64Store<2> {
  using type = StoreF64SU2;
};

// max_ij |(U U^dag - 1)_ij|
__device__ __forceinline__ double unitarity_defect(const SU3<double> &u) {
  double d = 0.0;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = i; j < 3; j++) {
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        re = fma(u.e[i][k].re, u.e[j][k].re, re);
        re = fma(u.e[i][k].im, u.e[j][k].im, re);
        im = fma(u.e[i][k].im, u.e[j][k].re, im);
        im = fma(-u.e[i][k].re, u.e[j][k].im, im);
      }
      if (i == j)
        re -= 1.0;
      d = fmax(d, fmax(fabs(re), fabs(im)));
    }
  return d;
}
// SU(2) quaternion a0 + i a.sigma: U U^dag = |a|^2 1
__device__ __forceinline__ double unitarity_defect(const SU2<double> &u) {
  return fabs(dot4(u.a0, u.a0, u.a1, u.a1, u.a2, u.a2, u.a3, u.a3) - 1.0);
}

// The temporal link the gauge lines are built from. FP64 links are unitary to
// rounding. An FP32 link's last projection step leaves its singular values
// 1 - O(d^2) (d the defect before that step, up to 2e-5), a shrink of up to a
// few 1e-10 with one sign; through G^dag G != 1 it entered every transformed
// link, and W's error against FP64 grew linearly in R and T (3.4e-8 at 24^4,
// R,T = 12, against 4.3e-9 for the exact product). One FP64 Newton-Schulz
// step (SU(2): a / |a|) makes the link unitary to FP64 rounding; it moves
// the link by that shrink only, well inside the FP32 rounding of the stored
// link.
template <class Store>
__device__ __forceinline__ typename Store::template M<double> gauge_time_link(
    const typename Store::template M<double> &u) {
  if constexpr (Store::kBytes == 48 || Store::kBytes == 72)
    return ns_step(u);
  else if constexpr (Store::kBytes == 16)
    return proj(u);
  else
    return u;
}

template <class Store>
__global__ void __launch_bounds__(128)
    gauge_lines_kernel(const __grid_constant__ Geom g, const void *Ut, void *GA, void *GB,
                       int h, double tol, int *flag) {
  using GS = typename F64Store<Store::NC>::type;
  using MD = typename Store::template M<double>;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.Vs)
    return;
  const size_t V = g.V;
  const int Lt = g.L[3];
  if (blockIdx.y == 0) {
    // cut A: G_A(s,0) = 1, G_A(s,t+1) = G_A(s,t) U_t(s,t); the defect check
    double dmax = 0.0;
    MD G = unit(MD());
#pragma unroll 1
    for (int t = 0; t < Lt; t++) {
      GS::template store<double>(GA, V, s + t * g.Vs, G);
      const MD u = Store::template load<double>(Ut, V, s + t * g.Vs);
      dmax = fmax(dmax, unitarity_defect(u));
      if (t + 1 < Lt)
        G = mul(G, gauge_time_link<Store>(u));
    }
    if (!(dmax <= tol)) // (a NaN link counts as not unitary)
      *flag = 1;
    return;
  }
  // cut B: G_B(s,h) = 1, forward through Lt-1 and around to h-1
  MD G = unit(MD());
  int t = h;
#pragma unroll 1
  for (int k = 0; k < Lt; k++) {
    GS::template store<double>(GB, V, s + t * g.Vs, G);
    if (k + 1 < Lt)
      G = mul(G, gauge_time_link<Store>(Store::template load<double>(Ut, V, s + t * g.Vs)));
    t = (t + 1 == Lt) ? 0 : t + 1;
  }
}

// U'_nu(x) = G(x) U_nu(x) G(x + nu)^dag for both cuts; thread per (site, nu).
template <class Store>
__global__ void __launch_bounds__(128)
    gauge_transform_kernel(const __grid_constant__ Geom g, const __grid_constant__ Fields4 U,
                           const void *GA, const void *GB, const __grid_constant__ Fields4 UA,
                           const __grid_constant__ Fields4 UB) {
  using GS = typename F64Store<Store::NC>::type;
  using MD = typename Store::template M<double>;
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  if (site >= g.V)
    return;
  const int nu = blockIdx.y;
  int x[4];
  site_coords(g, site, x);
  const int sn = site + step_off(g, sel4(x, nu), nu, +1);
  const size_t V = g.V;
  const MD u = Store::template load<double>(U.f[nu], V, site);
  Store::template store<double>(
      UA.f[nu], V, site,
      mul_ad(mul(GS::template load<double>(GA, V, site), u),
             GS::template load<double>(GA, V, sn)));
  Store::template store<double>(
      UB.f[nu], V, site,
      mul_ad(mul(GS::template load<double>(GB, V, site), u),
             GS::template load<double>(GB, V, sn)));
}

// The loop value from Tr[a b^dag] as loop_value (gc_wcol.cuh) computes it,
// with the sum split into one fused chain per row and the three rows added at
// the end: three independent chains instead of one of 18 dependent FMAs,
// which the trace loop below (a few warps per scheduler, shared-memory
// operands) needs to keep the FMA pipe fed.
// Per-thread sums of the loop values: FP32 for the fundamental loops of the
// mixed form (a thread adds at most a few loops; every loop value is an FP32
// dot product), FP64 otherwise; the block and the grid sum them in FP64.
template <bool ADJ, class CT>
using GAcc = typename std::conditional<!ADJ && std::is_same<CT, float>::value, float,
                                       double>::type;

template <bool ADJ, class T>
__device__ __forceinline__ GAcc<ADJ, T> gauge_trace(const SU3<T> &a, const SU3<T> &b, bool) {
  T re[3], im[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    re[i] = a.e[i][0].re * b.e[i][0].re;
    re[i] = GC_FMA(a.e[i][0].im, b.e[i][0].im, re[i]);
    if (ADJ) {
      im[i] = a.e[i][0].im * b.e[i][0].re;
      im[i] = GC_FMA(-a.e[i][0].re, b.e[i][0].im, im[i]);
    }
#pragma unroll
    for (int j = 1; j < 3; j++) {
      re[i] = GC_FMA(a.e[i][j].re, b.e[i][j].re, re[i]);
      re[i] = GC_FMA(a.e[i][j].im, b.e[i][j].im, re[i]);
      if (ADJ) {
        im[i] = GC_FMA(a.e[i][j].im, b.e[i][j].re, im[i]);
        im[i] = GC_FMA(-a.e[i][j].re, b.e[i][j].im, im[i]);
      }
    }
  }
  if (!ADJ)
    return (re[0] + re[1]) + re[2];
  const double r = double((re[0] + re[1]) + re[2]);
  const double m = double((im[0] + im[1]) + im[2]);
  return fma(r, r, fma(m, m, -1.0));
}
template <bool ADJ>
__device__ __forceinline__ GAcc<ADJ, float> gauge_trace(const SU3<f2> &a, const SU3<f2> &b,
                                                        bool lane1) {
  f2 re[3], im[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    re[i] = a.e[i][0].re * b.e[i][0].re;
    re[i] = fma(a.e[i][0].im, b.e[i][0].im, re[i]);
    if (ADJ) {
      im[i] = a.e[i][0].im * b.e[i][0].re;
      im[i] = fma(-a.e[i][0].re, b.e[i][0].im, im[i]);
    }
#pragma unroll
    for (int j = 1; j < 3; j++) {
      re[i] = fma(a.e[i][j].re, b.e[i][j].re, re[i]);
      re[i] = fma(a.e[i][j].im, b.e[i][j].im, re[i]);
      if (ADJ) {
        im[i] = fma(a.e[i][j].im, b.e[i][j].re, im[i]);
        im[i] = fma(-a.e[i][j].re, b.e[i][j].im, im[i]);
      }
    }
  }
  const float2 r = make_float2((re[0].v.x + re[1].v.x) + re[2].v.x,
                               (re[0].v.y + re[1].v.y) + re[2].v.y);
  if (!ADJ)
    return lane1 ? r.x + r.y : r.x;
  const float2 m = make_float2((im[0].v.x + im[1].v.x) + im[2].v.x,
                               (im[0].v.y + im[1].v.y) + im[2].v.y);
  const double r0 = double(r.x), i0 = double(m.x);
  const double v0 = fma(r0, r0, fma(i0, i0, -1.0));
  if (!lane1)
    return v0;
  const double r1 = double(r.y), i1 = double(m.y);
  return v0 + fma(r1, r1, fma(i1, i1, -1.0));
}
template <bool ADJ, class T>
__device__ __forceinline__ GAcc<ADJ, T> gauge_trace(const SU2<T> &a, const SU2<T> &b,
                                                    bool lane1) {
  if (!ADJ)
    return dot4(a.a0, b.a0, a.a1, b.a1, a.a2, b.a2, a.a3, b.a3);
  return loop_value<ADJ>(a, b, lane1);
}

// First spatial site of a column block. When the block's columns tile the x
// extent, consecutive blocks step along nu (for nu = y, z), so that the
// blocks running at the same time extend their space lines with the same
// transformed links (they hit L2 instead of each reading HBM); otherwise the
// blocks take consecutive runs of sites.
__device__ __forceinline__ int column_base(const Geom &g, int cb, int cols, int nu) {
  if (nu == 0 || g.L[0] % cols != 0)
    return cb * cols;
  const int nxc = g.L[0] / cols;
  int xc, y, z;
  if (nu == 1) {
    y = cb % g.L[1];
    const int rest = cb / g.L[1];
    xc = rest % nxc;
    z = rest / nxc;
  } else {
    z = cb % g.L[2];
    const int rest = cb / g.L[2];
    xc = rest % nxc;
    y = rest / nxc;
  }
  return xc * cols + g.L[0] * (y + g.L[1] * z);
}

// Shared memory of one block: per-thread loop sums red[nt][threads] (GAcc),
// then the space lines of cut A and of cut B, one slot per (t, column unit).
// KS > 1: a thread owns KS consecutive start slices t0 = KS row + m, m < KS
// (all of one cut: KS divides the cut slice h), and one shared-memory load of
// a top space line S(t) serves the loops of all of them that end on t
// (T = t - t0 - m): nt + KS - 1 loads for KS nt loops, the sums of the last
// KS values of T kept in registers. KS = 1: a thread owns the slices
// row + k rows and loads one line per loop.
// split = h is the first start slice of cut B: Lt/2, or Lt for a time slab,
// whose counted starts [0, tstarts) all take cut A. SLAB (the same in the
// one-column kernels below) compiles in the check that a start is counted;
// the whole-lattice kernels count every start.
template <class Store, class CT, bool ADJ, int KS, bool SLAB>
__global__ void __launch_bounds__(256)
    wilson_gauge_kernel(const __grid_constant__ Geom g, const __grid_constant__ Fields4 UA,
                        const __grid_constant__ Fields4 UB, int rmin, int rmax, int tmin,
                        int tmax, int cols, int rows, double *partials, const int *flag, int split, int tstarts) {
  // the exact product runs instead when a temporal link failed the check
  if (flag && *flag != 0)
    return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int LANES = wilson_lanes(Store::NC, sizeof(CT));
  using LL = LaneLoad<Store, CT, LANES>;
  using M = typename LL::M;
  using CS = ColSet<M>;
  const int Lt = g.L[3], h = split; // the first slice of cut B
  const int nt = tmax - tmin + 1;
  const int nthreads = blockDim.x;
  const int cs = wilson_col_stride(cols, LANES);
  const int units = cs / LANES;
  const int nslots = Lt * units;
  using Acc = GAcc<ADJ, CT>;
  Acc *red = reinterpret_cast<Acc *>(smem_raw); // [nt][nthreads]
  unsigned char *sa = smem_raw + ((sizeof(Acc) * nt * nthreads + 15) & ~(size_t)15);
  unsigned char *sb = sa + (size_t)CS::kBytes * nslots;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31, nwarps = nthreads >> 5;
  const int u = tid % units;
  const int row = tid / units;
  const int nu = blockIdx.y;
  const int s0 = column_base(g, blockIdx.x, cols, nu) + LANES * u;
  const bool active = (row < rows) && (s0 < g.Vs);
  const bool lane1 = LANES == 2 && active && (LANES * u + 1 < cols) && (s0 + 1 < g.Vs);
  const int s1 = lane1 ? s0 + 1 : s0;
  const int kt = Lt / rows;
  const int Ln = sel4(g.L, nu), stn = sel4(g.stride, nu);
  const int xn0 = (s0 / stn) % Ln, xn1 = (s1 / stn) % Ln;
  const size_t V = g.V;
  const int ne = (rmax - rmin + 1) * nt;
  double *part = partials + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * ne;

#pragma unroll 1
  for (int R = 1; R <= rmax; R++) {
    // extend the space lines of both cuts by the link at x + (R-1) nu
    if (active) {
      const int l0 = s0 + ((xn0 + R - 1) % Ln - xn0) * stn;
      const int l1 = s1 + ((xn1 + R - 1) % Ln - xn1) * stn;
#pragma unroll 1
      for (int k = 0; k < kt; k++) {
        const int t = KS > 1 ? KS * row + k : row + k * rows;
        const int i = t * units + u;
        // both cuts' links are loaded before either product needs them
        const M la = LL::load(UA.f[nu], V, l0 + t * g.Vs, l1 + t * g.Vs);
        const M lb = LL::load(UB.f[nu], V, l0 + t * g.Vs, l1 + t * g.Vs);
        if (R == 1) {
          CS::store(sa, nslots, i, la);
          CS::store(sb, nslots, i, lb);
        } else {
          CS::store(sa, nslots, i, mul(CS::load(sa, nslots, i), la));
          CS::store(sb, nslots, i, mul(CS::load(sb, nslots, i), lb));
        }
      }
    }
    __syncthreads();
    if (R >= rmin && KS > 1) {
      const int t0 = KS * row;
      const unsigned char *set = (t0 < h) ? sa : sb;
      M a[KS];
#pragma unroll
      for (int m = 0; m < KS; m++)
        a[m] = active ? CS::load(set, nslots, (t0 + m) * units + u) : unit(M());
      int tt = t0 + tmin;
      tt = (tt >= Lt) ? tt - Lt : tt;
      Acc acc[KS]; // acc[m]: the sum for T index j - m
#pragma unroll
      for (int m = 0; m < KS; m++)
        acc[m] = Acc(0);
      // One step of the sweep: the loops of all starts that end on top line
      // b (index j), then the completed sum of T index j - KS + 1.
      auto step = [&](int j, const M &b) {
        if (active) {
#pragma unroll
          for (int m = 0; m < KS; m++)
            if (j - m >= 0 && j - m < nt && (!SLAB || t0 + m < tstarts)) // T = tmin + j - m
              acc[m] += gauge_trace<ADJ>(a[m], b, lane1);
        }
        if (j - (KS - 1) >= 0) // T index j - KS + 1 has all KS starts
          red[(size_t)(j - (KS - 1)) * nthreads + tid] = acc[KS - 1];
#pragma unroll
        for (int m = KS - 1; m > 0; m--)
          acc[m] = acc[m - 1];
        acc[0] = Acc(0);
      };
      // two top lines in flight (b0, b1 alternate): the next line's load is
      // issued before the current line's traces (a slot past the last step
      // is still a slot of the column: its load is in bounds and unused;
      // inactive threads use no line)
      const int nsteps = nt + KS - 1;
      M b0, b1;
      if (active)
        b0 = CS::load(set, nslots, tt * units + u);
#pragma unroll 1
      for (int j = 0; j < nsteps; j += 2) {
        tt = (tt + 1 == Lt) ? 0 : tt + 1;
        if (active)
          b1 = CS::load(set, nslots, tt * units + u);
        step(j, b0);
        tt = (tt + 1 == Lt) ? 0 : tt + 1;
        if (active)
          b0 = CS::load(set, nslots, tt * units + u);
        if (j + 1 < nsteps)
          step(j + 1, b1);
      }
    } else if (R >= rmin) {
#pragma unroll 1
      for (int k = 0; k < kt; k++) {
        const int t0 = row + k * rows;
        // the cut this start slice's loops use
        const unsigned char *set = (t0 < h) ? sa : sb;
        const M a = active ? CS::load(set, nslots, t0 * units + u) : unit(M());
        int tt = t0 + tmin;
        tt = (tt >= Lt) ? tt - Lt : tt;
#pragma unroll 1
        for (int T = 0; T < nt; T++) {
          const Acc v =
              (active && (!SLAB || t0 < tstarts)) ? gauge_trace<ADJ>(a, CS::load(set, nslots, tt * units + u), lane1) : Acc(0);
          Acc *r = red + (size_t)T * nthreads + tid;
          *r = (k == 0) ? v : *r + v;
          tt = (tt + 1 == Lt) ? 0 : tt + 1;
        }
      }
    }
    if (R >= rmin) {
      __syncthreads();
      // fixed-order sum over the block's threads: warp w takes T = w, w +
      // nwarps, ...; each lane sums a strided subset, then a warp tree
#pragma unroll 1
      for (int T = warp; T < nt; T += nwarps) {
        double v = 0.0;
        for (int i = lane; i < nthreads; i += 32)
          v += double(red[(size_t)T * nthreads + i]);
        v = warp_sum(v);
        if (lane == 0)
          part[(R - rmin) * nt + T] = v;
      }
    }
    __syncthreads();
  }
}

// Shared-memory record of an FP32 SU(3) space line for the one-column kernel
// below: rows 0 and 1 (row 2 = conj(row0 x row1) is rebuilt where a trace
// needs it), 48 bytes moved as three 16-byte vectors at immediate offsets, in
// the element order of the stored links (StoreF32SU3). Consecutive threads
// hold consecutive records (a 12-word stride), so each quarter-warp phase of a
// 16-byte access covers the 32 banks once.
struct Rows01Set {
  static constexpr int kBytes = 48;
  __device__ __forceinline__ static void store(unsigned char *set, int i, const SU3<float> &m) {
    float4 *p = reinterpret_cast<float4 *>(set + (size_t)kBytes * i);
    p[0] = make_float4(m.e[0][0].re, m.e[0][0].im, m.e[0][1].re, m.e[0][1].im);
    p[1] = make_float4(m.e[0][2].re, m.e[0][2].im, m.e[1][0].re, m.e[1][0].im);
    p[2] = make_float4(m.e[1][1].re, m.e[1][1].im, m.e[1][2].re, m.e[1][2].im);
  }
  // rows 0 and 1 (row 2 not set)
  __device__ __forceinline__ static SU3<float> load(const unsigned char *set, int i) {
    const float4 *p = reinterpret_cast<const float4 *>(set + (size_t)kBytes * i);
    const float4 a = p[0], b = p[1], c = p[2];
    SU3<float> m;
    m.e[0][0] = {a.x, a.y};
    m.e[0][1] = {a.z, a.w};
    m.e[0][2] = {b.x, b.y};
    m.e[1][0] = {b.z, b.w};
    m.e[1][1] = {c.x, c.y};
    m.e[1][2] = {c.z, c.w};
    return m;
  }
};

// The fundamental loops of the mixed SU(3) form with one column per thread
// and KS consecutive start slices t0 = KS row + m (all of one cut: KS divides
// the cut slice h) whose space lines stay in registers from one R to the
// next. The trace sweep reads each top line once for the KS starts, as in
// wilson_gauge_kernel, but the lines are not lane-packed, so KS = 4 starts
// fit in the registers: twice the loops per shared-memory byte of the
// two-column, two-start form. Each R the thread extends its own starts' lines
// in registers (and stores them for the other threads' sweeps) and the other
// cut's lines of the same slices in shared memory. Lines are products of
// SU(3) links, so they are computed and kept in shared memory as rows 0 and 1
// (48 bytes a line instead of 72; 72 instead of 108 multiply-adds a product),
// and row 2 is rebuilt where a trace needs it. Compiled for 16 warps per SM
// (128 registers, a few spilled): at SU(3) 32^4 that ran 2.45 ms against 2.98
// ms at 175 registers (8 warps) and 3.01 ms for the two-column kernel.
// Partials, block sums and the per-thread FP32 loop sums as
// wilson_gauge_kernel.
template <int KS, bool SLAB>
__global__ void __launch_bounds__(256, 2)
    wilson_gauge_reg_kernel(const __grid_constant__ Geom g, const __grid_constant__ Fields4 UA,
                            const __grid_constant__ Fields4 UB, int rmin, int rmax, int tmin,
                            int tmax, int cols, int rows, double *partials, const int *flag, int split, int tstarts) {
  if (flag && *flag != 0)
    return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Lt = g.L[3], h = split; // the first slice of cut B
  const int nt = tmax - tmin + 1;
  const int nthreads = blockDim.x;
  const int nslots = Lt * cols;
  float *red = reinterpret_cast<float *>(smem_raw); // [nt][nthreads]
  unsigned char *sa = smem_raw + ((sizeof(float) * nt * nthreads + 15) & ~(size_t)15);
  unsigned char *sb = sa + (size_t)Rows01Set::kBytes * nslots;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31, nwarps = nthreads >> 5;
  const int u = tid % cols;
  const int row = tid / cols;
  const int nu = blockIdx.y;
  const int s0 = column_base(g, blockIdx.x, cols, nu) + u;
  const bool active = (row < rows) && (s0 < g.Vs);
  const int t0 = KS * row;
  // the cut of this thread's starts, and the other one
  const bool cut_a = t0 < h;
  unsigned char *own = cut_a ? sa : sb;
  unsigned char *other = cut_a ? sb : sa;
  const void *f_own = cut_a ? UA.f[nu] : UB.f[nu];
  const void *f_other = cut_a ? UB.f[nu] : UA.f[nu];
  const int Ln = sel4(g.L, nu), stn = sel4(g.stride, nu);
  const int xn = (s0 / stn) % Ln;
  const size_t V = g.V;
  const int ne = (rmax - rmin + 1) * nt;
  double *part = partials + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * ne;

  SU3<float> a[KS];
#pragma unroll 1
  for (int R = 1; R <= rmax; R++) {
    // extend both cuts' lines of slices t0 .. t0 + KS - 1 by the link at
    // x + (R-1) nu
    if (active) {
      const int l = s0 + ((xn + R - 1) % Ln - xn) * stn;
#pragma unroll
      for (int m = 0; m < KS; m++) {
        const int t = t0 + m;
        const int i = t * cols + u;
        const SU3<float> lo = StoreF32SU3::load<float>(f_own, V, l + t * g.Vs);
        const SU3<float> lx = StoreF32SU3::load<float>(f_other, V, l + t * g.Vs);
        if (R == 1) {
          a[m] = lo;
          Rows01Set::store(other, i, lx);
        } else {
          // rows 0 and 1 of the products; the own line's row 2 rebuilt for
          // its traces
          a[m] = mul01(a[m], lo);
          rebuild_row2(a[m]);
          Rows01Set::store(other, i, mul01(Rows01Set::load(other, i), lx));
        }
        Rows01Set::store(own, i, a[m]);
      }
    }
    __syncthreads();
    if (R >= rmin) {
      int tt = t0 + tmin;
      tt = (tt >= Lt) ? tt - Lt : tt;
      float acc[KS]; // acc[m]: the sum for T index j - m
#pragma unroll
      for (int m = 0; m < KS; m++)
        acc[m] = 0.f;
      // the loops of all starts that end on top line b (index j), then the
      // completed sum of T index j - KS + 1
      auto step = [&](int j, const SU3<float> &b) {
        if (active) {
#pragma unroll
          for (int m = 0; m < KS; m++)
            if (j - m >= 0 && j - m < nt && (!SLAB || t0 + m < tstarts)) // T = tmin + j - m
              acc[m] += gauge_trace<false>(a[m], b, false);
        }
        if (j - (KS - 1) >= 0)
          red[(size_t)(j - (KS - 1)) * nthreads + tid] = acc[KS - 1];
#pragma unroll
        for (int m = KS - 1; m > 0; m--)
          acc[m] = acc[m - 1];
        acc[0] = 0.f;
      };
      // two top lines in flight (b0, b1 alternate); a slot one past the last
      // step is still a slot of the column (in bounds, unused)
      const int nsteps = nt + KS - 1;
      SU3<float> b0, b1;
      if (active)
        b0 = Rows01Set::load(own, tt * cols + u);
#pragma unroll 1
      for (int j = 0; j < nsteps; j += 2) {
        tt = (tt + 1 == Lt) ? 0 : tt + 1;
        if (active)
          b1 = Rows01Set::load(own, tt * cols + u);
        rebuild_row2(b0);
        step(j, b0);
        tt = (tt + 1 == Lt) ? 0 : tt + 1;
        if (active)
          b0 = Rows01Set::load(own, tt * cols + u);
        if (j + 1 < nsteps) {
          rebuild_row2(b1);
          step(j + 1, b1);
        }
      }
      __syncthreads();
      // fixed-order sum over the block's threads (as wilson_gauge_kernel)
#pragma unroll 1
      for (int T = warp; T < nt; T += nwarps) {
        double v = 0.0;
        for (int i = lane; i < nthreads; i += 32)
          v += double(red[(size_t)T * nthreads + i]);
        v = warp_sum(v);
        if (lane == 0)
          part[(R - rmin) * nt + T] = v;
      }
    }
    __syncthreads();
  }
}

// Shared-memory records of SU(2) space lines (quaternions) for the SU(2)
// one-column kernel: FP32 one 16-byte vector per slot; FP64 two planes of
// 16-byte (a0, a1) and (a2, a3) pairs. A quarter-warp phase of 8 consecutive
// slots reads 128 contiguous bytes of a plane: conflict-free when the block's
// columns are a multiple of 8.
template <class T> struct QuatSet;
template <> struct QuatSet<float> {
  static constexpr int kBytes = 16;
  __device__ __forceinline__ static void store(unsigned char *set, int, int i,
                                               const SU2<float> &q) {
    reinterpret_cast<float4 *>(set)[i] = make_float4(q.a0, q.a1, q.a2, q.a3);
  }
  __device__ __forceinline__ static SU2<float> load(const unsigned char *set, int, int i) {
    const float4 v = reinterpret_cast<const float4 *>(set)[i];
    return {v.x, v.y, v.z, v.w};
  }
};
template <> struct QuatSet<double> {
  static constexpr int kBytes = 32;
  __device__ __forceinline__ static void store(unsigned char *set, int nslots, int i,
                                               const SU2<double> &q) {
    double2 *p = reinterpret_cast<double2 *>(set);
    p[i] = make_double2(q.a0, q.a1);
    p[nslots + i] = make_double2(q.a2, q.a3);
  }
  __device__ __forceinline__ static SU2<double> load(const unsigned char *set, int nslots,
                                                     int i) {
    const double2 *p = reinterpret_cast<const double2 *>(set);
    const double2 a = p[i], b = p[nslots + i];
    return {a.x, a.y, b.x, b.y};
  }
};

// The fundamental SU(2) loops with one column per thread and KS consecutive
// start slices of one cut whose space lines stay in registers (as
// wilson_gauge_reg_kernel for SU(3)). A quaternion loop is a 4-term dot
// product, so in the two-column kernel a step of the trace sweep spent more
// instructions on its shared-memory loads, bounds checks, rolling sums and
// index updates than on the loops themselves (0.87 instructions per cycle per
// scheduler, issue-bound). Here the sweep runs over T: each step loads one
// line into a register window and adds the KS loops of that T, with no checks
// and no moves. Per-thread sums in the compute type (FP32 for the mixed
// form), block and grid sums in FP64.
template <class Store, class CT, int KS, bool SLAB>
__global__ void __launch_bounds__(256)
    wilson_gauge_q_kernel(const __grid_constant__ Geom g, const __grid_constant__ Fields4 UA,
                          const __grid_constant__ Fields4 UB, int rmin, int rmax, int tmin,
                          int tmax, int cols, int rows, double *partials, const int *flag, int split, int tstarts) {
  if (flag && *flag != 0)
    return;
  using Q = SU2<CT>;
  using QS = QuatSet<CT>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Lt = g.L[3], h = split; // the first slice of cut B
  const int nt = tmax - tmin + 1;
  const int nthreads = blockDim.x;
  const int nslots = Lt * cols;
  CT *red = reinterpret_cast<CT *>(smem_raw); // [nt][nthreads]
  unsigned char *sa = smem_raw + ((sizeof(CT) * nt * nthreads + 15) & ~(size_t)15);
  unsigned char *sb = sa + (size_t)QS::kBytes * nslots;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31, nwarps = nthreads >> 5;
  const int u = tid % cols;
  const int row = tid / cols;
  const int nu = blockIdx.y;
  const int s0 = column_base(g, blockIdx.x, cols, nu) + u;
  const bool active = (row < rows) && (s0 < g.Vs);
  const int t0 = KS * row;
  const bool cut_a = t0 < h;
  unsigned char *own = cut_a ? sa : sb;
  unsigned char *other = cut_a ? sb : sa;
  const void *f_own = cut_a ? UA.f[nu] : UB.f[nu];
  const void *f_other = cut_a ? UB.f[nu] : UA.f[nu];
  const int Ln = sel4(g.L, nu), stn = sel4(g.stride, nu);
  const int xn = (s0 / stn) % Ln;
  const size_t V = g.V;
  const int ne = (rmax - rmin + 1) * nt;
  double *part = partials + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * ne;

  Q a[KS];
#pragma unroll 1
  for (int R = 1; R <= rmax; R++) {
    if (active) {
      const int l = s0 + ((xn + R - 1) % Ln - xn) * stn;
#pragma unroll
      for (int m = 0; m < KS; m++) {
        const int t = t0 + m;
        const int i = t * cols + u;
        const Q lo = Store::template load<CT>(f_own, V, l + t * g.Vs);
        const Q lx = Store::template load<CT>(f_other, V, l + t * g.Vs);
        if (R == 1) {
          a[m] = lo;
          QS::store(other, nslots, i, lx);
        } else {
          a[m] = mul(a[m], lo);
          QS::store(other, nslots, i, mul(QS::load(other, nslots, i), lx));
        }
        QS::store(own, nslots, i, a[m]);
      }
    }
    __syncthreads();
    if (R >= rmin) {
      // T-major sweep: the thread's sum for T index q is its KS loops of
      // starts t0 + m ending on the lines of relative index p = q + m
      // (slice t0 + tmin + p). A window of W = KS + 1 lines in registers
      // holds relative index p in w[p % W]; step q (unrolled by W, so every
      // slot index is a constant) loads the line p = q + KS that step q + 1
      // needs and adds the KS dot products of step q. Inactive threads load
      // nothing (zero lines) and write zero sums.
      constexpr int W = KS + 1;
      if (!active) {
#pragma unroll
        for (int m = 0; m < KS; m++)
          a[m] = Q{CT(0), CT(0), CT(0), CT(0)};
      }
      Q w[W];
      int tp = t0 + tmin; // slice of the next line to load
      tp = (tp >= Lt) ? tp - Lt : tp;
#pragma unroll
      for (int m = 0; m < KS; m++) {
        w[m] = active ? QS::load(own, nslots, tp * cols + u) : a[0];
        tp = (tp + 1 == Lt) ? 0 : tp + 1;
      }
#pragma unroll 1
      for (int q0 = 0; q0 < nt; q0 += W) {
#pragma unroll
        for (int r = 0; r < W; r++) {
          if (q0 + r < nt) {
            w[(r + KS) % W] = active ? QS::load(own, nslots, tp * cols + u) : a[0];
            tp = (tp + 1 == Lt) ? 0 : tp + 1;
            CT d[KS];
#pragma unroll
            for (int m = 0; m < KS; m++) {
              const Q &b = w[(r + m) % W];
              d[m] = (!SLAB || t0 + m < tstarts) ? dot4(a[m].a0, b.a0, a[m].a1, b.a1, a[m].a2, b.a2, a[m].a3, b.a3) : CT(0);
            }
#pragma unroll
            for (int k = 1; k < KS; k *= 2)
#pragma unroll
              for (int m = 0; m + k < KS; m += 2 * k)
                d[m] += d[m + k];
            red[(size_t)(q0 + r) * nthreads + tid] = d[0];
          }
        }
      }
      __syncthreads();
#pragma unroll 1
      for (int T = warp; T < nt; T += nwarps) {
        double v = 0.0;
        for (int i = lane; i < nthreads; i += 32)
          v += double(red[(size_t)T * nthreads + i]);
        v = warp_sum(v);
        if (lane == 0)
          part[(R - rmin) * nt + T] = v;
      }
    }
    __syncthreads();
  }
}

// The fixed-order tree over blocks (as reduce_partials_kernel in
// gc_wilson.cu) over the partials of whichever method ran.
__global__ void __launch_bounds__(256)
    reduce_select_kernel(const double *partials, int blocks_exact, int blocks_gauge,
                         const int *flag, int nr, int nt, double scale, double *out) {
  __shared__ double sh[256];
  const int e = blockIdx.x;
  const int nblocks = *flag ? blocks_exact : blocks_gauge;
  const int nentries = nr * nt;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    s += partials[(size_t)b * nentries + e];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int ir = e / nt, it = e % nt;
    out[it * nr + ir] = sh[0] * scale;
  }
}

// The one-column kernel runs the fundamental loops of the mixed SU(3) form
// when four consecutive start slices share a cut (8 divides Lt).
bool gauge_reg_applies(int Lt, int nc, int ct_bytes, bool adjoint) {
  return nc == 3 && ct_bytes == 4 && !adjoint && Lt % 8 == 0 && Lt / 4 <= 64;
}

// Start slices per thread of the SU(2) one-column kernel. Four in both
// forms: at SU(2) 48^4 mixed, R,T <= 24, eight starts (122 registers, 15
// warps per SM) took 5.68 ms against 5.15 ms for four (70 registers), which
// keep twice the threads per column resident.
constexpr int gauge_q_starts(int) { return 4; }
// The SU(2) one-column kernel runs the fundamental loops when a thread's
// consecutive start slices share a cut (2 x starts divides Lt).
// (at most 32 threads per column, so that a block of 8 columns fits)
bool gauge_q_applies(int Lt, int nc, int ct_bytes, bool adjoint) {
  const int ks = gauge_q_starts(ct_bytes);
  return nc == 2 && !adjoint && Lt % (2 * ks) == 0 && Lt / ks <= 32;
}

int largest_divisor_upto_g(int n, int cap) {
  for (int d = cap < n ? cap : n; d > 1; d--)
    if (n % d == 0)
      return d;
  return 1;
}

} // namespace

// Block shape: every start slice of a column has a thread (rows = Lt up to
// 64; beyond, the largest divisor of Lt up to 64 with Lt/rows slices each),
// and about 128 threads per block.
WilsonPlan wilson_gauge_plan(const Geom &g, int nt, int nc, int ct_bytes, int units_req,
                             bool adjoint) {
  WilsonPlan p{};
  const int Lt = g.L[3];
  const int ncomp = (nc == 3) ? 18 : 4;
  if (gauge_reg_applies(Lt, nc, ct_bytes, adjoint)) {
    // the one-column kernel: four starts per thread, columns of Lt/4 threads,
    // by default the largest power of two of columns with at most 128 threads
    // per block (SU(3) mixed, R,T <= L/2: 2.45 ms at 32^4 with 16 columns,
    // 0.59 ms at 24^4 with 16, 1.11 ms at 24^3 x 48 with 8; 2-15% slower
    // with twice or half the columns, 10-50% with a quarter)
    p.kernel = 1;
    p.starts = 4;
    p.rows = Lt / 4;
    int units = units_req;
    if (units <= 0)
      for (units = 1; 2 * units * p.rows <= 128;)
        units *= 2;
    p.cols_per_block = units;
    p.threads = wilson_threads(units, p.rows, 1);
    p.blocks = ((g.Vs + units - 1) / units) * 3;
    p.smem = ((size_t)nt * p.threads * sizeof(float) + 15) / 16 * 16 +
             2 * (size_t)Rows01Set::kBytes * Lt * units;
    p.fits = p.threads <= 256 && p.smem <= 200 * 1024;
    return p;
  }
  if (gauge_q_applies(Lt, nc, ct_bytes, adjoint)) {
    // the SU(2) one-column kernel: four starts per thread, columns of Lt / 4
    // threads, by default the largest power of two (at least 8) of columns
    // with at most 192 threads per block (48^4 mixed: 5.15 ms with 16
    // columns of 12 threads, 5.47 ms with 8)
    p.kernel = 2;
    p.starts = gauge_q_starts(ct_bytes);
    p.rows = Lt / p.starts;
    int units = units_req;
    if (units <= 0)
      for (units = 8; 2 * units * p.rows <= 192;)
        units *= 2;
    p.cols_per_block = units;
    p.threads = wilson_threads(units, p.rows, 1);
    p.blocks = ((g.Vs + units - 1) / units) * 3;
    p.smem = ((size_t)nt * p.threads * ct_bytes + 15) / 16 * 16 +
             2 * (size_t)(ct_bytes == 4 ? 16 : 32) * Lt * units;
    p.fits = p.threads <= 256 && p.smem <= 200 * 1024;
    return p;
  }
  const int lanes = wilson_lanes(nc, ct_bytes);
  // consecutive start slices per thread (a divisor of the cut slice h = Lt/2,
  // so that a thread's starts share a cut): 2 for SU(3) (its registers hold
  // two lane-packed matrices), 4 for SU(2) (quaternions are small)
  p.starts = 1;
  for (int ks : {nc == 2 ? 4 : 2, 2})
    if (p.starts == 1 && Lt % (2 * ks) == 0 && Lt / ks <= 64)
      p.starts = ks;
  p.rows = p.starts > 1 ? Lt / p.starts : largest_divisor_upto_g(Lt, 64);
  // (about 128 threads: at SU(3) 32^4 the paired kernel took 5.5, 4.6, 3.8,
  // 3.1, 3.1 ms mixed with 1, 2, 4, 8, 16 column units of 16 threads; wider
  // blocks coalesce the extension's link loads)
  const int units = units_req > 0 ? units_req : std::max(1, 128 / p.rows);
  p.cols_per_block = units * lanes;
  p.threads = wilson_threads(p.cols_per_block, p.rows, lanes);
  p.blocks = ((g.Vs + p.cols_per_block - 1) / p.cols_per_block) * 3;
  const size_t sets = 2 * (size_t)ncomp * Lt * wilson_col_stride(p.cols_per_block, lanes) *
                      ct_bytes;
  // (the per-thread sums: GAcc, FP32 for the mixed form's fundamental loops)
  const size_t acc = (!adjoint && ct_bytes == 4) ? 4 : 8;
  p.smem = ((size_t)nt * p.threads * acc + 15) / 16 * 16 + sets;
  p.fits = p.threads <= 256 && p.smem <= 200 * 1024;
  return p;
}

bool wilson_gauge_applies(const Geom &g, int tmax, int nt, int nc, int ct_bytes, int tstarts) {
  const int Lt = g.L[3];
  const bool slab = tstarts > 0 && tstarts < Lt;
  if (Lt < 2 || tmax > (slab ? Lt - tstarts : Lt / 2))
    return false;
  // (the fundamental and the adjoint loops may take different kernels)
  return wilson_gauge_plan(g, nt, nc, ct_bytes, 0, true).fits &&
         wilson_gauge_plan(g, nt, nc, ct_bytes, 0, false).fits;
}

double wilson_gauge_tolerance(int ct_bytes) { return ct_bytes == 8 ? 1e-14 : 1e-6; }

size_t wilson_gauge_line_bytes(const Geom &g, int nc) {
  return ((size_t)(nc == 3 ? 144 : 32) * (size_t)g.V + 255) / 256 * 256;
}

template <class Store, class CT>
int launch_wilson_gauge_prep(const Geom &g, const Fields4 &U, void *GA, void *GB,
                             const Fields4 &UA, const Fields4 &UB, int *flag,
                             cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), s);
  if (e != cudaSuccess)
    return launch_check("gauge flag reset");
  // (the two cuts' lines in separate blocks: blockIdx.y = 0 for cut A and
  // the defect check, 1 for cut B)
  gauge_lines_kernel<Store><<<dim3((g.Vs + 127) / 128, 2), 128, 0, s>>>(
      g, U.f[3], GA, GB, g.L[3] / 2, wilson_gauge_tolerance((int)sizeof(CT)), flag);
  int rc = launch_check("gauge_lines_kernel");
  if (rc)
    return rc;
  gauge_transform_kernel<Store><<<dim3((g.V + 127) / 128, 3), 128, 0, s>>>(g, U, GA, GB, UA,
                                                                          UB);
  return launch_check("gauge_transform_kernel");
}

template <class Store, class CT>
int launch_wilson_gauge_kernel(const Geom &g, const Fields4 &UA, const Fields4 &UB, int rmin,
                               int rmax, int tmin, int tmax, bool adjoint, const int *flag,
                               double *partials, int *blocks, cudaStream_t s, int units = 0,
                               int tstarts = 0) {
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  // every start slice in two cuts (A at slice 0, B at Lt/2), or the start
  // slices [0, tstarts) of a time slab in cut A alone
  const int Lt = g.L[3];
  const bool slab = tstarts > 0 && tstarts < Lt;
  const int split = slab ? Lt : Lt / 2;
  if (!slab)
    tstarts = Lt;
  if (tmax > (slab ? Lt - tstarts : Lt / 2))
    return plan_error(slab ? "wilson_gauge_kernel: time_max above Lt - t_starts"
                           : "wilson_gauge_kernel: time_max above Lt/2");
  const WilsonPlan p = wilson_gauge_plan(g, nt, Store::NC, (int)sizeof(CT), units, adjoint);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cap);
  const bool capturing = cap != cudaStreamCaptureStatusNone;
  if (!p.fits || nr * nt > kWilsonMaxEntries)
    return plan_error("wilson_gauge_kernel: block shape does not fit");
  auto go = [&](auto kernel) {
    int r = allow_large_smem(kernel, p.smem, capturing);
    if (r)
      return r;
    kernel<<<dim3(p.blocks / 3, 3), p.threads, p.smem, s>>>(
        g, UA, UB, rmin, rmax, tmin, tmax, p.cols_per_block, p.rows, partials, flag, split,
        tstarts);
    return GC_OK;
  };
  int rc;
  // (four starts per thread for SU(2), and in the one-column kernel for the
  // mixed SU(3) form's fundamental loops, as the plan chooses)
  constexpr int K4 = Store::NC == 2 ? 4 : 2;
  if constexpr (Store::NC == 2) {
    if (p.kernel == 2) {
      constexpr int KS = gauge_q_starts((int)sizeof(CT));
      rc = slab ? go(wilson_gauge_q_kernel<Store, CT, KS, true>)
                : go(wilson_gauge_q_kernel<Store, CT, KS, false>);
      if (rc)
        return rc;
      *blocks = p.blocks;
      return launch_check("wilson_gauge_q_kernel");
    }
  }
  if constexpr (std::is_same<Store, StoreF32SU3>::value) {
    if (p.kernel == 1) {
      rc = slab ? go(wilson_gauge_reg_kernel<4, true>) : go(wilson_gauge_reg_kernel<4, false>);
      if (rc)
        return rc;
      *blocks = p.blocks;
      return launch_check("wilson_gauge_reg_kernel");
    }
  }
  // (the start-slice checks of a t-slab compiled in only where they are used)
  auto go2 = [&](auto k_all, auto k_slab) { return slab ? go(k_slab) : go(k_all); };
  if (adjoint)
    rc = p.starts == 4   ? go2(wilson_gauge_kernel<Store, CT, true, K4, false>,
                               wilson_gauge_kernel<Store, CT, true, K4, true>)
         : p.starts == 2 ? go2(wilson_gauge_kernel<Store, CT, true, 2, false>,
                               wilson_gauge_kernel<Store, CT, true, 2, true>)
                         : go2(wilson_gauge_kernel<Store, CT, true, 1, false>,
                               wilson_gauge_kernel<Store, CT, true, 1, true>);
  else
    rc = p.starts == 4   ? go2(wilson_gauge_kernel<Store, CT, false, K4, false>,
                               wilson_gauge_kernel<Store, CT, false, K4, true>)
         : p.starts == 2 ? go2(wilson_gauge_kernel<Store, CT, false, 2, false>,
                               wilson_gauge_kernel<Store, CT, false, 2, true>)
                         : go2(wilson_gauge_kernel<Store, CT, false, 1, false>,
                               wilson_gauge_kernel<Store, CT, false, 1, true>);
  if (rc)
    return rc;
  *blocks = p.blocks;
  return launch_check("wilson_gauge_kernel");
}

template <class Store, class CT>
int launch_wilson_gauge(const Geom &g, const Fields4 &UA, const Fields4 &UB, int rmin,
                        int rmax, int tmin, int tmax, bool adjoint, double *partials,
                        double *out_dev, cudaStream_t s) {
  int blocks = 0;
  const int rc = launch_wilson_gauge_kernel<Store, CT>(g, UA, UB, rmin, rmax, tmin, tmax,
                                                       adjoint, nullptr, partials, &blocks, s);
  if (rc)
    return rc;
  return launch_reduce_wilson(partials, blocks, rmax - rmin + 1, tmax - tmin + 1,
                              wilson_scale(g.V, Store::NC, adjoint), out_dev, s);
}

template <class Store, class CT>
int launch_wilson_auto(const Geom &g, const Fields4 &U, const Fields4 &UA, const Fields4 &UB,
                       int rmin, int rmax, int tmin, int tmax, bool adjoint, const int *flag,
                       double *partials, double *out_dev, cudaStream_t s, int units,
                       int tstarts) {
  if (tstarts <= 0 || tstarts > g.L[3])
    tstarts = g.L[3];
  int b_exact = 0, b_gauge = 0;
  int rc = launch_wilson_exact_gated<Store, CT>(g, U, rmin, rmax, tmin, tmax, adjoint, flag,
                                                partials, &b_exact, s, tstarts);
  if (rc)
    return rc;
  rc = launch_wilson_gauge_kernel<Store, CT>(g, UA, UB, rmin, rmax, tmin, tmax, adjoint, flag,
                                             partials, &b_gauge, s, units, tstarts);
  if (rc)
    return rc;
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  // average over the loops counted: every site, or the tstarts slices
  reduce_select_kernel<<<nr * nt, 256, 0, s>>>(
      partials, b_exact, b_gauge, flag, nr, nt,
      wilson_scale((long long)g.Vs * tstarts, Store::NC, adjoint), out_dev);
  return launch_check("reduce_select_kernel");
}

size_t wilson_auto_partials_count(const Geom &g, int nr, int nt, int nc, int units) {
  int blocks = 0;
  for (int ct : {4, 8})
    for (bool adj : {false, true})
      blocks = std::max(blocks, wilson_gauge_plan(g, nt, nc, ct, units, adj).blocks);
  return std::max<size_t>(wilson_partials_count(g, nr, nt, nc), (size_t)blocks * nr * nt);
}

// Times one launch of the gauge W kernel of a lattice with `units` column
// units per block (the autotuner's candidate), from prepared transformed
// links; partials must hold wilson_auto_partials_count(.., units) doubles.
template <class Store, class CT>
int time_wilson_gauge(const Geom &g, const Fields4 &UA, const Fields4 &UB, int rmin, int rmax,
                      int tmin, int tmax, int units, double *partials, cudaStream_t s,
                      float *ms) {
  const WilsonPlan p =
      wilson_gauge_plan(g, tmax - tmin + 1, Store::NC, (int)sizeof(CT), units, false);
  if (!p.fits)
    return GC_ERR_ARG;
  int blocks = 0;
  int rc = launch_wilson_gauge_kernel<Store, CT>(g, UA, UB, rmin, rmax, tmin, tmax, false,
                                                 nullptr, partials, &blocks, s, units);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 3 && rc == GC_OK; rep++) {
    cudaEventRecord(e0, s);
    rc = launch_wilson_gauge_kernel<Store, CT>(g, UA, UB, rmin, rmax, tmin, tmax, false,
                                               nullptr, partials, &blocks, s, units);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    best = std::min(best, t);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = best;
  return rc;
}

#define GC_INSTANTIATE_WG(STORE, CT)                                                        \
  template int launch_wilson_gauge_prep<STORE, CT>(const Geom &, const Fields4 &, void *,   \
                                                   void *, const Fields4 &, const Fields4 &, \
                                                   int *, cudaStream_t);                    \
  template int launch_wilson_gauge<STORE, CT>(const Geom &, const Fields4 &, const Fields4 &, \
                                              int, int, int, int, bool, double *, double *,  \
                                              cudaStream_t);                                 \
  template int launch_wilson_auto<STORE, CT>(const Geom &, const Fields4 &, const Fields4 &,  \
                                             const Fields4 &, int, int, int, int, bool,       \
                                             const int *, double *, double *, cudaStream_t,   \
                                             int, int);                                       \
  template int time_wilson_gauge<STORE, CT>(const Geom &, const Fields4 &, const Fields4 &,   \
                                            int, int, int, int, int, double *, cudaStream_t,  \
                                            float *);

GC_INSTANTIATE_WG(StoreF64SU3, double)
GC_INSTANTIATE_WG(StoreF64SU2, double)
GC_INSTANTIATE_WG(StoreF32SU3, float)
GC_INSTANTIATE_WG(StoreF32SU2, float)

} // namespace gc
