// Off-axis Wilson loops (sm_100a kernels and the host-side plan).
//
// Reference: wilson_offaxis / wilson_offaxis_adjoint and their _result
// wrappers (lib/cpu/include/wilson_loops.h:313-663), the space lines along a
// step pattern (wilson_line_offaxis, wilson_lines_offaxis :113-137, 195-213),
// the per-loop sums (calculate_wilson_loop_offaxis[_adjoint] :241-310), and
// the direction, pattern, permutation, reflection and merge helpers
// (lib/cpu/src/basic_observables.cpp:167-186, 543-623, 754-840).
//
// A spatial direction d = (a1, a2, a3), a1 >= a2 >= a3, is walked as a
// staircase of unit links (Bresenham's pattern), and the staircase is taken
// in every permuted and reflected orientation and repeated m times for the
// lengths m |d| in the requested range. For one such space line S (pattern,
// displacement D) and time extent T the loop is
//     Re Tr[ L(x,T) S(x+T t) L(x+D,T)^dag S(x)^dag ] / N   (or |Tr|^2 - 1),
// averaged over all sites x.
//
// offaxis_fused_kernel: a block owns a few spatial columns over all t and a
// group of lines. Per line, a thread per (column, t) forms the product of
// the pattern's links (a negative step moves back first and multiplies by
// the link's adjoint) into shared memory, beside the columns' own time links
// (loaded once per block) and the displaced columns' time links; then the
// same exact recursion as the on-axis kernel, K_0 = S(x),
// K_T = U_t(x+(T-1)t)^dag K_{T-1} U_t(x+D+(T-1)t), value Re Tr[S(x+T t) K_T^dag],
// reads only shared memory. line_loop_kernel is that recursion over a line
// field in global memory, thread per site, for the spatial loops (any
// "time" axis). Fixed-order warp / block / grid sums (deterministic).
#include "gc_internal.cuh"
#include "gc_kernels.h"

#include <algorithm>
#include <cmath>

namespace gc {

namespace {

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Re Tr(a b^dag) (raw trace for SU(3), a.b = Re Tr / 2 for SU(2)) or the
// adjoint character from it.
template <bool ADJ, class T> __device__ __forceinline__ double offaxis_value(const SU3<T> &a,
                                                                            const SU3<T> &b) {
  double re = 0, im = 0;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const cx<T> x = a.e[k / 3][k % 3], y = b.e[k / 3][k % 3];
    re += double(GC_FMA(x.re, y.re, x.im * y.im));
    im += double(GC_FMA(x.im, y.re, -(x.re * y.im)));
  }
  return ADJ ? fma(re, re, fma(im, im, -1.0)) : re;
}
template <bool ADJ, class T> __device__ __forceinline__ double offaxis_value(const SU2<T> &a,
                                                                            const SU2<T> &b) {
  const double d = dot4(double(a.a0), double(b.a0), double(a.a1), double(b.a1),
                        double(a.a2), double(b.a2), double(a.a3), double(b.a3));
  return ADJ ? 4.0 * d * d - 1.0 : d;
}

// partials[block * nt + (T - tmin)]. The loop's "time" axis is ax (3 for the
// off-axis loops, a spatial axis for the spatial loops), with its links in
// the field Ut; d holds the displacement of the line's end as non-negative
// residues (d[ax] = 0).
template <class Store, class CT, bool ADJ>
__global__ void __launch_bounds__(256)
    line_loop_kernel(const __grid_constant__ Geom g, const void *Ut, int ax, const void *S,
                     int4 d, int tmin, int tmax, double *partials, int pstride) {
  using M = typename Store::template M<CT>;
  using IS = typename InterStore<Store>::type;
  extern __shared__ double wacc[]; // [nwarps][nt]
  const int nt = tmax - tmin + 1;
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < nwarps * nt; i += blockDim.x)
    wacc[i] = 0.0;
  __syncthreads();
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = site < g.V;
  const size_t V = g.V;
  const int La = sel4(g.L, ax), sta = sel4(g.stride, ax);
  int base = 0, baseD = 0, t = 0;
  if (active) {
    int x[4];
    site_coords(g, site, x);
    const int xd[4] = {(x[0] + d.x) % g.L[0], (x[1] + d.y) % g.L[1], (x[2] + d.z) % g.L[2],
                       (x[3] + d.w) % g.L[3]};
    const int siteD = xd[0] + g.L[0] * (xd[1] + g.L[1] * (xd[2] + g.L[2] * xd[3]));
    t = sel4(x, ax);
    base = site - t * sta;
    baseD = siteD - t * sta;
  }
  M K = active ? IS::template load<CT>(S, V, site) : unit(M());
  int tt = t; // (t + T - 1) mod La
#pragma unroll 1
  for (int T = 1; T <= tmax; T++) {
    int tu = tt + 1;
    tu = (tu == La) ? 0 : tu;
    if (active) {
      M a = Store::template load<CT>(Ut, V, base + tt * sta);
      M b = Store::template load<CT>(Ut, V, baseD + tt * sta);
      K = mul(mul_da(a, K), b);
    }
    if (T >= tmin) {
      double v = active ? offaxis_value<ADJ>(IS::template load<CT>(S, V, base + tu * sta), K)
                        : 0.0;
      v = warp_sum_d(v);
      if (lane == 0)
        wacc[warp * nt + (T - tmin)] += v;
    }
    tt = tu;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nt; e += blockDim.x) {
    double sum = 0.0;
    for (int w = 0; w < nwarps; w++)
      sum += wacc[w * nt + e];
    partials[(size_t)blockIdx.x * pstride + e] = sum;
  }
}

// S(x) <- (init ? F(x) : S(x)) * F(x + offset ax)^count, F a single-direction
// link field along ax (the straight-line helpers of the spatial loops,
// wilson_lines_single_direction_indexed / _prolong, wilson_loops.h:1268-1300).
template <class Store, class CT>
__global__ void __launch_bounds__(256)
    line_extend_kernel(const __grid_constant__ Geom g, const void *F, void *S, int ax,
                       int offset, int count, int init) {
  using M = typename Store::template M<CT>;
  using IS = typename InterStore<Store>::type;
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  if (site >= g.V)
    return;
  const size_t V = g.V;
  int x[4];
  site_coords(g, site, x);
  M A = init ? Store::template load<CT>(F, V, site) : IS::template load<CT>(S, V, site);
  if (count > 0) {
    const int fo = site + fwd_off(g, sel4(x, ax), ax, offset);
    const M u = Store::template load<CT>(F, V, fo);
#pragma unroll 1
    for (int i = 0; i < count; i++)
      A = mul(A, u);
  }
  IS::template store<CT>(S, V, site, A);
}

constexpr int kOffaxisBlock = 128;

// Matrices in shared memory as planes of complex entries (float2 / double2),
// [entry][slot], so that consecutive threads (consecutive slots) touch
// consecutive words and a matrix is 9 (SU(2): 2) vector loads.
template <class T> struct Vec2;
template <> struct Vec2<float> {
  using type = float2;
};
template <> struct Vec2<double> {
  using type = double2;
};

template <class T>
__device__ __forceinline__ void sm_store(T *a, int nslots, int i, const SU3<T> &m) {
  using V = typename Vec2<T>::type;
  V *p = reinterpret_cast<V *>(a) + i;
#pragma unroll
  for (int k = 0; k < 9; k++)
    p[k * nslots] = V{m.e[k / 3][k % 3].re, m.e[k / 3][k % 3].im};
}
template <class T> __device__ __forceinline__ SU3<T> sm_load(const T *a, int nslots, int i,
                                                             SU3<T> *) {
  using V = typename Vec2<T>::type;
  const V *p = reinterpret_cast<const V *>(a) + i;
  SU3<T> m;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const V v = p[k * nslots];
    m.e[k / 3][k % 3] = {v.x, v.y};
  }
  return m;
}
template <class T>
__device__ __forceinline__ void sm_store(T *a, int nslots, int i, const SU2<T> &m) {
  using V = typename Vec2<T>::type;
  V *p = reinterpret_cast<V *>(a) + i;
  p[0] = V{m.a0, m.a1};
  p[nslots] = V{m.a2, m.a3};
}
template <class T> __device__ __forceinline__ SU2<T> sm_load(const T *a, int nslots, int i,
                                                             SU2<T> *) {
  using V = typename Vec2<T>::type;
  const V *p = reinterpret_cast<const V *>(a) + i;
  const V u = p[0], v = p[nslots];
  return {u.x, u.y, v.x, v.y};
}

// One step of a space line from the site `cur` with spatial coordinates
// (x0, x1, x2): e = +a moves forward along axis a-1 and returns the link it
// crossed, e = -a moves back and returns the adjoint of the link it crossed.
template <class Store, class CT>
__device__ __forceinline__ typename Store::template M<CT>
step_link(const Geom &g, const Fields4 &U, int e, int &x0, int &x1, int &x2, int &cur) {
  using M = typename Store::template M<CT>;
  const size_t V = g.V;
  const int mu = (e > 0 ? e : -e) - 1;
  const int Lm = sel4(g.L, mu), st = sel4(g.stride, mu);
  int cm = mu == 0 ? x0 : (mu == 1 ? x1 : x2);
  // (a select, not U.f[mu]: an indexed parameter array goes to the stack)
  const void *f = mu == 0 ? U.f[0] : (mu == 1 ? U.f[1] : U.f[2]);
  M u;
  if (e > 0) {
    u = Store::template load<CT>(f, V, cur);
    cur += (cm == Lm - 1) ? -(Lm - 1) * st : st;
    cm = (cm == Lm - 1) ? 0 : cm + 1;
  } else {
    cur += (cm == 0) ? (Lm - 1) * st : -st;
    cm = (cm == 0) ? Lm - 1 : cm - 1;
    u = adjoint(Store::template load<CT>(f, V, cur));
  }
  if (mu == 0)
    x0 = cm;
  else if (mu == 1)
    x1 = cm;
  else
    x2 = cm;
  return u;
}

// Lines per block of the fused kernel (the block loads its columns' time
// links once for these).
constexpr int kOffaxisLinesPerBlock = 8;

// Block shape of the fused kernel: rows threads per column (one start slice
// each up to Lt = 64), cols columns, about 128 threads (256 when rows > 32),
// shared memory (three sets of Lt x cols matrices) at most ~100 KB.
struct FusedShape {
  int rows, cols, threads;
  size_t smem;
};
FusedShape fused_shape(const Geom &g, int nc, int ct_bytes, int nt) {
  FusedShape f;
  const int Lt = g.L[3];
  f.rows = 1;
  for (int d = 64; d >= 1; d--)
    if (d <= Lt && Lt % d == 0) {
      f.rows = d;
      break;
    }
  f.cols = std::max(1, (f.rows > 32 ? 256 : 128) / f.rows);
  const size_t nreal = nc == 3 ? 18 : 4;
  auto smem_of = [&](int cols, int threads) {
    return ((size_t)(threads / 32) * nt + 1) / 2 * 2 * sizeof(double) +
           3 * nreal * (size_t)Lt * cols * ct_bytes;
  };
  for (;;) {
    f.threads = (f.cols * f.rows + 31) / 32 * 32;
    f.smem = smem_of(f.cols, f.threads);
    if (f.cols == 1 || f.smem <= 100 * 1024)
      break;
    f.cols--;
  }
  return f;
}

// Off-axis loops, fused (see launch_offaxis_fused): line products walked
// from each (column, t), then the T walk of line_loop_kernel with every
// operand in shared memory.
template <class Store, class CT, bool ADJ>
__device__ __forceinline__ void offaxis_fused_body(const Geom &g, const Fields4 &U,
                                                   const OffaxisLineDesc *__restrict__ lines,
                                                   int nlines, int tmin, int tmax, int cols,
                                                   int rows, double *partials) {
  using M = typename Store::template M<CT>;
  constexpr int NREAL = Store::NC == 3 ? 18 : 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Lt = g.L[3];
  const int nt = tmax - tmin + 1;
  const int nslots = Lt * cols;
  const int nwarps = blockDim.x >> 5;
  double *wacc = reinterpret_cast<double *>(smem_raw); // [nwarps][nt]
  CT *ucol = reinterpret_cast<CT *>(wacc + ((nwarps * nt + 1) & ~1));
  CT *ncol = ucol + NREAL * nslots;
  CT *scol = ncol + NREAL * nslots;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int c = tid % cols, row = tid / cols;
  const int s = blockIdx.x * cols + c;
  const bool active = row < rows && s < g.Vs;
  const int kt = Lt / rows;
  const size_t V = g.V;
  const int xs0 = s % g.L[0], xs1 = (s / g.L[0]) % g.L[1], xs2 = s / (g.L[0] * g.L[1]);
  if (active) {
#pragma unroll 1
    for (int k = 0; k < kt; k++) {
      const int t = row + k * rows;
      sm_store(ucol, nslots, t * cols + c, Store::template load<CT>(U.f[3], V, s + t * g.Vs));
    }
  }
  const int l0 = blockIdx.y * kOffaxisLinesPerBlock;
  const int l1 = min(nlines, l0 + kOffaxisLinesPerBlock);
#pragma unroll 1
  for (int l = l0; l < l1; l++) {
    const OffaxisLineDesc *L = lines + l;
    const int n = __ldg(&L->n);
    for (int i = tid; i < nwarps * nt; i += blockDim.x)
      wacc[i] = 0.0;
    if (active) {
      const int sd = (xs0 + __ldg(&L->d[0])) % g.L[0] +
                     g.L[0] * ((xs1 + __ldg(&L->d[1])) % g.L[1] +
                               g.L[1] * ((xs2 + __ldg(&L->d[2])) % g.L[2]));
#pragma unroll 1
      for (int k = 0; k < kt; k++) {
        const int t = row + k * rows;
        const int i = t * cols + c;
        sm_store(ncol, nslots, i, Store::template load<CT>(U.f[3], V, sd + t * g.Vs));
        // the line from (s, t): steps along the spatial axes, periodic. The
        // link of step q+1 is loaded before step q's product (its address
        // needs only the step pattern), so the load's latency overlaps it.
        int x0 = xs0, x1 = xs1, x2 = xs2;
        int cur = s + t * g.Vs;
        // the first factor is taken as it is (identity times a link is exact)
        M A = step_link<Store, CT>(g, U, __ldg(&L->s[0]), x0, x1, x2, cur);
        M u = (n > 1) ? step_link<Store, CT>(g, U, __ldg(&L->s[1]), x0, x1, x2, cur) : A;
#pragma unroll 1
        for (int q = 1; q < n; q++) {
          const M cu = u;
          if (q + 1 < n)
            u = step_link<Store, CT>(g, U, __ldg(&L->s[q + 1]), x0, x1, x2, cur);
          A = mul(A, cu);
        }
        sm_store(scol, nslots, i, A);
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int k = 0; k < kt; k++) {
      const int t0 = row + k * rows;
      M K = active ? sm_load(scol, nslots, t0 * cols + c, (M *)nullptr) : unit(M());
      int tt = t0; // (t0 + T - 1) mod Lt
#pragma unroll 1
      for (int T = 1; T <= tmax; T++) {
        int tu = tt + 1;
        tu = (tu == Lt) ? 0 : tu;
        if (active) {
          const int i = tt * cols + c;
          K = mul(mul_da(sm_load(ucol, nslots, i, (M *)nullptr), K),
                  sm_load(ncol, nslots, i, (M *)nullptr));
        }
        if (T >= tmin) {
          double v = active ? offaxis_value<ADJ>(
                                  sm_load(scol, nslots, tu * cols + c, (M *)nullptr), K)
                            : 0.0;
          v = warp_sum_d(v);
          if (lane == 0)
            wacc[warp * nt + (T - tmin)] += v;
        }
        tt = tu;
      }
    }
    __syncthreads();
    for (int e = tid; e < nt; e += blockDim.x) {
      double sum = 0.0;
      for (int w = 0; w < nwarps; w++)
        sum += wacc[w * nt + e];
      partials[((size_t)blockIdx.x * nlines + l) * nt + e] = sum;
    }
    __syncthreads();
  }
}

// Two entry points: the FP32 form with its registers held to 85 per thread
// (three 256-thread blocks per SM: 79 registers, no spills, where the
// unbounded build took 105 and kept a third fewer warps resident, 36 -> 32
// ms per 24^4 call); the FP64 form without a minimum (an explicit minimum of
// one block made it take 180 registers instead of 154).
template <class Store, class CT, bool ADJ>
__global__ void __launch_bounds__(256, 3)
    offaxis_fused_kernel_f32(const __grid_constant__ Geom g, const __grid_constant__ Fields4 U,
                             const OffaxisLineDesc *__restrict__ lines, int nlines, int tmin,
                             int tmax, int cols, int rows, double *partials) {
  offaxis_fused_body<Store, CT, ADJ>(g, U, lines, nlines, tmin, tmax, cols, rows, partials);
}
template <class Store, class CT, bool ADJ>
__global__ void __launch_bounds__(256)
    offaxis_fused_kernel(const __grid_constant__ Geom g, const __grid_constant__ Fields4 U,
                         const OffaxisLineDesc *__restrict__ lines, int nlines, int tmin,
                         int tmax, int cols, int rows, double *partials) {
  offaxis_fused_body<Store, CT, ADJ>(g, U, lines, nlines, tmin, tmax, cols, rows, partials);
}

} // namespace

int offaxis_partials_count(const Geom &g, int nt) {
  return ((g.V + kOffaxisBlock - 1) / kOffaxisBlock) * nt;
}

int offaxis_fused_blocks(const Geom &g, int nc, int ct_bytes) {
  const FusedShape f = fused_shape(g, nc, ct_bytes, 1);
  return (g.Vs + f.cols - 1) / f.cols;
}

template <class Store, class CT>
int launch_offaxis_fused(const Geom &g, const Fields4 &U, const OffaxisLineDesc *lines,
                         int nlines, int tmin, int tmax, bool adjoint, double *partials,
                         int *blocks, cudaStream_t s) {
  const int nt = tmax - tmin + 1;
  if (nt < 1 || nt > kWilsonMaxEntries || nlines < 1)
    return plan_error("offaxis_fused_kernel: time range or line count");
  const FusedShape f = fused_shape(g, Store::NC, (int)sizeof(CT), nt);
  if (f.smem > 227 * 1024)
    return plan_error("offaxis_fused_kernel: time extent too large for shared memory");
  const int colblocks = (g.Vs + f.cols - 1) / f.cols;
  const dim3 grid(colblocks, (nlines + kOffaxisLinesPerBlock - 1) / kOffaxisLinesPerBlock);
  auto launch = [&](auto kernel) {
    int rc = allow_large_smem(kernel, f.smem);
    if (!rc)
      kernel<<<grid, f.threads, f.smem, s>>>(g, U, lines, nlines, tmin, tmax, f.cols, f.rows,
                                             partials);
    return rc;
  };
  int rc;
  if constexpr (sizeof(CT) == 4)
    rc = adjoint ? launch(offaxis_fused_kernel_f32<Store, CT, true>)
                 : launch(offaxis_fused_kernel_f32<Store, CT, false>);
  else
    rc = adjoint ? launch(offaxis_fused_kernel<Store, CT, true>)
                 : launch(offaxis_fused_kernel<Store, CT, false>);
  if (rc)
    return rc;
  if (blocks)
    *blocks = colblocks;
  return launch_check("offaxis_fused_kernel");
}

double line_loop_scale(const Geom &g, int nc, bool adjoint) {
  // averages over V sites (calculate_wilson_loop_offaxis and
  // wilson_spatial_plane_indexed divide by V); the fundamental SU(3) value is
  // Re Tr / 3 (tr_real, multiply_conj_tr)
  return 1.0 / ((double)g.V * ((!adjoint && nc == 3) ? 3.0 : 1.0));
}

template <class Store, class CT>
int launch_line_loops(const Geom &g, const void *Ut, int ax, const void *S, const int disp[4],
                      int tmin, int tmax, bool adjoint, double *partials, double *out_dev,
                      cudaStream_t s, int pstride) {
  const int nt = tmax - tmin + 1;
  if (nt < 1 || nt > kWilsonMaxEntries)
    return plan_error("line_loop_kernel: time range");
  if (ax < 0 || ax > 3 || disp[ax] != 0)
    return plan_error("line_loop_kernel: axis");
  const int blocks = (g.V + kOffaxisBlock - 1) / kOffaxisBlock;
  const size_t smem = (size_t)(kOffaxisBlock / 32) * nt * sizeof(double);
  // displacement as non-negative residues
  int d[4];
  for (int i = 0; i < 4; i++)
    d[i] = ((disp[i] % g.L[i]) + g.L[i]) % g.L[i];
  const int4 d4 = make_int4(d[0], d[1], d[2], d[3]);
  if (pstride < nt)
    pstride = nt;
  if (adjoint)
    line_loop_kernel<Store, CT, true><<<blocks, kOffaxisBlock, smem, s>>>(
        g, Ut, ax, S, d4, tmin, tmax, partials, pstride);
  else
    line_loop_kernel<Store, CT, false><<<blocks, kOffaxisBlock, smem, s>>>(
        g, Ut, ax, S, d4, tmin, tmax, partials, pstride);
  int rc = launch_check("line_loop_kernel");
  if (rc || !out_dev)
    return rc;
  return launch_reduce_rows(partials, blocks, nt, line_loop_scale(g, Store::NC, adjoint),
                            out_dev, s);
}

template <class Store, class CT>
int launch_line_extend(const Geom &g, const void *F, void *S, int ax, int offset, int count,
                       bool init, cudaStream_t s) {
  if (ax < 0 || ax > 3 || count < 0 || offset < 0)
    return plan_error("line_extend_kernel: arguments");
  line_extend_kernel<Store, CT><<<(g.V + 255) / 256, 256, 0, s>>>(g, F, S, ax, offset, count,
                                                                  init ? 1 : 0);
  return launch_check("line_extend_kernel");
}

#define GC_INSTANTIATE_O(STORE, CT)                                                        \
  template int launch_line_loops<STORE, CT>(const Geom &, const void *, int, const void *, \
                                            const int *, int, int, bool, double *,        \
                                            double *, cudaStream_t, int);                 \
  template int launch_line_extend<STORE, CT>(const Geom &, const void *, void *, int, int,  \
                                             int, bool, cudaStream_t);                     \
  template int launch_offaxis_fused<STORE, CT>(const Geom &, const Fields4 &,              \
                                               const OffaxisLineDesc *, int, int, int,     \
                                               bool, double *, int *, cudaStream_t);

GC_INSTANTIATE_O(StoreF64SU3, double)
GC_INSTANTIATE_O(StoreF64SU2, double)
GC_INSTANTIATE_O(StoreF32SU3, float)
GC_INSTANTIATE_O(StoreF32SU2, float)

// ------------------------------------------------------------------ host plan
// Spatial directions with a1 >= a2 >= a3, a1 in [1, length_max], one per
// slope: a candidate proportional to one already taken is skipped
// (generate_directions / is_direction_same, basic_observables.cpp:754-788).
std::vector<std::array<int, 3>> offaxis_directions(int length_max) {
  std::vector<std::array<int, 3>> dirs;
  for (int a1 = 1; a1 <= length_max; a1++)
    for (int a2 = 0; a2 <= length_max; a2++)
      for (int a3 = 0; a3 <= length_max; a3++) {
        if (!(a1 >= a2 && a2 >= a3))
          continue;
        bool fresh = true;
        for (const auto &d : dirs)
          if (d[0] * a2 == d[1] * a1 && d[0] * a3 == d[2] * a1)
            fresh = false;
        if (fresh)
          dirs.push_back({a1, a2, a3});
      }
  return dirs;
}

namespace {

// Bresenham staircase of a direction (make_offaxis_pattern,
// basic_observables.cpp:819-840): axis numbers 1..3, one 1 per unit of a1,
// with the 2s and 3s placed by the error terms of the two slopes.
std::vector<int> staircase(const std::array<int, 3> &d) {
  std::vector<int> p;
  int e1 = -d[1], e2 = -d[2];
  for (int i = 0; i < d[0]; i++) {
    e1 += 2 * d[1];
    e2 += 2 * d[2];
    if (e1 >= d[0]) {
      p.push_back(2);
      e1 -= 2 * d[0];
    }
    if (e2 >= d[0]) {
      p.push_back(3);
      e2 -= 2 * d[0];
    }
    p.push_back(1);
  }
  return p;
}

int zeros(const std::array<int, 3> &d) { return (d[0] == 0) + (d[1] == 0) + (d[2] == 0); }

// Axis permutations (generate_permutations, basic_observables.cpp:543-580):
// all six in lexicographic order, or three for an on-axis direction.
std::vector<std::array<int, 3>> permutations_of(const std::array<int, 3> &d) {
  if (zeros(d) == 2)
    return {{1, 2, 3}, {2, 1, 3}, {3, 1, 2}};
  std::vector<std::array<int, 3>> v;
  for (int p1 = 1; p1 <= 3; p1++)
    for (int p2 = 1; p2 <= 3; p2++)
      for (int p3 = 1; p3 <= 3; p3++)
        if (p1 != p2 && p2 != p3 && p3 != p1)
          v.push_back({p1, p2, p3});
  return v;
}

// Reflections (generate_reflections, basic_observables.cpp:582-623): with no
// zero component the signs of axes 2 and 3 and then the identity once more
// (the reference's one-zero test has an else branch that also runs for no
// zero, so that orientation is averaged twice); with one zero the sign of the
// first non-zero axis of the unpermuted direction; none otherwise.
std::vector<std::array<int, 3>> reflections_of(const std::array<int, 3> &d) {
  const int z = zeros(d);
  if (z == 0)
    return {{1, 1, 1}, {1, 1, -1}, {1, -1, 1}, {1, -1, -1}, {1, 1, 1}};
  if (z == 1) {
    int k = 0;
    while (d[k] == 0)
      k++;
    std::array<int, 3> a{1, 1, 1}, b{1, 1, 1};
    b[k] = -1;
    return {a, b};
  }
  return {{1, 1, 1}};
}

} // namespace

OffaxisPlan offaxis_plan(const std::vector<std::array<int, 3>> &directions, double r_min,
                         double r_max) {
  OffaxisPlan plan;
  for (const auto &d : directions) {
    const double len0 = std::sqrt((double)(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
    const std::vector<int> base = staircase(d);
    // length multipliers: r_min rounded up, r_max rounded down (wilson_loops.h:395-396)
    const int m_lo = (int)std::round(r_min / len0 + 0.5);
    const int m_hi = (int)std::round(r_max / len0 - 0.5);
    const int first_group = (int)plan.groups.size();
    for (int m = m_lo; m <= m_hi; m++)
      plan.groups.push_back({len0, m, {}});
    for (const auto &perm : permutations_of(d)) {
      std::vector<int> pp(base.size());
      for (size_t i = 0; i < base.size(); i++)
        pp[i] = perm[base[i] - 1]; // base steps are positive
      std::array<int, 3> dp{0, 0, 0};
      for (int k = 0; k < 3; k++)
        dp[perm[k] - 1] = d[k];
      for (const auto &refl : reflections_of(d)) {
        std::vector<int> pr(pp.size());
        for (size_t i = 0; i < pp.size(); i++)
          pr[i] = pp[i] * refl[pp[i] - 1];
        for (int m = m_lo; m <= m_hi; m++) {
          OffaxisLine line;
          for (int rep = 0; rep < m; rep++)
            line.pattern.insert(line.pattern.end(), pr.begin(), pr.end());
          for (int k = 0; k < 3; k++)
            line.disp[k] = dp[k] * refl[k] * m;
          plan.groups[first_group + (m - m_lo)].lines.push_back((int)plan.lines.size());
          plan.lines.push_back(std::move(line));
        }
      }
    }
  }
  return plan;
}

// Merge of equal (T, size) entries, step for step as wilson_offaxis_reduce
// (basic_observables.cpp:167-186) does it, including its traits: the merged
// entry keeps its own statistics count, the erase shifts later entries
// (including entry i when j < i), and the inner index advances past the
// entry that moves into the erased place.
void offaxis_reduce(std::vector<gc_wilson_result> &r) {
  for (int i = 0; i < (int)r.size(); i++)
    for (int j = 0; j < (int)r.size(); j++)
      if (r[i].space_size == r[j].space_size && r[i].time_size == r[j].time_size && i != j) {
        r[i].wilson_loop = (r[i].wilson_loop * r[i].statistics_size +
                            r[j].wilson_loop * r[j].statistics_size) /
                           (r[i].statistics_size + r[j].statistics_size);
        r.erase(r.begin() + j);
      }
}

} // namespace gc
