// On-axis Wilson loops W(R,T) and the average plaquette (sm_100a).
//
// Reference: wilson_loop (wilson_loops.h:1047-1074) builds time lines
// L(x,T) and space lines S_nu(x,R) as full-lattice fields and, for every
// (R,T), sums Re Tr[L(x,T) S_nu(x+T,R) L(x+R nu,T)^dag S_nu(x,R)^dag]/N over
// x and nu < 3, divided by 3V (:719-791).
//
// Here one block owns `cols` spatial columns (s, nu) over all t. The space
// lines S(s,t,R) of its columns live in shared memory and are extended by one
// link per R; the columns' own time links U_t(s,t) are staged in shared
// memory once and the neighbour columns' time links U_t(s+R nu,t) once per R,
// so the T walk reads only shared memory. For every corner (s,t0) a thread
// walks T with the exact
// recursion
//     K_0 = S(x,R),   K_T = U_t(x+(T-1)t)^dag K_{T-1} U_t(x+R nu+(T-1)t),
// so that K_T = L(x,T)^dag S(x,R) L(x+R nu,T), and the loop trace is
//     Re Tr[S(x+T t, R) K_T^dag] / N.
// This is the same product of links as the reference's, reassociated; it
// does not assume unitarity. Per (x,nu,R,T): two matrix products and one
// 9-element dot product. No line fields are written to HBM.
//
// Reductions are deterministic: warp shuffles into per-warp shared
// accumulators, a fixed-order sum over warps into one partial per block and
// (R,T), then a fixed-order tree over blocks.
#include "gc_internal.cuh"
#include "gc_kernels.h"

namespace gc {

namespace {

// Shared-memory matrices are stored element-major as 2-vectors: complex
// element k (or quaternion pair k) of matrix i at sm[k*stride + i], one
// 8-byte (FP32) or 16-byte (FP64) load per element, consecutive threads on
// consecutive addresses.
template <class T> struct V2;
template <> struct V2<double> {
  using type = double2;
};
template <> struct V2<float> {
  using type = float2;
};

template <class T>
__device__ __forceinline__ void sm_store(typename V2<T>::type *sm, int stride,
                                         int i, const SU3<T> &m) {
#pragma unroll
  for (int k = 0; k < 9; k++)
    sm[k * stride + i] = {m.e[k / 3][k % 3].re, m.e[k / 3][k % 3].im};
}
template <class T>
__device__ __forceinline__ SU3<T> sm_load(const typename V2<T>::type *sm,
                                          int stride, int i, SU3<T> *) {
  SU3<T> m;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const auto v = sm[k * stride + i];
    m.e[k / 3][k % 3] = {v.x, v.y};
  }
  return m;
}
template <class T>
__device__ __forceinline__ void sm_store(typename V2<T>::type *sm, int stride,
                                         int i, const SU2<T> &m) {
  sm[i] = {m.a0, m.a1};
  sm[stride + i] = {m.a2, m.a3};
}
template <class T>
__device__ __forceinline__ SU2<T> sm_load(const typename V2<T>::type *sm,
                                          int stride, int i, SU2<T> *) {
  const auto a = sm[i], b = sm[stride + i];
  return {a.x, a.y, b.x, b.y};
}
template <class M> struct Elems;
template <class T> struct Elems<SU3<T>> {
  static constexpr int n = 9;
};
template <class T> struct Elems<SU2<T>> {
  static constexpr int n = 2;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Re Tr(A B^dag)/N in the compute type, returned in FP64 for accumulation.
template <class T> __device__ __forceinline__ double conj_tr_d(const SU3<T> &a, const SU3<T> &b) {
  T s = a.e[0][0].re * b.e[0][0].re;
  s = GC_FMA(a.e[0][0].im, b.e[0][0].im, s);
#pragma unroll
  for (int k = 1; k < 9; k++) {
    s = GC_FMA(a.e[k / 3][k % 3].re, b.e[k / 3][k % 3].re, s);
    s = GC_FMA(a.e[k / 3][k % 3].im, b.e[k / 3][k % 3].im, s);
  }
  return double(s) / 3.0;
}
template <class T> __device__ __forceinline__ double conj_tr_d(const SU2<T> &a, const SU2<T> &b) {
  T s = a.a0 * b.a0;
  s = GC_FMA(a.a1, b.a1, s);
  s = GC_FMA(a.a2, b.a2, s);
  s = GC_FMA(a.a3, b.a3, s);
  return double(s);
}

// The per-loop quantity, from the loop's trace Tr[S K^dag]: the fundamental
// Re Tr W / N (multiply_conj_tr, matrix.h:54-56, 260-262) or, with ADJ, the
// adjoint character |Tr W|^2 - 1 (multiply_conj_tr_adjoint / tr_adjoint,
// matrix.h:62-65, 264-270; SU(2): 4 (a.b)^2 - 1).
template <bool ADJ, class T>
__device__ __forceinline__ double loop_value(const SU3<T> &a, const SU3<T> &b) {
  if (!ADJ)
    return conj_tr_d(a, b);
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
  return r * r + i * i - 1.0;
}
template <bool ADJ, class T>
__device__ __forceinline__ double loop_value(const SU2<T> &a, const SU2<T> &b) {
  const double d = conj_tr_d(a, b);
  return ADJ ? 4.0 * d * d - 1.0 : d;
}

// One block of the W computation: `cols` spatial columns starting at
// colblock*cols, direction nu; writes its nr*nt partial sums to part.
template <class Store, class CT, bool ADJ = false>
__device__ __forceinline__ void wilson_block(const Geom &g, const Fields4 &U, int rmin,
                                             int rmax, int tmin, int tmax, int cols,
                                             int rows, int colblock, int nu,
                                             double *part, unsigned char *smem_raw) {
  using M = typename Store::template M<CT>;
  using VT = typename V2<CT>::type;
  constexpr int NE = Elems<M>::n;
  const int Lt = g.L[3];
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  const int nwarps = blockDim.x >> 5;
  double *wacc = reinterpret_cast<double *>(smem_raw);         // [nwarps][nr*nt]
  const int sstride = Lt * cols;                                // matrices per set
  // space lines S(s,t,R) of the block's columns
  // (the accumulator block is rounded up to an even number of doubles so the
  // 16-byte double2 arrays after it stay 16-byte aligned)
  VT *scol = reinterpret_cast<VT *>(wacc + wacc_doubles(nwarps, nr, nt));
  // the block's own time links U_t(s, t), reused for every R and T
  VT *ucol = scol + (size_t)NE * sstride;
  // the time links of the neighbour columns U_t(s + R nu, t), one R at a time
  VT *ncol = ucol + (size_t)NE * sstride;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < nwarps * nr * nt; i += blockDim.x)
    wacc[i] = 0.0;

  const int c = tid % cols;
  const int row = tid / cols;
  const int s = colblock * cols + c;
  const bool active = (row < rows) && (s < g.Vs);
  const int kt = Lt / rows;
  int xs[4] = {0, 0, 0, 0};
  if (active)
    site_coords(g, s, xs);
  const size_t V = g.V;
  const void *Unu = U.f[nu];
  const void *Ut = U.f[3];
  if (active) {
#pragma unroll 1
    for (int k = 0; k < kt; k++) {
      const int t0 = row + k * rows;
      sm_store(ucol, sstride, t0 * cols + c,
               Store::template load<CT>(Ut, V, s + t0 * g.Vs));
    }
  }
  __syncthreads();

#pragma unroll 1
  for (int R = 1; R <= rmax; R++) {
    // Extend the space lines of this thread's corners by one link, and stage
    // the neighbour column's time links for this R.
    if (active) {
      const int sl = s + fwd_off(g, xs[nu], nu, R - 1);
      const int sR = s + fwd_off(g, xs[nu], nu, R);
#pragma unroll 1
      for (int k = 0; k < kt; k++) {
        const int t0 = row + k * rows;
        M u = Store::template load<CT>(Unu, V, sl + t0 * g.Vs);
        M sn = (R == 1) ? u : mul(sm_load(scol, sstride, t0 * cols + c, (M *)nullptr), u);
        sm_store(scol, sstride, t0 * cols + c, sn);
        if (R >= rmin)
          sm_store(ncol, sstride, t0 * cols + c,
                   Store::template load<CT>(Ut, V, sR + t0 * g.Vs));
      }
    }
    __syncthreads();
    if (R >= rmin) {
      double *wrow = wacc + (size_t)warp * nr * nt + (R - rmin) * nt;
#pragma unroll 1
      for (int k = 0; k < kt; k++) {
        const int t0 = row + k * rows;
        M K = active ? sm_load(scol, sstride, t0 * cols + c, (M *)nullptr)
                     : unit(M());
        int tt = t0; // (t0 + T - 1) mod Lt
#pragma unroll 1
        for (int T = 1; T <= tmax; T++) {
          int tu = tt + 1; // (t0 + T) mod Lt
          tu = (tu == Lt) ? 0 : tu;
          if (active) {
            M a = sm_load(ucol, sstride, tt * cols + c, (M *)nullptr);
            M b = sm_load(ncol, sstride, tt * cols + c, (M *)nullptr);
            K = mul(mul_da(a, K), b);
          }
          if (T >= tmin) {
            double term = active
                ? loop_value<ADJ>(sm_load(scol, sstride, tu * cols + c, (M *)nullptr), K)
                : 0.0;
            term = warp_sum(term);
            if (lane == 0)
              wrow[T - tmin] += term;
          }
          tt = tu;
        }
      }
    }
    __syncthreads();
  }

  // Fixed-order sum over warps -> one partial per (block, R, T).
  for (int e = tid; e < nr * nt; e += blockDim.x) {
    double sum = 0.0;
    for (int w = 0; w < nwarps; w++)
      sum += wacc[(size_t)w * nr * nt + e];
    part[e] = sum;
  }
}

template <class Store, class CT, bool ADJ>
__global__ void __launch_bounds__(256)
    wilson_kernel(Geom g, const __grid_constant__ Fields4 U, int rmin, int rmax, int tmin,
                  int tmax, int cols, int rows, double *partials) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const size_t blk = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
  const int ne = (rmax - rmin + 1) * (tmax - tmin + 1);
  wilson_block<Store, CT, ADJ>(g, U, rmin, rmax, tmin, tmax, cols, rows, blockIdx.x, blockIdx.y,
                          partials + blk * ne, smem_raw);
}

// Several lattices in one launch. A block finds its lattice by binary search
// over block_start; nu varies fastest over a lattice's blocks, and each block
// writes its partials at the index the single-lattice kernel uses
// (nu * colblocks + colblock), so the fixed-order sums are the same.
template <class Store, class CT>
__global__ void __launch_bounds__(256)
    wilson_batch_kernel(const WJob *__restrict__ jobs, int njobs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].block_start <= (int)blockIdx.x)
      lo = mid;
    else
      hi = mid - 1;
  }
  const WJob &jb = jobs[lo];
  const int local = blockIdx.x - jb.block_start;
  const int nu = local % 3, colblock = local / 3;
  const int colblocks = jb.blocks / 3;
  const int ne = (jb.rmax - jb.rmin + 1) * (jb.tmax - jb.tmin + 1);
  if (jb.cols * jb.rows > (int)blockDim.x)
    return; // a lattice whose shape needs more threads than the launch has
  wilson_block<Store, CT>(jb.g, jb.U, jb.rmin, jb.rmax, jb.tmin, jb.tmax, jb.cols, jb.rows,
                          colblock, nu,
                          jb.partials + ((size_t)nu * colblocks + colblock) * ne, smem_raw);
}

// Fixed-order reduction of several lattices' partials; block = (lattice,
// entry), the same tree as reduce_partials_kernel.
__global__ void __launch_bounds__(256)
    reduce_batch_kernel(const RJob *__restrict__ jobs, int njobs) {
  __shared__ double sh[256];
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].entry_start <= (int)blockIdx.x)
      lo = mid;
    else
      hi = mid - 1;
  }
  const RJob &jb = jobs[lo];
  const int e = blockIdx.x - jb.entry_start;
  const int nentries = jb.nr * jb.nt;
  double s = 0.0;
  for (int b = threadIdx.x; b < jb.nblocks; b += blockDim.x)
    s += jb.partials[(size_t)b * nentries + e];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int ir = e / jb.nt, it = e % jb.nt;
    jb.out[it * jb.nr + ir] = sh[0] * jb.scale;
  }
}

// out[(T-tmin)*nr + (R-rmin)] = (sum over blocks of partial e=(R-rmin)*nt+(T-tmin)) * scale
__global__ void __launch_bounds__(256)
    reduce_partials_kernel(const double *partials, int nblocks, int nentries,
                           int nr, int nt, double scale, double *out) {
  __shared__ double sh[256];
  const int e = blockIdx.x;
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

// Average plaquette: thread per site, six planes (plaket.h:24-42), fixed-order
// block sums.
template <class Store, class CT>
__global__ void __launch_bounds__(256)
    plaquette_kernel(Geom g, const __grid_constant__ Fields4 U, double *partials) {
  using M = typename Store::template M<CT>;
  __shared__ double sh[256];
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  double p = 0.0;
  if (site < g.V) {
    int x[4];
    site_coords(g, site, x);
    const size_t V = g.V;
    double acc = 0.0;
#pragma unroll 1
    for (int mu = 0; mu < 3; mu++) {
#pragma unroll 1
      for (int nu = mu + 1; nu < 4; nu++) {
        const int pm = site + step_off(g, x[mu], mu, +1);
        const int pn = site + step_off(g, x[nu], nu, +1);
        M a = mul(Store::template load<CT>(U.f[mu], V, site),
                  Store::template load<CT>(U.f[nu], V, pm));
        a = mul_ad(a, Store::template load<CT>(U.f[mu], V, pn));
        acc += conj_tr_d(a, Store::template load<CT>(U.f[nu], V, site));
      }
    }
    p = acc / 6.0;
  }
  sh[threadIdx.x] = p;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    partials[blockIdx.x] = sh[0];
}

int largest_divisor_upto(int n, int cap) {
  for (int d = cap < n ? cap : n; d > 1; d--)
    if (n % d == 0)
      return d;
  return 1;
}

} // namespace

// The block shape depends only on Lt and the group, never on the R/T ranges
// or the compute type, so every caller that sizes the per-block partials
// from a plan gets the same block count as the launch. Columns per block are
// limited so that the shared column storage (FP64 worst case) plus the
// largest per-warp accumulator set (8 warps x 1024 (R,T) entries) fits in a
// block's shared memory.
WilsonPlan wilson_plan(const Geom &g, int nr, int nt, int nc, int ct_bytes) {
  WilsonPlan p;
  const int Lt = g.L[3];
  const int ncomp = (nc == 3) ? 18 : 4;
  p.rows = largest_divisor_upto(Lt, 32);
  p.cols_per_block = 256 / p.rows;
  if (p.cols_per_block < 1)
    p.cols_per_block = 1;
  const size_t col_bytes = 3 * (size_t)ncomp * Lt * sizeof(double);
  while (p.cols_per_block > 1 && p.cols_per_block * col_bytes > kWilsonColumnBudget)
    p.cols_per_block--;
  const int active = p.cols_per_block * p.rows;
  p.threads = ((active + 31) / 32) * 32;
  const int colblocks = (g.Vs + p.cols_per_block - 1) / p.cols_per_block;
  p.blocks = colblocks * 3;
  const int nwarps = p.threads / 32;
  // per-warp accumulators + space lines + own and neighbour time links
  p.smem = wacc_doubles(nwarps, nr, nt) * sizeof(double) +
           3 * (size_t)ncomp * Lt * p.cols_per_block * ct_bytes;
  p.fits = p.cols_per_block * col_bytes <= kWilsonColumnBudget;
  return p;
}

size_t wilson_partials_count(const Geom &g, int nr, int nt, int nc) {
  return (size_t)wilson_plan(g, nr, nt, nc, 8).blocks * nr * nt;
}

int plaquette_partials_count(const Geom &g) { return (g.V + 255) / 256; }

template <class Store, class CT>
int launch_wilson(const Geom &g, const Fields4 &U, int rmin, int rmax,
                  int tmin, int tmax, double *partials, double *out_dev,
                  cudaStream_t s, bool adjoint) {
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  WilsonPlan p = wilson_plan(g, nr, nt, Store::NC, (int)sizeof(CT));
  if (!p.fits || nr * nt > kWilsonMaxEntries)
    return plan_error("wilson_kernel: time extent or (R,T) range too large for "
                      "one block's shared memory");
  if (p.smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(
        adjoint ? wilson_kernel<Store, CT, true> : wilson_kernel<Store, CT, false>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem);
    if (e != cudaSuccess)
      return launch_check("wilson_kernel smem attribute");
  }
  dim3 grid(p.blocks / 3, 3);
  auto kern = adjoint ? wilson_kernel<Store, CT, true> : wilson_kernel<Store, CT, false>;
  kern<<<grid, p.threads, p.smem, s>>>(
      g, U, rmin, rmax, tmin, tmax, p.cols_per_block, p.rows, partials);
  int rc = launch_check("wilson_kernel");
  if (rc)
    return rc;
  reduce_partials_kernel<<<nr * nt, 256, 0, s>>>(
      partials, p.blocks, nr * nt, nr, nt, 1.0 / (3.0 * (double)g.V), out_dev);
  return launch_check("reduce_partials_kernel");
}

template <class Store, class CT>
int launch_plaquette(const Geom &g, const Fields4 &U, double *partials,
                     double *out_dev, cudaStream_t s) {
  const int nb = plaquette_partials_count(g);
  plaquette_kernel<Store, CT><<<nb, 256, 0, s>>>(g, U, partials);
  int rc = launch_check("plaquette_kernel");
  if (rc)
    return rc;
  reduce_partials_kernel<<<1, 256, 0, s>>>(partials, nb, 1, 1, 1,
                                           1.0 / (double)g.V, out_dev);
  return launch_check("reduce_partials_kernel");
}

WilsonPlan wilson_plan_shape(const Geom &g, int nr, int nt, int nc, int ct_bytes, int rows,
                             int cols) {
  WilsonPlan p;
  const int ncomp = (nc == 3) ? 18 : 4;
  p.rows = rows;
  p.cols_per_block = cols;
  p.threads = ((rows * cols + 31) / 32) * 32;
  p.blocks = ((g.Vs + cols - 1) / cols) * 3;
  const int nwarps = p.threads / 32;
  p.smem = wacc_doubles(nwarps, nr, nt) * sizeof(double) +
           3 * (size_t)ncomp * g.L[3] * cols * ct_bytes;
  p.fits = (g.L[3] % rows == 0) && rows * cols <= 256 && p.smem <= 227 * 1024;
  return p;
}

template <class Store, class CT>
int launch_wilson_plan(const Geom &g, const Fields4 &U, int rmin, int rmax, int tmin,
                       int tmax, const WilsonPlan &p, double *partials, double *out_dev,
                       cudaStream_t s) {
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  if (!p.fits)
    return plan_error("wilson_kernel: block shape does not fit");
  if (p.smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(
        wilson_kernel<Store, CT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)p.smem);
    if (e != cudaSuccess)
      return launch_check("wilson_kernel smem attribute");
  }
  wilson_kernel<Store, CT, false><<<dim3(p.blocks / 3, 3), p.threads, p.smem, s>>>(
      g, U, rmin, rmax, tmin, tmax, p.cols_per_block, p.rows, partials);
  int rc = launch_check("wilson_kernel");
  if (rc)
    return rc;
  if (!out_dev)
    return GC_OK;
  reduce_partials_kernel<<<nr * nt, 256, 0, s>>>(
      partials, p.blocks, nr * nt, nr, nt, 1.0 / (3.0 * (double)g.V), out_dev);
  return launch_check("reduce_partials_kernel");
}

size_t wilson_job_smem(const WJob &j, int nc, int ct_bytes) {
  const int nwarps = 256 / 32;
  const int ncomp = (nc == 3) ? 18 : 4;
  return wacc_doubles(nwarps, j.rmax - j.rmin + 1, j.tmax - j.tmin + 1) * sizeof(double) +
         3 * (size_t)ncomp * j.g.L[3] * j.cols * ct_bytes;
}

template <class Store, class CT>
int launch_wilson_batch(const WJob *jobs, int njobs, int blocks, size_t smem,
                        cudaStream_t s) {
  if (njobs <= 0 || blocks <= 0)
    return GC_OK;
  if (smem > 227 * 1024)
    return plan_error("wilson_batch_kernel: shared memory above 227 KB");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cap);
  // (while a stream is captured the attribute set by an earlier eager launch
  // of the same schedule stays in force)
  if (smem > 48 * 1024 && cap == cudaStreamCaptureStatusNone) {
    cudaError_t e = cudaFuncSetAttribute(wilson_batch_kernel<Store, CT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess)
      return launch_check("wilson_batch_kernel smem attribute");
  }
  wilson_batch_kernel<Store, CT><<<blocks, 256, smem, s>>>(jobs, njobs);
  return launch_check("wilson_batch_kernel");
}

int launch_reduce_batch(const RJob *jobs, int njobs, int entries, cudaStream_t s) {
  if (njobs <= 0 || entries <= 0)
    return GC_OK;
  reduce_batch_kernel<<<entries, 256, 0, s>>>(jobs, njobs);
  return launch_check("reduce_batch_kernel");
}

#define GC_INSTANTIATE_W(STORE, CT)                                            \
  template int launch_wilson<STORE, CT>(const Geom &, const Fields4 &, int,   \
                                        int, int, int, double *, double *,    \
                                        cudaStream_t, bool);                  \
  template int launch_plaquette<STORE, CT>(const Geom &, const Fields4 &,     \
                                           double *, double *, cudaStream_t);  \
  template int launch_wilson_batch<STORE, CT>(const WJob *, int, int, size_t, \
                                              cudaStream_t);                  \
  template int launch_wilson_plan<STORE, CT>(const Geom &, const Fields4 &,   \
                                             int, int, int, int,              \
                                             const WilsonPlan &, double *,    \
                                             double *, cudaStream_t);

GC_INSTANTIATE_W(StoreF64SU3, double)
GC_INSTANTIATE_W(StoreF64SU2, double)
GC_INSTANTIATE_W(StoreF32SU3, float)
GC_INSTANTIATE_W(StoreF32SU2, float)

} // namespace gc
