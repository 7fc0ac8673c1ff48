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
#include "gc_pair.cuh"
#include "gc_wcol.cuh"

#include <algorithm>
#include <mutex>
#include <set>
#include <type_traits>
#include <utility>

namespace gc {

namespace {

// ---------------------------------------------------------------- W block
// One block of the W computation: `cols` spatial columns starting at
// colblock*cols, direction nu; writes its nr*nt partial sums to part. Each
// thread carries LANES adjacent columns: LANES = 2 for FP32 SU(3), whose
// matrices are SU3<f2> so that every product and dot-product term is one
// packed FP32x2 instruction for both columns. Lane 1 of a pair that runs past
// the block's columns or the lattice duplicates lane 0's site and contributes
// nothing.
//
// GEVP (wilson_gevp_indexed, wilson_loops.h:1202-1233; per-plane sums
// :867-955, adjoint :957-1045): the space lines come from two
// configurations, U (S1) and U2 (S2), the time links from U, and every loop
// is counted twice, with S1 on top and S2 at the bottom and the other way
// round. The block keeps a fourth set (S2) and walks T once per ordering.
template <class Store, class CT, bool ADJ = false, bool GEVP = false>
__device__ __forceinline__ void wilson_block(const Geom &g, const Fields4 &U, const Fields4 &U2,
                                             int rmin, int rmax, int tmin, int tmax, int cols,
                                             int rows, int colblock, int nu,
                                             double *part, unsigned char *smem_raw,
                                             int tstarts) {
  constexpr int LANES = wilson_lanes(Store::NC, sizeof(CT));
  using LL = LaneLoad<Store, CT, LANES>;
  using M = typename LL::M;
  using CS = ColSet<M>;
  const int Lt = g.L[3];
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  const int nwarps = blockDim.x >> 5;
  const int cs = wilson_col_stride(cols, LANES); // slot units per t (x LANES columns)
  const int units = cs / LANES;
  const int nslots = Lt * units;
  double *wacc = reinterpret_cast<double *>(smem_raw); // [nwarps][nr*nt]
  // (the accumulator block is rounded up to an even number of doubles so the
  // 16-byte vectors after it stay 16-byte aligned; set sizes are multiples of
  // 16 bytes)
  unsigned char *scol = reinterpret_cast<unsigned char *>(wacc + wacc_doubles(nwarps, nr, nt));
  unsigned char *ucol = scol + (size_t)CS::kBytes * nslots; // own time links U_t(s, t)
  unsigned char *ncol = ucol + (size_t)CS::kBytes * nslots; // U_t(s + R nu, t), per R
  unsigned char *scol2 = ncol + (size_t)CS::kBytes * nslots; // GEVP: S2 lines

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < nwarps * nr * nt; i += blockDim.x)
    wacc[i] = 0.0;

  const int u = tid % units;
  const int row = tid / units;
  const int s0 = colblock * cols + LANES * u;
  const bool active = (row < rows) && (s0 < g.Vs);
  const bool lane1 = LANES == 2 && active && (LANES * u + 1 < cols) && (s0 + 1 < g.Vs);
  const int s1 = lane1 ? s0 + 1 : s0;
  const int kt = Lt / rows;
  // coordinates of the columns along nu, and the lattice's extent and stride
  // along nu (scalars: no dynamically indexed local arrays)
  const int Ln = sel4(g.L, nu), stn = sel4(g.stride, nu);
  const int xn0 = (s0 / stn) % Ln, xn1 = (s1 / stn) % Ln;
  const size_t V = g.V;
  const void *Unu = U.f[nu];
  const void *Ut = U.f[3];
  if (active) {
#pragma unroll 1
    for (int k = 0; k < kt; k++) {
      const int t0 = row + k * rows;
      CS::store(ucol, nslots, t0 * units + u, LL::load(Ut, V, s0 + t0 * g.Vs, s1 + t0 * g.Vs));
    }
  }
  __syncthreads();

#pragma unroll 1
  for (int R = 1; R <= rmax; R++) {
    // Extend the space lines of this thread's corners by one link, and stage
    // the neighbour columns' time links for this R.
    if (active) {
      const int l0 = s0 + ((xn0 + R - 1) % Ln - xn0) * stn;
      const int l1 = s1 + ((xn1 + R - 1) % Ln - xn1) * stn;
      const int r0 = s0 + ((xn0 + R) % Ln - xn0) * stn;
      const int r1 = s1 + ((xn1 + R) % Ln - xn1) * stn;
#pragma unroll 1
      for (int k = 0; k < kt; k++) {
        const int t0 = row + k * rows;
        const int i = t0 * units + u;
        M lnk = LL::load(Unu, V, l0 + t0 * g.Vs, l1 + t0 * g.Vs);
        M sn = (R == 1) ? lnk : mul(CS::load(scol, nslots, i), lnk);
        CS::store(scol, nslots, i, sn);
        if (GEVP) {
          M lnk2 = LL::load(U2.f[nu], V, l0 + t0 * g.Vs, l1 + t0 * g.Vs);
          M sn2 = (R == 1) ? lnk2 : mul(CS::load(scol2, nslots, i), lnk2);
          CS::store(scol2, nslots, i, sn2);
        }
        if (R >= rmin)
          CS::store(ncol, nslots, i, LL::load(Ut, V, r0 + t0 * g.Vs, r1 + t0 * g.Vs));
      }
    }
    __syncthreads();
    if (R >= rmin) {
      double *wrow = wacc + (size_t)warp * nr * nt + (R - rmin) * nt;
#pragma unroll 1
      for (int pass = 0; pass < (GEVP ? 2 : 1); pass++) {
        // bottom and top space lines of this pass (GEVP: S2 below S1, then S1
        // below S2)
        const unsigned char *sbot = (GEVP && pass == 0) ? scol2 : scol;
        const unsigned char *stop = (GEVP && pass == 1) ? scol2 : scol;
#pragma unroll 1
        for (int k = 0; k < kt; k++) {
          const int t0 = row + k * rows;
          // loops start on the slices [0, tstarts) only (all of them unless
          // the lattice is a t-slab with its forward halo)
          const bool counted = active && t0 < tstarts;
          if (!__any_sync(0xffffffffu, counted))
            continue; // warp-uniform
          M K = counted ? CS::load(sbot, nslots, t0 * units + u) : unit(M());
          int tt = t0; // (t0 + T - 1) mod Lt
#pragma unroll 1
          for (int T = 1; T <= tmax; T++) {
            int tu = tt + 1; // (t0 + T) mod Lt
            tu = (tu == Lt) ? 0 : tu;
            if (counted) {
              const int i = tt * units + u;
              K = mul(mul_da(CS::load(ucol, nslots, i), K), CS::load(ncol, nslots, i));
            }
            if (T >= tmin) {
              double term = counted
                  ? loop_value<ADJ>(CS::load(stop, nslots, tu * units + u), K, lane1)
                  : 0.0;
              term = warp_sum(term);
              if (lane == 0)
                wrow[T - tmin] += term;
            }
            tt = tu;
          }
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

template <class Store, class CT, bool ADJ, bool GEVP>
__global__ void __launch_bounds__(256)
    wilson_kernel(const __grid_constant__ Geom g, const __grid_constant__ Fields4 U,
                  const __grid_constant__ Fields4 U2, int rmin, int rmax, int tmin, int tmax,
                  int cols, int rows, double *partials, int tstarts,
                  const int *gate = nullptr) {
  // gate: the temporal-gauge form's unitarity flag; this launch is the exact
  // fallback and computes nothing when the flag says the gauge form ran
  if (gate && *gate == 0)
    return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const size_t blk = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
  const int ne = (rmax - rmin + 1) * (tmax - tmin + 1);
  wilson_block<Store, CT, ADJ, GEVP>(g, U, U2, rmin, rmax, tmin, tmax, cols, rows, blockIdx.x,
                                     blockIdx.y, partials + blk * ne, smem_raw, tstarts);
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
  if (wilson_threads(jb.cols, jb.rows, wilson_lanes(Store::NC, sizeof(CT))) > (int)blockDim.x) {
    // a lattice whose shape needs more threads than the launch has: its table
    // would be wrong, so the batch reports an error instead of a result
    if (threadIdx.x == 0 && jb.status)
      *jb.status = 1;
    return;
  }
  wilson_block<Store, CT, false>(jb.g, jb.U, jb.U, jb.rmin, jb.rmax, jb.tmin, jb.tmax, jb.cols,
                                 jb.rows, colblock, nu,
                                 jb.partials + ((size_t)nu * colblocks + colblock) * ne,
                                 smem_raw, jb.g.L[3]);
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

// Plaquette sums: thread per site over the six planes (plaket.h:24-42),
// split into the three spatial planes (plaket_site_space, :63-81) and the
// three (mu, t) planes (plaket_site_time, :44-61); raw traces, fixed-order
// block sums into partials[2 * block + {0: space, 1: time}].
template <class Store, class CT>
__global__ void __launch_bounds__(256)
    plaquette_kernel(const __grid_constant__ Geom g, const __grid_constant__ Fields4 U,
                     double *partials) {
  using M = typename Store::template M<CT>;
  __shared__ double sh[2][256];
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  double sp = 0.0, tm = 0.0;
  if (site < g.V) {
    int x[4];
    site_coords(g, site, x);
    const size_t V = g.V;
#pragma unroll 1
    for (int mu = 0; mu < 3; mu++) {
#pragma unroll 1
      for (int nu = mu + 1; nu < 4; nu++) {
        const int pm = site + step_off(g, sel4(x, mu), mu, +1);
        const int pn = site + step_off(g, sel4(x, nu), nu, +1);
        M a = mul(Store::template load<CT>(U.f[mu], V, site),
                  Store::template load<CT>(U.f[nu], V, pm));
        a = mul_ad(a, Store::template load<CT>(U.f[mu], V, pn));
        const double v = loop_value<false>(a, Store::template load<CT>(U.f[nu], V, site), false);
        if (nu == 3)
          tm += v;
        else
          sp += v;
      }
    }
  }
  sh[0][threadIdx.x] = sp;
  sh[1][threadIdx.x] = tm;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = sh[0][0];
    partials[2 * blockIdx.x + 1] = sh[1][0];
  }
}

int largest_divisor_upto(int n, int cap) {
  for (int d = cap < n ? cap : n; d > 1; d--)
    if (n % d == 0)
      return d;
  return 1;
}

} // namespace

// The block shape depends only on Lt, the group and the compute type, never
// on the R/T ranges (callers size the partial sums before they know the
// ranges of later launches). rows = the largest divisor of Lt up to 64
// threads per column, so one start slice per thread up to Lt = 64 (a thread
// walking several starts needs that many times the shared memory per
// thread); each thread carries `lanes` columns; about 128 threads per block,
// 256 when rows > 32. Columns are limited so that the column storage fits
// kWilsonColumnBudget. (Choosing the columns instead for the most resident
// threads per SM -- smaller blocks at Lt = 16 and 32 -- measured slower:
// 32^4 W 9.06 -> 9.60 ms mixed, 18.2 -> 19.1 ms FP64.)
WilsonPlan wilson_plan(const Geom &g, int nr, int nt, int nc, int ct_bytes, int sets) {
  WilsonPlan p;
  const int Lt = g.L[3];
  const int ncomp = (nc == 3) ? 18 : 4;
  const int lanes = wilson_lanes(nc, ct_bytes);
  p.rows = largest_divisor_upto(Lt, 64);
  p.cols_per_block = lanes * ((p.rows > 32 ? 256 : 128) / p.rows);
  if (p.cols_per_block < 1)
    p.cols_per_block = 1;
  const size_t col_bytes = (size_t)sets * ncomp * Lt * ct_bytes;
  while (p.cols_per_block > 1 &&
         wilson_col_stride(p.cols_per_block, lanes) * col_bytes > kWilsonColumnBudget)
    p.cols_per_block--;
  p.threads = wilson_threads(p.cols_per_block, p.rows, lanes);
  const int colblocks = (g.Vs + p.cols_per_block - 1) / p.cols_per_block;
  p.blocks = colblocks * 3;
  const int nwarps = p.threads / 32;
  // per-warp accumulators + space lines + own and neighbour time links
  // (+ the second configuration's space lines)
  p.smem = wacc_doubles(nwarps, nr, nt) * sizeof(double) +
           wilson_col_stride(p.cols_per_block, lanes) * col_bytes;
  p.fits = wilson_col_stride(p.cols_per_block, lanes) * col_bytes <= kWilsonColumnBudget;
  return p;
}

// Blocks of the W plan for either compute type, whichever has more: the
// size of per-block partial sums a handle needs before its form is known.
int wilson_max_blocks(const Geom &g, int nc, int sets) {
  return std::max(wilson_plan(g, 1, 1, nc, 4, sets).blocks,
                  wilson_plan(g, 1, 1, nc, 8, sets).blocks);
}

size_t wilson_partials_count(const Geom &g, int nr, int nt, int nc, int sets) {
  return (size_t)wilson_max_blocks(g, nc, sets) * nr * nt;
}

int plaquette_partials_count(const Geom &g) { return 2 * ((g.V + 255) / 256); }

template <class Store, class CT, bool ADJ, bool GEVP>
int launch_wilson_mode(const Geom &g, const Fields4 &U, const Fields4 &U2, int rmin, int rmax,
                       int tmin, int tmax, double *partials, double *out_dev, cudaStream_t s,
                       int tstarts) {
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  if (tstarts <= 0 || tstarts > g.L[3])
    tstarts = g.L[3];
  WilsonPlan p = wilson_plan(g, nr, nt, Store::NC, (int)sizeof(CT), GEVP ? 4 : 3);
  if (!p.fits || nr * nt > kWilsonMaxEntries)
    return plan_error("wilson_kernel: time extent or (R,T) range too large for "
                      "one block's shared memory");
  int rc = allow_large_smem(wilson_kernel<Store, CT, ADJ, GEVP>, p.smem);
  if (rc)
    return rc;
  wilson_kernel<Store, CT, ADJ, GEVP><<<dim3(p.blocks / 3, 3), p.threads, p.smem, s>>>(
      g, U, U2, rmin, rmax, tmin, tmax, p.cols_per_block, p.rows, partials, tstarts);
  rc = launch_check("wilson_kernel");
  if (rc)
    return rc;
  // average over the loops counted (all V sites, or the tstarts slices);
  // GEVP counts every loop twice (the / (6 V) of wilson_loops.h:910, 954)
  const double scale =
      wilson_scale((long long)g.Vs * tstarts, Store::NC, ADJ) / (GEVP ? 2.0 : 1.0);
  reduce_partials_kernel<<<nr * nt, 256, 0, s>>>(partials, p.blocks, nr * nt, nr, nt, scale,
                                                 out_dev);
  return launch_check("reduce_partials_kernel");
}

template <class Store, class CT>
int launch_wilson_exact_gated(const Geom &g, const Fields4 &U, int rmin, int rmax, int tmin,
                              int tmax, bool adjoint, const int *gate, double *partials,
                              int *blocks, cudaStream_t s, int tstarts) {
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  if (tstarts <= 0 || tstarts > g.L[3])
    tstarts = g.L[3];
  WilsonPlan p = wilson_plan(g, nr, nt, Store::NC, (int)sizeof(CT), 3);
  if (!p.fits || nr * nt > kWilsonMaxEntries)
    return plan_error("wilson_kernel: time extent or (R,T) range too large for "
                      "one block's shared memory");
  int rc;
  if (adjoint) {
    rc = allow_large_smem(wilson_kernel<Store, CT, true, false>, p.smem);
    if (rc)
      return rc;
    wilson_kernel<Store, CT, true, false><<<dim3(p.blocks / 3, 3), p.threads, p.smem, s>>>(
        g, U, U, rmin, rmax, tmin, tmax, p.cols_per_block, p.rows, partials, tstarts, gate);
  } else {
    rc = allow_large_smem(wilson_kernel<Store, CT, false, false>, p.smem);
    if (rc)
      return rc;
    wilson_kernel<Store, CT, false, false><<<dim3(p.blocks / 3, 3), p.threads, p.smem, s>>>(
        g, U, U, rmin, rmax, tmin, tmax, p.cols_per_block, p.rows, partials, tstarts, gate);
  }
  *blocks = p.blocks;
  return launch_check("wilson_kernel");
}

template <class Store, class CT>
int launch_wilson(const Geom &g, const Fields4 &U, int rmin, int rmax,
                  int tmin, int tmax, double *partials, double *out_dev,
                  cudaStream_t s, bool adjoint, const Fields4 *second, int tstarts) {
  if (second)
    return adjoint ? launch_wilson_mode<Store, CT, true, true>(
                         g, U, *second, rmin, rmax, tmin, tmax, partials, out_dev, s, tstarts)
                   : launch_wilson_mode<Store, CT, false, true>(
                         g, U, *second, rmin, rmax, tmin, tmax, partials, out_dev, s, tstarts);
  return adjoint ? launch_wilson_mode<Store, CT, true, false>(g, U, U, rmin, rmax, tmin, tmax,
                                                              partials, out_dev, s, tstarts)
                 : launch_wilson_mode<Store, CT, false, false>(g, U, U, rmin, rmax, tmin, tmax,
                                                               partials, out_dev, s, tstarts);
}

// out_dev[0] = spatial-plane average (plaket_space), out_dev[1] = (mu, t)
// average (plaket_time); the full plaquette is their mean.
template <class Store, class CT>
int launch_plaquette(const Geom &g, const Fields4 &U, double *partials,
                     double *out_dev, cudaStream_t s) {
  const int nb = (g.V + 255) / 256;
  plaquette_kernel<Store, CT><<<nb, 256, 0, s>>>(g, U, partials);
  int rc = launch_check("plaquette_kernel");
  if (rc)
    return rc;
  reduce_partials_kernel<<<2, 256, 0, s>>>(partials, nb, 2, 2, 1,
                                           1.0 / (3.0 * (double)g.V *
                                                  wilson_trace_norm(Store::NC)),
                                           out_dev);
  return launch_check("reduce_partials_kernel");
}

WilsonPlan wilson_plan_shape(const Geom &g, int nr, int nt, int nc, int ct_bytes, int rows,
                             int cols) {
  WilsonPlan p;
  const int ncomp = (nc == 3) ? 18 : 4;
  const int lanes = wilson_lanes(nc, ct_bytes);
  p.rows = rows;
  p.cols_per_block = cols;
  p.threads = wilson_threads(cols, rows, lanes);
  p.blocks = ((g.Vs + cols - 1) / cols) * 3;
  const int nwarps = p.threads / 32;
  p.smem = wacc_doubles(nwarps, nr, nt) * sizeof(double) +
           3 * (size_t)ncomp * g.L[3] * wilson_col_stride(cols, lanes) * ct_bytes;
  p.fits = (g.L[3] % rows == 0) && p.threads <= 256 && p.smem <= 227 * 1024;
  return p;
}

template <class Store, class CT>
int launch_wilson_plan(const Geom &g, const Fields4 &U, int rmin, int rmax, int tmin,
                       int tmax, const WilsonPlan &p, double *partials, double *out_dev,
                       cudaStream_t s) {
  const int nr = rmax - rmin + 1, nt = tmax - tmin + 1;
  if (!p.fits)
    return plan_error("wilson_kernel: block shape does not fit");
  int rc = allow_large_smem(wilson_kernel<Store, CT, false, false>, p.smem);
  if (rc)
    return rc;
  wilson_kernel<Store, CT, false, false><<<dim3(p.blocks / 3, 3), p.threads, p.smem, s>>>(
      g, U, U, rmin, rmax, tmin, tmax, p.cols_per_block, p.rows, partials, g.L[3]);
  rc = launch_check("wilson_kernel");
  if (rc)
    return rc;
  if (!out_dev)
    return GC_OK;
  reduce_partials_kernel<<<nr * nt, 256, 0, s>>>(
      partials, p.blocks, nr * nt, nr, nt, wilson_scale(g.V, Store::NC, false), out_dev);
  return launch_check("reduce_partials_kernel");
}

// (for a launch of `threads` threads: the per-warp accumulators are sized by
// the launch's warps)
size_t wilson_job_smem(const WJob &j, int nc, int ct_bytes, int threads) {
  const int nwarps = threads / 32;
  const int ncomp = (nc == 3) ? 18 : 4;
  const int lanes = wilson_lanes(nc, ct_bytes);
  return wacc_doubles(nwarps, j.rmax - j.rmin + 1, j.tmax - j.tmin + 1) * sizeof(double) +
         3 * (size_t)ncomp * j.g.L[3] * wilson_col_stride(j.cols, lanes) * ct_bytes;
}

template <class Store, class CT>
int launch_wilson_batch(const WJob *jobs, int njobs, int blocks, int threads, size_t smem,
                        cudaStream_t s) {
  if (njobs <= 0 || blocks <= 0)
    return GC_OK;
  if (threads <= 0 || threads > 256 || threads % 32)
    return plan_error("wilson_batch_kernel: thread count");
  if (smem > 227 * 1024)
    return plan_error("wilson_batch_kernel: shared memory above 227 KB");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cap);
  int rc = allow_large_smem(wilson_batch_kernel<Store, CT>, smem,
                            cap != cudaStreamCaptureStatusNone);
  if (rc)
    return rc;
  wilson_batch_kernel<Store, CT><<<blocks, threads, smem, s>>>(jobs, njobs);
  return launch_check("wilson_batch_kernel");
}

int launch_reduce_sum(const double *partials, int n, double scale, double *out_dev,
                      cudaStream_t s) {
  reduce_partials_kernel<<<1, 256, 0, s>>>(partials, n, 1, 1, 1, scale, out_dev);
  return launch_check("reduce_partials_kernel");
}

int launch_reduce_rows(const double *partials, int blocks, int n, double scale,
                       double *out_dev, cudaStream_t s) {
  reduce_partials_kernel<<<n, 256, 0, s>>>(partials, blocks, n, 1, n, scale, out_dev);
  return launch_check("reduce_partials_kernel");
}

int launch_reduce_wilson(const double *partials, int blocks, int nr, int nt, double scale,
                         double *out_dev, cudaStream_t s) {
  reduce_partials_kernel<<<nr * nt, 256, 0, s>>>(partials, blocks, nr * nt, nr, nt, scale,
                                                 out_dev);
  return launch_check("reduce_partials_kernel");
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
                                        cudaStream_t, bool, const Fields4 *,  \
                                        int);                                 \
  template int launch_plaquette<STORE, CT>(const Geom &, const Fields4 &,     \
                                           double *, double *, cudaStream_t);  \
  template int launch_wilson_batch<STORE, CT>(const WJob *, int, int, int,     \
                                              size_t, cudaStream_t);          \
  template int launch_wilson_plan<STORE, CT>(const Geom &, const Fields4 &,   \
                                             int, int, int, int,              \
                                             const WilsonPlan &, double *,    \
                                             double *, cudaStream_t);         \
  template int launch_wilson_exact_gated<STORE, CT>(                          \
      const Geom &, const Fields4 &, int, int, int, int, bool, const int *,   \
      double *, int *, cudaStream_t, int);

GC_INSTANTIATE_W(StoreF64SU3, double)
GC_INSTANTIATE_W(StoreF64SU2, double)
GC_INSTANTIATE_W(StoreF32SU3, float)
GC_INSTANTIATE_W(StoreF32SU2, float)

} // namespace gc
