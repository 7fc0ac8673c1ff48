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
// offaxis_line_kernel: thread per site, the product of the pattern's links
// (a negative step moves back first and multiplies by the link's adjoint)
// into a field of V matrices. line_loop_kernel: thread per site, the same
// exact recursion as the on-axis kernel, K_0 = S(x),
// K_T = U_t(x+(T-1)t)^dag K_{T-1} U_t(x+D+(T-1)t), value Re Tr[S(x+T t) K_T^dag],
// with fixed-order warp / block / grid sums (deterministic).
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

template <class Store, class CT>
__global__ void __launch_bounds__(256)
    offaxis_line_kernel(const __grid_constant__ Geom g, const __grid_constant__ Fields4 U,
                        const __grid_constant__ OffaxisSteps steps, void *S) {
  using M = typename Store::template M<CT>;
  using IS = typename InterStore<Store>::type;
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  if (site >= g.V)
    return;
  const size_t V = g.V;
  int x[4];
  site_coords(g, site, x);
  int cur = site;
  M A = unit(M());
#pragma unroll 1
  for (int i = 0; i < steps.n; i++) {
    const int e = steps.s[i];
    const int mu = (e > 0 ? e : -e) - 1;
    const int L = sel4(g.L, mu), st = sel4(g.stride, mu);
    int c = mu == 0 ? x[0] : (mu == 1 ? x[1] : x[2]);
    M u;
    if (e > 0) {
      u = Store::template load<CT>(U.f[mu], V, cur);
      cur += (c == L - 1) ? -(L - 1) * st : st;
      c = (c == L - 1) ? 0 : c + 1;
    } else {
      cur += (c == 0) ? (L - 1) * st : -st;
      c = (c == 0) ? L - 1 : c - 1;
      u = adjoint(Store::template load<CT>(U.f[mu], V, cur));
    }
    if (mu == 0)
      x[0] = c;
    else if (mu == 1)
      x[1] = c;
    else
      x[2] = c;
    // the first factor is taken as it is (identity times a link is exact)
    A = (i == 0) ? u : mul(A, u);
  }
  IS::template store<CT>(S, V, site, A);
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

} // namespace

int offaxis_partials_count(const Geom &g, int nt) {
  return ((g.V + kOffaxisBlock - 1) / kOffaxisBlock) * nt;
}

template <class Store, class CT>
int launch_offaxis_line(const Geom &g, const Fields4 &U, const OffaxisSteps &steps, void *S,
                        cudaStream_t s) {
  if (steps.n < 1 || steps.n > kOffaxisMaxSteps)
    return plan_error("offaxis_line_kernel: pattern length");
  offaxis_line_kernel<Store, CT><<<(g.V + 255) / 256, 256, 0, s>>>(g, U, steps, S);
  return launch_check("offaxis_line_kernel");
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
int launch_offaxis_loops(const Geom &g, const Fields4 &U, const void *S, const int disp[3],
                         int tmin, int tmax, bool adjoint, double *partials, double *out_dev,
                         cudaStream_t s, int pstride) {
  const int d4[4] = {disp[0], disp[1], disp[2], 0};
  return launch_line_loops<Store, CT>(g, U.f[3], 3, S, d4, tmin, tmax, adjoint, partials,
                                      out_dev, s, pstride);
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
  template int launch_offaxis_line<STORE, CT>(const Geom &, const Fields4 &,              \
                                              const OffaxisSteps &, void *, cudaStream_t); \
  template int launch_line_loops<STORE, CT>(const Geom &, const void *, int, const void *, \
                                            const int *, int, int, bool, double *,        \
                                            double *, cudaStream_t, int);                 \
  template int launch_line_extend<STORE, CT>(const Geom &, const void *, void *, int, int,  \
                                             int, bool, cudaStream_t);                     \
  template int launch_offaxis_loops<STORE, CT>(const Geom &, const Fields4 &, const void *, \
                                               const int *, int, int, bool, double *,      \
                                               double *, cudaStream_t, int);

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
