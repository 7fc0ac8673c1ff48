// Host-side declarations of the kernel launchers (implemented in the .cu files).
#pragma once

#include <mutex>
#include <set>
#include <utility>

#include "../../include/gc_lattice.h"
#include "gc_internal.cuh"

#include <array>
#include <vector>

namespace gc {

struct HypL1 {
  void *f[9];
};
struct HypL2 {
  void *f[6];
};

// Per-lattice descriptors of the multi-lattice ("batch") launches. One launch
// covers the blocks of every lattice in its table; block_start/start* is the
// first block of the lattice in that launch (tables are sorted by it).
struct ApeJob {
  Geom g;
  Fields4 in, out;
  double alpha;
  int block_start;
};
struct HypL1;
struct HypL2;

template <class Store, class CT>
int launch_ape(const Geom &g, const Fields4 &in, const Fields4 &out,
               double alpha, cudaStream_t s);

template <class Store, class CT>
int launch_hyp(const Geom &g, const Fields4 &U, const HypL1 &l1,
               const HypL2 &l2, void *out_t, double a1, double a2, double a3,
               cudaStream_t s);
// HYP as a pipeline over time slices (Lt >= 3): Lt + 3 launches, the
// decorated links in rings of 3 slices inside l1/l2's fields; the same links
// as launch_hyp bit for bit.
template <class Store, class CT>
int launch_hyp_slices(const Geom &g, const Fields4 &U, const HypL1 &l1, const HypL2 &l2,
                      void *out_t, double a1, double a2, double a3, cudaStream_t s);

struct HypJob {
  Geom g;
  Fields4 U;
  HypL1 l1;
  HypL2 l2;
  void *out_t;
  double a1, a2, a3;
  int start1, start2, start3; // first block in the level-1/2/3 launches
};

// jobs: device array (njobs entries, sorted by block_start); blocks: total.
template <class Store, class CT>
int launch_ape_batch(const ApeJob *jobs, int njobs, int blocks, cudaStream_t s);
template <class Store, class CT>
int launch_hyp_batch(const HypJob *jobs, int njobs, const int blocks[3],
                     cudaStream_t s);

struct WJob {
  Geom g;
  Fields4 U;
  int rmin, rmax, tmin, tmax;
  int cols, rows;       // block shape (columns x threads per column)
  double *partials;     // this lattice's per-block partials
  int block_start;      // first block (blocks = colblocks * 3, nu fastest)
  int blocks;
  int *status;          // set to 1 when the launch cannot run this lattice's shape
};
struct RJob {           // fixed-order reduction of one lattice's partials
  const double *partials;
  int nblocks, nr, nt;
  double scale;
  double *out;          // (T-tmin)*nr + (R-rmin)
  int entry_start;      // first block of the reduction launch
};
template <class Store, class CT>
int launch_wilson_batch(const WJob *jobs, int njobs, int blocks, int threads, size_t smem,
                        cudaStream_t s);
int launch_reduce_batch(const RJob *jobs, int njobs, int entries, cudaStream_t s);
// Shared memory one lattice's W blocks need.
size_t wilson_job_smem(const WJob &j, int nc, int ct_bytes, int threads);

// Wilson loops: per-block partial sums into `partials` (device, sized by
// wilson_partials_count), then a fixed-order reduction into `out_dev`
// ((tmax-tmin+1)*(rmax-rmin+1) doubles, index (T-tmin)*nR + (R-rmin)).
struct WilsonPlan {
  int cols_per_block; // spatial columns per block
  int rows;           // threads per column (a divisor of Lt, <= 64)
  int threads;        // ceil(cols_per_block / lanes) * rows, whole warps
  int blocks;         // ceil(Vs / cols_per_block) * 3
  size_t smem;        // dynamic shared memory bytes
  bool fits;          // false when even one column exceeds the budget
  int starts = 1;     // temporal-gauge form: consecutive start slices per thread
  // temporal-gauge form: 0 wilson_gauge_kernel; one column per thread with
  // the lines of its starts in registers: 1 wilson_gauge_reg_kernel (mixed
  // SU(3)), 2 wilson_gauge_q_kernel (SU(2))
  int kernel = 0;
};
// Doubles of a W block's per-warp accumulators in shared memory, rounded up
// to an even count so the 16-byte arrays placed after them stay aligned.
__host__ __device__ inline size_t wacc_doubles(int nwarps, int nr, int nt) {
  return ((size_t)nwarps * nr * nt + 1) & ~(size_t)1;
}
// Spatial columns one W thread carries: two adjacent columns (packed FP32x2
// arithmetic) for FP32 SU(3), one otherwise.
__host__ __device__ constexpr int wilson_lanes(int nc, int ct_bytes) {
  return (nc == 3 && ct_bytes == 4) ? 2 : 1;
}
// The W kernels sum raw traces Re Tr W (SU(3)) or a.b = Re Tr W / 2 (SU(2),
// quaternion form); the fundamental normalisation 1/N of the reference's
// multiply_conj_tr is applied once, with the 1/(3V) average, to the sums.
__host__ __device__ inline double wilson_trace_norm(int nc) { return nc == 3 ? 3.0 : 1.0; }
// Scale of the summed per-block partials: 1/(3V) over sites and the three
// spatial directions, times 1/N for the fundamental SU(3) trace (the adjoint
// character |Tr W|^2 - 1 is summed as is).
inline double wilson_scale(long long V, int nc, bool adjoint) {
  return 1.0 / (3.0 * (double)V * (adjoint ? 1.0 : wilson_trace_norm(nc)));
}
// Row stride of a W block's shared column arrays: cols rounded up to a
// multiple of the lane count.
__host__ __device__ inline int wilson_col_stride(int cols, int lanes) {
  return (cols + lanes - 1) / lanes * lanes;
}
// Threads of a W block shape (whole warps).
__host__ __device__ inline int wilson_threads(int cols, int rows, int lanes) {
  return ((wilson_col_stride(cols, lanes) / lanes * rows + 31) / 32) * 32;
}
// At most this many (R,T) entries per launch (callers split R into chunks).
constexpr int kWilsonMaxEntries = 1024;
// Shared-memory budget for the column storage of one block (bytes), sized
// so that two blocks fit on an SM with their per-warp accumulators (a
// 256-thread block with 12 x 12 (R,T) entries: 2 x (104 + 9) KB).
constexpr size_t kWilsonColumnBudget = 104 * 1024;

// sets: shared column sets of the block (3; 4 for the two-configuration
// GEVP loops).
WilsonPlan wilson_plan(const Geom &g, int nr, int nt, int nc, int ct_bytes, int sets = 3);

// adjoint: the adjoint-representation loop |Tr W|^2 - 1 instead of Re Tr W/N.
// second: a second configuration of the same lattice for the GEVP loops
// (wilson_gevp_indexed): its space lines pair with U's, time lines from U.
// tstarts > 0: only loops whose lower edge lies on the slices [0, tstarts)
// are counted, and the result is their average (a t-slab whose forward halo
// occupies the slices above).
template <class Store, class CT>
int launch_wilson(const Geom &g, const Fields4 &U, int rmin, int rmax,
                  int tmin, int tmax, double *partials, double *out_dev,
                  cudaStream_t s, bool adjoint = false, const Fields4 *second = nullptr,
                  int tstarts = 0);

// W(R,T) in the temporal gauge (gc_wilson_gauge.cu): applies to one
// configuration's loops over the whole lattice with T <= Lt/2 when the block
// shape fits; exact to rounding when the temporal links are unitary.
// units: column units (threads per time row) per block; 0 = about 128 threads.
WilsonPlan wilson_gauge_plan(const Geom &g, int nt, int nc, int ct_bytes, int units = 0,
                             bool adjoint = false);
// tstarts in (0, Lt): the start slices [0, tstarts) of a time slab, in one
// cut (time_max <= Lt - tstarts); otherwise every start slice (T <= Lt/2).
bool wilson_gauge_applies(const Geom &g, int tmax, int nt, int nc, int ct_bytes,
                          int tstarts = 0);
// Largest unitarity defect max |U U^dag - 1| of a temporal link for which the
// form is used (FP64: ct_bytes 8; mixed: 4).
double wilson_gauge_tolerance(int ct_bytes);
// Bytes of one field of gauge time lines (FP64 matrices, 256-byte aligned).
size_t wilson_gauge_line_bytes(const Geom &g, int nc);
// Gauge time lines GA, GB (cuts at slices 0 and Lt/2) and the transformed
// spatial links UA.f[0..2], UB.f[0..2] (the link storage format); *flag (a
// device int) is set to 1 when a temporal link's defect exceeds the
// tolerance, else left 0.
template <class Store, class CT>
int launch_wilson_gauge_prep(const Geom &g, const Fields4 &U, void *GA, void *GB,
                             const Fields4 &UA, const Fields4 &UB, int *flag, cudaStream_t s);
// The W table from the transformed links (partials: blocks of
// wilson_gauge_plan x nr x nt doubles), reduced into out_dev.
template <class Store, class CT>
int launch_wilson_gauge(const Geom &g, const Fields4 &UA, const Fields4 &UB, int rmin,
                        int rmax, int tmin, int tmax, bool adjoint, double *partials,
                        double *out_dev, cudaStream_t s);

// Both methods with the choice made on the device: the exact W kernel runs
// (and the gauge one returns at once) when *flag != 0, else the other way
// round; the fixed-order reduction then sums the partials of the method that
// ran. No host synchronisation (usable inside stream capture once each
// kernel's shared-memory attribute has been set by an earlier launch).
// partials: wilson_auto_partials_count doubles. tstarts in (0, Lt): the
// loops of the start slices [0, tstarts) only (a time slab's lattice of its
// own slices and the ones above them), in one cut at slice 0; the caller
// guarantees time_max <= Lt - tstarts (no loop passes the lattice's end).
template <class Store, class CT>
int launch_wilson_auto(const Geom &g, const Fields4 &U, const Fields4 &UA, const Fields4 &UB,
                       int rmin, int rmax, int tmin, int tmax, bool adjoint, const int *flag,
                       double *partials, double *out_dev, cudaStream_t s, int units = 0,
                       int tstarts = 0);
size_t wilson_auto_partials_count(const Geom &g, int nr, int nt, int nc, int units = 0);
template <class Store, class CT>
int time_wilson_gauge(const Geom &g, const Fields4 &UA, const Fields4 &UB, int rmin, int rmax,
                      int tmin, int tmax, int units, double *partials, cudaStream_t s,
                      float *ms);
// The exact W kernel, gated on *gate != 0, without the reduction; *blocks
// receives the number of blocks (rows of partials). tstarts as for
// launch_wilson_auto (0: every start slice).
template <class Store, class CT>
int launch_wilson_exact_gated(const Geom &g, const Fields4 &U, int rmin, int rmax, int tmin,
                              int tmax, bool adjoint, const int *gate, double *partials,
                              int *blocks, cudaStream_t s, int tstarts = 0);

// An explicit block shape (rows must divide Lt, at most 256 threads).
WilsonPlan wilson_plan_shape(const Geom &g, int nr, int nt, int nc, int ct_bytes, int rows,
                             int cols);
// W with an explicit plan; out_dev == nullptr skips the reduction.
template <class Store, class CT>
int launch_wilson_plan(const Geom &g, const Fields4 &U, int rmin, int rmax, int tmin,
                       int tmax, const WilsonPlan &p, double *partials, double *out_dev,
                       cudaStream_t s);

template <class Store, class CT>
int launch_plaquette(const Geom &g, const Fields4 &U, double *partials,
                     double *out_dev, cudaStream_t s);

int plaquette_partials_count(const Geom &g);

// out_dev[0] = scale * (fixed-order sum of partials[0..n)).
int launch_reduce_sum(const double *partials, int n, double scale, double *out_dev,
                      cudaStream_t s);

// out_dev[e] = scale * (fixed-order sum over blocks b of partials[b * n + e]),
// e < n.
// out_dev[(T-tmin)*nr + (R-rmin)] = scale * (fixed-order sum over blocks b of
// partials[b * nr * nt + (R-rmin) * nt + (T-tmin)]).
int launch_reduce_wilson(const double *partials, int blocks, int nr, int nt, double scale,
                         double *out_dev, cudaStream_t s);

int launch_reduce_rows(const double *partials, int blocks, int n, double scale,
                       double *out_dev, cudaStream_t s);

// ------------------------------------------------------------ off-axis loops
constexpr int kOffaxisMaxSteps = 256;
// A space line's links, in order (OffaxisLine::pattern, OffaxisLineDesc::s):
// +a steps forward along axis a-1 (1..3), -a steps back and takes the
// link's adjoint.
struct OffaxisLine {
  std::vector<int> pattern;
  int disp[3];
};
// Device table entry of one line for the fused kernel: its steps and the
// displacement of its end as non-negative residues.
struct OffaxisLineDesc {
  int n;
  int d[3];
  signed char s[kOffaxisMaxSteps];
};
// The lines of one (direction, length multiplier), in the order whose
// values are averaged.
struct OffaxisGroup {
  double length; // |direction|
  int multiplier;
  std::vector<int> lines;
};
struct OffaxisPlan {
  std::vector<OffaxisLine> lines;
  std::vector<OffaxisGroup> groups; // output order
};
std::vector<std::array<int, 3>> offaxis_directions(int length_max);
OffaxisPlan offaxis_plan(const std::vector<std::array<int, 3>> &directions, double r_min,
                         double r_max);
void offaxis_reduce(std::vector<gc_wilson_result> &results);
int offaxis_partials_count(const Geom &g, int nt);
// Scale of the summed partials of the line loops (1/V, and 1/N for the
// fundamental SU(3) trace).
double line_loop_scale(const Geom &g, int nc, bool adjoint);
// Off-axis loops of nlines lines (device table `lines`) in one launch: a
// block owns a few spatial columns over all t and a group of lines; the
// line products, the columns' time links and the displaced columns' time
// links sit in shared memory and the T walk reads only those. Per-block
// partial sums at partials[(block * nlines + line) * nt + (T - tmin)];
// returns the number of blocks (rows of partials) in *blocks.
template <class Store, class CT>
int launch_offaxis_fused(const Geom &g, const Fields4 &U, const OffaxisLineDesc *lines,
                         int nlines, int tmin, int tmax, bool adjoint, double *partials,
                         int *blocks, cudaStream_t s);
// Column blocks of the fused launch (rows of its partials) for a lattice.
int offaxis_fused_blocks(const Geom &g, int nc, int ct_bytes);

// Loops of a line field S (decorated-link storage) whose end is displaced
// by disp (disp[ax] = 0) with "time" axis ax and time links Ut:
// out_dev[T - tmin] = mean over sites of Re Tr[L(x,T) S(x+T ax) L(x+D,T)^dag
// S(x)^dag] / N (or the adjoint character).
template <class Store, class CT>
int launch_line_loops(const Geom &g, const void *Ut, int ax, const void *S, const int disp[4],
                      int tmin, int tmax, bool adjoint, double *partials, double *out_dev,
                      cudaStream_t s, int pstride = 0);
// S <- (init ? F : S) * F(x + offset ax)^count for a single-direction field F.
template <class Store, class CT>
int launch_line_extend(const Geom &g, const void *F, void *S, int ax, int offset, int count,
                       bool init, cudaStream_t s);
// One two-dimensional APE step of the single-direction fields f1 (axis a)
// and f2 (axis b) into o1, o2.
template <class Store, class CT>
int launch_ape_plane(const Geom &g, const void *f1, const void *f2, void *o1, void *o2, int a,
                     int b, double alpha, cudaStream_t s);

// Polyakov lines P(s) of every spatial site into `lines` (FP64 element
// planes: 9 (SU(3)) or 2 (SU(2)) double2 planes of Vs entries), block sums of
// Re Tr P / N into partials ((Vs + 255) / 256 of them) and, if out_dev is
// given, the Polyakov loop (their mean) into out_dev[0].
template <class Store, class CT>
int launch_polyakov_lines(const Geom &g, const Fields4 &U, double2 *lines, double *partials,
                          double *out_dev, cudaStream_t s);
// Correlator entries out_dev[offsets[i].w] for the offsets (x, y, z) of the
// table; singlet: Re Tr(P P'^dag)/N, else Re(tr P conj(tr P')).
int launch_polyakov_correlator(const Geom &g, int nc, const double2 *lines, const int4 *offsets,
                               int noffsets, bool singlet, double *out_dev, cudaStream_t s);
size_t wilson_partials_count(const Geom &g, int nr, int nt, int nc, int sets = 3);
int wilson_max_blocks(const Geom &g, int nc, int sets = 3);

// Host AoS (uploaded raw to a device staging buffer) <-> device SoA fields.
// The upload converts the sites [site0, site0 + nsites) (all of them when
// nsites < 0); the staging buffer holds exactly those sites' links.
int launch_aos_to_soa(const Geom &g, int nc, int prec, int layout,
                      const double *staging, const Fields4 &U, cudaStream_t s,
                      int site0 = 0, int nsites = -1);
int launch_soa_to_aos(const Geom &g, int nc, int prec, int layout,
                      const Fields4 &U, double *staging, cudaStream_t s);

// Lets `kernel` use up to the device's opt-in shared memory per block. Set
// once per (kernel, device) rather than before every launch: concurrent
// request threads would otherwise call cudaFuncSetAttribute on every W
// launch. The attribute only raises the allowed maximum; each launch still
// asks for the shared memory it needs.
template <class K> inline int allow_large_smem(K *kernel, size_t smem, bool capturing = false) {
  if (smem <= 48 * 1024)
    return GC_OK;
  static std::mutex mu;
  static std::set<std::pair<const void *, int>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({(const void *)kernel, dev}))
    return GC_OK;
  // (while a stream is captured the attribute set by an earlier eager launch
  // of the same schedule stays in force)
  if (capturing)
    return GC_OK;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if ((size_t)optin < smem)
    return plan_error("kernel: shared memory above the device's limit");
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) !=
      cudaSuccess)
    return launch_check("shared-memory attribute");
  done.insert({(const void *)kernel, dev});
  return GC_OK;
}


} // namespace gc
