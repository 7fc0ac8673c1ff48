/*
 * general_code_b200 — C ABI for APE/HYP link smearing and on-axis Wilson loops
 * W(R,T) on SU(2)/SU(3) gauge configurations, computed by sm_100a kernels.
 *
 * The reference ("general_code", lib/cpu) exposes this path as C++ templates
 * on Data::LatticeData<DataPatternLexicographical, MatrixType>; it has no FFI.
 * Each entry point below names the reference interface it replaces. The C++
 * drop-in overloads with the reference's own signatures live in gc_dropin.hpp
 * and are thin wrappers over these functions.
 *
 * Conventions
 *  - Plain pointers and sizes only. Every function returns GC_OK (0) or a
 *    GC_ERR_* code; the message of the last failure on a handle is returned by
 *    gc_last_error(handle) (gc_last_error(NULL) gives the last failure of a
 *    call that had no handle). Nothing throws across the ABI.
 *  - Lattice geometry: dims = {Lx, Ly, Lz, Lt}; site = x + Lx*(y + Ly*(z +
 *    Lz*t)); directions mu = 0,1,2 (space), 3 (time); link index 4*site+mu
 *    (reference indexing.h:71-126, DataPatternLexicographical).
 *  - Host link arrays hold 4*V links in that order. Per link:
 *      SU(2): 4 doubles (a0,a1,a2,a3), U = a0 + i a.sigma   (matrix.h:8-13)
 *      SU(3): 18 doubles; GC_LAYOUT_ROWMAJOR stores element (i,j) at
 *             (3i+j)*2 (re), +1 (im) — the reference's file / get_data order
 *             (matrix.h:228-243); GC_LAYOUT_EIGEN_COLMAJOR stores it at
 *             (i+3j)*2 — the in-memory image of std::vector<su3> (an
 *             Eigen::Matrix3cd per link).
 *  - Links stay resident on the device between calls. Calls on one handle are
 *    serialised on the handle's CUDA stream; functions that return results to
 *    host memory synchronise that stream. A handle may be used from one host
 *    thread at a time per call (calls are internally locked).
 */
#ifndef GC_LATTICE_H
#define GC_LATTICE_H

#ifdef __cplusplus
extern "C" {
#endif

#define GC_OK 0
#define GC_ERR_ARG 1       /* invalid argument (sizes, ranges, null pointers) */
#define GC_ERR_CUDA 2      /* a CUDA runtime call or kernel launch failed     */
#define GC_ERR_NOMEM 3     /* device or pinned-host allocation failed         */
#define GC_ERR_NODEVICE 4  /* no CUDA device, or not an sm_100 device         */
#define GC_ERR_IO 5        /* configuration file could not be read/written    */
#define GC_ERR_STATE 6     /* handle not initialised with links yet           */
#define GC_ERR_TIMEOUT 7   /* a bounded device-side wait expired              */
#define GC_ERR_BUSY 8      /* admission refused (no free slot or memory)      */

#define GC_PREC_FP64 0     /* links stored and computed in FP64               */
#define GC_PREC_MIXED 1    /* FP32 links (SU(3): 12 reals, third row rebuilt),
                              FP64 projection and FP64 trace accumulation     */

/* Methods of the on-axis Wilson loops (gc_set_wilson_method). */
#define GC_WILSON_AUTO 0   /* temporal gauge where it applies, else exact     */
#define GC_WILSON_EXACT 1  /* always the exact product of links               */
#define GC_WILSON_GAUGE 2  /* (reported by gc_wilson_method_used)             */

/* Methods of HYP smearing (gc_set_hyp_method). */
#define GC_HYP_AUTO 0    /* the library's choice (the level kernels)          */
#define GC_HYP_LEVELS 1  /* one launch per decoration level, whole-lattice    */
                         /* decorated-link fields                             */
#define GC_HYP_SLICES 2  /* a pipeline over time slices, decorated links in   */
                         /* rings of three slices (Lt >= 3)                   */

#define GC_LAYOUT_ROWMAJOR 0
#define GC_LAYOUT_EIGEN_COLMAJOR 1

typedef struct gc_lattice gc_lattice;

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int gc_version(void);

/* Text for the last failure on h (or of a handle-less call when h == NULL).
 * The pointer stays valid until the next failing call on the same handle. */
const char *gc_last_error(const gc_lattice *h);

/* Creates a device-resident lattice (no links yet; upload or generate next).
 * Replaces: Data::LatticeData<DP,MT>::LatticeData(lat_dim) (data.h:84-87).
 * nc is 2 or 3; precision is GC_PREC_FP64 or GC_PREC_MIXED. */
int gc_lattice_create(const int dims[4], int nc, int precision,
                      gc_lattice **out);

/* As gc_lattice_create, but all of the handle's device memory is allocated
 * and freed stream-ordered (cudaMallocAsync/cudaFreeAsync) on cuda_stream
 * (a cudaStream_t as void*), and all its work runs there: creating and
 * destroying handles then never synchronises the device, so handles of
 * concurrent jobs on different streams overlap. gc_set_stream is refused for
 * such a handle. */
int gc_lattice_create_on_stream(const int dims[4], int nc, int precision,
                                void *cuda_stream, gc_lattice **out);

/* Frees all device memory of h. NULL is accepted. */
int gc_lattice_destroy(gc_lattice *h);

/* Runs h's work on an existing CUDA stream (a cudaStream_t passed as void*).
 * NULL selects the handle's own stream. */
int gc_set_stream(gc_lattice *h, void *cuda_stream);

/* Blocks until all work queued on h has finished. */
int gc_synchronize(gc_lattice *h);

/* Copies 4*V host links (layout GC_LAYOUT_*) to the device.
 * Replaces: filling LatticeData::array (data.h:95-112) before a call. */
int gc_upload(gc_lattice *h, const double *host_links, int layout);

/* Copies the device links back into 4*V host links (layout GC_LAYOUT_*). */
int gc_download(gc_lattice *h, double *host_links, int layout);

/* Device-to-device copy of all links of src into dst (same dims, nc and
 * precision), queued on dst's stream after src's queued work. Replaces:
 * copy-assignment of LatticeData (data.h:78-93), e.g. `smeared = conf`. */
int gc_copy_links(gc_lattice *dst, gc_lattice *src);

/* ---- time slices (t-slab decomposition of one lattice over several GPUs).
 * The reference has no domain decomposition (it runs one lattice on the
 * OpenMP threads of one node); these entry points are the pieces a
 * decomposition over time slabs needs: a slab lattice of Lt_slab slices is
 * filled from the slices of a larger lattice, smeared, its smeared slices
 * exchanged with the neighbouring slabs, and its Wilson loops counted from
 * its own slices only (gc_wilson_onaxis_tslab). Slices are whole time
 * slices t = const of all four directions (sites with t varying slowest, as
 * in the reference's lexicographic order, indexing.h:71-126). */

/* Uploads nt time slices of host links (layout GC_LAYOUT_*) into the slices
 * [t0, t0 + nt) of the lattice: host_links holds the 4 * nt * Lx*Ly*Lz links
 * of those slices, i.e. the run of a larger lattice's host array starting at
 * its slice (link index 4*site+mu, site of the first slice = 0). */
int gc_upload_slices(gc_lattice *h, int t0, int nt, const double *host_links, int layout);

/* Bytes of nt time slices of all four directions in the handle's device
 * form (the size of a gc_pack_slices buffer); -1 for a bad argument. */
long long gc_slice_bytes(const gc_lattice *h, int nt);

/* Packs the device links of the slices [t0, t0 + nt) into the device buffer
 * dev_buf (gc_slice_bytes(h, nt) bytes, 16-byte aligned), queued on the
 * handle's stream; gc_unpack_slices is the inverse. The packed form is the
 * handle's own (FP64 or mixed), for an exchange between handles of the same
 * spatial extents, group and precision (e.g. over NCCL). */
int gc_pack_slices(gc_lattice *h, int t0, int nt, void *dev_buf);
int gc_unpack_slices(gc_lattice *h, int t0, int nt, const void *dev_buf);

/* Device-to-device copy of the slices [src_t0, src_t0 + nt) of src into the
 * slices [dst_t0, dst_t0 + nt) of dst (same Lx, Ly, Lz, group and precision;
 * Lt may differ), queued on dst's stream after src's queued work. */
int gc_copy_slices(gc_lattice *dst, int dst_t0, gc_lattice *src, int src_t0, int nt);

/* On-axis Wilson loops (adjoint != 0: the adjoint representation) counted
 * only from the lower-edge slices t in [0, t_starts), averaged over those
 * loops (3 * Lx*Ly*Lz * t_starts of them); the slices above hold the forward
 * halo of a t-slab, at least time_max slices deep so no loop wraps. The
 * global average over slabs is sum_slab W_slab * t_starts / Lt. Same output
 * layout as gc_wilson_onaxis. With t_starts = Lt it is gc_wilson_onaxis
 * (wilson_loops.h:1047-1074). Methods as gc_wilson_onaxis: for
 * time_max <= Lt - t_starts (no counted loop passes slice Lt - 1) the
 * temporal gauge with one cut at slice 0 where the device finds the temporal
 * links unitary, else the exact product. */
int gc_wilson_onaxis_tslab(gc_lattice *h, int t_starts, int r_min, int r_max, int time_min,
                           int time_max, int adjoint, double *out);

/* One or more APE steps on the spatial links (temporal links unchanged):
 * U'_i = Proj[(1-alpha) U_i + alpha/4 sum_{j != i, j < 3} staples].
 * Replaces: smearing_APE(conf, alpha) (smearing.h:115-161), called steps
 * times. */
int gc_ape(gc_lattice *h, double alpha, int steps);

/* One or more HYP steps; only temporal links change (three decoration levels
 * with alpha1/alpha2/alpha3, divisors 6/4/2).
 * Replaces: smearing_HYP(conf, alpha1, alpha2, alpha3) (smearing.h:480-516),
 * called steps times. */
int gc_hyp(gc_lattice *h, double alpha1, double alpha2, double alpha3,
           int steps);

/* Selects how gc_hyp runs on this handle: GC_HYP_AUTO (default), GC_HYP_LEVELS
 * or GC_HYP_SLICES (GC_ERR_ARG if Lt < 3). Both give the same links bit for
 * bit; the slice pipeline keeps the decorated links of three time slices at a
 * time instead of fifteen whole-lattice fields (less DRAM traffic, more time:
 * Lt + 3 launches). No counterpart in the reference. */
int gc_set_hyp_method(gc_lattice *h, int method);

/* On-axis Wilson loops averaged over sites and the three spatial directions,
 * for R in [r_min, r_max] (space) and T in [time_min, time_max] (time).
 * out (host) receives (time_max-time_min+1)*(r_max-r_min+1) doubles:
 * out[(T-time_min)*(r_max-r_min+1) + (R-r_min)] = W(R,T), i.e. the entries of
 * the reference's std::map keyed (T,R), in the map's iteration order.
 * Two methods give the same table: the exact product of links (walked in T
 * for every corner), and, for T <= Lt/2 when the temporal links are unitary
 * (checked on the device for every call: defect max |U U^dag - 1| at most
 * 1e-14 in FP64, 1e-6 in the mixed form), the same loops in the temporal
 * gauge (one trace per loop instead of two matrix products); see
 * gc_set_wilson_method. A block keeps one column's lines of all Lt slices in
 * shared memory: GC_ERR_ARG when they do not fit (SU(3): Lt > 246).
 * Replaces: wilson_loop(conf, r_min, r_max, time_min, time_max)
 * (wilson_loops.h:1047-1074) and the legacy vector overload
 * (basic_observables.h:108-111). */
int gc_wilson_onaxis(gc_lattice *h, int r_min, int r_max, int time_min,
                     int time_max, double *out);

/* On-axis Wilson loops in the adjoint representation: per loop W,
 * |Tr W|^2 - 1 (SU(2): 4 (Re Tr W / 2)^2 - 1), averaged like
 * gc_wilson_onaxis, same output layout.
 * Replaces: wilson_loop_adjoint(conf, r_min, r_max, time_min, time_max)
 * (wilson_loops.h:1173-1200, plane sums :793-861). */
int gc_wilson_adjoint_onaxis(gc_lattice *h, int r_min, int r_max, int time_min,
                             int time_max, double *out);

/* Selects the method of gc_wilson_onaxis and gc_wilson_adjoint_onaxis on this
 * handle: GC_WILSON_AUTO (default) or GC_WILSON_EXACT. No counterpart in the
 * reference (which has one method, the exact product). */
int gc_set_wilson_method(gc_lattice *h, int method);

/* The method the last on-axis W call of the handle ran: GC_WILSON_EXACT or
 * GC_WILSON_GAUGE (0 before the first call). */
int gc_wilson_method_used(gc_lattice *h, int *method);

/* On-axis Wilson loops between two configurations of the same lattice (for
 * a generalised eigenvalue problem over smearing levels): time lines from
 * h1, and each loop counted with h1's space line on top and h2's at the
 * bottom and the other way round, averaged over 6V. h1 and h2 must have the
 * same sizes, group and precision (h2 == h1 is allowed); h1's stream waits
 * for h2's queued work. Same output layout as gc_wilson_onaxis.
 * Replaces: wilson_gevp_indexed(conf1, conf2, r_min, r_max, time_min,
 * time_max) (wilson_loops.h:1202-1233, plane sums :867-955). */
int gc_wilson_gevp_onaxis(gc_lattice *h1, gc_lattice *h2, int r_min, int r_max,
                          int time_min, int time_max, double *out);

/* The same in the adjoint representation (|Tr W|^2 - 1 per loop).
 * Replaces: wilson_gevp_adjoint_indexed (wilson_loops.h:1235-1266, plane
 * sums :957-1045). */
int gc_wilson_gevp_adjoint_onaxis(gc_lattice *h1, gc_lattice *h2, int r_min, int r_max,
                                  int time_min, int time_max, double *out);

/* The W(R,T) table of gc_wilson_onaxis for callers that cannot allocate
 * device memory (an application whose allocator owns the whole device budget,
 * or a timing-critical loop where cudaMalloc/cudaFree would synchronise the
 * device). It has no counterpart in the reference. Nothing is allocated: the
 * caller passes the links as four device buffers it owns (fields[mu], mu =
 * 0..3, in this library's device layout: FP64 SU(3) = 9 planes of V double2,
 * plane k = element (k/3, k%3) as (re, im); FP64 SU(2) = 2 planes of V double2,
 * (a0,a1) then (a2,a3); mixed SU(3) = 3 planes of V float4, (u00,u01),
 * (u02,u10), (u11,u12); mixed SU(2) = 1 plane of V float4) and a device
 * buffer out_dev of (time_max-time_min+1)*(r_max-r_min+1) doubles, filled as
 * gc_wilson_onaxis fills `out` with the exact product of links
 * (GC_WILSON_EXACT). The work is queued on cuda_stream (a
 * cudaStream_t as void*, NULL = default stream) and the call returns without
 * waiting. Working memory is a fixed 16 MiB array in the library's static
 * device memory. The CUDA runtime loads the library's device module lazily,
 * so the 16 MiB are taken on a device at the first call there (if no other
 * entry point of the library ran on it before) and held until exit: make one
 * call before an allocator that owns the device budget claims it; without
 * room for the array the call fails with GC_ERR_NOMEM. A lattice for which
 * one value of R does not fit in the array is rejected with GC_ERR_ARG. Every
 * call looks up the array's device address with the caller's device current
 * (so cudaDeviceReset does not leave a stale address behind); the first call
 * for each group and precision on a device also sets a kernel attribute, so
 * make it outside stream capture. All calls share the array: calls whose
 * work overlaps on the GPU race and must be serialised by the caller.
 * Errors: gc_last_error(NULL). */
int gc_wilson_onaxis_noalloc(const int dims[4], int nc, int precision,
                             const void *const fields[4], int r_min, int r_max,
                             int time_min, int time_max, double *out_dev,
                             void *cuda_stream);

/* Average plaquette over the 6 planes (1 for unit links).
 * Replaces: plaket(conf) (plaket.h:83-101). */
int gc_plaquette(gc_lattice *h, double *out);

/* One off-axis Wilson-loop entry (the reference's wilson_result,
 * basic_observables.h:18-23). */
typedef struct {
  double wilson_loop;  /* average over the orientations of the entry */
  int time_size;       /* T */
  double space_size;   /* |direction| * multiplier */
  int statistics_size; /* orientations averaged */
} gc_wilson_result;

/* Off-axis Wilson loops for the given spatial directions (ndirections x 3
 * ints, each a1 >= a2 >= a3 >= 0, a1 > 0): every permuted and reflected
 * orientation of each direction's staircase, lengths |d| m in
 * [r_min, r_max] (m rounded inwards), T in [time_min, time_max]; one entry per
 * (direction, m, T) in the reference's order. adjoint != 0: |Tr W|^2 - 1 per
 * loop. out has room for capacity entries; *count receives the number of
 * entries (GC_ERR_ARG, with *count set, when capacity is too small). A line
 * may have at most 256 links.
 * Replaces: wilson_offaxis / wilson_offaxis_adjoint (wilson_loops.h:313-467,
 * 487-645). */
int gc_wilson_offaxis(gc_lattice *h, const int *directions, int ndirections, double r_min,
                      double r_max, int time_min, int time_max, int adjoint,
                      gc_wilson_result *out, int capacity, int *count);

/* gc_wilson_offaxis over the directions of length up to 4 with the range
 * widened by 0.1 on each side, then entries of equal (T, size) merged as
 * the reference's wilson_offaxis_reduce does; a caller keys the entries by
 * (time_size, space_size) in order, later entries replacing earlier ones.
 * Replaces: wilson_offaxis_result / wilson_offaxis_adjoint_result
 * (wilson_loops.h:470-485, 648-663; reduce basic_observables.cpp:167-186). */
int gc_wilson_offaxis_result(gc_lattice *h, double r_min, double r_max, int time_min,
                             int time_max, int adjoint, gc_wilson_result *out, int capacity,
                             int *count);

/* One two-dimensional APE step (steps times) of the link fields of
 * directions a and b of h, in place, with the staples of the (a, b) plane
 * only; the other directions are unchanged.
 * Replaces: smearing_APE_2d(conf1, conf2, data_pattern, a, b, alpha)
 * (smearing.h:223-277) applied to h's fields of directions a and b. */
int gc_ape_plane(gc_lattice *h, int a, int b, double alpha, int steps);

/* One entry of the spatial Wilson-loop table. */
typedef struct {
  int smearing;       /* two-dimensional APE steps taken before the entry */
  int time_size;      /* length along the loop's spatial "time" axis */
  int space_size;     /* length along the smeared axis */
  double wilson_loop;
} gc_wilson_spatial_result;

/* Spatial (three-dimensional) Wilson loops with two-dimensional APE
 * smearing of the transverse links, as the reference computes them: for each
 * spatial plane (nu, eta) the links of nu and eta are smeared in that plane
 * (smearing_end steps), the loops have their "time" extent along the third
 * spatial axis (unsmeared links) and their space extent along nu or eta
 * (smeared links), measured before smearing and after the steps s with
 * (s - smearing_start) % smearing_step == 0 while smearing_step >=
 * smearing_start; every entry is the sum over the three planes and both axes
 * / 6. The space lines follow the reference's construction step for step
 * (wilson_lines_single_direction_indexed starts them with length time_min).
 * Entries in (smearing, T, R) order; capacity and *count as
 * gc_wilson_offaxis. Needs 1 <= r_min <= r_max, 1 <= time_min <= time_max,
 * smearing_step >= 1, smearing_end >= 0.
 * Replaces: wilson_spatial_3d_indexed(conf, r_min, r_max, time_min,
 * time_max, alpha, smearing_start, smearing_end, smearing_step)
 * (wilson_loops.h:1384-1428, helpers :1268-1382). */
int gc_wilson_spatial_3d(gc_lattice *h, int r_min, int r_max, int time_min, int time_max,
                         double alpha, int smearing_start, int smearing_end, int smearing_step,
                         gc_wilson_spatial_result *out, int capacity, int *count);

/* Average of the three spatial plaquettes per site.
 * Replaces: plaket_space(conf) (plaket.h:123-141, sites :63-81). */
int gc_plaquette_space(gc_lattice *h, double *out);

/* Average of the three (mu, t) plaquettes per site.
 * Replaces: plaket_time(conf) (plaket.h:103-121, sites :44-61). */
int gc_plaquette_time(gc_lattice *h, double *out);

/* Polyakov loop: mean over spatial sites of Re Tr P / N, P the product of
 * the Lt time links of the site's column.
 * Replaces: polyakov_loop(conf) (polyakov_loops.h:24-41, lines :10-22). */
int gc_polyakov_loop(gc_lattice *h, double *out);

#define GC_POLYAKOV_COLOR_AVERAGE 0
#define GC_POLYAKOV_SINGLET 1
/* Polyakov-loop correlator table of (2 d_max + 1)^3 doubles, entry
 * (Dz+d_max)(2d_max+1)^2 + (Dy+d_max)(2d_max+1) + Dx+d_max, for the offsets
 * the reference visits (|D| <= d_max; Dx >= 0 when Dy, Dz are both non-zero),
 * other entries 0. kind GC_POLYAKOV_COLOR_AVERAGE: mean of
 * Re[tr P(s) conj(tr P(s+D))], tr = Tr/N; GC_POLYAKOV_SINGLET: mean of
 * Re Tr[P(s) P(s+D)^dag]/N.
 * Replaces: polyakov_loop_correlator_color_average (polyakov_loops.h:83-145)
 * and polyakov_loop_correlator_singlet (:147-206). */
int gc_polyakov_correlator(gc_lattice *h, int d_max, int kind, double *out);

/* Reads a configuration file straight into h's device links.
 * format: "lexicographical" (link index 4*site+mu, get_data element order),
 * "qcdstag" (direction-major with t first; SU(2) elements a0,a3,a2,a1) or
 * "ildg" (LIME container, record "ildg-binary-data", big-endian doubles);
 * precision: "float" or "double" (ignored for ildg, which is read as
 * doubles); bytes_skip: header bytes before the links (not for ildg);
 * convert != 0 applies the reference's MatrixConverter<MT,MT> (diagonal phase
 * removal). Files shorter than the lattice are an error (GC_ERR_IO).
 * Replaces: Data::read_data_convert(conf, path, format, bytes_skip,
 * precision, convert) (data.h:265-338; patterns indexing.h:190-351). */
int gc_read_config(gc_lattice *h, const char *path, const char *format,
                   long long bytes_skip, const char *precision, int convert);

/* Writes h's links as doubles in the lexicographical pattern.
 * Replaces: conf.write_data(path, FilePatternLexicographical) (data.h:193-205),
 * the format apps/smearing saves smeared configurations in. */
int gc_write_config(gc_lattice *h, const char *path);

/* Host-only check of a configuration file (no device needed): the byte
 * offset and length of the link payload, or GC_ERR_IO with the reason
 * (missing file, too short, not a LIME file, no ildg-binary-data record). */
int gc_probe_config(const int dims[4], int nc, const char *path,
                    const char *format, long long bytes_skip,
                    const char *precision, long long *offset,
                    long long *length);

/* Fills h with the seeded synthetic configuration used by the benchmarks:
 *   SU(2): U = (cos th, sin th a/|a|), th = eps*|a|, a_k ~ N(0,1);
 *   SU(3): U = exp(i eps sum_a c_a lambda_a), c_a ~ N(0,1), reunitarised;
 * then, if gauge != 0, a Haar-random gauge transformation
 * U_mu(x) <- g(x) U_mu(x) g(x+mu)^dag. Randomness: Philox-4x32-10 with key
 * (seed, config_index); identical on every host and thread count. The links
 * are generated on the host and uploaded. */
int gc_generate(gc_lattice *h, double eps, unsigned int seed,
                unsigned int config_index, int gauge);

/* Host-only generator (no device needed): writes 4*V links in layout
 * GC_LAYOUT_ROWMAJOR to host_links. Same stream of numbers as gc_generate. */
int gc_generate_host(const int dims[4], int nc, double eps, unsigned int seed,
                     unsigned int config_index, int gauge, double *host_links);

/* ---------------------------------------------------------------- batches
 * Many independent smear-and-measure jobs of uneven sizes (SU(2) and SU(3)
 * mixed), run together. The reference runs one configuration per program
 * invocation (apps/smearing/smearing.cpp:228-301); a batch is that loop for
 * many configurations at once: HYP x hyp_steps, APE x ape_steps, then the
 * W(R,T) table, per job. Each phase is one launch over all jobs of a group;
 * the first gc_batch_run captures the schedule into a CUDA graph and later
 * runs replay it. */
typedef struct gc_batch gc_batch;

typedef struct {
  int dims[4];          /* Lx, Ly, Lz, Lt */
  int nc;               /* 2 or 3 */
  int hyp_steps;        /* >= 0 */
  double hyp_alpha[3];  /* alpha1, alpha2, alpha3 */
  int ape_steps;        /* >= 0 */
  double ape_alpha;
  int r_min, r_max;     /* W ranges; r_max = time_max = 0: no W table */
  int time_min, time_max;
} gc_job;

/* Plans the batch and allocates all its device memory (links, working
 * fields, W partial sums and tables). */
int gc_batch_create(const gc_job *jobs, int njobs, int precision,
                    gc_batch **out);
int gc_batch_destroy(gc_batch *b);
/* Sets job j's input links (host array, GC_LAYOUT_*). Every run starts from
 * the inputs. */
int gc_batch_upload(gc_batch *b, int job, const double *host_links,
                    int layout);
/* Sets every job's input to the seeded synthetic configuration of
 * gc_generate (eps by group), config index first_index + job. */
int gc_batch_generate(gc_batch *b, double eps_su2, double eps_su3,
                      unsigned int seed, unsigned int first_index);
/* Optional: times the candidate W block shapes for each distinct (time
 * extent, group, R/T range) of the batch on this GPU and keeps the fastest. */
int gc_batch_autotune(gc_batch *b);
/* Runs the whole batch on cuda_stream (NULL: the batch's own stream) and
 * returns after enqueueing. The first run executes eagerly and captures the
 * schedule into a CUDA graph; later runs launch the graph. */
int gc_batch_run(gc_batch *b, void *cuda_stream);
/* Waits for the last run. */
int gc_batch_synchronize(gc_batch *b);
/* Job j's W table of the last run (waits for it), laid out like
 * gc_wilson_onaxis's output. */
int gc_batch_wilson(gc_batch *b, int job, double *out);
/* Job j's smeared links of the last run (host array, GC_LAYOUT_*). */
int gc_batch_download(gc_batch *b, int job, double *host_links, int layout);
/* Device bytes of the batch, kernel nodes of its graph (0 before the first
 * run) and kernel launches per run. */
int gc_batch_info(const gc_batch *b, long long *device_bytes, int *graph_nodes,
                  int *launches);
/* The W block shape (threads per column, columns per block) used for job j. */
int gc_batch_job_shape(const gc_batch *b, int job, int *rows, int *cols);
/* What gc_batch_autotune measured: one line per candidate block shape timed
 * ("<job class> <kernel> <shape> <ms>"), the chosen ones marked; copied into
 * buf (at most len bytes, NUL-terminated). No counterpart in the reference. */
int gc_batch_autotune_report(const gc_batch *b, char *buf, int len);

/* ---------------------------------------------------------------- serving
 * A request loop: each request is one configuration (a gc_job and its host
 * links). Requests wait in a FIFO queue; `slots` workers, each on its own
 * CUDA stream, take the head as soon as a worker is free and the head's
 * device memory (gc_job_device_bytes) fits in the rest of the memory budget
 * (and, if a free-memory provider is given, in the free memory it reports).
 * Requests run concurrently on the GPU with stream-ordered memory; a
 * request's result is bitwise the same alone and among others. No
 * counterpart in the reference (its programs process one configuration per
 * invocation). */
typedef struct gc_server gc_server;

typedef struct {
  int slots;                 /* requests on the GPU at once (1..256) */
  int precision;             /* GC_PREC_FP64 or GC_PREC_MIXED */
  long long memory_budget;   /* bytes admitted requests may hold together;
                                0: 90% of the free device memory at creation */
  int queue_capacity;        /* pending requests before GC_ERR_BUSY; 0: no limit */
  long long (*free_bytes)(void *ctx); /* optional free-memory provider */
  void *free_bytes_ctx;
  int simulate_us;           /* > 0: no GPU work, each request sleeps this many
                                microseconds (tests of the admission logic) */
  long long reserve_bytes;   /* device memory the requests' stream-ordered pool
                                (the device's default pool) takes at creation
                                and keeps, so that running requests allocate
                                without mapping new memory (a mapping stalls
                                every stream on the device); 0: min(budget,
                                16 GiB); < 0: none. With a free-memory provider,
                                the pool's reserved but unused bytes count as
                                free for admission (other users of the default
                                pool share them) */
} gc_server_opts;

typedef struct {
  long long submitted, completed, rejected, failed, pending;
  int inflight, peak_inflight;
  long long peak_bytes, budget;
  double p50_ms, p99_ms, mean_ms; /* submit-to-result latency of completed requests */
  double sites_per_s;             /* completed sites / (last result - first submit) */
  double queue_p50_ms, queue_p99_ms; /* submit-to-admission part of the latency */
  double run_p50_ms, run_p99_ms;     /* admission-to-result part */
} gc_server_metrics;

int gc_server_create(const gc_server_opts *opts, gc_server **out);
/* Queues a request. host_links (4V links, GC_LAYOUT_*) must stay valid until
 * the request completes. GC_ERR_NOMEM: the job alone exceeds the memory
 * budget; GC_ERR_BUSY: the queue is full. */
int gc_server_submit(gc_server *s, const gc_job *job, const double *host_links,
                     int layout, unsigned long long *id);
/* Waits up to timeout_s seconds for request id and copies its W table to
 * out_w (as gc_wilson_onaxis lays it out). GC_ERR_TIMEOUT leaves the request
 * in place (wait again); any other return releases it. */
int gc_server_wait(gc_server *s, unsigned long long id, double *out_w,
                   double timeout_s);
/* Removes a request that has not started (GC_ERR_STATE if it has). */
int gc_server_cancel(gc_server *s, unsigned long long id);
int gc_server_stats(gc_server *s, gc_server_metrics *stats);
/* Cancels pending requests, waits for running ones, frees everything. */
int gc_server_destroy(gc_server *s);

/* Bytes of device memory a handle of this shape uses for links plus working
 * buffers of a full HYP + APE + W job (for admission control). */
long long gc_job_device_bytes(const int dims[4], int nc, int precision,
                              int r_max, int time_max);

/* Measured vector FMA throughput of the current device in TFLOP/s: packed
 * FP32x2 fused multiply-adds (precision GC_PREC_MIXED) or FP64 ones
 * (GC_PREC_FP64) on every SM, best of three timed launches on the legacy
 * default stream (so it waits for, and is not overlapped by, other work on
 * the device). The compute roofline denominator of the smearing and
 * Wilson-loop kernels, which are bound by the FP32 or FP64 pipe rather than
 * by HBM. No reference counterpart. */
int gc_fma_peak(int precision, double *tflops);

#ifdef __cplusplus
}
#endif

#endif /* GC_LATTICE_H */
