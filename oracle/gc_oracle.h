/*
 * CPU restatement of the reference's APE/HYP smearing, on-axis Wilson loops
 * and plaquette, in plain C (FP64).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as the checker. The product never links it.
 * Parity pinned against golden fixtures produced by the reference's own code
 * (oracle/_ref, tests/golden/make_golden.py).
 *
 * Links: host array of 4*V links, link index 4*site+mu, site = x + Lx*(y +
 * Ly*(z + Lz*t)); SU(2) 4 doubles (a0..a3), SU(3) 18 doubles row-major
 * (element (i,j) at (3i+j)*2 re, +1 im).
 */
#ifndef GC_ORACLE_H
#define GC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

int or_ape(int nc, const int dims[4], double *links, double alpha, int steps);
int or_hyp(int nc, const int dims[4], double *links, double alpha1,
           double alpha2, double alpha3, int steps);
int or_wilson(int nc, const int dims[4], const double *links, int r_min,
              int r_max, int time_min, int time_max, double *out);
int or_wilson_adjoint(int nc, const int dims[4], const double *links, int r_min,
                      int r_max, int time_min, int time_max, double *out);
/* Two-configuration (GEVP) loops; adjoint selects the adjoint trace. */
int or_wilson_gevp(int nc, const int dims[4], const double *links1, const double *links2,
                   int r_min, int r_max, int time_min, int time_max, int adjoint,
                   double *out);
/* Off-axis Wilson loops; entries as the reference's wilson_result. Return
 * the entry count (entries past capacity are not written) or -1. */
typedef struct {
  double wilson_loop;
  int time_size;
  double space_size;
  int statistics_size;
} or_wilson_result;
int or_wilson_offaxis(int nc, const int dims[4], const double *links, const int *directions,
                      int ndirections, double r_min, double r_max, int time_min, int time_max,
                      int adjoint, or_wilson_result *out, int capacity);
int or_wilson_offaxis_result(int nc, const int dims[4], const double *links, double r_min,
                             double r_max, int time_min, int time_max, int adjoint,
                             or_wilson_result *out, int capacity);
/* smearing_APE_2d of the direction fields a, b (in place). */
int or_ape_plane(int nc, const int dims[4], double *links, int a, int b, double alpha,
                 int steps);
/* wilson_spatial_3d_indexed: entries (smearing, T, R, W); returns the count. */
int or_wilson_spatial_3d(int nc, const int dims[4], const double *links, int rmin, int rmax,
                         int tmin, int tmax, double alpha, int sm_start, int sm_end,
                         int sm_step, int *out_s, int *out_t, int *out_r, double *out_w,
                         int cap);
double or_plaquette(int nc, const int dims[4], const double *links);
double or_plaquette_time(int nc, const int dims[4], const double *links);
double or_plaquette_space(int nc, const int dims[4], const double *links);
double or_polyakov_loop(int nc, const int dims[4], const double *links);
/* kind 0: color average, 1: singlet; out: (2 D + 1)^3 doubles. */
int or_polyakov_correlator(int nc, const int dims[4], const double *links, int D, int kind,
                           double *out);
/* Applies proj() to every link (test helper for the projection alone). */
int or_proj_all(int nc, long long nlinks, double *links);
void or_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
