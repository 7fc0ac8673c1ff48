// C-ABI harness around the reference's OWN templated CPU path, compiled from
// the reference sources by oracle/Makefile into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline): the
// product never links this. Every entry point calls the reference functions
// unchanged:
//   smearing_APE          lib/cpu/include/smearing.h:115-161
//   smearing_HYP          lib/cpu/include/smearing.h:480-516
//   wilson_loop           lib/cpu/include/wilson_loops.h:1047-1074
//   wilson_loop_adjoint   lib/cpu/include/wilson_loops.h:1173-1200
//   plaket_site           lib/cpu/include/plaket.h:24-42
//   plaket_site_time / plaket_site_space   plaket.h:44-61, 63-81
//   wilson_gevp_indexed / wilson_gevp_adjoint_indexed  wilson_loops.h:1202-1266
//   get_polyakov_loop, polyakov_loop_correlator_{color_average,singlet}
//                         lib/cpu/include/polyakov_loops.h:10-22, 83-206
//   polyakov_average_directions            lib/cpu/src/polyakov_loops.cpp:6-40
//   wilson_offaxis[_adjoint], wilson_offaxis[_adjoint]_result
//                         lib/cpu/include/wilson_loops.h:313-663
//   smearing_APE_2d       lib/cpu/include/smearing.h:223-277
//   wilson_spatial_3d_indexed              lib/cpu/include/wilson_loops.h:1384-1428
//   Data::read_data_convert / write_data   lib/cpu/include/data.h:193-205,265-338
//
// Link exchange layout ("row-major"): link index 4*site+mu with
// site = x + Lx*(y + Ly*(z + Lz*t)) (indexing.h:111-123); per link the
// matrix's get_data() order: su2 = (a0,a1,a2,a3), su3 = 18 doubles,
// element (i,j) at (3*i+j)*2 (re) and +1 (im) (matrix.h:236-243).
#include "data.h"
#include "indexing.h"
#include "matrix.h"
#include "plaket.h"
#include "polyakov_loops.h"
#include "smearing.h"
#include "wilson_loops.h"

#include <chrono>
#include <cstring>
#include <omp.h>
#include <string>

// The legacy headers declare these as extern (indexing.h:8-13); each reference
// app defines them in its main translation unit.
int x_size;
int y_size;
int z_size;
int t_size;
int size1;
int size2;

namespace {

typedef DataPatternLexicographical DP;

void set_globals(const int *dims) {
  x_size = dims[0];
  y_size = dims[1];
  z_size = dims[2];
  t_size = dims[3];
  size1 = x_size * y_size;
  size2 = x_size * y_size * z_size;
}

template <class MT>
Data::LatticeData<DP, MT> make_conf(const int *dims, const double *links) {
  Data::LatticeData<DP, MT> conf({dims[0], dims[1], dims[2], dims[3]});
  const int ds = MT::data_size;
  std::vector<double> buf(ds);
  for (size_t i = 0; i < conf.array.size(); i++) {
    for (int k = 0; k < ds; k++)
      buf[k] = links[i * ds + k];
    conf.array[i] = MT(buf);
  }
  return conf;
}

template <class MT>
void export_conf(Data::LatticeData<DP, MT> &conf, double *links) {
  const int ds = MT::data_size;
  for (size_t i = 0; i < conf.array.size(); i++) {
    std::vector<double> buf = conf.array[i].get_data();
    for (int k = 0; k < ds; k++)
      links[i * ds + k] = buf[k];
  }
}

template <class MT>
void wilson_to_table(const std::map<std::tuple<int, int>, double> &w, int rmin,
                     int rmax, int tmin, int tmax, double *out) {
  const int nr = rmax - rmin + 1;
  for (int t = tmin; t <= tmax; t++)
    for (int r = rmin; r <= rmax; r++)
      out[(t - tmin) * nr + (r - rmin)] = w.at(std::tuple<int, int>(t, r));
}

// The reference's plaket() leaves its OpenMP reduction variable uninitialised
// (plaket.h:85), so its result depends on stack contents. The harness sums the
// reference's own per-site function plaket_site (plaket.h:24-42) into a zeroed
// accumulator instead, in the same site order.
template <class MT> double plaquette(const Data::LatticeData<DP, MT> &conf) {
  DP dp(conf.lat_dim);
  double sum = 0;
#pragma omp parallel for collapse(4) firstprivate(dp) reduction(+ : sum)
  for (int t = 0; t < dp.lat_dim[3]; t++)
    for (int z = 0; z < dp.lat_dim[2]; z++)
      for (int y = 0; y < dp.lat_dim[1]; y++)
        for (int x = 0; x < dp.lat_dim[0]; x++) {
          dp.lat_coord = {x, y, z, t};
          sum += plaket_site(conf, dp);
        }
  return sum / dp.get_lattice_size();
}

// plaket_time / plaket_space (plaket.h:103-141) and polyakov_loop
// (polyakov_loops.h:24-41) have the same uninitialised reduction variable;
// the harness sums the reference's per-site functions into zeroed
// accumulators. which: 1 time, 2 space.
template <class MT> double plaquette_part(const Data::LatticeData<DP, MT> &conf, int which) {
  DP dp(conf.lat_dim);
  double sum = 0;
#pragma omp parallel for collapse(4) firstprivate(dp) reduction(+ : sum)
  for (int t = 0; t < dp.lat_dim[3]; t++)
    for (int z = 0; z < dp.lat_dim[2]; z++)
      for (int y = 0; y < dp.lat_dim[1]; y++)
        for (int x = 0; x < dp.lat_dim[0]; x++) {
          dp.lat_coord = {x, y, z, t};
          sum += which == 1 ? plaket_site_time(conf, dp) : plaket_site_space(conf, dp);
        }
  return sum / dp.get_lattice_size();
}

template <class MT> double polyakov_mean(const Data::LatticeData<DP, MT> &conf) {
  DP dp(conf.lat_dim);
  double sum = 0;
  for (int z = 0; z < dp.lat_dim[2]; z++)
    for (int y = 0; y < dp.lat_dim[1]; y++)
      for (int x = 0; x < dp.lat_dim[0]; x++) {
        dp.lat_coord = {x, y, z, 0};
        sum += get_polyakov_loop(conf, dp).tr_real();
      }
  return sum / (dp.lat_dim[0] * dp.lat_dim[1] * dp.lat_dim[2]);
}

double now() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

template <class MT>
int job(const int *dims, double *links, int hyp_steps, double a1, double a2,
        double a3, int ape_steps, double alpha, int rmin, int rmax, int tmin,
        int tmax, double *out, double *times) {
  set_globals(dims);
  Data::LatticeData<DP, MT> conf = make_conf<MT>(dims, links);
  double t0 = now();
  for (int i = 0; i < hyp_steps; i++)
    smearing_HYP(conf, a1, a2, a3);
  double t1 = now();
  for (int i = 0; i < ape_steps; i++)
    smearing_APE(conf, alpha);
  double t2 = now();
  if (rmax >= rmin && tmax >= tmin) {
    std::map<std::tuple<int, int>, double> w =
        wilson_loop(conf, rmin, rmax, tmin, tmax);
    wilson_to_table<MT>(w, rmin, rmax, tmin, tmax, out);
  }
  double t3 = now();
  if (times) {
    times[0] = t1 - t0;
    times[1] = t2 - t1;
    times[2] = t3 - t2;
  }
  export_conf(conf, links);
  return 0;
}

template <class MT>
int read_conf(const int *dims, const char *path, const char *format,
              int bytes_skip, const char *precision, int convert,
              double *links) {
  set_globals(dims);
  Data::LatticeData<DP, MT> conf({dims[0], dims[1], dims[2], dims[3]});
  Data::read_data_convert(conf, std::string(path), std::string(format),
                          bytes_skip, std::string(precision), convert != 0);
  export_conf(conf, links);
  return 0;
}

template <class MT>
int ape_plane(const int *dims, double *links, int a, int b, double alpha, int steps) {
  Data::LatticeData<DP, MT> conf = make_conf<MT>(dims, links);
  DP dp(conf.lat_dim);
  std::vector<MT> f1 = get_data_single_direction(conf, a);
  std::vector<MT> f2 = get_data_single_direction(conf, b);
  for (int i = 0; i < steps; i++)
    smearing_APE_2d(f1, f2, dp, a, b, alpha);
  for (size_t x = 0; x < f1.size(); x++) {
    conf.array[4 * x + a] = f1[x];
    conf.array[4 * x + b] = f2[x];
  }
  export_conf(conf, links);
  return 0;
}

} // namespace

extern "C" {

int ref_num_threads() { return omp_get_max_threads(); }

void ref_set_threads(int n) {
  if (n > 0)
    omp_set_num_threads(n);
}

int ref_ape(int nc, const int *dims, double *links, double alpha, int steps) {
  double dummy = 0;
  if (nc == 2)
    return job<su2>(dims, links, 0, 0, 0, 0, steps, alpha, 1, 0, 1, 0, &dummy,
                    nullptr);
  if (nc == 3)
    return job<su3>(dims, links, 0, 0, 0, 0, steps, alpha, 1, 0, 1, 0, &dummy,
                    nullptr);
  return -1;
}

int ref_hyp(int nc, const int *dims, double *links, double a1, double a2,
            double a3, int steps) {
  double dummy = 0;
  if (nc == 2)
    return job<su2>(dims, links, steps, a1, a2, a3, 0, 0, 1, 0, 1, 0, &dummy,
                    nullptr);
  if (nc == 3)
    return job<su3>(dims, links, steps, a1, a2, a3, 0, 0, 1, 0, 1, 0, &dummy,
                    nullptr);
  return -1;
}

int ref_wilson(int nc, const int *dims, const double *links, int rmin,
               int rmax, int tmin, int tmax, double *out) {
  set_globals(dims);
  if (nc == 2) {
    Data::LatticeData<DP, su2> conf = make_conf<su2>(dims, links);
    wilson_to_table<su2>(wilson_loop(conf, rmin, rmax, tmin, tmax), rmin, rmax,
                         tmin, tmax, out);
    return 0;
  }
  if (nc == 3) {
    Data::LatticeData<DP, su3> conf = make_conf<su3>(dims, links);
    wilson_to_table<su3>(wilson_loop(conf, rmin, rmax, tmin, tmax), rmin, rmax,
                         tmin, tmax, out);
    return 0;
  }
  return -1;
}

// wilson_loop_adjoint (wilson_loops.h:1173-1200)
int ref_wilson_adjoint(int nc, const int *dims, const double *links, int rmin,
                       int rmax, int tmin, int tmax, double *out) {
  set_globals(dims);
  if (nc == 2) {
    Data::LatticeData<DP, su2> conf = make_conf<su2>(dims, links);
    wilson_to_table<su2>(wilson_loop_adjoint(conf, rmin, rmax, tmin, tmax), rmin,
                         rmax, tmin, tmax, out);
    return 0;
  }
  if (nc == 3) {
    Data::LatticeData<DP, su3> conf = make_conf<su3>(dims, links);
    wilson_to_table<su3>(wilson_loop_adjoint(conf, rmin, rmax, tmin, tmax), rmin,
                         rmax, tmin, tmax, out);
    return 0;
  }
  return -1;
}

int ref_wilson_gevp(int nc, const int *dims, const double *links1, const double *links2,
                    int rmin, int rmax, int tmin, int tmax, int adjoint, double *out) {
  set_globals(dims);
  if (nc == 2) {
    Data::LatticeData<DP, su2> c1 = make_conf<su2>(dims, links1), c2 = make_conf<su2>(dims, links2);
    wilson_to_table<su2>(adjoint ? wilson_gevp_adjoint_indexed(c1, c2, rmin, rmax, tmin, tmax)
                                 : wilson_gevp_indexed(c1, c2, rmin, rmax, tmin, tmax),
                         rmin, rmax, tmin, tmax, out);
    return 0;
  }
  if (nc == 3) {
    Data::LatticeData<DP, su3> c1 = make_conf<su3>(dims, links1), c2 = make_conf<su3>(dims, links2);
    wilson_to_table<su3>(adjoint ? wilson_gevp_adjoint_indexed(c1, c2, rmin, rmax, tmin, tmax)
                                 : wilson_gevp_indexed(c1, c2, rmin, rmax, tmin, tmax),
                         rmin, rmax, tmin, tmax, out);
    return 0;
  }
  return -1;
}

double ref_plaquette_part(int nc, const int *dims, const double *links, int which) {
  set_globals(dims);
  if (nc == 2)
    return plaquette_part(make_conf<su2>(dims, links), which);
  if (nc == 3)
    return plaquette_part(make_conf<su3>(dims, links), which);
  return 0.0;
}

double ref_polyakov_loop(int nc, const int *dims, const double *links) {
  set_globals(dims);
  if (nc == 2)
    return polyakov_mean(make_conf<su2>(dims, links));
  if (nc == 3)
    return polyakov_mean(make_conf<su3>(dims, links));
  return 0.0;
}

// kind 0: color average, 1: singlet; out: (2 D + 1)^3 doubles.
int ref_polyakov_correlator(int nc, const int *dims, const double *links, int D, int kind,
                            double *out) {
  set_globals(dims);
  std::vector<double> v;
  if (nc == 2) {
    Data::LatticeData<DP, su2> c = make_conf<su2>(dims, links);
    v = kind ? polyakov_loop_correlator_singlet(c, D) : polyakov_loop_correlator_color_average(c, D);
  } else if (nc == 3) {
    Data::LatticeData<DP, su3> c = make_conf<su3>(dims, links);
    v = kind ? polyakov_loop_correlator_singlet(c, D) : polyakov_loop_correlator_color_average(c, D);
  } else {
    return -1;
  }
  std::memcpy(out, v.data(), v.size() * sizeof(double));
  return 0;
}

// polyakov_average_directions: distances (ascending) and averages; returns
// the number of distances (at most cap).
int ref_polyakov_average_directions(const double *table, int D, double *dist, double *avg,
                                    int cap) {
  const int n = (2 * D + 1) * (2 * D + 1) * (2 * D + 1);
  std::map<double, double> m = polyakov_average_directions(std::vector<double>(table, table + n), D);
  int i = 0;
  for (auto &kv : m) {
    if (i >= cap)
      break;
    dist[i] = kv.first;
    avg[i] = kv.second;
    i++;
  }
  return i;
}

// Off-axis loops. mode 0: wilson_offaxis with the given directions;
// mode 1: wilson_offaxis_result (directions of length <= 4, merged, as the
// map it returns). adjoint selects the _adjoint forms (su3 only: the
// reference's su2 has no tr_adjoint). Entries go to w/t/s/n (capacity cap);
// returns the count.
int ref_wilson_offaxis(int nc, const int *dims, const double *links, int mode,
                       const int *directions, int ndirections, double rmin, double rmax,
                       int tmin, int tmax, int adjoint, double *w, int *t, double *s, int *n,
                       int cap) {
  set_globals(dims);
  std::vector<std::vector<int>> dirs;
  for (int i = 0; i < ndirections; i++)
    dirs.push_back({directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]});
  std::vector<wilson_result> raw;
  std::map<std::tuple<int, double>, double> merged;
  if (nc == 2 && !adjoint) {
    Data::LatticeData<DP, su2> c = make_conf<su2>(dims, links);
    if (mode == 0)
      raw = wilson_offaxis(c, dirs, rmin, rmax, tmin, tmax);
    else
      merged = wilson_offaxis_result(c, rmin, rmax, tmin, tmax);
  } else if (nc == 3) {
    Data::LatticeData<DP, su3> c = make_conf<su3>(dims, links);
    if (mode == 0)
      raw = adjoint ? wilson_offaxis_adjoint(c, dirs, rmin, rmax, tmin, tmax)
                    : wilson_offaxis(c, dirs, rmin, rmax, tmin, tmax);
    else
      merged = adjoint ? wilson_offaxis_adjoint_result(c, rmin, rmax, tmin, tmax)
                       : wilson_offaxis_result(c, rmin, rmax, tmin, tmax);
  } else {
    return -1;
  }
  int k = 0;
  if (mode == 0) {
    for (const auto &r : raw) {
      if (k < cap) {
        w[k] = r.wilson_loop;
        t[k] = r.time_size;
        s[k] = r.space_size;
        n[k] = r.statistics_size;
      }
      k++;
    }
  } else {
    for (const auto &kv : merged) {
      if (k < cap) {
        w[k] = kv.second;
        t[k] = std::get<0>(kv.first);
        s[k] = std::get<1>(kv.first);
        n[k] = 0;
      }
      k++;
    }
  }
  return k;
}

// smearing_APE_2d on the direction fields a, b of a configuration (in place)
int ref_ape_plane(int nc, const int *dims, double *links, int a, int b, double alpha,
                  int steps) {
  set_globals(dims);
  if (nc == 2)
    return ape_plane<su2>(dims, links, a, b, alpha, steps);
  if (nc == 3)
    return ape_plane<su3>(dims, links, a, b, alpha, steps);
  return -1;
}

// wilson_spatial_3d_indexed: entries (smearing, T, R, W) in map order
int ref_wilson_spatial_3d(int nc, const int *dims, const double *links, int rmin, int rmax,
                          int tmin, int tmax, double alpha, int sm_start, int sm_end,
                          int sm_step, int *out_s, int *out_t, int *out_r, double *out_w,
                          int cap) {
  set_globals(dims);
  std::map<std::tuple<int, int, int>, double> m;
  if (nc == 2)
    m = wilson_spatial_3d_indexed(make_conf<su2>(dims, links), rmin, rmax, tmin, tmax, alpha,
                                  sm_start, sm_end, sm_step);
  else if (nc == 3)
    m = wilson_spatial_3d_indexed(make_conf<su3>(dims, links), rmin, rmax, tmin, tmax, alpha,
                                  sm_start, sm_end, sm_step);
  else
    return -1;
  int k = 0;
  for (const auto &kv : m) {
    if (k < cap) {
      out_s[k] = std::get<0>(kv.first);
      out_t[k] = std::get<1>(kv.first);
      out_r[k] = std::get<2>(kv.first);
      out_w[k] = kv.second;
    }
    k++;
  }
  return k;
}

double ref_plaquette(int nc, const int *dims, const double *links) {
  set_globals(dims);
  if (nc == 2)
    return plaquette(make_conf<su2>(dims, links));
  if (nc == 3)
    return plaquette(make_conf<su3>(dims, links));
  return 0.0;
}

// Full smear-and-measure job as apps/smearing/smearing.cpp:228-301 runs it
// (HYP steps, then APE steps, then one W table), without the app's extra W at
// smearing step 0. times[0..2] = seconds in HYP, APE, W.
int ref_job(int nc, const int *dims, double *links, int hyp_steps, double a1,
            double a2, double a3, int ape_steps, double alpha, int rmin,
            int rmax, int tmin, int tmax, double *out, double *times) {
  if (nc == 2)
    return job<su2>(dims, links, hyp_steps, a1, a2, a3, ape_steps, alpha, rmin,
                    rmax, tmin, tmax, out, times);
  if (nc == 3)
    return job<su3>(dims, links, hyp_steps, a1, a2, a3, ape_steps, alpha, rmin,
                    rmax, tmin, tmax, out, times);
  return -1;
}

int ref_read(int nc, const int *dims, const char *path, const char *format,
             int bytes_skip, const char *precision, int convert,
             double *links) {
  if (nc == 2)
    return read_conf<su2>(dims, path, format, bytes_skip, precision, convert,
                          links);
  if (nc == 3)
    return read_conf<su3>(dims, path, format, bytes_skip, precision, convert,
                          links);
  return -1;
}

// write_data with the lexicographical file pattern, as apps/smearing writes a
// smeared configuration (smearing.cpp:336-339).
int ref_write_lexicographical(int nc, const int *dims, const double *links,
                              const char *path) {
  set_globals(dims);
  if (nc == 2) {
    Data::LatticeData<DP, su2> conf = make_conf<su2>(dims, links);
    FilePatternLexicographical<4, su2> fp;
    conf.write_data(std::string(path), fp);
    return 0;
  }
  if (nc == 3) {
    Data::LatticeData<DP, su3> conf = make_conf<su3>(dims, links);
    FilePatternLexicographical<4, su3> fp;
    conf.write_data(std::string(path), fp);
    return 0;
  }
  return -1;
}

} // extern "C"

