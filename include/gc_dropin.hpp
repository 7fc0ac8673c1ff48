// general_code_b200 — C++ drop-in for the reference's smearing / Wilson-loop
// path. Include this header AFTER the reference's own headers
// (lib/cpu/include/smearing.h, wilson_loops.h, plaket.h, data.h): it adds
// non-template overloads with the reference's exact signatures for
// Data::LatticeData<DataPatternLexicographical, su2|su3>. Overload resolution
// prefers a non-template function over a template of equal match, so the
// existing call sites in apps/smearing/smearing.cpp and
// apps/observables/wilson_loops/wilson_loops.cpp bind to these without
// further edits.
//
// Each call uploads conf.array to the GPU, runs the sm_100a kernels and copies
// the result back, keeping the reference's semantics (in-place smearing; W
// returned as std::map keyed (T, R)). There is no CPU fallback: a failure
// (no sm_100 device, out of memory, ...) throws std::runtime_error with the
// library's message. Link with libgc_b200.so.
//
//   reference signature                                   file:line
//   smearing_APE(LatticeData&, double)                    smearing.h:115-117
//   smearing_HYP(LatticeData&, double, double, double)    smearing.h:480-482
//   wilson_loop(const LatticeData&, int, int, int, int)   wilson_loops.h:1047-1050
//   wilson_loop_adjoint(const LatticeData&, int x4)       wilson_loops.h:1173-1176
//   wilson_loop(const std::vector<T>&, int, int, int, int)
//                                              basic_observables.h:108-111
//   plaket(const LatticeData&)                            plaket.h:83-84
//   plaket_time / plaket_space(const LatticeData&)        plaket.h:103-141
//   wilson_gevp_indexed / wilson_gevp_adjoint_indexed(const LatticeData&,
//       const LatticeData&, int, int, int, int)           wilson_loops.h:1202-1266
//   polyakov_loop(const LatticeData&)                     polyakov_loops.h:24-41
//   polyakov_loop_correlator_color_average / _singlet(const LatticeData&, int)
//                                                         polyakov_loops.h:83-206
//   Data::read_data_convert(LatticeData&, std::string, std::string, int,
//       std::string, bool)                                data.h:265-338
//   wilson_offaxis / wilson_offaxis_adjoint(const LatticeData&,
//       std::vector<std::vector<int>>, double, double, int, int)
//                                                         wilson_loops.h:313-317, 487-491
//   wilson_offaxis_result / wilson_offaxis_adjoint_result(const LatticeData&,
//       double, double, int, int)                         wilson_loops.h:470-473, 648-651
//   wilson_offaxis_result / wilson_offaxis_adjoint_result(const std::vector<T>&,
//       double, double, int, int)                         basic_observables.h:34-36, 45-48
//   wilson_spatial_3d_indexed(const LatticeData&, int, int, int, int, double,
//       int, int, int)                                    wilson_loops.h:1384-1388
//
// Helpers the reference templates call internally (wilson_offaxis from
// wilson_offaxis_result, smearing_APE_2d from wilson_spatial_3d_indexed) are
// found by argument-dependent lookup inside those templates too; the
// overloads below take over whole observables, and smearing_APE_2d has no
// overload (gc_ape_plane in gc_lattice.h is its C entry point).
#pragma once

#include "gc_lattice.h"

#include <array>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

namespace gc_dropin {

template <class MT> struct traits;
template <> struct traits<su2> {
  static constexpr int nc = 2;
  static constexpr int layout = GC_LAYOUT_ROWMAJOR; // a0, a1, a2, a3
};
template <> struct traits<su3> {
  static constexpr int nc = 3;
  // std::vector<su3> holds one Eigen::Matrix3cd (column-major) per link
  static constexpr int layout = GC_LAYOUT_EIGEN_COLMAJOR;
};

inline void check(int rc, gc_lattice *h, const char *what) {
  if (rc != GC_OK)
    throw std::runtime_error(std::string("general_code_b200 ") + what + ": " +
                             gc_last_error(h));
}

// One device-resident copy of a configuration for the duration of a call.
template <class MT> class Session {
public:
  static_assert(sizeof(MT) == (traits<MT>::nc == 3 ? 18 : 4) * sizeof(double),
                "link type must be a plain array of doubles");
  // an empty FP64 handle (links to be read from a file)
  explicit Session(const std::array<int, 4> &dims) {
    check(gc_lattice_create(dims.data(), traits<MT>::nc, GC_PREC_FP64, &h_),
          nullptr, "create");
  }
  Session(const std::array<int, 4> &dims, const MT *links) {
    check(gc_lattice_create(dims.data(), traits<MT>::nc, GC_PREC_FP64, &h_),
          nullptr, "create");
    int rc = gc_upload(h_, reinterpret_cast<const double *>(links),
                       traits<MT>::layout);
    if (rc != GC_OK) {
      std::string msg = gc_last_error(h_);
      gc_lattice_destroy(h_);
      throw std::runtime_error("general_code_b200 upload: " + msg);
    }
  }
  ~Session() { gc_lattice_destroy(h_); }
  Session(const Session &) = delete;
  Session &operator=(const Session &) = delete;
  gc_lattice *get() const { return h_; }
  void download(MT *links) {
    check(gc_download(h_, reinterpret_cast<double *>(links), traits<MT>::layout),
          h_, "download");
  }

private:
  gc_lattice *h_ = nullptr;
};

template <class MT>
void ape(Data::LatticeData<DataPatternLexicographical, MT> &conf, double alpha) {
  Session<MT> s(conf.lat_dim, conf.array.data());
  check(gc_ape(s.get(), alpha, 1), s.get(), "APE");
  s.download(conf.array.data());
}

template <class MT>
void hyp(Data::LatticeData<DataPatternLexicographical, MT> &conf, double a1,
         double a2, double a3) {
  Session<MT> s(conf.lat_dim, conf.array.data());
  check(gc_hyp(s.get(), a1, a2, a3, 1), s.get(), "HYP");
  s.download(conf.array.data());
}

template <class MT>
std::map<std::tuple<int, int>, double>
wilson(const std::array<int, 4> &dims, const MT *links, int r_min, int r_max,
       int time_min, int time_max, bool adjoint = false) {
  std::map<std::tuple<int, int>, double> result;
  if (r_max < r_min || time_max < time_min)
    return result;
  Session<MT> s(dims, links);
  const int nr = r_max - r_min + 1, nt = time_max - time_min + 1;
  std::vector<double> w((size_t)nr * nt);
  if (adjoint)
    check(gc_wilson_adjoint_onaxis(s.get(), r_min, r_max, time_min, time_max, w.data()),
          s.get(), "wilson_loop_adjoint");
  else
    check(gc_wilson_onaxis(s.get(), r_min, r_max, time_min, time_max, w.data()),
          s.get(), "wilson_loop");
  for (int t = time_min; t <= time_max; t++)
    for (int r = r_min; r <= r_max; r++)
      result[std::tuple<int, int>(t, r)] = w[(t - time_min) * nr + (r - r_min)];
  return result;
}

// which: 0 all planes, 1 (mu, t) planes, 2 spatial planes.
template <class MT>
double plaquette(const Data::LatticeData<DataPatternLexicographical, MT> &conf, int which = 0) {
  Session<MT> s(conf.lat_dim, conf.array.data());
  double p = 0;
  if (which == 1)
    check(gc_plaquette_time(s.get(), &p), s.get(), "plaket_time");
  else if (which == 2)
    check(gc_plaquette_space(s.get(), &p), s.get(), "plaket_space");
  else
    check(gc_plaquette(s.get(), &p), s.get(), "plaket");
  return p;
}

template <class MT>
std::map<std::tuple<int, int>, double>
gevp(const Data::LatticeData<DataPatternLexicographical, MT> &conf1,
     const Data::LatticeData<DataPatternLexicographical, MT> &conf2, int r_min, int r_max,
     int time_min, int time_max, bool adjoint) {
  std::map<std::tuple<int, int>, double> result;
  if (r_max < r_min || time_max < time_min)
    return result;
  if (conf1.lat_dim != conf2.lat_dim)
    throw std::runtime_error("general_code_b200 wilson_gevp: lattice sizes differ");
  Session<MT> a(conf1.lat_dim, conf1.array.data()), b(conf2.lat_dim, conf2.array.data());
  const int nr = r_max - r_min + 1, nt = time_max - time_min + 1;
  std::vector<double> w((size_t)nr * nt);
  if (adjoint)
    check(gc_wilson_gevp_adjoint_onaxis(a.get(), b.get(), r_min, r_max, time_min, time_max,
                                        w.data()),
          a.get(), "wilson_gevp_adjoint_indexed");
  else
    check(gc_wilson_gevp_onaxis(a.get(), b.get(), r_min, r_max, time_min, time_max, w.data()),
          a.get(), "wilson_gevp_indexed");
  for (int t = time_min; t <= time_max; t++)
    for (int r = r_min; r <= r_max; r++)
      result[std::tuple<int, int>(t, r)] = w[(t - time_min) * nr + (r - r_min)];
  return result;
}

// The file is read by the library's reader straight into device links
// (gc_read_config), then copied into conf.array.
template <class MT>
void read(Data::LatticeData<DataPatternLexicographical, MT> &conf, const std::string &path,
          const std::string &format, int bytes_skip, const std::string &precision,
          bool convert) {
  Session<MT> s(conf.lat_dim);
  check(gc_read_config(s.get(), path.c_str(), format.c_str(), bytes_skip, precision.c_str(),
                       convert ? 1 : 0),
        s.get(), "read_data_convert");
  s.download(conf.array.data());
}

// Off-axis entries of one call (gc_wilson_offaxis[_result]) as the
// reference's wilson_result list.
template <class MT>
std::vector<wilson_result> offaxis(const std::array<int, 4> &dims, const MT *links,
                                   const std::vector<std::vector<int>> *directions,
                                   double r_min, double r_max, int time_min, int time_max,
                                   bool adjoint) {
  Session<MT> s(dims, links);
  std::vector<int> flat;
  if (directions)
    for (const auto &d : *directions) {
      if (d.size() != 3)
        throw std::runtime_error("general_code_b200 wilson_offaxis: directions need 3 ints");
      flat.insert(flat.end(), d.begin(), d.end());
    }
  std::vector<gc_wilson_result> out(4096);
  int count = 0;
  for (int attempt = 0; attempt < 2; attempt++) {
    const int rc =
        directions ? gc_wilson_offaxis(s.get(), flat.data(), (int)directions->size(), r_min,
                                       r_max, time_min, time_max, adjoint ? 1 : 0, out.data(),
                                       (int)out.size(), &count)
                   : gc_wilson_offaxis_result(s.get(), r_min, r_max, time_min, time_max,
                                              adjoint ? 1 : 0, out.data(), (int)out.size(),
                                              &count);
    if (rc == GC_ERR_ARG && count > (int)out.size()) {
      out.resize(count);
      continue;
    }
    check(rc, s.get(), "wilson_offaxis");
    break;
  }
  std::vector<wilson_result> res(count);
  for (int i = 0; i < count; i++) {
    res[i].wilson_loop = out[i].wilson_loop;
    res[i].time_size = out[i].time_size;
    res[i].space_size = out[i].space_size;
    res[i].statistics_size = out[i].statistics_size;
  }
  return res;
}

// The merged entries keyed (T, size), later entries replacing earlier ones
// (as the reference builds its map).
inline std::map<std::tuple<int, double>, double>
offaxis_map(const std::vector<wilson_result> &entries) {
  std::map<std::tuple<int, double>, double> m;
  for (const auto &e : entries)
    m[std::tuple<int, double>(e.time_size, e.space_size)] = e.wilson_loop;
  return m;
}

template <class MT>
std::map<std::tuple<int, int, int>, double>
spatial(const Data::LatticeData<DataPatternLexicographical, MT> &conf, int r_min, int r_max,
        int time_min, int time_max, double alpha, int smearing_start, int smearing_end,
        int smearing_step) {
  Session<MT> s(conf.lat_dim, conf.array.data());
  std::vector<gc_wilson_spatial_result> out(4096);
  int count = 0;
  for (int attempt = 0; attempt < 2; attempt++) {
    const int rc = gc_wilson_spatial_3d(s.get(), r_min, r_max, time_min, time_max, alpha,
                                        smearing_start, smearing_end, smearing_step,
                                        out.data(), (int)out.size(), &count);
    if (rc == GC_ERR_ARG && count > (int)out.size()) {
      out.resize(count);
      continue;
    }
    check(rc, s.get(), "wilson_spatial_3d_indexed");
    break;
  }
  std::map<std::tuple<int, int, int>, double> m;
  for (int i = 0; i < count; i++)
    m[std::tuple<int, int, int>(out[i].smearing, out[i].time_size, out[i].space_size)] =
        out[i].wilson_loop;
  return m;
}

template <class MT>
double polyakov(const Data::LatticeData<DataPatternLexicographical, MT> &conf) {
  Session<MT> s(conf.lat_dim, conf.array.data());
  double p = 0;
  check(gc_polyakov_loop(s.get(), &p), s.get(), "polyakov_loop");
  return p;
}

template <class MT>
std::vector<double> polyakov_correlator(const Data::LatticeData<DataPatternLexicographical, MT> &conf,
                                        int D_max, int kind) {
  Session<MT> s(conf.lat_dim, conf.array.data());
  const size_t n = (size_t)(2 * D_max + 1) * (2 * D_max + 1) * (2 * D_max + 1);
  std::vector<double> out(n);
  check(gc_polyakov_correlator(s.get(), D_max, kind, out.data()), s.get(),
        kind == GC_POLYAKOV_SINGLET ? "polyakov_loop_correlator_singlet"
                                    : "polyakov_loop_correlator_color_average");
  return out;
}

} // namespace gc_dropin

// ---------------------------------------------------------------- overloads
inline void smearing_APE(Data::LatticeData<DataPatternLexicographical, su2> &conf,
                         double alpha) {
  gc_dropin::ape(conf, alpha);
}
inline void smearing_APE(Data::LatticeData<DataPatternLexicographical, su3> &conf,
                         double alpha) {
  gc_dropin::ape(conf, alpha);
}
inline void smearing_HYP(Data::LatticeData<DataPatternLexicographical, su2> &conf,
                         double alpha1, double alpha2, double alpha3) {
  gc_dropin::hyp(conf, alpha1, alpha2, alpha3);
}
inline void smearing_HYP(Data::LatticeData<DataPatternLexicographical, su3> &conf,
                         double alpha1, double alpha2, double alpha3) {
  gc_dropin::hyp(conf, alpha1, alpha2, alpha3);
}
inline std::map<std::tuple<int, int>, double>
wilson_loop(const Data::LatticeData<DataPatternLexicographical, su2> &conf,
            int r_min, int r_max, int time_min, int time_max) {
  return gc_dropin::wilson(conf.lat_dim, conf.array.data(), r_min, r_max,
                           time_min, time_max);
}
inline std::map<std::tuple<int, int>, double>
wilson_loop(const Data::LatticeData<DataPatternLexicographical, su3> &conf,
            int r_min, int r_max, int time_min, int time_max) {
  return gc_dropin::wilson(conf.lat_dim, conf.array.data(), r_min, r_max,
                           time_min, time_max);
}
// Adjoint representation (wilson_loops.h:1173-1200).
inline std::map<std::tuple<int, int>, double>
wilson_loop_adjoint(const Data::LatticeData<DataPatternLexicographical, su2> &conf,
                    int r_min, int r_max, int time_min, int time_max) {
  return gc_dropin::wilson(conf.lat_dim, conf.array.data(), r_min, r_max,
                           time_min, time_max, true);
}
inline std::map<std::tuple<int, int>, double>
wilson_loop_adjoint(const Data::LatticeData<DataPatternLexicographical, su3> &conf,
                    int r_min, int r_max, int time_min, int time_max) {
  return gc_dropin::wilson(conf.lat_dim, conf.array.data(), r_min, r_max,
                           time_min, time_max, true);
}
// Legacy vector form (basic_observables.h:108-111). The reference reads the
// lattice size from the globals x_size, y_size, z_size, t_size
// (indexing.h:8-11), which the calling program must set; so does this one.
inline std::map<std::tuple<int, int>, double>
wilson_loop(const std::vector<su2> &conf, int r_min, int r_max, int time_min,
            int time_max) {
  return gc_dropin::wilson(std::array<int, 4>{x_size, y_size, z_size, t_size},
                           conf.data(), r_min, r_max, time_min, time_max);
}
inline std::map<std::tuple<int, int>, double>
wilson_loop(const std::vector<su3> &conf, int r_min, int r_max, int time_min,
            int time_max) {
  return gc_dropin::wilson(std::array<int, 4>{x_size, y_size, z_size, t_size},
                           conf.data(), r_min, r_max, time_min, time_max);
}
inline double plaket(const Data::LatticeData<DataPatternLexicographical, su2> &conf) {
  return gc_dropin::plaquette(conf);
}
inline double plaket(const Data::LatticeData<DataPatternLexicographical, su3> &conf) {
  return gc_dropin::plaquette(conf);
}
inline double plaket_time(const Data::LatticeData<DataPatternLexicographical, su2> &conf) {
  return gc_dropin::plaquette(conf, 1);
}
inline double plaket_time(const Data::LatticeData<DataPatternLexicographical, su3> &conf) {
  return gc_dropin::plaquette(conf, 1);
}
inline double plaket_space(const Data::LatticeData<DataPatternLexicographical, su2> &conf) {
  return gc_dropin::plaquette(conf, 2);
}
inline double plaket_space(const Data::LatticeData<DataPatternLexicographical, su3> &conf) {
  return gc_dropin::plaquette(conf, 2);
}
// Two-configuration loops (wilson_loops.h:1202-1266), as
// apps/smearing/smearing_wilson_gevp.cpp:200-203 calls them.
inline std::map<std::tuple<int, int>, double>
wilson_gevp_indexed(const Data::LatticeData<DataPatternLexicographical, su2> &conf1,
                    const Data::LatticeData<DataPatternLexicographical, su2> &conf2, int r_min,
                    int r_max, int time_min, int time_max) {
  return gc_dropin::gevp(conf1, conf2, r_min, r_max, time_min, time_max, false);
}
inline std::map<std::tuple<int, int>, double>
wilson_gevp_indexed(const Data::LatticeData<DataPatternLexicographical, su3> &conf1,
                    const Data::LatticeData<DataPatternLexicographical, su3> &conf2, int r_min,
                    int r_max, int time_min, int time_max) {
  return gc_dropin::gevp(conf1, conf2, r_min, r_max, time_min, time_max, false);
}
inline std::map<std::tuple<int, int>, double>
wilson_gevp_adjoint_indexed(const Data::LatticeData<DataPatternLexicographical, su2> &conf1,
                            const Data::LatticeData<DataPatternLexicographical, su2> &conf2,
                            int r_min, int r_max, int time_min, int time_max) {
  return gc_dropin::gevp(conf1, conf2, r_min, r_max, time_min, time_max, true);
}
inline std::map<std::tuple<int, int>, double>
wilson_gevp_adjoint_indexed(const Data::LatticeData<DataPatternLexicographical, su3> &conf1,
                            const Data::LatticeData<DataPatternLexicographical, su3> &conf2,
                            int r_min, int r_max, int time_min, int time_max) {
  return gc_dropin::gevp(conf1, conf2, r_min, r_max, time_min, time_max, true);
}
// Polyakov loops (polyakov_loops.h:24-41, 83-206); with polyakov_loops.h
// included before this header, as apps/smearing/smearing.cpp:5 does.
inline double polyakov_loop(const Data::LatticeData<DataPatternLexicographical, su2> &conf) {
  return gc_dropin::polyakov(conf);
}
inline double polyakov_loop(const Data::LatticeData<DataPatternLexicographical, su3> &conf) {
  return gc_dropin::polyakov(conf);
}
inline std::vector<double>
polyakov_loop_correlator_singlet(const Data::LatticeData<DataPatternLexicographical, su2> &conf,
                                 int D_max) {
  return gc_dropin::polyakov_correlator(conf, D_max, GC_POLYAKOV_SINGLET);
}
inline std::vector<double>
polyakov_loop_correlator_singlet(const Data::LatticeData<DataPatternLexicographical, su3> &conf,
                                 int D_max) {
  return gc_dropin::polyakov_correlator(conf, D_max, GC_POLYAKOV_SINGLET);
}
inline std::vector<double> polyakov_loop_correlator_color_average(
    const Data::LatticeData<DataPatternLexicographical, su2> &conf, int D_max) {
  return gc_dropin::polyakov_correlator(conf, D_max, GC_POLYAKOV_COLOR_AVERAGE);
}
inline std::vector<double> polyakov_loop_correlator_color_average(
    const Data::LatticeData<DataPatternLexicographical, su3> &conf, int D_max) {
  return gc_dropin::polyakov_correlator(conf, D_max, GC_POLYAKOV_COLOR_AVERAGE);
}
// Off-axis loops (wilson_loops.h:313-663), and the legacy vector form of the
// merged results that apps/observables/wilson_loops/wilson_loops.cpp:135-140
// calls (basic_observables.h:34-36, 45-48; lattice size from the globals
// x_size, y_size, z_size, t_size, which the program must set).
#define GC_DROPIN_OFFAXIS(MT)                                                                  \
  inline std::vector<wilson_result> wilson_offaxis(                                            \
      const Data::LatticeData<DataPatternLexicographical, MT> &conf,                           \
      const std::vector<std::vector<int>> directions, double r_min, double r_max,              \
      int time_min, int time_max) {                                                            \
    return gc_dropin::offaxis(conf.lat_dim, conf.array.data(), &directions, r_min, r_max,      \
                              time_min, time_max, false);                                      \
  }                                                                                            \
  inline std::vector<wilson_result> wilson_offaxis_adjoint(                                    \
      const Data::LatticeData<DataPatternLexicographical, MT> &conf,                           \
      const std::vector<std::vector<int>> directions, double r_min, double r_max,              \
      int time_min, int time_max) {                                                            \
    return gc_dropin::offaxis(conf.lat_dim, conf.array.data(), &directions, r_min, r_max,      \
                              time_min, time_max, true);                                       \
  }                                                                                            \
  inline std::map<std::tuple<int, double>, double> wilson_offaxis_result(                      \
      const Data::LatticeData<DataPatternLexicographical, MT> &conf, double r_min,             \
      double r_max, int time_min, int time_max) {                                              \
    return gc_dropin::offaxis_map(gc_dropin::offaxis(conf.lat_dim, conf.array.data(),          \
                                                     nullptr, r_min, r_max, time_min,          \
                                                     time_max, false));                        \
  }                                                                                            \
  inline std::map<std::tuple<int, double>, double> wilson_offaxis_adjoint_result(              \
      const Data::LatticeData<DataPatternLexicographical, MT> &conf, double r_min,             \
      double r_max, int time_min, int time_max) {                                              \
    return gc_dropin::offaxis_map(gc_dropin::offaxis(conf.lat_dim, conf.array.data(),          \
                                                     nullptr, r_min, r_max, time_min,          \
                                                     time_max, true));                         \
  }                                                                                            \
  inline std::map<std::tuple<int, double>, double> wilson_offaxis_result(                      \
      const std::vector<MT> &array, double r_min, double r_max, int time_min, int time_max) {  \
    return gc_dropin::offaxis_map(gc_dropin::offaxis(                                          \
        std::array<int, 4>{x_size, y_size, z_size, t_size}, array.data(), nullptr, r_min,      \
        r_max, time_min, time_max, false));                                                    \
  }                                                                                            \
  inline std::map<std::tuple<int, double>, double> wilson_offaxis_adjoint_result(              \
      const std::vector<MT> &array, double r_min, double r_max, int time_min, int time_max) {  \
    return gc_dropin::offaxis_map(gc_dropin::offaxis(                                          \
        std::array<int, 4>{x_size, y_size, z_size, t_size}, array.data(), nullptr, r_min,      \
        r_max, time_min, time_max, true));                                                     \
  }
GC_DROPIN_OFFAXIS(su2)
GC_DROPIN_OFFAXIS(su3)
#undef GC_DROPIN_OFFAXIS

// Spatial Wilson loops with two-dimensional APE smearing
// (wilson_loops.h:1384-1428), as apps/observables/wilson_loops_spatial calls
// them (wilson_loops_spatial.cpp:117-119).
#define GC_DROPIN_SPATIAL(MT)                                                                  \
  inline std::map<std::tuple<int, int, int>, double> wilson_spatial_3d_indexed(                \
      const Data::LatticeData<DataPatternLexicographical, MT> &conf, int r_min, int r_max,     \
      int time_min, int time_max, double alpha, int smearing_start, int smearing_end,          \
      int smearing_step) {                                                                     \
    return gc_dropin::spatial(conf, r_min, r_max, time_min, time_max, alpha, smearing_start,   \
                              smearing_end, smearing_step);                                    \
  }
GC_DROPIN_SPATIAL(su2)
GC_DROPIN_SPATIAL(su3)
#undef GC_DROPIN_SPATIAL

// Configuration reader (data.h:265-338), as apps/smearing/smearing.cpp:188
// calls it (qualified, Data::read_data_convert).
namespace Data {
inline void read_data_convert(LatticeData<DataPatternLexicographical, su2> &conf,
                              std::string file_path, std::string conf_format, int bytes_skip,
                              std::string file_precision, bool convert) {
  gc_dropin::read(conf, file_path, conf_format, bytes_skip, file_precision, convert);
}
inline void read_data_convert(LatticeData<DataPatternLexicographical, su3> &conf,
                              std::string file_path, std::string conf_format, int bytes_skip,
                              std::string file_precision, bool convert) {
  gc_dropin::read(conf, file_path, conf_format, bytes_skip, file_precision, convert);
}
} // namespace Data
