// Drop-in check (TEST INFRASTRUCTURE ONLY): compiles the reference's own
// headers together with include/gc_dropin.hpp, then runs the sequence of
// apps/smearing/smearing.cpp:186-301 (plaket, Polyakov loop and correlators,
// HYP, APE, wilson_loop), and the observables of
// apps/smearing/smearing_wilson_gevp.cpp (wilson_loop_adjoint,
// wilson_gevp_indexed, wilson_gevp_adjoint_indexed of the HYP and HYP+APE
// configurations), plaket_time / plaket_space, the reader, and the merged
// off-axis loops of apps/observables/wilson_loops (wilson_offaxis_result and,
// for su3, wilson_offaxis_adjoint_result) and the spatial loops of
// apps/observables/wilson_loops_spatial (wilson_spatial_3d_indexed), twice on
// the same seeded configuration:
//   - with unqualified calls, exactly as the app writes them, which overload
//     resolution binds to the drop-in (GPU) functions;
//   - with the reference templates named explicitly (CPU).
// Prints the largest differences and exits 0 when they are within the FP64
// tolerance (links 1e-12, W and plaquette 1e-12 relative + 1e-14). Exits 3
// when the drop-in reports that no GPU is present (it throws; the reference
// templates never throw, so this also shows that the drop-in was called).
//
// Usage: dropin_check [--time] <nc 2|3> <L> <T> <ape_steps> <r_max> <t_max>
// (--time: the app's HYP + APE + W job timed through both, see time_app)
#include "data.h"
#include "indexing.h"
#include "matrix.h"
#include "plaket.h"
#include "polyakov_loops.h"
#include "smearing.h"
#include "wilson_loops.h"

#include "gc_dropin.hpp"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <string>
#include <cstdlib>
#include <type_traits>
#include <unistd.h>

int x_size, y_size, z_size, t_size, size1, size2;

namespace {

typedef DataPatternLexicographical DP;

// which: 0 plaket_site, 1 plaket_site_time, 2 plaket_site_space, summed into
// a zeroed accumulator (the reference's plaket / plaket_time / plaket_space
// leave theirs uninitialised, plaket.h:85, 105, 125).
template <class MT> double ref_plaquette(const Data::LatticeData<DP, MT> &conf, int which = 0) {
  DP dp(conf.lat_dim);
  double sum = 0;
  for (int t = 0; t < dp.lat_dim[3]; t++)
    for (int z = 0; z < dp.lat_dim[2]; z++)
      for (int y = 0; y < dp.lat_dim[1]; y++)
        for (int x = 0; x < dp.lat_dim[0]; x++) {
          dp.lat_coord = {x, y, z, t};
          sum += which == 1   ? plaket_site_time(conf, dp)
                 : which == 2 ? plaket_site_space(conf, dp)
                              : plaket_site(conf, dp);
        }
  return sum / dp.get_lattice_size();
}

// polyakov_loop (polyakov_loops.h:24-41) with a zeroed accumulator (the
// reference's is uninitialised).
template <class MT> double ref_polyakov(const Data::LatticeData<DP, MT> &conf) {
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

// The reference's wilson_offaxis[_adjoint]_result (wilson_loops.h:470-485,
// 648-663) with its own steps: the templates are named with explicit
// arguments, so the drop-in overload of wilson_offaxis cannot take over the
// call that the result function would otherwise make by name.
template <class MT>
std::map<std::tuple<int, double>, double>
ref_offaxis_result(const Data::LatticeData<DP, MT> &conf, double r_min, double r_max,
                   int time_min, int time_max, bool adjoint) {
  const std::vector<std::vector<int>> dirs = generate_directions(4);
  std::vector<wilson_result> r;
  if (adjoint) {
    if constexpr (std::is_same<MT, su3>::value)
      r = ::wilson_offaxis_adjoint<DP, MT>(conf, dirs, r_min - 0.1, r_max + 0.1, time_min,
                                           time_max);
  } else {
    r = ::wilson_offaxis<DP, MT>(conf, dirs, r_min - 0.1, r_max + 0.1, time_min, time_max);
  }
  wilson_offaxis_reduce(r);
  std::map<std::tuple<int, double>, double> m;
  for (const auto &e : r)
    m[std::tuple<int, double>(e.time_size, e.space_size)] = e.wilson_loop;
  return m;
}

double max_rel(const std::map<std::tuple<int, int>, double> &a,
               const std::map<std::tuple<int, int>, double> &b, bool *ok) {
  double d = 0;
  for (auto &kv : b) {
    const double e = std::fabs(a.at(kv.first) - kv.second);
    d = std::fmax(d, e / (std::fabs(kv.second) + 1e-300));
    *ok = *ok && e <= 1e-12 * std::fabs(kv.second) + 1e-14;
  }
  return d;
}

double max_abs_vec(const std::vector<double> &a, const std::vector<double> &b, bool *ok) {
  double d = 0;
  for (size_t i = 0; i < b.size(); i++) {
    const double e = std::fabs(a.at(i) - b[i]);
    d = std::fmax(d, e);
    *ok = *ok && e <= 1e-12 * std::fabs(b[i]) + 1e-14;
  }
  *ok = *ok && a.size() == b.size();
  return d;
}

template <class MT>
int run(const std::array<int, 4> &dims, int ape_steps, int rmax, int tmax) {
  const int ds = MT::data_size;
  Data::LatticeData<DP, MT> a(dims), b(dims);
  std::vector<double> host((size_t)4 * dims[0] * dims[1] * dims[2] * dims[3] * ds);
  if (gc_generate_host(dims.data(), ds == 4 ? 2 : 3, ds == 4 ? 0.3 : 0.25,
                       20261203, 0, 1, host.data()) != GC_OK) {
    std::printf("generator failed: %s\n", gc_last_error(nullptr));
    return 1;
  }
  std::vector<double> buf(ds);
  for (size_t i = 0; i < a.array.size(); i++) {
    for (int k = 0; k < ds; k++)
      buf[k] = host[i * ds + k];
    a.array[i] = MT(buf);
    b.array[i] = MT(buf);
  }
  double pa, pb, pta, ptb, psa, psb, la, lb;
  std::map<std::tuple<int, int>, double> wa, wb, aa, ab, ga, gb, gaa, gab;
  std::map<std::tuple<int, double>, double> oa, ob, ooa, oob;
  std::map<std::tuple<int, int, int>, double> sa, sb;
  std::vector<double> csa, csb, cca, ccb;
  const int D = 2;
  Data::LatticeData<DP, MT> ha(dims), hb(dims); // configurations after HYP
  try {
    pa = plaket(a); // drop-in
    smearing_HYP(a, 1, 0.75, 0.6);
    ha.array = a.array;
    la = polyakov_loop(a);
    csa = polyakov_loop_correlator_singlet(a, D);
    cca = polyakov_loop_correlator_color_average(a, D);
    for (int i = 0; i < ape_steps; i++)
      smearing_APE(a, 0.5);
    wa = wilson_loop(a, 1, rmax, 1, tmax);
    aa = wilson_loop_adjoint(a, 1, rmax, 1, tmax);
    ga = wilson_gevp_indexed(a, ha, 1, rmax, 1, tmax);
    gaa = wilson_gevp_adjoint_indexed(a, ha, 1, rmax, 1, tmax);
    oa = wilson_offaxis_result(a, 1, rmax, 1, tmax);
    if (ds == 18)
      ooa = wilson_offaxis_adjoint_result(a, 1, rmax, 1, tmax);
    sa = wilson_spatial_3d_indexed(a, 1, 2, 1, 2, 0.5, 1, 2, 1);
    pta = plaket_time(a);
    psa = plaket_space(a);
  } catch (const std::exception &e) {
    std::printf("drop-in raised: %s\n", e.what());
    return 3;
  }
  pb = ref_plaquette(b);
  ::smearing_HYP<DP, MT>(b, 1, 0.75, 0.6);
  hb.array = b.array;
  // reader: the HYP-smeared links written as the app writes them
  // (smearing.cpp:336-339), read back through the drop-in (qualified call, as
  // smearing.cpp:188) and through the reference's template
  double dread = -1;
  {
    char path[] = "/tmp/gc_dropin_conf_XXXXXX";
    const int fd = mkstemp(path);
    if (fd >= 0) {
      close(fd);
      FilePatternLexicographical<4, MT> fp;
      hb.write_data(std::string(path), fp);
      Data::LatticeData<DP, MT> ra(dims), rb(dims);
      try {
        Data::read_data_convert(ra, std::string(path), "lexicographical", 0, "double", false);
      } catch (const std::exception &e) {
        std::printf("drop-in reader raised: %s\n", e.what());
        std::remove(path);
        return 3;
      }
      Data::read_data_convert<DP>(rb, std::string(path), "lexicographical", 0, "double", false);
      std::remove(path);
      dread = 0;
      for (size_t i = 0; i < ra.array.size(); i++) {
        std::vector<double> x = ra.array[i].get_data(), y = rb.array[i].get_data();
        for (size_t k = 0; k < x.size(); k++)
          dread = std::fmax(dread, std::fabs(x[k] - y[k]));
      }
    }
  }
  lb = ref_polyakov(b);
  csb = ::polyakov_loop_correlator_singlet<DP, MT>(b, D);
  ccb = ::polyakov_loop_correlator_color_average<DP, MT>(b, D);
  for (int i = 0; i < ape_steps; i++)
    ::smearing_APE<DP, MT>(b, 0.5);
  wb = ::wilson_loop<DP, MT>(b, 1, rmax, 1, tmax);
  ab = ::wilson_loop_adjoint<DP, MT>(b, 1, rmax, 1, tmax);
  gb = ::wilson_gevp_indexed<DP, MT>(b, hb, 1, rmax, 1, tmax);
  gab = ::wilson_gevp_adjoint_indexed<DP, MT>(b, hb, 1, rmax, 1, tmax);
  ob = ref_offaxis_result(b, 1, rmax, 1, tmax, false);
  if (ds == 18)
    oob = ref_offaxis_result(b, 1, rmax, 1, tmax, true);
  sb = ::wilson_spatial_3d_indexed<DP, MT>(b, 1, 2, 1, 2, 0.5, 1, 2, 1);
  ptb = ref_plaquette(b, 1);
  psb = ref_plaquette(b, 2);
  double dl = 0;
  for (size_t i = 0; i < a.array.size(); i++) {
    std::vector<double> x = a.array[i].get_data(), y = b.array[i].get_data();
    for (int k = 0; k < ds; k++)
      dl = std::fmax(dl, std::fabs(x[k] - y[k]));
  }
  bool ok = dl <= 1e-12 && dread == 0.0;
  for (auto pr : {std::make_pair(pa, pb), std::make_pair(pta, ptb), std::make_pair(psa, psb),
                  std::make_pair(la, lb)})
    ok = ok && std::fabs(pr.first - pr.second) <= 1e-12 * std::fabs(pr.second) + 1e-14;
  double dw = max_rel(wa, wb, &ok);
  dw = std::fmax(dw, max_rel(aa, ab, &ok));
  const double dg = std::fmax(max_rel(ga, gb, &ok), max_rel(gaa, gab, &ok));
  const double dc = std::fmax(max_abs_vec(csa, csb, &ok), max_abs_vec(cca, ccb, &ok));
  double doff = 0;
  for (const auto *pr : {&oa, &ooa}) {
    const auto &got = *pr, &want = (pr == &oa) ? ob : oob;
    ok = ok && got.size() == want.size();
    for (auto &kv : want) {
      auto it = got.find(kv.first);
      if (it == got.end()) {
        ok = false;
        continue;
      }
      const double e = std::fabs(it->second - kv.second);
      doff = std::fmax(doff, e / (std::fabs(kv.second) + 1e-300));
      ok = ok && e <= 1e-12 * std::fabs(kv.second) + 1e-14;
    }
  }
  double dsp = 0;
  ok = ok && sa.size() == sb.size();
  for (auto &kv : sb) {
    auto it = sa.find(kv.first);
    if (it == sa.end()) {
      ok = false;
      continue;
    }
    const double e = std::fabs(it->second - kv.second);
    dsp = std::fmax(dsp, e / (std::fabs(kv.second) + 1e-300));
    ok = ok && e <= 1e-12 * std::fabs(kv.second) + 1e-14;
  }
  std::printf("links max|diff| %.3e  plaquette diff %.3e (time %.3e space %.3e)  W max rel "
              "diff %.3e  GEVP %.3e  Polyakov %.3e, correlators %.3e  reader %.3e  "
              "off-axis %.3e (%zu entries)  spatial %.3e (%zu entries)  entries %zu  %s\n",
              dl, std::fabs(pa - pb), std::fabs(pta - ptb), std::fabs(psa - psb), dw, dg,
              std::fabs(la - lb), dc, dread, doff, ob.size(), dsp, sb.size(), wb.size(),
              ok ? "OK" : "MISMATCH");
  return ok ? 0 : 1;
}

// Timing mode: the job of apps/smearing/smearing.cpp:228-301 as the app runs
// it (HYP once, APE ape_steps times, then the W table), on the same seeded
// configuration, once through the drop-in overloads (unqualified calls: each
// uploads the whole configuration, runs on the GPU and downloads the result,
// as gc_dropin.hpp does for every call) and once through the reference
// templates named explicitly (CPU). Wall-clock seconds of each, one line.
template <class MT>
int time_app(const std::array<int, 4> &dims, int ape_steps, int rmax, int tmax) {
  const int ds = MT::data_size;
  Data::LatticeData<DP, MT> a(dims), b(dims);
  std::vector<double> host((size_t)4 * dims[0] * dims[1] * dims[2] * dims[3] * ds);
  if (gc_generate_host(dims.data(), ds == 4 ? 2 : 3, ds == 4 ? 0.3 : 0.25,
                       20261203, 0, 1, host.data()) != GC_OK) {
    std::printf("generator failed: %s\n", gc_last_error(nullptr));
    return 1;
  }
  std::vector<double> buf(ds);
  for (size_t i = 0; i < a.array.size(); i++) {
    for (int k = 0; k < ds; k++)
      buf[k] = host[i * ds + k];
    a.array[i] = MT(buf);
    b.array[i] = MT(buf);
  }
  using clk = std::chrono::steady_clock;
  std::map<std::tuple<int, int>, double> wa, wb;
  double t_hyp = 0, t_ape = 0, t_w = 0;
  try {
    plaket(a); // first call: CUDA context and library set-up, not timed
    auto t0 = clk::now();
    smearing_HYP(a, 1, 0.75, 0.6);
    auto t1 = clk::now();
    for (int i = 0; i < ape_steps; i++)
      smearing_APE(a, 0.5);
    auto t2 = clk::now();
    wa = wilson_loop(a, 1, rmax, 1, tmax);
    auto t3 = clk::now();
    t_hyp = std::chrono::duration<double>(t1 - t0).count();
    t_ape = std::chrono::duration<double>(t2 - t1).count();
    t_w = std::chrono::duration<double>(t3 - t2).count();
  } catch (const std::exception &e) {
    std::printf("drop-in raised: %s\n", e.what());
    return 3;
  }
  auto r0 = clk::now();
  ::smearing_HYP<DP, MT>(b, 1, 0.75, 0.6);
  auto r1 = clk::now();
  for (int i = 0; i < ape_steps; i++)
    ::smearing_APE<DP, MT>(b, 0.5);
  auto r2 = clk::now();
  wb = ::wilson_loop<DP, MT>(b, 1, rmax, 1, tmax);
  auto r3 = clk::now();
  bool ok = wa.size() == wb.size();
  double dw = 0;
  for (const auto &kv : wb) {
    const double e = std::fabs(wa[kv.first] - kv.second);
    dw = std::fmax(dw, e / std::fabs(kv.second));
    ok = ok && e <= 1e-12 * std::fabs(kv.second) + 1e-14;
  }
  const double bytes = (double)a.array.size() * ds * 8;
  std::printf("{\"dropin_s\": {\"hyp\": %.6f, \"ape_total\": %.6f, \"wilson\": %.6f}, "
              "\"reference_s\": {\"hyp\": %.6f, \"ape_total\": %.6f, \"wilson\": %.6f}, "
              "\"config_bytes\": %.0f, \"calls\": %d, \"w_max_rel_diff\": %.3e, "
              "\"ok\": %s}\n",
              t_hyp, t_ape, t_w, std::chrono::duration<double>(r1 - r0).count(),
              std::chrono::duration<double>(r2 - r1).count(),
              std::chrono::duration<double>(r3 - r2).count(), bytes, ape_steps + 2, dw,
              ok ? "true" : "false");
  return ok ? 0 : 1;
}

} // namespace

int main(int argc, char **argv) {
  bool timing = argc > 1 && std::string(argv[1]) == "--time";
  if (timing) {
    argv++;
    argc--;
  }
  if (argc < 7) {
    std::printf("usage: %s [--time] nc L T ape_steps r_max t_max\n", argv[0]);
    return 2;
  }
  const int nc = std::atoi(argv[1]), L = std::atoi(argv[2]), T = std::atoi(argv[3]);
  const int n_ape = std::atoi(argv[4]), rmax = std::atoi(argv[5]), tmax = std::atoi(argv[6]);
  if (timing) {
    std::array<int, 4> dims = {L, L, L, T};
    x_size = y_size = z_size = L;
    t_size = T;
    size1 = L * L;
    size2 = L * L * L;
    return nc == 2 ? time_app<su2>(dims, n_ape, rmax, tmax)
                   : time_app<su3>(dims, n_ape, rmax, tmax);
  }
  std::array<int, 4> dims = {L, L, L, T};
  x_size = y_size = z_size = L;
  t_size = T;
  size1 = L * L;
  size2 = L * L * L;
  return nc == 2 ? run<su2>(dims, n_ape, rmax, tmax) : run<su3>(dims, n_ape, rmax, tmax);
}
