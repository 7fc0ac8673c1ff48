// Drop-in check (TEST INFRASTRUCTURE ONLY): compiles the reference's own
// headers together with include/gc_dropin.hpp, then runs the sequence of
// apps/smearing/smearing.cpp:186-301 (plaket, HYP, APE, wilson_loop, and
// wilson_loop_adjoint as apps/smearing/smearing_wilson_gevp.cpp uses it) twice on
// the same seeded configuration:
//   - with unqualified calls, exactly as the app writes them, which overload
//     resolution binds to the drop-in (GPU) functions;
//   - with the reference templates named explicitly (CPU).
// Prints the largest differences and exits 0 when they are within the FP64
// tolerance (links 1e-12, W and plaquette 1e-12 relative + 1e-14). Exits 3
// when the drop-in reports that no GPU is present (it throws; the reference
// templates never throw, so this also shows that the drop-in was called).
//
// Usage: dropin_check <nc 2|3> <L> <T> <ape_steps> <r_max> <t_max>
#include "data.h"
#include "indexing.h"
#include "matrix.h"
#include "plaket.h"
#include "smearing.h"
#include "wilson_loops.h"

#include "gc_dropin.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>

int x_size, y_size, z_size, t_size, size1, size2;

namespace {

typedef DataPatternLexicographical DP;

template <class MT> double ref_plaquette(const Data::LatticeData<DP, MT> &conf) {
  DP dp(conf.lat_dim);
  double sum = 0;
  for (int t = 0; t < dp.lat_dim[3]; t++)
    for (int z = 0; z < dp.lat_dim[2]; z++)
      for (int y = 0; y < dp.lat_dim[1]; y++)
        for (int x = 0; x < dp.lat_dim[0]; x++) {
          dp.lat_coord = {x, y, z, t};
          sum += plaket_site(conf, dp);
        }
  return sum / dp.get_lattice_size();
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
  double pa, pb;
  std::map<std::tuple<int, int>, double> wa, wb, aa, ab;
  try {
    pa = plaket(a); // drop-in
    smearing_HYP(a, 1, 0.75, 0.6);
    for (int i = 0; i < ape_steps; i++)
      smearing_APE(a, 0.5);
    wa = wilson_loop(a, 1, rmax, 1, tmax);
    aa = wilson_loop_adjoint(a, 1, rmax, 1, tmax);
  } catch (const std::exception &e) {
    std::printf("drop-in raised: %s\n", e.what());
    return 3;
  }
  pb = ref_plaquette(b);
  ::smearing_HYP<DP, MT>(b, 1, 0.75, 0.6);
  for (int i = 0; i < ape_steps; i++)
    ::smearing_APE<DP, MT>(b, 0.5);
  wb = ::wilson_loop<DP, MT>(b, 1, rmax, 1, tmax);
  ab = ::wilson_loop_adjoint<DP, MT>(b, 1, rmax, 1, tmax);
  double dl = 0;
  for (size_t i = 0; i < a.array.size(); i++) {
    std::vector<double> x = a.array[i].get_data(), y = b.array[i].get_data();
    for (int k = 0; k < ds; k++)
      dl = std::fmax(dl, std::fabs(x[k] - y[k]));
  }
  double dw = 0;
  bool ok = dl <= 1e-12 && std::fabs(pa - pb) <= 1e-12 * std::fabs(pb) + 1e-14;
  for (auto &kv : wb) {
    double d = std::fabs(wa.at(kv.first) - kv.second);
    dw = std::fmax(dw, d / (std::fabs(kv.second) + 1e-300));
    ok = ok && d <= 1e-12 * std::fabs(kv.second) + 1e-14;
  }
  for (auto &kv : ab) {
    double d = std::fabs(aa.at(kv.first) - kv.second);
    dw = std::fmax(dw, d / (std::fabs(kv.second) + 1e-300));
    ok = ok && d <= 1e-12 * std::fabs(kv.second) + 1e-14;
  }
  std::printf("links max|diff| %.3e  plaquette diff %.3e  W max rel diff %.3e  "
              "entries %zu  %s\n",
              dl, std::fabs(pa - pb), dw, wb.size(), ok ? "OK" : "MISMATCH");
  return ok ? 0 : 1;
}

} // namespace

int main(int argc, char **argv) {
  if (argc < 7) {
    std::printf("usage: %s nc L T ape_steps r_max t_max\n", argv[0]);
    return 2;
  }
  const int nc = std::atoi(argv[1]), L = std::atoi(argv[2]), T = std::atoi(argv[3]);
  const int n_ape = std::atoi(argv[4]), rmax = std::atoi(argv[5]), tmax = std::atoi(argv[6]);
  std::array<int, 4> dims = {L, L, L, T};
  x_size = y_size = z_size = L;
  t_size = T;
  size1 = L * L;
  size2 = L * L * L;
  return nc == 2 ? run<su2>(dims, n_ape, rmax, tmax) : run<su3>(dims, n_ape, rmax, tmax);
}
