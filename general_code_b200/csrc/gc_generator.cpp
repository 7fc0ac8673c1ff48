// Seeded synthetic gauge configurations (host side, multithreaded).
//
//   SU(2): a_k ~ N(0,1), theta = eps*|a|, U = (cos theta, sin theta a/|a|),
//          normalised to a unit quaternion.
//   SU(3): H = eps * sum_a c_a lambda_a (Gell-Mann matrices in the order of
//          the reference's get_generators_su3, matrix.h:987-1046), c_a ~
//          N(0,1); U = exp(iH) by Taylor series with scaling and squaring
//          (Moler & Van Loan, "Nineteen dubious ways...", 2003, method 3),
//          then Gram-Schmidt reunitarisation.
//   Gauge: g(x) Haar random (SU(2): normalised 4-Gaussian; SU(3): Gram-Schmidt
//          of two complex Gaussian rows, third row = conj(row0 x row1)),
//          U_mu(x) <- g(x) U_mu(x) g(x+mu)^dag.
// Random numbers: Philox-4x32-10 with key (seed, config_index); links use
// stream 0 and item = link index 4*site+mu, the gauge field stream 1 and
// item = site. Output: host array, link index 4*site+mu, row-major layout.
#include "gc_algebra.cuh"
#include "gc_philox.h"

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace gc {

namespace {

SU3<double> su3_exp_i(const double c[8], double eps) {
  const double s3 = 1.0 / std::sqrt(3.0);
  // H (Hermitian, traceless)
  cx<double> H[3][3];
  H[0][0] = {eps * (c[2] + c[7] * s3), 0};
  H[1][1] = {eps * (-c[2] + c[7] * s3), 0};
  H[2][2] = {eps * (-2.0 * c[7] * s3), 0};
  H[0][1] = {eps * c[0], -eps * c[1]};
  H[1][0] = {eps * c[0], eps * c[1]};
  H[0][2] = {eps * c[3], -eps * c[4]};
  H[2][0] = {eps * c[3], eps * c[4]};
  H[1][2] = {eps * c[5], -eps * c[6]};
  H[2][1] = {eps * c[5], eps * c[6]};
  // X = i H
  SU3<double> X;
  double nrm = 0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      X.e[i][j] = {-H[i][j].im, H[i][j].re};
      nrm += H[i][j].re * H[i][j].re + H[i][j].im * H[i][j].im;
    }
  nrm = std::sqrt(nrm);
  int sq = 0;
  while (nrm > 0.125) {
    nrm *= 0.5;
    sq++;
  }
  X = scale(X, std::ldexp(1.0, -sq));
  // Horner: E = I + X(I + X/2(I + X/3(... (I + X/n))))
  const int order = 16;
  SU3<double> I = unit(SU3<double>());
  SU3<double> E = I;
  for (int k = order; k >= 1; k--)
    E = add(I, scale(mul(X, E), 1.0 / k));
  for (int k = 0; k < sq; k++)
    E = mul(E, E);
  return reunitarize_gs(E);
}

SU3<double> haar_su3(NormalStream &ns) {
  SU3<double> A;
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 3; j++) {
      double re = ns.next();
      double im = ns.next();
      A.e[i][j] = {re, im};
    }
  for (int j = 0; j < 3; j++)
    A.e[2][j] = {0, 0};
  return reunitarize_gs(A);
}

SU2<double> haar_su2(NormalStream &ns) {
  double a[4];
  for (int k = 0; k < 4; k++)
    a[k] = ns.next();
  return proj_div(SU2<double>{a[0], a[1], a[2], a[3]});
}

void store_link(double *out, long long l, const SU3<double> &U) {
  double *p = out + l * 18;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      p[(3 * i + j) * 2] = U.e[i][j].re;
      p[(3 * i + j) * 2 + 1] = U.e[i][j].im;
    }
}
void store_link(double *out, long long l, const SU2<double> &U) {
  double *p = out + l * 4;
  p[0] = U.a0;
  p[1] = U.a1;
  p[2] = U.a2;
  p[3] = U.a3;
}

template <class F> void parallel_for(long long n, F f) {
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0)
    nt = 1;
  nt = std::min<unsigned>(nt, 64);
  if (n < 4096)
    nt = 1;
  std::vector<std::thread> th;
  const long long chunk = (n + nt - 1) / nt;
  for (unsigned t = 0; t < nt; t++) {
    const long long b = t * chunk, e = std::min<long long>(n, b + chunk);
    if (b >= e)
      break;
    th.emplace_back([=]() {
      for (long long i = b; i < e; i++)
        f(i);
    });
  }
  for (auto &t : th)
    t.join();
}

int neighbour(const int dims[4], int site, int mu) {
  int x[4];
  int r = site;
  for (int d = 0; d < 4; d++) {
    x[d] = r % dims[d];
    r /= dims[d];
  }
  x[mu] = (x[mu] + 1) % dims[mu];
  return x[0] + dims[0] * (x[1] + dims[1] * (x[2] + dims[2] * x[3]));
}

} // namespace

int generate_host(const int dims[4], int nc, double eps, unsigned seed,
                  unsigned cfg, int gauge, double *out) {
  const long long V = (long long)dims[0] * dims[1] * dims[2] * dims[3];
  if (nc == 3) {
    std::vector<SU3<double>> g;
    if (gauge) {
      g.resize(V);
      parallel_for(V, [&](long long s) {
        NormalStream ns(seed, cfg, 1, (uint64_t)s);
        g[s] = haar_su3(ns);
      });
    }
    parallel_for(4 * V, [&](long long l) {
      NormalStream ns(seed, cfg, 0, (uint64_t)l);
      double c[8];
      for (int a = 0; a < 8; a++)
        c[a] = ns.next();
      SU3<double> U = su3_exp_i(c, eps);
      if (gauge) {
        const int site = (int)(l >> 2), mu = (int)(l & 3);
        U = mul_ad(mul(g[site], U), g[neighbour(dims, site, mu)]);
        U = reunitarize_gs(U);
      }
      store_link(out, l, U);
    });
  } else {
    std::vector<SU2<double>> g;
    if (gauge) {
      g.resize(V);
      parallel_for(V, [&](long long s) {
        NormalStream ns(seed, cfg, 1, (uint64_t)s);
        g[s] = haar_su2(ns);
      });
    }
    parallel_for(4 * V, [&](long long l) {
      NormalStream ns(seed, cfg, 0, (uint64_t)l);
      double a1 = ns.next(), a2 = ns.next(), a3 = ns.next();
      double n = std::sqrt(a1 * a1 + a2 * a2 + a3 * a3);
      double th = eps * n;
      double sn = (n > 0) ? std::sin(th) / n : 0.0;
      SU2<double> U = proj_div(SU2<double>{std::cos(th), sn * a1, sn * a2, sn * a3});
      if (gauge) {
        const int site = (int)(l >> 2), mu = (int)(l & 3);
        U = proj_div(mul_ad(mul(g[site], U), g[neighbour(dims, site, mu)]));
      }
      store_link(out, l, U);
    });
  }
  return 0;
}

} // namespace gc
