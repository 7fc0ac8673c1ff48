/*
 * CPU restatement of the reference's smear-and-measure path (FP64, plain C).
 *
 * TEST INFRASTRUCTURE ONLY — the checker for tests/, smoke() and the CPU
 * baseline leg of bench.py. The product never calls it.
 *
 * Followed reference code (general_code, lib/cpu):
 *   su2 algebra            include/matrix.h:54-110
 *   su3 algebra, proj      include/matrix.h:256-292, :348-358 (Eigen products)
 *   periodic indexing      include/indexing.h:71-126
 *   smearing_APE           include/smearing.h:115-161
 *   smearing_plane_HYP     include/smearing.h:283-378 (both overloads)
 *   HYP_initialize_vector  include/smearing.h:380-399
 *   make_step1/make_step2  include/smearing.h:401-467
 *   smearing_HYP           include/smearing.h:480-516, make_indices3 src/smearing.cpp:333-350
 *   wilson lines           include/wilson_loops.h:665-717
 *   W(R,T) plane sums      include/wilson_loops.h:719-791
 *   wilson_loop driver     include/wilson_loops.h:1047-1074
 *   plaquette              include/plaket.h:24-42, :83-101 (accumulator zeroed)
 * The operation order of every staple and product is the reference's.
 */
#include "gc_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int L[4];
  long long V;
} geom_t;

static void geom_init(geom_t *g, const int dims[4]) {
  g->V = 1;
  for (int d = 0; d < 4; d++) {
    g->L[d] = dims[d];
    g->V *= dims[d];
  }
}

static void coords(const geom_t *g, long long s, int x[4]) {
  for (int d = 0; d < 4; d++) {
    x[d] = (int)(s % g->L[d]);
    s /= g->L[d];
  }
}

static long long index_of(const geom_t *g, const int x[4]) {
  return x[0] + (long long)g->L[0] * (x[1] + (long long)g->L[1] * (x[2] + (long long)g->L[2] * x[3]));
}

/* Site reached from s by n steps (any sign, any length) in direction mu. */
static long long shift(const geom_t *g, long long s, int mu, int n) {
  int x[4];
  coords(g, s, x);
  int m = (x[mu] + n) % g->L[mu];
  if (m < 0)
    m += g->L[mu];
  x[mu] = m;
  return index_of(g, x);
}

/* ------------------------------------------------------------ su2 */
static void su2_mul(double *c, const double *a, const double *b) {
  double r0 = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  double r1 = a[0] * b[1] + b[0] * a[1] + a[3] * b[2] - a[2] * b[3];
  double r2 = a[0] * b[2] + b[0] * a[2] + a[1] * b[3] - a[3] * b[1];
  double r3 = a[0] * b[3] + b[0] * a[3] + a[2] * b[1] - a[1] * b[2];
  c[0] = r0; c[1] = r1; c[2] = r2; c[3] = r3;
}
static void su2_mul_ad(double *c, const double *a, const double *b) {
  double r0 = a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
  double r1 = -a[0] * b[1] + b[0] * a[1] - a[3] * b[2] + a[2] * b[3];
  double r2 = -a[0] * b[2] + b[0] * a[2] - a[1] * b[3] + a[3] * b[1];
  double r3 = -a[0] * b[3] + b[0] * a[3] - a[2] * b[1] + a[1] * b[2];
  c[0] = r0; c[1] = r1; c[2] = r2; c[3] = r3;
}
static void su2_mul_da(double *c, const double *a, const double *b) {
  double r0 = a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
  double r1 = a[0] * b[1] - b[0] * a[1] - a[3] * b[2] + a[2] * b[3];
  double r2 = a[0] * b[2] - b[0] * a[2] - a[1] * b[3] + a[3] * b[1];
  double r3 = a[0] * b[3] - b[0] * a[3] - a[2] * b[1] + a[1] * b[2];
  c[0] = r0; c[1] = r1; c[2] = r2; c[3] = r3;
}
static void su2_proj(double *a) {
  double rho = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3]);
  for (int k = 0; k < 4; k++)
    a[k] = a[k] / rho;
}
static double su2_conj_tr(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}

/* ------------------------------------------------------------ su3 */
#define RE(m, i, j) (m)[(3 * (i) + (j)) * 2]
#define IM(m, i, j) (m)[(3 * (i) + (j)) * 2 + 1]

static void su3_mul(double *c, const double *a, const double *b) {
  double r[18];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double sr = 0, si = 0;
      for (int k = 0; k < 3; k++) {
        double ar = RE(a, i, k), ai = IM(a, i, k), br = RE(b, k, j), bi = IM(b, k, j);
        sr += ar * br - ai * bi;
        si += ar * bi + ai * br;
      }
      RE(r, i, j) = sr;
      IM(r, i, j) = si;
    }
  memcpy(c, r, sizeof(r));
}
static void su3_adjoint(double *c, const double *a) {
  double r[18];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      RE(r, i, j) = RE(a, j, i);
      IM(r, i, j) = -IM(a, j, i);
    }
  memcpy(c, r, sizeof(r));
}
/* A * B^dag, as Eigen evaluates A * B.adjoint().eval() */
static void su3_mul_ad(double *c, const double *a, const double *b) {
  double bd[18];
  su3_adjoint(bd, b);
  su3_mul(c, a, bd);
}
/* A^dag * B */
static void su3_mul_da(double *c, const double *a, const double *b) {
  double ad[18];
  su3_adjoint(ad, a);
  su3_mul(c, ad, b);
}
static void su3_det(const double *m, double *dr, double *di) {
  /* cofactor expansion along the first column */
#define CM(ar, ai, br, bi, rr, ri) do { rr = (ar) * (br) - (ai) * (bi); ri = (ar) * (bi) + (ai) * (br); } while (0)
  double p1r, p1i, p2r, p2i, c0r, c0i, c1r, c1i, c2r, c2i, tr, ti;
  CM(RE(m, 1, 1), IM(m, 1, 1), RE(m, 2, 2), IM(m, 2, 2), p1r, p1i);
  CM(RE(m, 2, 1), IM(m, 2, 1), RE(m, 1, 2), IM(m, 1, 2), p2r, p2i);
  c0r = p1r - p2r; c0i = p1i - p2i;
  CM(RE(m, 0, 1), IM(m, 0, 1), RE(m, 2, 2), IM(m, 2, 2), p1r, p1i);
  CM(RE(m, 2, 1), IM(m, 2, 1), RE(m, 0, 2), IM(m, 0, 2), p2r, p2i);
  c1r = p1r - p2r; c1i = p1i - p2i;
  CM(RE(m, 0, 1), IM(m, 0, 1), RE(m, 1, 2), IM(m, 1, 2), p1r, p1i);
  CM(RE(m, 1, 1), IM(m, 1, 1), RE(m, 0, 2), IM(m, 0, 2), p2r, p2i);
  c2r = p1r - p2r; c2i = p1i - p2i;
  CM(RE(m, 0, 0), IM(m, 0, 0), c0r, c0i, *dr, *di);
  CM(RE(m, 1, 0), IM(m, 1, 0), c1r, c1i, tr, ti);
  *dr -= tr; *di -= ti;
  CM(RE(m, 2, 0), IM(m, 2, 0), c2r, c2i, tr, ti);
  *dr += tr; *di += ti;
#undef CM
}
/* matrix.h:279-292: 6 x [A = 3/2 M - 1/2 M M^dag M; A = (1 - (det A - 1)/3) A] */
static void su3_proj(double *m) {
  double a[18], h[18], md[18], t[18];
  memcpy(a, m, sizeof(a));
  for (int it = 0; it < 6; it++) {
    su3_adjoint(md, a);
    for (int k = 0; k < 18; k++)
      t[k] = 0.5 * a[k];
    su3_mul(h, t, md);  /* (0.5 M) M^dag */
    su3_mul(h, h, a);   /* ... M */
    for (int k = 0; k < 18; k++)
      a[k] = 1.5 * a[k] - h[k];
    double dr, di;
    su3_det(a, &dr, &di);
    const double third = 1. / 3;
    double cr = 1.0 - third * (dr - 1.0), ci = -third * di;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        double xr = RE(a, i, j), xi = IM(a, i, j);
        RE(a, i, j) = cr * xr - ci * xi;
        IM(a, i, j) = cr * xi + ci * xr;
      }
  }
  memcpy(m, a, sizeof(a));
}
static double su3_conj_tr(const double *a, const double *b) {
  double c[18];
  su3_mul_ad(c, a, b);
  return (RE(c, 0, 0) + RE(c, 1, 1) + RE(c, 2, 2)) / 3;
}
static double su3_tr_real(const double *a) {
  return (RE(a, 0, 0) + RE(a, 1, 1) + RE(a, 2, 2)) / 3.;
}

/* ------------------------------------------------------------ group table */
typedef struct {
  int ds;
  void (*mul)(double *, const double *, const double *);
  void (*mul_ad)(double *, const double *, const double *);
  void (*mul_da)(double *, const double *, const double *);
  void (*proj)(double *);
} group_t;

static const group_t SU2G = {4, su2_mul, su2_mul_ad, su2_mul_da, su2_proj};
static const group_t SU3G = {18, su3_mul, su3_mul_ad, su3_mul_da, su3_proj};

static const group_t *group_of(int nc) {
  return nc == 2 ? &SU2G : (nc == 3 ? &SU3G : NULL);
}

static void axpy(int ds, double *s, double c, const double *a) {
  for (int k = 0; k < ds; k++)
    s[k] += c * a[k];
}

/* staple of smearing_plane_HYP / smearing_APE, added to sum:
 *  sum += ((alpha/div * (Fnu(x) Fmu(x+nu))) ^ Fnu(x+mu))
 *  sum += ((alpha/div * (Fnu(x-nu) % Fmu(x-nu))) * Fnu(x-nu+mu))
 * F*(site) returns the link of a field at a site. */
typedef const double *(*field_fn)(const void *ctx, long long site);

static void add_staples(const group_t *G, const geom_t *g, double *sum,
                        long long x, int mu, int nu, field_fn fmu,
                        const void *cmu, field_fn fnu, const void *cnu,
                        double coef) {
  double st[18], t2[18];
  const int ds = G->ds;
  long long x_pnu = shift(g, x, nu, 1), x_pmu = shift(g, x, mu, 1);
  long long x_mnu = shift(g, x, nu, -1), x_mnu_pmu = shift(g, x_mnu, mu, 1);
  G->mul(st, fnu(cnu, x), fmu(cmu, x_pnu));
  for (int k = 0; k < ds; k++)
    st[k] = coef * st[k];
  G->mul_ad(t2, st, fnu(cnu, x_pmu));
  for (int k = 0; k < ds; k++)
    sum[k] = sum[k] + t2[k];
  G->mul_da(st, fnu(cnu, x_mnu), fmu(cmu, x_mnu));
  for (int k = 0; k < ds; k++)
    st[k] = coef * st[k];
  G->mul(t2, st, fnu(cnu, x_mnu_pmu));
  for (int k = 0; k < ds; k++)
    sum[k] = sum[k] + t2[k];
}

typedef struct {
  const double *links;
  int mu;
  int ds;
} conf_ctx;
static const double *conf_link(const void *c, long long site) {
  const conf_ctx *cc = (const conf_ctx *)c;
  return cc->links + (4 * site + cc->mu) * cc->ds;
}
typedef struct {
  const double *f;
  int ds;
} vec_ctx;
static const double *vec_link(const void *c, long long site) {
  const vec_ctx *vc = (const vec_ctx *)c;
  return vc->f + site * vc->ds;
}

void or_set_threads(int n) {
  if (n > 0)
    omp_set_num_threads(n);
}

int or_proj_all(int nc, long long n, double *links) {
  const group_t *G = group_of(nc);
  if (!G)
    return -1;
#pragma omp parallel for
  for (long long i = 0; i < n; i++)
    G->proj(links + i * G->ds);
  return 0;
}

/* ------------------------------------------------------------ APE */
int or_ape(int nc, const int dims[4], double *links, double alpha, int steps) {
  const group_t *G = group_of(nc);
  if (!G)
    return -1;
  geom_t g;
  geom_init(&g, dims);
  const int ds = G->ds;
  const size_t n = (size_t)(4 * g.V * ds);
  double *sm = (double *)malloc(n * sizeof(double));
  for (int st = 0; st < steps; st++) {
    memcpy(sm, links, n * sizeof(double));
#pragma omp parallel for
    for (long long x = 0; x < g.V; x++) {
      for (int mu = 0; mu < 3; mu++) {
        double S[18];
        const double *u = links + (4 * x + mu) * ds;
        for (int k = 0; k < ds; k++)
          S[k] = (1 - alpha) * u[k];
        for (int nu = 0; nu < 3; nu++) {
          if (nu == mu)
            continue;
          conf_ctx cmu = {links, mu, ds}, cnu = {links, nu, ds};
          add_staples(G, &g, S, x, mu, nu, conf_link, &cmu, conf_link, &cnu,
                      alpha / 4);
        }
        G->proj(S);
        memcpy(sm + (4 * x + mu) * ds, S, ds * sizeof(double));
      }
    }
    memcpy(links, sm, n * sizeof(double));
  }
  free(sm);
  return 0;
}

/* ------------------------------------------------------------ HYP */
/* (1-alpha) * U_mu as a per-site vector (HYP_initialize_vector). */
static double *init_vector(const group_t *G, const geom_t *g, const double *links,
                           int mu, double alpha) {
  const int ds = G->ds;
  double *v = (double *)malloc((size_t)g->V * ds * sizeof(double));
#pragma omp parallel for
  for (long long x = 0; x < g->V; x++)
    for (int k = 0; k < ds; k++)
      v[x * ds + k] = (1 - alpha) * links[(4 * x + mu) * ds + k];
  return v;
}

static void proj_vector(const group_t *G, const geom_t *g, double *v) {
#pragma omp parallel for
  for (long long x = 0; x < g->V; x++)
    G->proj(v + x * G->ds);
}

/* smearing_plane_HYP on two per-site vectors (smearing.h:343-378). */
static void plane_vec(const group_t *G, const geom_t *g, double *sm,
                      const double *fmu, const double *fnu, int mu, int nu,
                      double alpha, double divisor) {
  vec_ctx cmu = {fmu, G->ds}, cnu = {fnu, G->ds};
#pragma omp parallel for
  for (long long x = 0; x < g->V; x++)
    add_staples(G, g, sm + x * G->ds, x, mu, nu, vec_link, &cmu, vec_link, &cnu,
                alpha / divisor);
}

/* Level-1 field Vbar for tuple (mu, a, b): the one staple direction eta < 3
 * not in {mu, a, b} (make_step1, smearing.h:401-425). */
static double *level1(const group_t *G, const geom_t *g, const double *links,
                      int mu, int a, int b, double alpha3) {
  double *v = init_vector(G, g, links, mu, alpha3);
  for (int eta = 0; eta < 3; eta++) {
    if (eta == mu || eta == a || eta == b)
      continue;
    conf_ctx cmu = {links, mu, G->ds}, cnu = {links, eta, G->ds};
#pragma omp parallel for
    for (long long x = 0; x < g->V; x++)
      add_staples(G, g, v + x * G->ds, x, mu, eta, conf_link, &cmu, conf_link,
                  &cnu, alpha3 / 2);
  }
  proj_vector(G, g, v);
  return v;
}

int or_hyp(int nc, const int dims[4], double *links, double a1, double a2,
           double a3, int steps) {
  const group_t *G = group_of(nc);
  if (!G)
    return -1;
  geom_t g;
  geom_init(&g, dims);
  const int ds = G->ds;
  for (int st = 0; st < steps; st++) {
    /* level-1 fields: s1[mu][nu] = (mu; nu, t) for spatial mu != nu,
     * t1[eta] = (t; the two spatial directions other than eta) */
    double *s1[3][3] = {{0}};
    double *t1[3] = {0};
    for (int mu = 0; mu < 3; mu++)
      for (int nu = 0; nu < 3; nu++)
        if (mu != nu)
          s1[mu][nu] = level1(G, &g, links, mu, nu, 3, a3);
    for (int eta = 0; eta < 3; eta++) {
      int a = (eta == 0) ? 1 : 0, b = (eta == 2) ? 1 : 2;
      t1[eta] = level1(G, &g, links, 3, a, b, a3);
    }
    double *sm = init_vector(G, &g, links, 3, a1);
    for (int nu = 0; nu < 3; nu++) {
      double *l20 = init_vector(G, &g, links, 3, a2);
      for (int rho = 0; rho < 3; rho++) {
        if (rho == nu)
          continue;
        plane_vec(G, &g, l20, t1[3 - nu - rho], s1[rho][nu], 3, rho, a2, 4);
      }
      proj_vector(G, &g, l20);
      double *l21 = init_vector(G, &g, links, nu, a2);
      for (int rho = 0; rho < 3; rho++) {
        if (rho == nu)
          continue;
        plane_vec(G, &g, l21, s1[nu][rho], s1[rho][nu], nu, rho, a2, 4);
      }
      proj_vector(G, &g, l21);
      plane_vec(G, &g, sm, l20, l21, 3, nu, a1, 6);
      free(l20);
      free(l21);
    }
    proj_vector(G, &g, sm);
#pragma omp parallel for
    for (long long x = 0; x < g.V; x++)
      memcpy(links + (4 * x + 3) * ds, sm + x * ds, ds * sizeof(double));
    free(sm);
    for (int mu = 0; mu < 3; mu++)
      for (int nu = 0; nu < 3; nu++)
        free(s1[mu][nu]);
    for (int eta = 0; eta < 3; eta++)
      free(t1[eta]);
  }
  return 0;
}

/* ------------------------------------------------------------ Wilson loops */
/* lines[x] <- lines[x] * U_mu(x + length mu)  (wilson_lines_prolong) */
static void prolong(const group_t *G, const geom_t *g, const double *links,
                    double *lines, int length, int mu) {
  const int ds = G->ds;
#pragma omp parallel for
  for (long long x = 0; x < g->V; x++) {
    long long y = shift(g, x, mu, length);
    G->mul(lines + x * ds, lines + x * ds, links + (4 * y + mu) * ds);
  }
}

static double *lines_indexed(const group_t *G, const geom_t *g,
                             const double *links, int length, int mu) {
  const int ds = G->ds;
  double *l = (double *)malloc((size_t)g->V * ds * sizeof(double));
#pragma omp parallel for
  for (long long x = 0; x < g->V; x++)
    memcpy(l + x * ds, links + (4 * x + mu) * ds, ds * sizeof(double));
  for (int i = 1; i < length; i++)
    prolong(G, g, links, l, i, mu);
  return l;
}

/* Value of one loop: L(x) * S_top(x+T) * L(x+R)^dag * S_bot(x)^dag, its
 * real trace / N, or the adjoint |Tr|^2 - 1 (su3 tr_adjoint, matrix.h:258)
 * / 4 (w.s)^2 - 1 (su2 multiply_conj_tr_adjoint, matrix.h:62-65). */
static double loop_value(int nc, int ds, const double *L, const double *stop,
                         const double *L3, const double *sbot, int adjoint) {
  double w[18];
  if (nc == 3) {
    /* (L(x) * S(x+T) * L(x+R)^dag * S(x)^dag).tr_real()  (:781-784) */
    su3_mul(w, L, stop);
    su3_mul_ad(w, w, L3);
    su3_mul_ad(w, w, sbot);
    if (adjoint) {
      double tr = RE(w, 0, 0) + RE(w, 1, 1) + RE(w, 2, 2);
      double ti = IM(w, 0, 0) + IM(w, 1, 1) + IM(w, 2, 2);
      return tr * tr + ti * ti - 1;
    }
    return su3_tr_real(w);
  }
  (void)ds;
  /* generic form (:735-748) */
  su2_mul(w, L, stop);
  su2_mul_ad(w, w, L3);
  double d = su2_conj_tr(w, sbot);
  return adjoint ? 4 * d * d - 1 : d;
}

/* adjoint = 0: wilson_loop (wilson_loops.h:1047-1074, plane sums :719-791);
 * adjoint = 1: wilson_loop_adjoint (:1173-1200, plane sums :793-861).
 * links2 != NULL: wilson_gevp_indexed / wilson_gevp_adjoint_indexed
 * (:1202-1266, plane sums :867-1045): time lines from links, space lines S1
 * from links and S2 from links2, each loop taken as (top S1, bottom S2) and
 * (top S2, bottom S1), the sum divided by 6V. */
static int wilson_impl(int nc, const int dims[4], const double *links, const double *links2,
                       int rmin, int rmax, int tmin, int tmax, double *out, int adjoint) {
  const group_t *G = group_of(nc);
  if (!G || rmin < 1 || tmin < 1 || rmax < rmin || tmax < tmin)
    return -1;
  geom_t g;
  geom_init(&g, dims);
  const int ds = G->ds;
  const int nt = tmax - tmin + 1, nr = rmax - rmin + 1;
  double **tl = (double **)malloc(nt * sizeof(double *));
  tl[0] = lines_indexed(G, &g, links, tmin, 3);
  for (int t = tmin + 1; t <= tmax; t++) {
    tl[t - tmin] = (double *)malloc((size_t)g.V * ds * sizeof(double));
    memcpy(tl[t - tmin], tl[t - tmin - 1], (size_t)g.V * ds * sizeof(double));
    prolong(G, &g, links, tl[t - tmin], t - 1, 3);
  }
  double *sl[3], *sl2[3] = {NULL, NULL, NULL};
  for (int mu = 0; mu < 3; mu++) {
    sl[mu] = lines_indexed(G, &g, links, rmin, mu);
    if (links2)
      sl2[mu] = lines_indexed(G, &g, links2, rmin, mu);
  }
  for (int r = rmin; r <= rmax; r++) {
    for (int t = tmin; t <= tmax; t++) {
      const double *L = tl[t - tmin];
      double result = 0;
#pragma omp parallel for reduction(+ : result)
      for (long long x = 0; x < g.V; x++) {
        long long x2 = shift(&g, x, 3, t);
        for (int nu = 0; nu < 3; nu++) {
          long long x3 = shift(&g, x, nu, r);
          if (!links2) {
            result += loop_value(nc, ds, L + x * ds, sl[nu] + x2 * ds, L + x3 * ds,
                                 sl[nu] + x * ds, adjoint);
          } else {
            result += loop_value(nc, ds, L + x * ds, sl[nu] + x2 * ds, L + x3 * ds,
                                 sl2[nu] + x * ds, adjoint);
            result += loop_value(nc, ds, L + x * ds, sl2[nu] + x2 * ds, L + x3 * ds,
                                 sl[nu] + x * ds, adjoint);
          }
        }
      }
      out[(t - tmin) * nr + (r - rmin)] = result / (g.V * (links2 ? 6 : 3));
    }
    for (int mu = 0; mu < 3; mu++) {
      prolong(G, &g, links, sl[mu], r, mu);
      if (links2)
        prolong(G, &g, links2, sl2[mu], r, mu);
    }
  }
  for (int i = 0; i < nt; i++)
    free(tl[i]);
  free(tl);
  for (int mu = 0; mu < 3; mu++) {
    free(sl[mu]);
    free(sl2[mu]);
  }
  return 0;
}

int or_wilson(int nc, const int dims[4], const double *links, int rmin,
              int rmax, int tmin, int tmax, double *out) {
  return wilson_impl(nc, dims, links, NULL, rmin, rmax, tmin, tmax, out, 0);
}

int or_wilson_adjoint(int nc, const int dims[4], const double *links, int rmin,
                      int rmax, int tmin, int tmax, double *out) {
  return wilson_impl(nc, dims, links, NULL, rmin, rmax, tmin, tmax, out, 1);
}

int or_wilson_gevp(int nc, const int dims[4], const double *links1, const double *links2,
                   int rmin, int rmax, int tmin, int tmax, int adjoint, double *out) {
  if (!links2)
    return -1;
  return wilson_impl(nc, dims, links1, links2, rmin, rmax, tmin, tmax, out, adjoint);
}

/* ------------------------------------------------------------ off-axis loops */
/* wilson_offaxis (wilson_loops.h:313-467) and the _adjoint / _result forms
 * (:470-485, 487-663) with the helpers of basic_observables.cpp:167-186,
 * 543-623, 754-840, restated for host arrays. */

/* generate_directions: a1 >= a2 >= a3, one per slope; returns the count. */
static int offaxis_dirs(int lmax, int (*dirs)[3], int cap) {
  int n = 0;
  for (int a1 = 1; a1 <= lmax; a1++)
    for (int a2 = 0; a2 <= lmax; a2++)
      for (int a3 = 0; a3 <= lmax; a3++) {
        if (!(a1 >= a2 && a2 >= a3))
          continue;
        int fresh = 1;
        for (int i = 0; i < n; i++)
          if (dirs[i][0] * a2 == dirs[i][1] * a1 && dirs[i][0] * a3 == dirs[i][2] * a1)
            fresh = 0;
        if (fresh && n < cap) {
          dirs[n][0] = a1;
          dirs[n][1] = a2;
          dirs[n][2] = a3;
          n++;
        }
      }
  return n;
}

/* make_offaxis_pattern (Bresenham): returns the pattern length. */
static int offaxis_pattern(const int d[3], int *p) {
  int n = 0, e1 = -d[1], e2 = -d[2];
  for (int i = 0; i < d[0]; i++) {
    e1 += 2 * d[1];
    e2 += 2 * d[2];
    if (e1 >= d[0]) {
      p[n++] = 2;
      e1 -= 2 * d[0];
    }
    if (e2 >= d[0]) {
      p[n++] = 3;
      e2 -= 2 * d[0];
    }
    p[n++] = 1;
  }
  return n;
}

static int nzeros(const int d[3]) { return (d[0] == 0) + (d[1] == 0) + (d[2] == 0); }

/* generate_permutations */
static int offaxis_perms(const int d[3], int (*perm)[3]) {
  if (nzeros(d) == 2) {
    const int q[3][3] = {{1, 2, 3}, {2, 1, 3}, {3, 1, 2}};
    memcpy(perm, q, sizeof q);
    return 3;
  }
  int n = 0;
  for (int p1 = 1; p1 <= 3; p1++)
    for (int p2 = 1; p2 <= 3; p2++)
      for (int p3 = 1; p3 <= 3; p3++)
        if (p1 != p2 && p2 != p3 && p3 != p1) {
          perm[n][0] = p1;
          perm[n][1] = p2;
          perm[n][2] = p3;
          n++;
        }
  return n;
}

/* generate_reflections */
static int offaxis_refls(const int d[3], int (*refl)[3]) {
  const int z = nzeros(d);
  if (z == 0) {
    /* the four sign choices of axes 2, 3, then the identity again (the
     * reference's else branch of its one-zero test also runs here) */
    int n = 0;
    for (int r1 = 0; r1 < 2; r1++)
      for (int r2 = 0; r2 < 2; r2++) {
        refl[n][0] = 1;
        refl[n][1] = r1 ? -1 : 1;
        refl[n][2] = r2 ? -1 : 1;
        n++;
      }
    refl[n][0] = refl[n][1] = refl[n][2] = 1;
    return n + 1;
  }
  if (z == 1) {
    int k = 0;
    while (d[k] == 0)
      k++;
    for (int r1 = 0; r1 < 2; r1++) {
      refl[r1][0] = refl[r1][1] = refl[r1][2] = 1;
      refl[r1][k] = r1 ? -1 : 1;
    }
    return 2;
  }
  refl[0][0] = refl[0][1] = refl[0][2] = 1;
  return 1;
}

/* wilson_lines_offaxis: product of the pattern's links from every site
 * (starting from the identity, as wilson_line_offaxis does) */
static void offaxis_lines(const group_t *G, const geom_t *g, const double *links,
                          const int *pat, int n, double *S) {
  const int ds = G->ds;
#pragma omp parallel for
  for (long long x = 0; x < g->V; x++) {
    double A[18];
    memset(A, 0, sizeof A);
    if (ds == 4)
      A[0] = 1;
    else
      A[0] = A[8] = A[16] = 1;
    long long cur = x;
    for (int i = 0; i < n; i++) {
      const int mu = abs(pat[i]) - 1;
      if (pat[i] > 0) {
        G->mul(A, A, links + (4 * cur + mu) * ds);
        cur = shift(g, cur, mu, 1);
      } else {
        cur = shift(g, cur, mu, -1);
        G->mul_ad(A, A, links + (4 * cur + mu) * ds);
      }
    }
    memcpy(S + x * ds, A, ds * sizeof(double));
  }
}

/* calculate_wilson_loop_offaxis[_adjoint]: mean over x of the loop
 * L(x,T) S(x+T) L(x+D,T)^dag S(x)^dag (tr_real or tr_adjoint). */
static double offaxis_loop(int nc, const group_t *G, const geom_t *g, const double *L,
                           int T, const double *S, const int D[3], int adjoint) {
  const int ds = G->ds;
  double result = 0;
#pragma omp parallel for reduction(+ : result)
  for (long long x = 0; x < g->V; x++) {
    long long xT = shift(g, x, 3, T), xD = x;
    for (int i = 0; i < 3; i++)
      xD = shift(g, xD, i, D[i]);
    double w[18];
    G->mul(w, L + x * ds, S + xT * ds);
    G->mul_ad(w, w, L + xD * ds);
    G->mul_ad(w, w, S + x * ds);
    if (nc == 3) {
      if (adjoint) {
        double tr = RE(w, 0, 0) + RE(w, 1, 1) + RE(w, 2, 2);
        double ti = IM(w, 0, 0) + IM(w, 1, 1) + IM(w, 2, 2);
        result += tr * tr + ti * ti - 1;
      } else {
        result += su3_tr_real(w);
      }
    } else {
      result += adjoint ? 4 * w[0] * w[0] - 1 : w[0];
    }
  }
  return result / g->V;
}

/* One entry per (direction, multiplier, T); returns the count (or -1). */
static int offaxis_raw(int nc, const int dims[4], const double *links, const int (*dirs)[3],
                       int ndirs, double rmin, double rmax, int tmin, int tmax, int adjoint,
                       or_wilson_result *out, int cap) {
  const group_t *G = group_of(nc);
  if (!G || tmin < 1 || tmax < tmin)
    return -1;
  geom_t g;
  geom_init(&g, dims);
  const int ds = G->ds, nt = tmax - tmin + 1;
  double **tl = (double **)malloc(nt * sizeof(double *));
  for (int t = tmin; t <= tmax; t++)
    tl[t - tmin] = lines_indexed(G, &g, links, t, 3);
  double *S = (double *)malloc((size_t)g.V * ds * sizeof(double));
  int count = 0;
  for (int di = 0; di < ndirs; di++) {
    const int *d = dirs[di];
    const double len0 = sqrt((double)(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
    int base[64], perm[6][3], refl[5][3];
    const int nb = offaxis_pattern(d, base);
    const int np = offaxis_perms(d, perm), nrf = offaxis_refls(d, refl);
    const int mlo = (int)round(rmin / len0 + 0.5), mhi = (int)round(rmax / len0 - 0.5);
    const int nm = mhi - mlo + 1;
    if (nm <= 0)
      continue;
    /* sums[m][T] over the orientations, in the reference's order */
    double *sums = (double *)calloc((size_t)nm * nt, sizeof(double));
    int stats = 0;
    for (int p = 0; p < np; p++) {
      int pp[64], dp[3];
      for (int i = 0; i < nb; i++)
        pp[i] = perm[p][base[i] - 1];
      for (int k = 0; k < 3; k++)
        dp[perm[p][k] - 1] = d[k];
      for (int r = 0; r < nrf; r++) {
        int pr[64], dr[3];
        for (int i = 0; i < nb; i++)
          pr[i] = pp[i] * refl[r][pp[i] - 1];
        for (int k = 0; k < 3; k++)
          dr[k] = dp[k] * refl[r][k];
        stats++;
        for (int m = mlo; m <= mhi; m++) {
          int *pat = (int *)malloc((size_t)nb * m * sizeof(int)), D[3];
          for (int rep = 0; rep < m; rep++)
            memcpy(pat + rep * nb, pr, nb * sizeof(int));
          for (int k = 0; k < 3; k++)
            D[k] = dr[k] * m;
          offaxis_lines(G, &g, links, pat, nb * m, S);
          free(pat);
          for (int t = tmin; t <= tmax; t++)
            sums[(m - mlo) * nt + (t - tmin)] +=
                offaxis_loop(nc, G, &g, tl[t - tmin], t, S, D, adjoint);
        }
      }
    }
    for (int m = mlo; m <= mhi; m++)
      for (int t = tmin; t <= tmax; t++) {
        if (count < cap) {
          out[count].wilson_loop = sums[(m - mlo) * nt + (t - tmin)] / stats;
          out[count].time_size = t;
          out[count].space_size = len0 * m;
          out[count].statistics_size = stats;
        }
        count++;
      }
    free(sums);
  }
  free(S);
  for (int i = 0; i < nt; i++)
    free(tl[i]);
  free(tl);
  return count;
}

int or_wilson_offaxis(int nc, const int dims[4], const double *links, const int *directions,
                      int ndirections, double r_min, double r_max, int time_min, int time_max,
                      int adjoint, or_wilson_result *out, int capacity) {
  return offaxis_raw(nc, dims, links, (const int(*)[3])directions, ndirections, r_min, r_max,
                     time_min, time_max, adjoint, out, capacity);
}

/* wilson_offaxis_result: length-4 directions, range widened by 0.1, then
 * wilson_offaxis_reduce (step for step, basic_observables.cpp:167-186). */
int or_wilson_offaxis_result(int nc, const int dims[4], const double *links, double r_min,
                             double r_max, int time_min, int time_max, int adjoint,
                             or_wilson_result *out, int capacity) {
  int dirs[128][3];
  const int nd = offaxis_dirs(4, dirs, 128);
  int n = offaxis_raw(nc, dims, links, (const int(*)[3])dirs, nd, r_min - 0.1, r_max + 0.1,
                      time_min, time_max, adjoint, out, capacity);
  if (n < 0 || n > capacity)
    return n;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      if (out[i].space_size == out[j].space_size && out[i].time_size == out[j].time_size &&
          i != j) {
        out[i].wilson_loop = (out[i].wilson_loop * out[i].statistics_size +
                              out[j].wilson_loop * out[j].statistics_size) /
                             (out[i].statistics_size + out[j].statistics_size);
        memmove(out + j, out + j + 1, (size_t)(n - j - 1) * sizeof(or_wilson_result));
        n--;
      }
  return n;
}

/* ------------------------------------------------------------ spatial loops */
/* smearing_APE_2d (smearing.h:223-277) of the single-direction fields f1
 * (axis a) and f2 (axis b), in the reference's operation order. */
static void ape2d(const group_t *G, const geom_t *g, double *f1, double *f2, int a, int b,
                  double alpha) {
  const int ds = G->ds;
  double *o1 = (double *)malloc((size_t)g->V * ds * sizeof(double));
  double *o2 = (double *)malloc((size_t)g->V * ds * sizeof(double));
#pragma omp parallel for
  for (long long x = 0; x < g->V; x++) {
    double A[18], B[18], st[18], t[18], r[18];
    const long long xb = shift(g, x, b, 1), xa = shift(g, x, a, 1);
    G->mul_ad(A, f2 + xa * ds, f1 + xb * ds); /* A = f2(x+a) ^ f1(x+b) */
    G->mul_ad(B, f2 + x * ds, A);             /* B = f2(x) ^ A */
    G->mul(A, f1 + x * ds, A);                /* A = f1(x) * A */
    const long long xmb = shift(g, x, b, -1), xmb_pa = shift(g, xmb, a, 1);
    G->mul_da(st, f2 + xmb * ds, f1 + xmb * ds); /* staple = f2(x-b) % f1(x-b) */
    G->mul(t, st, f2 + xmb_pa * ds);
    for (int k = 0; k < ds; k++)
      r[k] = (1 - alpha) * f1[x * ds + k] + (alpha / 2) * (B[k] + t[k]);
    G->proj(r);
    memcpy(o1 + x * ds, r, ds * sizeof(double));
    const long long xma = shift(g, x, a, -1), xma_pb = shift(g, xma, b, 1);
    G->mul_da(B, f1 + xma * ds, f2 + xma * ds); /* B = f1(x-a) % f2(x-a) */
    G->mul(t, B, f1 + xma_pb * ds);
    for (int k = 0; k < ds; k++)
      r[k] = (1 - alpha) * f2[x * ds + k] + (alpha / 2) * (A[k] + t[k]);
    G->proj(r);
    memcpy(o2 + x * ds, r, ds * sizeof(double));
  }
  memcpy(f1, o1, (size_t)g->V * ds * sizeof(double));
  memcpy(f2, o2, (size_t)g->V * ds * sizeof(double));
  free(o1);
  free(o2);
}

/* smearing_APE_2d applied to the direction fields a, b of a configuration */
int or_ape_plane(int nc, const int dims[4], double *links, int a, int b, double alpha,
                 int steps) {
  const group_t *G = group_of(nc);
  if (!G || a < 0 || a > 3 || b < 0 || b > 3 || a == b)
    return -1;
  geom_t g;
  geom_init(&g, dims);
  const int ds = G->ds;
  double *f1 = (double *)malloc((size_t)g.V * ds * sizeof(double));
  double *f2 = (double *)malloc((size_t)g.V * ds * sizeof(double));
  for (long long x = 0; x < g.V; x++) {
    memcpy(f1 + x * ds, links + (4 * x + a) * ds, ds * sizeof(double));
    memcpy(f2 + x * ds, links + (4 * x + b) * ds, ds * sizeof(double));
  }
  for (int i = 0; i < steps; i++)
    ape2d(G, &g, f1, f2, a, b, alpha);
  for (long long x = 0; x < g.V; x++) {
    memcpy(links + (4 * x + a) * ds, f1 + x * ds, ds * sizeof(double));
    memcpy(links + (4 * x + b) * ds, f2 + x * ds, ds * sizeof(double));
  }
  free(f1);
  free(f2);
  return 0;
}

/* wilson_lines_single_direction_prolong (wilson_loops.h:1268-1287):
 * S(x) <- S(x) F(x + length mu) */
static void sd_prolong(const group_t *G, const geom_t *g, const double *F, double *S,
                       int length, int mu) {
  const int ds = G->ds;
#pragma omp parallel for
  for (long long x = 0; x < g->V; x++)
    G->mul(S + x * ds, S + x * ds, F + shift(g, x, mu, length) * ds);
}

/* wilson_spatial_plane_indexed (wilson_loops.h:1303-1334): mean over x of
 * Re Tr[Q(x) S(x + lm mu) Q(x + ln nu)^dag S(x)^dag] / N */
static double spatial_plane(int nc, const group_t *G, const geom_t *g, const double *Q,
                            const double *S, int mu, int nu, int lm, int ln) {
  const int ds = G->ds;
  double result = 0;
#pragma omp parallel for reduction(+ : result)
  for (long long x = 0; x < g->V; x++) {
    double w[18];
    G->mul(w, Q + x * ds, S + shift(g, x, mu, lm) * ds);
    G->mul_ad(w, w, Q + shift(g, x, nu, ln) * ds);
    result += (nc == 3) ? su3_conj_tr(w, S + x * ds) : su2_conj_tr(w, S + x * ds);
  }
  return result / g->V;
}

/* wilson_spatial_3d_indexed (wilson_loops.h:1384-1428) with its helpers,
 * step for step (space lines start with length time_min, see
 * wilson_lines_single_direction_indexed :1289-1301). Entries (smearing, T, R,
 * W) in (smearing, T, R) order; returns the count or -1. */
int or_wilson_spatial_3d(int nc, const int dims[4], const double *links, int rmin, int rmax,
                         int tmin, int tmax, double alpha, int sm_start, int sm_end,
                         int sm_step, int *out_s, int *out_t, int *out_r, double *out_w,
                         int cap) {
  const group_t *G = group_of(nc);
  if (!G || rmin < 1 || rmax < rmin || tmin < 1 || tmax < tmin || sm_step < 1 || sm_end < 0)
    return -1;
  geom_t g;
  geom_init(&g, dims);
  const int ds = G->ds, nt = tmax - tmin + 1, nr = rmax - rmin + 1;
  int *meas = (int *)malloc((sm_end + 1) * sizeof(int));
  int nm = 0;
  meas[nm++] = 0;
  for (int sm = 1; sm <= sm_end; sm++)
    if ((sm - sm_start) % sm_step == 0 && sm_step >= sm_start)
      meas[nm++] = sm;
  double *acc = (double *)calloc((size_t)nm * nt * nr, sizeof(double)); /* [m][t][r] */
  const size_t fsz = (size_t)g.V * ds * sizeof(double);
  double *F1 = (double *)malloc(fsz), *F2 = (double *)malloc(fsz);
  double *S1 = (double *)malloc(fsz), *S2 = (double *)malloc(fsz);
  const int planes[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int p = 0; p < 3; p++) {
    const int nu = planes[p][0], eta = planes[p][1], mu = 3 - nu - eta;
    for (long long x = 0; x < g.V; x++) {
      memcpy(F1 + x * ds, links + (4 * x + nu) * ds, ds * sizeof(double));
      memcpy(F2 + x * ds, links + (4 * x + eta) * ds, ds * sizeof(double));
    }
    /* quark lines along mu, lengths tmin..tmax */
    double **Q = (double **)malloc(nt * sizeof(double *));
    Q[0] = lines_indexed(G, &g, links, tmin, mu);
    for (int t = tmin + 1; t <= tmax; t++) {
      Q[t - tmin] = (double *)malloc(fsz);
      memcpy(Q[t - tmin], Q[t - tmin - 1], fsz);
      prolong(G, &g, links, Q[t - tmin], t - 1, mu);
    }
    int mi = 0;
    for (int sm = 0; sm <= sm_end; sm++) {
      if (sm > 0)
        ape2d(G, &g, F1, F2, nu, eta, alpha);
      if (mi >= nm || meas[mi] != sm)
        continue;
      memcpy(S1, F1, fsz);
      memcpy(S2, F2, fsz);
      for (int i = 1; i < tmin; i++) {
        sd_prolong(G, &g, F1, S1, tmin, nu);
        sd_prolong(G, &g, F2, S2, tmin, eta);
      }
      for (int r = rmin; r <= rmax; r++) {
        for (int t = tmin; t <= tmax; t++) {
          double *a = acc + ((size_t)mi * nt + (t - tmin)) * nr + (r - rmin);
          *a += spatial_plane(nc, G, &g, Q[t - tmin], S1, mu, nu, t, r);
          *a += spatial_plane(nc, G, &g, Q[t - tmin], S2, mu, eta, t, r);
        }
        sd_prolong(G, &g, F1, S1, r, nu);
        sd_prolong(G, &g, F2, S2, r, eta);
      }
      mi++;
    }
    for (int i = 0; i < nt; i++)
      free(Q[i]);
    free(Q);
  }
  int n = 0;
  for (int m = 0; m < nm; m++)
    for (int t = tmin; t <= tmax; t++)
      for (int r = rmin; r <= rmax; r++) {
        if (n < cap) {
          out_s[n] = meas[m];
          out_t[n] = t;
          out_r[n] = r;
          out_w[n] = acc[((size_t)m * nt + (t - tmin)) * nr + (r - rmin)] / 6;
        }
        n++;
      }
  free(F1);
  free(F2);
  free(S1);
  free(S2);
  free(acc);
  free(meas);
  return n;
}

/* ------------------------------------------------------------ plaquette */
/* which = 0: all six planes / 6 (plaket_site, plaket.h:24-42);
 * 1: (mu, t) planes / 3 (plaket_site_time, :44-61);
 * 2: spatial planes / 3 (plaket_site_space, :63-81). */
static double plaquette_kind(int nc, const int dims[4], const double *links, int which) {
  const group_t *G = group_of(nc);
  if (!G)
    return 0;
  geom_t g;
  geom_init(&g, dims);
  const int ds = G->ds;
  double sum = 0;
#pragma omp parallel for reduction(+ : sum)
  for (long long x = 0; x < g.V; x++) {
    double p = 0, a[18];
    for (int mu = 0; mu < 3; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        if ((which == 1 && nu != 3) || (which == 2 && nu == 3))
          continue;
        long long xm = shift(&g, x, mu, 1), xn = shift(&g, x, nu, 1);
        G->mul(a, links + (4 * x + mu) * ds, links + (4 * xm + nu) * ds);
        G->mul_ad(a, a, links + (4 * xn + mu) * ds);
        p += (nc == 3) ? su3_conj_tr(a, links + (4 * x + nu) * ds)
                       : su2_conj_tr(a, links + (4 * x + nu) * ds);
      }
    sum += p / (which == 0 ? 6 : 3);
  }
  return sum / g.V;
}

double or_plaquette_time(int nc, const int dims[4], const double *links) {
  return plaquette_kind(nc, dims, links, 1);
}

double or_plaquette_space(int nc, const int dims[4], const double *links) {
  return plaquette_kind(nc, dims, links, 2);
}

/* ------------------------------------------------------------ Polyakov loops */
/* P(s) = U_t(s,0) ... U_t(s,Lt-1) for spatial site s (get_polyakov_loop,
 * polyakov_loops.h:10-22); lines: Vs matrices. */
static double *polyakov_lines(const group_t *G, const geom_t *g, const double *links) {
  const int ds = G->ds;
  const long long Vs = g->V / g->L[3];
  double *P = (double *)malloc((size_t)Vs * ds * sizeof(double));
#pragma omp parallel for
  for (long long s = 0; s < Vs; s++) {
    double *A = P + s * ds;
    memcpy(A, links + (4 * s + 3) * ds, ds * sizeof(double));
    for (int t = 1; t < g->L[3]; t++)
      G->mul(A, A, links + (4 * (s + t * Vs) + 3) * ds);
  }
  return P;
}

/* tr P = Tr P / N (su3 tr(), matrix.h:256; su2 a0): re, im. */
static void norm_trace(int nc, const double *m, double *re, double *im) {
  if (nc == 3) {
    *re = (RE(m, 0, 0) + RE(m, 1, 1) + RE(m, 2, 2)) / 3;
    *im = (IM(m, 0, 0) + IM(m, 1, 1) + IM(m, 2, 2)) / 3;
  } else {
    *re = m[0];
    *im = 0;
  }
}

/* polyakov_loop (polyakov_loops.h:24-41) */
double or_polyakov_loop(int nc, const int dims[4], const double *links) {
  const group_t *G = group_of(nc);
  if (!G)
    return 0;
  geom_t g;
  geom_init(&g, dims);
  const long long Vs = g.V / g.L[3];
  double *P = polyakov_lines(G, &g, links);
  double sum = 0;
  for (long long s = 0; s < Vs; s++) {
    double re, im;
    norm_trace(nc, P + s * G->ds, &re, &im);
    sum += re;
  }
  free(P);
  return sum / Vs;
}

/* polyakov_loop_correlator_color_average (kind 0, polyakov_loops.h:83-145)
 * and polyakov_loop_correlator_singlet (kind 1, :147-206): out has
 * (2 D + 1)^3 entries, zero where the reference visits no offset. */
int or_polyakov_correlator(int nc, const int dims[4], const double *links, int D, int kind,
                           double *out) {
  const group_t *G = group_of(nc);
  if (!G || D < 0)
    return -1;
  geom_t g;
  geom_init(&g, dims);
  const int ds = G->ds;
  const long long Vs = g.V / g.L[3];
  const int n = 2 * D + 1;
  double *P = polyakov_lines(G, &g, links);
  memset(out, 0, (size_t)n * n * n * sizeof(double));
  for (int dz = -D; dz <= D; dz++)
    for (int dy = -D; dy <= D; dy++) {
      const int dx_min = (dy != 0 && dz != 0) ? 0 : -D;
      for (int dx = dx_min; dx <= D; dx++) {
        if (sqrt((double)(dx * dx + dy * dy + dz * dz)) > D)
          continue;
        double acc = 0;
#pragma omp parallel for reduction(+ : acc)
        for (long long s = 0; s < Vs; s++) {
          const int x = (int)(s % g.L[0]), y = (int)((s / g.L[0]) % g.L[1]),
                    z = (int)(s / ((long long)g.L[0] * g.L[1]));
          const int x2 = ((x + dx) % g.L[0] + g.L[0]) % g.L[0];
          const int y2 = ((y + dy) % g.L[1] + g.L[1]) % g.L[1];
          const int z2 = ((z + dz) % g.L[2] + g.L[2]) % g.L[2];
          const long long s2 = x2 + (long long)g.L[0] * (y2 + (long long)g.L[1] * z2);
          const double *a = P + s * ds, *b = P + s2 * ds;
          if (kind == 1) {
            acc += (nc == 3) ? su3_conj_tr(a, b) : su2_conj_tr(a, b);
          } else {
            double pr, pi, qr, qi;
            norm_trace(nc, a, &pr, &pi);
            norm_trace(nc, b, &qr, &qi);
            acc += pr * qr + pi * qi;
          }
        }
        out[(dz + D) * n * n + (dy + D) * n + dx + D] = acc / Vs;
      }
    }
  free(P);
  return 0;
}

double or_plaquette(int nc, const int dims[4], const double *links) {
  const group_t *G = group_of(nc);
  if (!G)
    return 0;
  geom_t g;
  geom_init(&g, dims);
  const int ds = G->ds;
  double sum = 0;
#pragma omp parallel for reduction(+ : sum)
  for (long long x = 0; x < g.V; x++) {
    double p = 0, a[18];
    for (int mu = 0; mu < 3; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        long long xm = shift(&g, x, mu, 1), xn = shift(&g, x, nu, 1);
        G->mul(a, links + (4 * x + mu) * ds, links + (4 * xm + nu) * ds);
        G->mul_ad(a, a, links + (4 * xn + mu) * ds);
        p += (nc == 3) ? su3_conj_tr(a, links + (4 * x + nu) * ds)
                       : su2_conj_tr(a, links + (4 * x + nu) * ds);
      }
    sum += p / 6;
  }
  return sum / g.V;
}
