// APE and HYP smearing kernels (sm_100a).
//
// APE  (reference smearing.h:115-161): thread per (site, spatial mu); reads
//      the current links, writes the smeared spatial links into a second
//      buffer (Jacobi update, no copy: the host swaps the field pointers).
// HYP  (reference smearing.h:305-516, smearing.cpp:333-350): three kernels,
//      one per decoration level, with the reference's staple order:
//        level 1: 9 fields   Vbar_{mu;nu rho}  (one staple direction each,
//                 alpha3/2)  — thread per (site, field)
//        level 2: 6 fields   Vtilde_{t;nu}, Vtilde_{nu;t}  (alpha2/4)
//        level 3: U_t'       (alpha1/6), written to a second temporal buffer.
//      or, as an option, one kernel per time slice that runs the three
//      levels of three consecutive slices (hyp_slices_kernel), with the
//      decorated links in rings of slices that stay in L2.
// The staple sums use the compute type CT (FP64 for the plain form, FP32 for
// the mixed form). The projection: FP64 SU(3) runs the reference's
// Newton-Schulz iteration in FP64; mixed SU(3) runs FP32 steps and a last
// FP64 step (proj_store); SU(2) normalises with |a|^2 and 1/|a| in FP64.
#include "gc_internal.cuh"
#include "gc_kernels.h"
#include "gc_rows01.cuh"

#include <type_traits>

namespace gc {

namespace {

// S += ((c * (Fnu(x) Fmu(x+nu))) Fnu(x+mu)^dag)                  upper staple
//    + ((c * (Fnu(x-nu)^dag Fmu(x-nu))) Fnu(x-nu+mu))             lower staple
// exactly in the operation order of smearing.h:134-149 / :305-318 / :343-356.
// The storage indices of Fnu's and Fmu's links are given separately (they
// differ when the two fields are kept in different slice rings).
template <class Store, class CT, class M>
__device__ __forceinline__ void add_staples2(M &S, const void *fmu, const void *fnu, size_t V,
                                             int nu_x, int mu_pnu, int nu_pmu, int nu_mnu,
                                             int mu_mnu, int nu_mnu_pmu, CT c) {
  M a = mul(Store::template load<CT>(fnu, V, nu_x),
            Store::template load<CT>(fmu, V, mu_pnu));
  S = add(S, mul_ad(scale(a, c), Store::template load<CT>(fnu, V, nu_pmu)));
  M b = mul_da(Store::template load<CT>(fnu, V, nu_mnu),
               Store::template load<CT>(fmu, V, mu_mnu));
  S = add(S, mul(scale(b, c), Store::template load<CT>(fnu, V, nu_mnu_pmu)));
}

template <class Store, class CT, class M>
__device__ __forceinline__ void add_staples(M &S, const void *fmu,
                                            const void *fnu, size_t V, int x,
                                            int x_pnu, int x_pmu, int x_mnu,
                                            int x_mnu_pmu, CT c) {
  add_staples2<Store, CT>(S, fmu, fnu, V, x, x_pnu, x_pmu, x_mnu, x_mnu, x_mnu_pmu, c);
}

// Projection tolerance of the FP64 iteration: an update below it ends the
// iteration early (see proj in gc_algebra.cuh); 1e-14, so the result equals
// the full six-step iteration to rounding. (SU(2) projection is a single
// normalisation and FP32-stored SU(3) uses proj_store's split iteration.)
template <class Store> struct ProjTol {
  static constexpr double value = 1e-14;
};
// HYP's decorated links of the mixed form are kept in FP32 with all 18 reals
// (InterStore): the reference's six-step projection of a level-1 or level-2
// sum need not reach SU(3) (e.g. 0.4 U + 0.3 x staples can be nearly
// singular), and the 12-real form would replace such a matrix's third row.

// FP32-stored SU(3) (the mixed form): Newton-Schulz steps in FP32 while the
// unitarity defect exceeds 2e-5 (at most five), then one FP64 step, whose
// result is stored (ns_until). Other storage: the reference's iteration in
// FP64 with the early exit of proj(A, tol).
template <class Store> struct SplitProj {
  static constexpr bool value = Store::NC == 3 && (Store::kBytes == 48 || Store::kBytes == 72);
};

// NORM (APE): the FP32 iteration starts from S scaled to sum_ij |S_ij|^2 = 3
// (mean squared singular value 1). A Newton-Schulz step and the determinant
// phase fix commute with a positive real factor, so a converging iteration
// ends at the same SU(3) matrix; it gets there in fewer steps (APE sums of a
// smeared field are close to a multiple of a unitary matrix: about one FP32
// step instead of one to two). HYP's level-1 and level-2 sums, which need
// not converge, keep the reference's trajectory (NORM false).
template <class Store, class CT, bool NORM = false, class M>
__device__ __forceinline__ void proj_store(void *out, size_t V, int site,
                                           const M &S) {
  using MD = typename Store::template M<double>;
  if constexpr (SplitProj<Store>::value) {
    using MF = typename Store::template M<float>;
    int n;
    MF a = convert(S, (MF *)nullptr);
    if constexpr (NORM) {
      float f2 = 0.f;
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
          f2 = fmaf(a.e[i][j].re, a.e[i][j].re, f2);
          f2 = fmaf(a.e[i][j].im, a.e[i][j].im, f2);
        }
      if (f2 > 0.f)
        a = scale(a, rsqrtf(f2 * (1.f / 3.f)));
    }
    const MF f = ns_until(a, 2e-5f, 5, &n);
    Store::template store<double>(out, V, site, ns_step(convert(f, (MD *)nullptr)));
  } else if constexpr (Store::NC == 2 && Store::kBytes == 16) {
    // FP32-stored SU(2): a / |a| with |a|^2 and 1/|a| in FP64 (one
    // reciprocal square root instead of a square root and four divisions),
    // each element rounded to FP32 on its own. (1/|a| in FP32 scales all four
    // elements by the same rounding error; over R + T links of a loop that
    // grew W's error against FP64 from 3e-9 to 2e-7 at SU(2) 48^4.)
    const SU2<double> a = convert(S, (SU2<double> *)nullptr);
    const double r = rsqrt(dot4(a.a0, a.a0, a.a1, a.a1, a.a2, a.a2, a.a3, a.a3));
    Store::template store<double>(out, V, site, SU2<double>{a.a0 * r, a.a1 * r, a.a2 * r, a.a3 * r});
  } else {
    MD d = convert(S, (MD *)nullptr);
    Store::template store<double>(out, V, site, proj(d, ProjTol<Store>::value));
  }
}

struct Nbr {
  int pnu, pmu, mnu, mnu_pmu;
};

__device__ __forceinline__ Nbr neighbours(const Geom &g, int site,
                                          const int x[4], int mu, int nu) {
  Nbr n;
  const int dpn = step_off(g, sel4(x, nu), nu, +1);
  const int dmn = step_off(g, sel4(x, nu), nu, -1);
  const int dpm = step_off(g, sel4(x, mu), mu, +1);
  n.pnu = site + dpn;
  n.pmu = site + dpm;
  n.mnu = site + dmn;
  n.mnu_pmu = site + dmn + dpm;
  return n;
}

constexpr int kSmearBlock = 128;

// ---------------------------------------------------- mixed SU(3) staples
// The mixed form stores two rows of an SU(3) link and rebuilds the third as
// conj(row0 x row1); a product of such links is again in SU(3), so a staple
// needs only its first two rows computed, and its third row is rebuilt the
// same way. Rows 0 and 1 of a product take 2/3 of its multiply-adds, and the
// left factor of a product needs no rebuilt row.
// rows 0 and 1 of a stored link (row 2 not set)
__device__ __forceinline__ SU3<float> load_rows01(const void *f, size_t V, int site) {
  const float4 *p = reinterpret_cast<const float4 *>(f) + site;
  const float4 a = __ldg(p), b = __ldg(p + V), c = __ldg(p + 2 * V);
  SU3<float> u;
  u.e[0][0] = {a.x, a.y};
  u.e[0][1] = {a.z, a.w};
  u.e[0][2] = {b.x, b.y};
  u.e[1][0] = {b.z, b.w};
  u.e[1][1] = {c.x, c.y};
  u.e[1][2] = {c.z, c.w};
  return u;
}
// rows 0 and 1 of A B^dag (A: rows 0, 1; B: all rows)
__device__ __forceinline__ SU3<float> mul_ad01(const SU3<float> &A, const SU3<float> &B) {
  SU3<float> C;
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      float re = A.e[i][0].re * B.e[j][0].re;
      float im = A.e[i][0].im * B.e[j][0].re;
      re = fmaf(A.e[i][0].im, B.e[j][0].im, re);
      im = fmaf(-A.e[i][0].re, B.e[j][0].im, im);
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = fmaf(A.e[i][k].re, B.e[j][k].re, re);
        re = fmaf(A.e[i][k].im, B.e[j][k].im, re);
        im = fmaf(A.e[i][k].im, B.e[j][k].re, im);
        im = fmaf(-A.e[i][k].re, B.e[j][k].im, im);
      }
      C.e[i][j] = {re, im};
    }
  return C;
}
// rows 0 and 1 of A^dag B (A, B: all rows)
__device__ __forceinline__ SU3<float> mul_da01(const SU3<float> &A, const SU3<float> &B) {
  SU3<float> C;
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      float re = A.e[0][i].re * B.e[0][j].re;
      float im = A.e[0][i].re * B.e[0][j].im;
      re = fmaf(A.e[0][i].im, B.e[0][j].im, re);
      im = fmaf(-A.e[0][i].im, B.e[0][j].re, im);
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = fmaf(A.e[k][i].re, B.e[k][j].re, re);
        re = fmaf(A.e[k][i].im, B.e[k][j].im, re);
        im = fmaf(A.e[k][i].re, B.e[k][j].im, im);
        im = fmaf(-A.e[k][i].im, B.e[k][j].re, im);
      }
      C.e[i][j] = {re, im};
    }
  return C;
}
// S += c T, T's row 2 rebuilt from its rows 0 and 1
__device__ __forceinline__ void add_staple01(SU3<float> &S, SU3<float> T, float c) {
  rebuild_row2(T);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      S.e[i][j].re = fmaf(c, T.e[i][j].re, S.e[i][j].re);
      S.e[i][j].im = fmaf(c, T.e[i][j].im, S.e[i][j].im);
    }
}

// One (site, mu) of an APE step of the mixed SU(3) form: the reference's
// staples (smearing.h:134-149), each computed in its first two rows; alpha/4
// is applied as each staple is added (the reference scales its first
// product).
__device__ __forceinline__ void ape_site_mixed_su3(const Geom &g, const Fields4 &in,
                                                   const Fields4 &out, double alpha,
                                                   int site, int mu) {
  int x[4];
  site_coords(g, site, x);
  const size_t V = g.V;
  const float c = float(alpha / 4);
  SU3<float> S = scale(StoreF32SU3::load<float>(in.f[mu], V, site), float(1 - alpha));
#pragma unroll 1
  for (int nu = 0; nu < 3; nu++) {
    if (nu == mu)
      continue;
    const Nbr n = neighbours(g, site, x, mu, nu);
    // upper staple Fnu(x) Fmu(x+nu) Fnu(x+mu)^dag
    SU3<float> a = mul01(load_rows01(in.f[nu], V, site),
                         StoreF32SU3::load<float>(in.f[mu], V, n.pnu));
    add_staple01(S, mul_ad01(a, StoreF32SU3::load<float>(in.f[nu], V, n.pmu)), c);
    // lower staple Fnu(x-nu)^dag Fmu(x-nu) Fnu(x-nu+mu)
    a = mul_da01(StoreF32SU3::load<float>(in.f[nu], V, n.mnu),
                 StoreF32SU3::load<float>(in.f[mu], V, n.mnu));
    add_staple01(S, mul01(a, StoreF32SU3::load<float>(in.f[nu], V, n.mnu_pmu)), c);
  }
  proj_store<StoreF32SU3, float, true>(out.f[mu], V, site, S);
}

// One (site, mu) of an APE step (smearing.h:121-155).
template <class Store, class CT>
__device__ __forceinline__ void ape_site(const Geom &g, const Fields4 &in,
                                         const Fields4 &out, double alpha,
                                         int site, int mu) {
  if constexpr (std::is_same<Store, StoreF32SU3>::value) {
    ape_site_mixed_su3(g, in, out, alpha, site, mu);
    return;
  }
  using M = typename Store::template M<CT>;
  int x[4];
  site_coords(g, site, x);
  const size_t V = g.V;
  M S = scale(Store::template load<CT>(in.f[mu], V, site), CT(1 - alpha));
  const CT c = CT(alpha / 4);
#pragma unroll 1
  for (int nu = 0; nu < 3; nu++) {
    if (nu == mu)
      continue;
    Nbr n = neighbours(g, site, x, mu, nu);
    add_staples<Store, CT>(S, in.f[mu], in.f[nu], V, site, n.pnu, n.pmu,
                           n.mnu, n.mnu_pmu, c);
  }
  proj_store<Store, CT, true>(out.f[mu], V, site, S);
}

// Level-1 decorated links. Field index f:
//   0..5 : spatial mu with excluded spatial nu, pairs (0,1),(0,2),(1,0),(1,2),
//          (2,0),(2,1); staple direction eta = 3 - mu - nu
//   6..8 : temporal, staple direction eta = f - 6
__constant__ int kL1Mu[9] = {0, 0, 1, 1, 2, 2, 3, 3, 3};
__constant__ int kL1Eta[9] = {2, 1, 2, 0, 1, 0, 0, 1, 2};

// Where a site's decorated links are kept. The whole-lattice kernels keep a
// field per decoration over all V sites (index = site, plane stride V); the
// slice pipeline keeps them in rings of slices (plane stride VR = 3 Vs):
// index = site + o0 for the site's own slice and site' + o1 for a site' on the
// slice above, in the fields that the next level reads on two slices (level-1
// spatial, level-2 spatial: three ring slots), and site + q0 in the fields
// read on one slice (level-1 and level-2 temporal: two ring slots).
struct DecAddr {
  size_t VR;
  int o0, o1, q0;
};
__device__ __forceinline__ DecAddr whole_lattice(const Geom &g) { return {(size_t)g.V, 0, 0, 0}; }

template <class Store, class CT>
__device__ __forceinline__ void hyp_l1_site(const Geom &g, const Fields4 &U,
                                            const HypL1 &out, double alpha3,
                                            int site, int f, const DecAddr &d) {
  const int oi = site + (f < 6 ? d.o0 : d.q0); // storage index of the result
  if constexpr (std::is_same<Store, StoreF32SU3>::value) {
    // the mixed form's staples of stored (SU(3)) links, in two rows as in
    // ape_site_mixed_su3
    int x[4];
    site_coords(g, site, x);
    const size_t V = g.V;
    const int mu = kL1Mu[f], eta = kL1Eta[f];
    SU3<float> S = scale(StoreF32SU3::load<float>(U.f[mu], V, site), float(1 - alpha3));
    const Nbr n = neighbours(g, site, x, mu, eta);
    const float c = float(alpha3 / 2);
    SU3<float> a = mul01(load_rows01(U.f[eta], V, site),
                         StoreF32SU3::load<float>(U.f[mu], V, n.pnu));
    add_staple01(S, mul_ad01(a, StoreF32SU3::load<float>(U.f[eta], V, n.pmu)), c);
    a = mul_da01(StoreF32SU3::load<float>(U.f[eta], V, n.mnu),
                 StoreF32SU3::load<float>(U.f[mu], V, n.mnu));
    add_staple01(S, mul01(a, StoreF32SU3::load<float>(U.f[eta], V, n.mnu_pmu)), c);
    proj_store<StoreF32SU3Full, float>(out.f[f], d.VR, oi, S);
    return;
  }
  using M = typename Store::template M<CT>;
  int x[4];
  site_coords(g, site, x);
  const size_t V = g.V;
  const int mu = kL1Mu[f], eta = kL1Eta[f];
  M S = scale(Store::template load<CT>(U.f[mu], V, site), CT(1 - alpha3));
  Nbr n = neighbours(g, site, x, mu, eta);
  add_staples<Store, CT>(S, U.f[mu], U.f[eta], V, site, n.pnu, n.pmu, n.mnu,
                         n.mnu_pmu, CT(alpha3 / 2));
  proj_store<typename InterStore<Store>::type, CT>(out.f[f], d.VR, oi, S);
}

// Level-1 field holding Vbar_{mu; nu, t} for spatial mu != nu.
__device__ __forceinline__ int l1_spatial(int mu, int nu) {
  return 2 * mu + (nu > mu ? nu - 1 : nu);
}
// Level-1 field holding Vbar_{t; a, b} (a, b spatial): staple dir 3 - a - b.
__device__ __forceinline__ int l1_temporal(int a, int b) { return 6 + (3 - a - b); }

// Level-2 decorated links. Field index f:
//   0..2 : Vtilde_{t;nu}, nu = f       (smearing.h:433-450)
//   3..5 : Vtilde_{nu;t}, nu = f - 3   (smearing.h:455-466)
// Vtilde_{t;nu} reads level-1 temporal links on the site's slice and level-1
// spatial links on it and on the slice above; Vtilde_{nu;t} reads level-1
// spatial links of the site's slice only.
template <class Store, class CT>
__device__ __forceinline__ void hyp_l2_site(const Geom &g, const Fields4 &U,
                                            const HypL1 &l1, const HypL2 &out,
                                            double alpha2, int site, int f,
                                            const DecAddr &d) {
  using M = typename Store::template M<CT>;
  using I = typename InterStore<Store>::type;
  int x[4];
  site_coords(g, site, x);
  const size_t V = g.V;
  const bool temporal = f < 3;
  const int nu = temporal ? f : f - 3;
  const int mu = temporal ? 3 : nu;
  M S = scale(Store::template load<CT>(U.f[mu], V, site), CT(1 - alpha2));
  const CT c = CT(alpha2 / 4);
  // offsets of the level-1 fields' links: Fmu's on this slice, Fnu's on this
  // slice and (x + mu, x - nu + mu) on the slice above when mu = t
  const int om = temporal ? d.q0 : d.o0;
  const int on1 = temporal ? d.o1 : d.o0;
#pragma unroll 1
  for (int rho = 0; rho < 3; rho++) {
    if (rho == nu)
      continue;
    const void *fmu = temporal ? l1.f[l1_temporal(nu, rho)]
                               : l1.f[l1_spatial(nu, rho)];
    const void *fnu = l1.f[l1_spatial(rho, nu)];
    Nbr n = neighbours(g, site, x, mu, rho);
    add_staples2<I, CT>(S, fmu, fnu, d.VR, site + d.o0, n.pnu + om, n.pmu + on1,
                        n.mnu + d.o0, n.mnu + om, n.mnu_pmu + on1, c);
  }
  proj_store<I, CT>(out.f[f], d.VR, site + (temporal ? d.q0 : d.o0), S);
}

// Level 3: the new temporal link (smearing.h:484-503). Reads the level-2
// temporal links on the site's slice and the level-2 spatial links on it and
// on the slice above.
template <class Store, class CT>
__device__ __forceinline__ void hyp_l3_site(const Geom &g, const void *Ut,
                                            const HypL2 &l2, void *out_t,
                                            double alpha1, int site, const DecAddr &d) {
  using M = typename Store::template M<CT>;
  int x[4];
  site_coords(g, site, x);
  const size_t V = g.V;
  M S = scale(Store::template load<CT>(Ut, V, site), CT(1 - alpha1));
  const CT c = CT(alpha1 / 6);
#pragma unroll 1
  for (int nu = 0; nu < 3; nu++) {
    Nbr n = neighbours(g, site, x, 3, nu);
    add_staples2<typename InterStore<Store>::type, CT>(
        S, l2.f[nu], l2.f[3 + nu], d.VR, site + d.o0, n.pnu + d.q0, n.pmu + d.o1,
        n.mnu + d.o0, n.mnu + d.q0, n.mnu_pmu + d.o1, c);
  }
  proj_store<Store, CT>(out_t, V, site, S);
}

// One APE step of SU(2) at a site, all three spatial links: the staples of
// the three links read 24 distinct links (the three own links, the six
// U_a(x + b) with a != b, each used by two staples, and the backward ones),
// which one thread loads once, against 39 loads for three threads of one
// link each. Per link the staples are added in the order of ape_site, with
// the same operations, so the links are those of ape_site bit for bit.
template <class Store, class CT>
__device__ __forceinline__ void ape_site_su2(const Geom &g, const Fields4 &in,
                                             const Fields4 &out, double alpha, int site) {
  using M = SU2<CT>;
  int x[4];
  site_coords(g, site, x);
  const size_t V = g.V;
  int fwd[3], bwd[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    fwd[d] = site + step_off(g, sel4(x, d), d, +1);
    bwd[d] = site + step_off(g, sel4(x, d), d, -1);
  }
  M own[3], F[3][3]; // F[a][b] = U_a(x + b), a != b
#pragma unroll
  for (int a = 0; a < 3; a++) {
    own[a] = Store::template load<CT>(in.f[a], V, site);
#pragma unroll
    for (int b = 0; b < 3; b++)
      if (a != b)
        F[a][b] = Store::template load<CT>(in.f[a], V, fwd[b]);
  }
  const CT c = CT(alpha / 4);
#pragma unroll
  for (int mu = 0; mu < 3; mu++) {
    M S = scale(own[mu], CT(1 - alpha));
#pragma unroll
    for (int nu = 0; nu < 3; nu++) {
      if (nu == mu)
        continue;
      // x - nu and x - nu + mu (x - nu has x's coordinate along mu)
      const int mnu = bwd[nu];
      const int mnu_pmu = mnu + (fwd[mu] - site);
      // upper: Fnu(x) Fmu(x+nu) Fnu(x+mu)^dag (add_staples' operations)
      const M a = mul(own[nu], F[mu][nu]);
      S = add(S, mul_ad(scale(a, c), F[nu][mu]));
      const M b = mul_da(Store::template load<CT>(in.f[nu], V, mnu),
                         Store::template load<CT>(in.f[mu], V, mnu));
      S = add(S, mul(scale(b, c), Store::template load<CT>(in.f[nu], V, mnu_pmu)));
    }
    proj_store<Store, CT, true>(out.f[mu], V, site, S);
  }
}

// Work items of an APE launch per site: three links (one thread each) for
// SU(3), one thread for all three for SU(2).
template <class Store> constexpr int ape_items() { return Store::NC == 2 ? 1 : 3; }

// Resident blocks of 128 threads per SM that an APE kernel is compiled for:
// 6 (80 registers) in FP32, 4 in FP64. The FP32 kernels wait on the links'
// loads at 4 blocks: SU(2) site kernel at 48^4 0.174 -> 0.163 ms per step
// (0.166 at 8 blocks, where it spills), SU(3) at 32^4 0.248 -> 0.238 ms
// (0.244 at 5 blocks). The FP64 kernels need their 128 registers.
template <class Store, class CT> constexpr int ape_min_blocks() {
  return sizeof(CT) == 4 ? 6 : 4;
}

// ---------------------------------------------------------- single lattice
// The field / direction index varies fastest over blocks, so all fields of
// a block of sites are computed back to back while their inputs are in L2.
template <class Store, class CT>
__global__ void __launch_bounds__(128, ape_min_blocks<Store, CT>())
    ape_kernel(Geom g, const __grid_constant__ Fields4 in,
               const __grid_constant__ Fields4 out, double alpha) {
  if constexpr (Store::NC == 2) {
    const int site = blockIdx.x * blockDim.x + threadIdx.x;
    if (site < g.V)
      ape_site_su2<Store, CT>(g, in, out, alpha, site);
    return;
  }
  const int mu = blockIdx.x % 3;
  const int site = (blockIdx.x / 3) * blockDim.x + threadIdx.x;
  if (site < g.V)
    ape_site<Store, CT>(g, in, out, alpha, site, mu);
}

template <class Store, class CT>
__global__ void __launch_bounds__(128, 4)
    hyp_level1_kernel(Geom g, const __grid_constant__ Fields4 U,
                      const __grid_constant__ HypL1 out, double alpha3) {
  const int f = blockIdx.x % 9;
  const int site = (blockIdx.x / 9) * blockDim.x + threadIdx.x;
  if (site < g.V)
    hyp_l1_site<Store, CT>(g, U, out, alpha3, site, f, whole_lattice(g));
}

template <class Store, class CT>
__global__ void __launch_bounds__(128, 4)
    hyp_level2_kernel(Geom g, const __grid_constant__ Fields4 U,
                      const __grid_constant__ HypL1 l1,
                      const __grid_constant__ HypL2 out, double alpha2) {
  const int f = blockIdx.x % 6;
  const int site = (blockIdx.x / 6) * blockDim.x + threadIdx.x;
  if (site < g.V)
    hyp_l2_site<Store, CT>(g, U, l1, out, alpha2, site, f, whole_lattice(g));
}

template <class Store, class CT>
__global__ void __launch_bounds__(128)
    hyp_level3_kernel(Geom g, const void *Ut, const __grid_constant__ HypL2 l2,
                      void *out_t, double alpha1) {
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  if (site < g.V)
    hyp_l3_site<Store, CT>(g, Ut, l2, out_t, alpha1, site, whole_lattice(g));
}

// ------------------------------------------------------ HYP slice pipeline
// HYP as a pipeline over time slices, with the decorated links in rings of
// slices instead of whole-lattice fields, so that they stay in L2 between the
// level that writes them and the levels that read them. What a slice needs
// lies on it and on the slice above: level 3 of slice k reads level-2
// temporal links of k and level-2 spatial links of k and k + 1; level-2
// temporal of k reads level-1 temporal of k and level-1 spatial of k, k + 1;
// level-2 spatial and level-1 spatial read their own slice; level 1 reads
// the links of its slice and the one above. Launch m computes
//   part 0: level-1 spatial of slice m       part 1: level-1 temporal of m-1
//   part 2: level-2 spatial of slice m - 1   part 3: level-2 temporal of m-2
//   part 4: level 3 of slice m - 3
// for m = 0 .. Lt + 2, each part whose slice is in range. Slices are counted
// without wrapping: slice Lt is slice 0 computed again, for level 3 of slice
// Lt - 1. A spatial level's ring slot is j mod 3 and a temporal level's
// j mod 2: a slot is rewritten three (two) launches after it was written,
// after its last reader, and no part reads what another part of the same
// launch writes. Each site is computed by the same site functions as in the
// level kernels, so the links are the same bit for bit.
struct HypStage {
  int start[6]; // first block of part p (start[5] = blocks of the launch)
  int slice[5]; // slice of part p (unwrapped, 0 .. Lt), -1 if absent
};

template <class Store, class CT>
__global__ void __launch_bounds__(128, 4)
    hyp_slices_kernel(Geom g, const __grid_constant__ Fields4 U,
                      const __grid_constant__ HypL1 l1, const __grid_constant__ HypL2 l2,
                      void *out_t, double a1, double a2, double a3,
                      const __grid_constant__ HypStage st) {
  const int b = blockIdx.x;
  const int p = b < st.start[1] ? 0 : b < st.start[2] ? 1 : b < st.start[3] ? 2
              : b < st.start[4] ? 3 : 4;
  const int nf = p == 0 ? 6 : p == 4 ? 1 : 3;
  const int local = b - st.start[p];
  const int fl = local % nf;
  const int s = (local / nf) * blockDim.x + threadIdx.x;
  if (s >= g.Vs)
    return;
  const int Lt = g.L[3], Vs = g.Vs;
  const int j = st.slice[p];
  const int t = j == Lt ? 0 : j;
  const int t1 = t + 1 == Lt ? 0 : t + 1;
  const int site = s + t * Vs;
  const DecAddr d{3 * (size_t)Vs, (j % 3 - t) * Vs, ((j + 1) % 3 - t1) * Vs, (j % 2 - t) * Vs};
  switch (p) {
  case 0: hyp_l1_site<Store, CT>(g, U, l1, a3, site, fl, d); break;
  case 1: hyp_l1_site<Store, CT>(g, U, l1, a3, site, 6 + fl, d); break;
  case 2: hyp_l2_site<Store, CT>(g, U, l1, l2, a2, site, 3 + fl, d); break;
  case 3: hyp_l2_site<Store, CT>(g, U, l1, l2, a2, site, fl, d); break;
  default: hyp_l3_site<Store, CT>(g, U.f[3], l2, out_t, a1, site, d); break;
  }
}

// ---------------------------------------------------------- many lattices
// One launch covers the blocks of several lattices; a block finds its
// lattice by binary search over the jobs' first block indices.
template <class J, int (*Start)(const J &)>
__device__ __forceinline__ int find_job(const J *jobs, int njobs, int b) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (Start(jobs[mid]) <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ int ape_start(const ApeJob &j) { return j.block_start; }
__device__ __forceinline__ int hyp_start1(const HypJob &j) { return j.start1; }
__device__ __forceinline__ int hyp_start2(const HypJob &j) { return j.start2; }
__device__ __forceinline__ int hyp_start3(const HypJob &j) { return j.start3; }

template <class Store, class CT>
__global__ void __launch_bounds__(128, ape_min_blocks<Store, CT>())
    ape_batch_kernel(const ApeJob *__restrict__ jobs, int njobs) {
  const int j = find_job<ApeJob, ape_start>(jobs, njobs, blockIdx.x);
  const ApeJob &jb = jobs[j];
  const int local = blockIdx.x - jb.block_start;
  if constexpr (Store::NC == 2) {
    const int site = local * blockDim.x + threadIdx.x;
    if (site < jb.g.V)
      ape_site_su2<Store, CT>(jb.g, jb.in, jb.out, jb.alpha, site);
    return;
  }
  const int mu = local % 3;
  const int site = (local / 3) * blockDim.x + threadIdx.x;
  if (site < jb.g.V)
    ape_site<Store, CT>(jb.g, jb.in, jb.out, jb.alpha, site, mu);
}

template <class Store, class CT>
__global__ void __launch_bounds__(128, 4)
    hyp_level1_batch_kernel(const HypJob *__restrict__ jobs, int njobs) {
  const int j = find_job<HypJob, hyp_start1>(jobs, njobs, blockIdx.x);
  const HypJob &jb = jobs[j];
  const int local = blockIdx.x - jb.start1;
  const int site = (local / 9) * blockDim.x + threadIdx.x;
  if (site < jb.g.V)
    hyp_l1_site<Store, CT>(jb.g, jb.U, jb.l1, jb.a3, site, local % 9, whole_lattice(jb.g));
}

template <class Store, class CT>
__global__ void __launch_bounds__(128, 4)
    hyp_level2_batch_kernel(const HypJob *__restrict__ jobs, int njobs) {
  const int j = find_job<HypJob, hyp_start2>(jobs, njobs, blockIdx.x);
  const HypJob &jb = jobs[j];
  const int local = blockIdx.x - jb.start2;
  const int site = (local / 6) * blockDim.x + threadIdx.x;
  if (site < jb.g.V)
    hyp_l2_site<Store, CT>(jb.g, jb.U, jb.l1, jb.l2, jb.a2, site, local % 6,
                           whole_lattice(jb.g));
}

template <class Store, class CT>
__global__ void __launch_bounds__(128)
    hyp_level3_batch_kernel(const HypJob *__restrict__ jobs, int njobs) {
  const int j = find_job<HypJob, hyp_start3>(jobs, njobs, blockIdx.x);
  const HypJob &jb = jobs[j];
  const int site = (blockIdx.x - jb.start3) * blockDim.x + threadIdx.x;
  if (site < jb.g.V)
    hyp_l3_site<Store, CT>(jb.g, jb.U.f[3], jb.l2, jb.out_t, jb.a1, site, whole_lattice(jb.g));
}

// Two-dimensional APE step of two single-direction fields, links along axes
// a (f1) and b (f2), with the staples of the (a, b) plane only
// (smearing_APE_2d, smearing.h:223-277): per site
//   f1'(x) = Proj[(1-alpha) f1(x) + alpha/2 (f2(x) f1(x+b) f2(x+a)^dag
//                                    + f2(x-b)^dag f1(x-b) f2(x-b+a))]
//   f2'(x) = Proj[(1-alpha) f2(x) + alpha/2 (f1(x) f2(x+a) f1(x+b)^dag
//                                    + f1(x-a)^dag f2(x-a) f1(x-a+b))]
template <class Store, class CT>
__global__ void __launch_bounds__(128, 4)
    ape_plane_kernel(const __grid_constant__ Geom g, const void *f1, const void *f2, void *o1,
                     void *o2, int a, int b, double alpha) {
  using M = typename Store::template M<CT>;
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  if (site >= g.V)
    return;
  const size_t V = g.V;
  int x[4];
  site_coords(g, site, x);
  const int pa = site + step_off(g, sel4(x, a), a, +1);
  const int pb = site + step_off(g, sel4(x, b), b, +1);
  const int mb = site + step_off(g, sel4(x, b), b, -1);
  const int ma = site + step_off(g, sel4(x, a), a, -1);
  const int mb_pa = mb + step_off(g, sel4(x, a), a, +1);
  const int ma_pb = ma + step_off(g, sel4(x, b), b, +1);
  const CT c = CT(alpha / 2);
  const M u1 = Store::template load<CT>(f1, V, site), u2 = Store::template load<CT>(f2, V, site);
  // upper staples: A = f2(x+a) f1(x+b)^dag
  const M A = mul_ad(Store::template load<CT>(f2, V, pa), Store::template load<CT>(f1, V, pb));
  M S1 = add(scale(u1, CT(1 - alpha)), scale(mul_ad(u2, A), c));
  M S2 = add(scale(u2, CT(1 - alpha)), scale(mul(u1, A), c));
  // lower staples
  const M l1 = mul_da(Store::template load<CT>(f2, V, mb), Store::template load<CT>(f1, V, mb));
  S1 = add(S1, scale(mul(l1, Store::template load<CT>(f2, V, mb_pa)), c));
  const M l2 = mul_da(Store::template load<CT>(f1, V, ma), Store::template load<CT>(f2, V, ma));
  S2 = add(S2, scale(mul(l2, Store::template load<CT>(f1, V, ma_pb)), c));
  proj_store<Store, CT>(o1, V, site, S1);
  proj_store<Store, CT>(o2, V, site, S2);
}

} // namespace

template <class Store, class CT>
int launch_ape(const Geom &g, const Fields4 &in, const Fields4 &out,
               double alpha, cudaStream_t s) {
  const unsigned nb = (g.V + kSmearBlock - 1) / kSmearBlock;
  ape_kernel<Store, CT><<<nb * ape_items<Store>(), kSmearBlock, 0, s>>>(g, in, out, alpha);
  return launch_check("ape_kernel");
}

template <class Store, class CT>
int launch_hyp(const Geom &g, const Fields4 &U, const HypL1 &l1,
               const HypL2 &l2, void *out_t, double a1, double a2, double a3,
               cudaStream_t s) {
  const int nb = (g.V + kSmearBlock - 1) / kSmearBlock;
  hyp_level1_kernel<Store, CT><<<nb * 9, kSmearBlock, 0, s>>>(g, U, l1, a3);
  int rc = launch_check("hyp_level1_kernel");
  if (rc)
    return rc;
  hyp_level2_kernel<Store, CT><<<nb * 6, kSmearBlock, 0, s>>>(g, U, l1, l2, a2);
  rc = launch_check("hyp_level2_kernel");
  if (rc)
    return rc;
  hyp_level3_kernel<Store, CT><<<nb, kSmearBlock, 0, s>>>(g, U.f[3], l2, out_t, a1);
  return launch_check("hyp_level3_kernel");
}

// Lattices with Lt >= 3 (the rings' 3 Vs sites per field fit in the
// whole-lattice fields' V).
template <class Store, class CT>
int launch_hyp_slices(const Geom &g, const Fields4 &U, const HypL1 &l1, const HypL2 &l2,
                      void *out_t, double a1, double a2, double a3, cudaStream_t s) {
  const int Lt = g.L[3];
  if (Lt < 3)
    return plan_error("hyp_slices_kernel: needs Lt >= 3");
  const int nbs = (g.Vs + kSmearBlock - 1) / kSmearBlock;
  static constexpr int kFields[5] = {6, 3, 3, 3, 1};
  for (int m = 0; m <= Lt + 2; m++) {
    HypStage st;
    const int slice[5] = {m <= Lt ? m : -1, m >= 1 && m <= Lt ? m - 1 : -1,
                          m >= 1 && m <= Lt + 1 ? m - 1 : -1,
                          m >= 2 && m <= Lt + 1 ? m - 2 : -1, m >= 3 ? m - 3 : -1};
    int blocks = 0;
    for (int p = 0; p < 5; p++) {
      st.start[p] = blocks;
      st.slice[p] = slice[p];
      if (slice[p] >= 0)
        blocks += kFields[p] * nbs;
    }
    st.start[5] = blocks;
    hyp_slices_kernel<Store, CT><<<blocks, kSmearBlock, 0, s>>>(g, U, l1, l2, out_t, a1, a2,
                                                                 a3, st);
    const int rc = launch_check("hyp_slices_kernel");
    if (rc)
      return rc;
  }
  return GC_OK;
}

template <class Store, class CT>
int launch_ape_batch(const ApeJob *jobs, int njobs, int blocks, cudaStream_t s) {
  if (njobs <= 0 || blocks <= 0)
    return GC_OK;
  ape_batch_kernel<Store, CT><<<blocks, kSmearBlock, 0, s>>>(jobs, njobs);
  return launch_check("ape_batch_kernel");
}

template <class Store, class CT>
int launch_hyp_batch(const HypJob *jobs, int njobs, const int blocks[3],
                     cudaStream_t s) {
  if (njobs <= 0)
    return GC_OK;
  hyp_level1_batch_kernel<Store, CT><<<blocks[0], kSmearBlock, 0, s>>>(jobs, njobs);
  int rc = launch_check("hyp_level1_batch_kernel");
  if (rc)
    return rc;
  hyp_level2_batch_kernel<Store, CT><<<blocks[1], kSmearBlock, 0, s>>>(jobs, njobs);
  rc = launch_check("hyp_level2_batch_kernel");
  if (rc)
    return rc;
  hyp_level3_batch_kernel<Store, CT><<<blocks[2], kSmearBlock, 0, s>>>(jobs, njobs);
  return launch_check("hyp_level3_batch_kernel");
}

template <class Store, class CT>
int launch_ape_plane(const Geom &g, const void *f1, const void *f2, void *o1, void *o2, int a,
                     int b, double alpha, cudaStream_t s) {
  if (a < 0 || a > 3 || b < 0 || b > 3 || a == b)
    return plan_error("ape_plane_kernel: directions");
  const unsigned nb = (g.V + kSmearBlock - 1) / kSmearBlock;
  ape_plane_kernel<Store, CT><<<nb, kSmearBlock, 0, s>>>(g, f1, f2, o1, o2, a, b, alpha);
  return launch_check("ape_plane_kernel");
}

#define GC_INSTANTIATE_SMEAR(STORE, CT)                                        \
  template int launch_ape_plane<STORE, CT>(const Geom &, const void *,        \
                                           const void *, void *, void *, int, \
                                           int, double, cudaStream_t);        \
  template int launch_ape<STORE, CT>(const Geom &, const Fields4 &,           \
                                     const Fields4 &, double, cudaStream_t);  \
  template int launch_hyp<STORE, CT>(const Geom &, const Fields4 &,           \
                                     const HypL1 &, const HypL2 &, void *,    \
                                     double, double, double, cudaStream_t);   \
  template int launch_hyp_slices<STORE, CT>(const Geom &, const Fields4 &,    \
                                            const HypL1 &, const HypL2 &,      \
                                            void *, double, double, double,    \
                                            cudaStream_t);                     \
  template int launch_ape_batch<STORE, CT>(const ApeJob *, int, int,          \
                                           cudaStream_t);                     \
  template int launch_hyp_batch<STORE, CT>(const HypJob *, int, const int *,  \
                                           cudaStream_t);

GC_INSTANTIATE_SMEAR(StoreF64SU3, double)
GC_INSTANTIATE_SMEAR(StoreF64SU2, double)
GC_INSTANTIATE_SMEAR(StoreF32SU3, float)
GC_INSTANTIATE_SMEAR(StoreF32SU2, float)

} // namespace gc
