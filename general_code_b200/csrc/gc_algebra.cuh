// Group algebra for SU(2) (quaternion a0 + i a.sigma) and SU(3) (3x3 complex),
// usable on host and device, templated on the arithmetic type (double/float).
//
// Semantics follow the reference's matrix types (lib/cpu/include/matrix.h):
//   mul(A,B)      = A*B        su2 :93-98,  su3 :348-350
//   mul_ad(A,B)   = A*B^dag    ("A ^ B")  su2 :99-104,  su3 :352-354
//   mul_da(A,B)   = A^dag*B    ("A % B")  su2 :105-110, su3 :356-358
//   conj_tr(A,B)  = Re Tr(A B^dag)/N  ("multiply_conj_tr") su2 :54-56, su3 :260-262
//   proj(A)       su2 :74-77 (a/|a|); su3 :279-292 (6 x [Newton-Schulz step,
//                 determinant phase fix])
// The quaternion product formulas and the projection iteration are the
// algebra itself and therefore have the same form as the reference's.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define GC_HD __host__ __device__ __forceinline__
#else
#define GC_HD inline
#endif

// Fused multiply-add on the device; a*b+c on the host (the host generator is
// built without FMA instructions, where fma() would be a slow library call).
#if defined(__CUDA_ARCH__)
#define GC_FMA(a, b, c) fma((a), (b), (c))
#else
#define GC_FMA(a, b, c) ((a) * (b) + (c))
#endif

namespace gc {

template <class T> struct cx {
  T re, im;
};

// Every product-sum below is an explicit fused multiply-add chain: left to
// the compiler, `a*b + c*d` may be contracted into either fma(a, b, c*d) or
// fma(c, d, a*b) depending on the surrounding code, so the same function
// inlined into two kernels could round differently. Written out, one
// function rounds one way everywhere (the batch, serving and single-lattice
// paths give bitwise equal results).
template <class T> GC_HD cx<T> cmul(cx<T> a, cx<T> b) {
  return {GC_FMA(-a.im, b.im, a.re * b.re), GC_FMA(a.im, b.re, a.re * b.im)};
}
// conj(a) * b
template <class T> GC_HD cx<T> cmulc(cx<T> a, cx<T> b) {
  return {GC_FMA(a.im, b.im, a.re * b.re), GC_FMA(-a.im, b.re, a.re * b.im)};
}
// a * conj(b)
template <class T> GC_HD cx<T> cmul_c(cx<T> a, cx<T> b) {
  return {GC_FMA(a.im, b.im, a.re * b.re), GC_FMA(-a.re, b.im, a.im * b.re)};
}
template <class T> GC_HD cx<T> cadd(cx<T> a, cx<T> b) {
  return {a.re + b.re, a.im + b.im};
}
template <class T> GC_HD cx<T> csub(cx<T> a, cx<T> b) {
  return {a.re - b.re, a.im - b.im};
}

// ----------------------------------------------------------------- SU(2)
template <class T> struct SU2 {
  T a0, a1, a2, a3;
  static constexpr int N = 2;
};

template <class T> GC_HD SU2<T> unit(SU2<T>) { return {T(1), T(0), T(0), T(0)}; }

// sum of four products p0 + s1 p1 + s2 p2 + s3 p3 as one fused chain
template <class T> GC_HD T dot4(T x0, T y0, T x1, T y1, T x2, T y2, T x3, T y3) {
  return GC_FMA(x3, y3, GC_FMA(x2, y2, GC_FMA(x1, y1, x0 * y0)));
}
template <class T> GC_HD SU2<T> mul(const SU2<T> &A, const SU2<T> &B) {
  return {dot4(A.a0, B.a0, -A.a1, B.a1, -A.a2, B.a2, -A.a3, B.a3),
          dot4(A.a0, B.a1, B.a0, A.a1, A.a3, B.a2, -A.a2, B.a3),
          dot4(A.a0, B.a2, B.a0, A.a2, A.a1, B.a3, -A.a3, B.a1),
          dot4(A.a0, B.a3, B.a0, A.a3, A.a2, B.a1, -A.a1, B.a2)};
}
template <class T> GC_HD SU2<T> mul_ad(const SU2<T> &A, const SU2<T> &B) {
  return {dot4(A.a0, B.a0, A.a1, B.a1, A.a2, B.a2, A.a3, B.a3),
          dot4(-A.a0, B.a1, B.a0, A.a1, -A.a3, B.a2, A.a2, B.a3),
          dot4(-A.a0, B.a2, B.a0, A.a2, -A.a1, B.a3, A.a3, B.a1),
          dot4(-A.a0, B.a3, B.a0, A.a3, -A.a2, B.a1, A.a1, B.a2)};
}
template <class T> GC_HD SU2<T> mul_da(const SU2<T> &A, const SU2<T> &B) {
  return {dot4(A.a0, B.a0, A.a1, B.a1, A.a2, B.a2, A.a3, B.a3),
          dot4(A.a0, B.a1, -B.a0, A.a1, -A.a3, B.a2, A.a2, B.a3),
          dot4(A.a0, B.a2, -B.a0, A.a2, -A.a1, B.a3, A.a3, B.a1),
          dot4(A.a0, B.a3, -B.a0, A.a3, -A.a2, B.a1, A.a1, B.a2)};
}
template <class T> GC_HD SU2<T> scale(const SU2<T> &A, T s) {
  return {A.a0 * s, A.a1 * s, A.a2 * s, A.a3 * s};
}
template <class T> GC_HD SU2<T> add(const SU2<T> &A, const SU2<T> &B) {
  return {A.a0 + B.a0, A.a1 + B.a1, A.a2 + B.a2, A.a3 + B.a3};
}
template <class T> GC_HD T conj_tr(const SU2<T> &A, const SU2<T> &B) {
  return dot4(A.a0, B.a0, A.a1, B.a1, A.a2, B.a2, A.a3, B.a3);
}
template <class T> GC_HD T tr_real(const SU2<T> &A) { return A.a0; }
template <class T> GC_HD SU2<T> adjoint(const SU2<T> &A) {
  return {A.a0, -A.a1, -A.a2, -A.a3};
}
// a / |a| by four divisions, as the reference writes it (the seeded
// configuration generator keeps this form, so that its links stay bit for
// bit those of the committed fixtures).
template <class T> GC_HD SU2<T> proj_div(const SU2<T> &A) {
  const T rho = sqrt(dot4(A.a0, A.a0, A.a1, A.a1, A.a2, A.a2, A.a3, A.a3));
  return {A.a0 / rho, A.a1 / rho, A.a2 / rho, A.a3 / rho};
}
// a / |a| as a times one reciprocal (four divisions cost more than the
// link's loads in FP64: SU(2) APE at 48^4 0.365 -> 0.311 ms per step; each
// element within an ulp of the quotient).
template <class T> GC_HD SU2<T> proj(const SU2<T> &A) {
  const T inv = T(1) / sqrt(dot4(A.a0, A.a0, A.a1, A.a1, A.a2, A.a2, A.a3, A.a3));
  return {A.a0 * inv, A.a1 * inv, A.a2 * inv, A.a3 * inv};
}

// ----------------------------------------------------------------- SU(3)
// Row-major: e[i][j] is the element in row i, column j.
template <class T> struct SU3 {
  cx<T> e[3][3];
  static constexpr int N = 3;
};

template <class T> GC_HD SU3<T> unit(SU3<T>) {
  SU3<T> U;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      U.e[i][j] = {i == j ? T(1) : T(0), T(0)};
  return U;
}

// The complex multiply-accumulates below are written as explicit fused
// multiply-add chains (one rounding per term instead of a product and an add).
// This is a different but equally accurate rounding order from the
// reference's separate product and sum.
template <class T> GC_HD SU3<T> mul(const SU3<T> &A, const SU3<T> &B) {
  SU3<T> C;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T re = A.e[i][0].re * B.e[0][j].re;
      T im = A.e[i][0].re * B.e[0][j].im;
      re = GC_FMA(-A.e[i][0].im, B.e[0][j].im, re);
      im = GC_FMA(A.e[i][0].im, B.e[0][j].re, im);
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = GC_FMA(A.e[i][k].re, B.e[k][j].re, re);
        re = GC_FMA(-A.e[i][k].im, B.e[k][j].im, re);
        im = GC_FMA(A.e[i][k].re, B.e[k][j].im, im);
        im = GC_FMA(A.e[i][k].im, B.e[k][j].re, im);
      }
      C.e[i][j] = {re, im};
    }
  return C;
}
// A * B^dag : C_ij = sum_k A_ik conj(B_jk)
template <class T> GC_HD SU3<T> mul_ad(const SU3<T> &A, const SU3<T> &B) {
  SU3<T> C;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T re = A.e[i][0].re * B.e[j][0].re;
      T im = A.e[i][0].im * B.e[j][0].re;
      re = GC_FMA(A.e[i][0].im, B.e[j][0].im, re);
      im = GC_FMA(-A.e[i][0].re, B.e[j][0].im, im);
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = GC_FMA(A.e[i][k].re, B.e[j][k].re, re);
        re = GC_FMA(A.e[i][k].im, B.e[j][k].im, re);
        im = GC_FMA(A.e[i][k].im, B.e[j][k].re, im);
        im = GC_FMA(-A.e[i][k].re, B.e[j][k].im, im);
      }
      C.e[i][j] = {re, im};
    }
  return C;
}
// A^dag * B : C_ij = sum_k conj(A_ki) B_kj
template <class T> GC_HD SU3<T> mul_da(const SU3<T> &A, const SU3<T> &B) {
  SU3<T> C;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T re = A.e[0][i].re * B.e[0][j].re;
      T im = A.e[0][i].re * B.e[0][j].im;
      re = GC_FMA(A.e[0][i].im, B.e[0][j].im, re);
      im = GC_FMA(-A.e[0][i].im, B.e[0][j].re, im);
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = GC_FMA(A.e[k][i].re, B.e[k][j].re, re);
        re = GC_FMA(A.e[k][i].im, B.e[k][j].im, re);
        im = GC_FMA(A.e[k][i].re, B.e[k][j].im, im);
        im = GC_FMA(-A.e[k][i].im, B.e[k][j].re, im);
      }
      C.e[i][j] = {re, im};
    }
  return C;
}
template <class T> GC_HD SU3<T> scale(const SU3<T> &A, T s) {
  SU3<T> C;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      C.e[i][j] = {A.e[i][j].re * s, A.e[i][j].im * s};
  return C;
}
template <class T> GC_HD SU3<T> add(const SU3<T> &A, const SU3<T> &B) {
  SU3<T> C;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      C.e[i][j] = cadd(A.e[i][j], B.e[i][j]);
  return C;
}
template <class T> GC_HD SU3<T> adjoint(const SU3<T> &A) {
  SU3<T> C;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      C.e[i][j] = {A.e[j][i].re, -A.e[j][i].im};
  return C;
}
// Re Tr(A B^dag) / 3
template <class T> GC_HD T conj_tr(const SU3<T> &A, const SU3<T> &B) {
  T s = T(0);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      s = GC_FMA(A.e[i][j].im, B.e[i][j].im, GC_FMA(A.e[i][j].re, B.e[i][j].re, s));
  return s / T(3);
}
template <class T> GC_HD T tr_real(const SU3<T> &A) {
  return (A.e[0][0].re + A.e[1][1].re + A.e[2][2].re) / T(3);
}
// a*b - c*d for complex numbers, as fused chains
template <class T> GC_HD cx<T> cmul_sub(cx<T> a, cx<T> b, cx<T> c, cx<T> d) {
  T re = a.re * b.re;
  T im = a.re * b.im;
  re = GC_FMA(-a.im, b.im, re);
  im = GC_FMA(a.im, b.re, im);
  re = GC_FMA(-c.re, d.re, re);
  re = GC_FMA(c.im, d.im, re);
  im = GC_FMA(-c.re, d.im, im);
  im = GC_FMA(-c.im, d.re, im);
  return {re, im};
}
// acc + a*b (complex)
template <class T> GC_HD cx<T> cmadd(cx<T> acc, cx<T> a, cx<T> b) {
  T re = GC_FMA(a.re, b.re, acc.re);
  T im = GC_FMA(a.re, b.im, acc.im);
  re = GC_FMA(-a.im, b.im, re);
  im = GC_FMA(a.im, b.re, im);
  return {re, im};
}
template <class T> GC_HD cx<T> det(const SU3<T> &m) {
  // cofactor expansion along the first column
  cx<T> c0 = cmul_sub(m.e[1][1], m.e[2][2], m.e[2][1], m.e[1][2]);
  cx<T> c1 = cmul_sub(m.e[0][1], m.e[2][2], m.e[2][1], m.e[0][2]);
  cx<T> c2 = cmul_sub(m.e[0][1], m.e[1][2], m.e[1][1], m.e[0][2]);
  cx<T> d = cmul(m.e[0][0], c0);
  d = cmadd(d, {-m.e[1][0].re, -m.e[1][0].im}, c1);
  d = cmadd(d, m.e[2][0], c2);
  return d;
}

// One Newton-Schulz step toward the unitary polar factor,
// A <- 3/2 A - 1/2 (A A^dag) A, followed by the determinant phase fix
// A <- (1 - (det A - 1)/3) A.  H = A A^dag is Hermitian: its upper triangle
// is computed and mirrored. The factor -1/2 is folded into H (exact: a power
// of two), so B = 3/2 A + (-H/2) A is one fused chain per element.
// H = -1/2 A A^dag (Hermitian; entries below the diagonal mirrored).
template <class T> GC_HD void ns_gram(const SU3<T> &A, cx<T> H[3][3]) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    T d = A.e[i][0].re * A.e[i][0].re;
    d = GC_FMA(A.e[i][0].im, A.e[i][0].im, d);
    d = GC_FMA(A.e[i][1].re, A.e[i][1].re, d);
    d = GC_FMA(A.e[i][1].im, A.e[i][1].im, d);
    d = GC_FMA(A.e[i][2].re, A.e[i][2].re, d);
    d = GC_FMA(A.e[i][2].im, A.e[i][2].im, d);
    H[i][i] = {T(-0.5) * d, T(0)};
#pragma unroll
    for (int j = i + 1; j < 3; j++) {
      T re = A.e[i][0].re * A.e[j][0].re;
      T im = A.e[i][0].im * A.e[j][0].re;
      re = GC_FMA(A.e[i][0].im, A.e[j][0].im, re);
      im = GC_FMA(-A.e[i][0].re, A.e[j][0].im, im);
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = GC_FMA(A.e[i][k].re, A.e[j][k].re, re);
        re = GC_FMA(A.e[i][k].im, A.e[j][k].im, re);
        im = GC_FMA(A.e[i][k].im, A.e[j][k].re, im);
        im = GC_FMA(-A.e[i][k].re, A.e[j][k].im, im);
      }
      H[i][j] = {T(-0.5) * re, T(-0.5) * im};
      H[j][i] = {T(-0.5) * re, T(0.5) * im};
    }
  }
}

// B = 3/2 A + H A with H from ns_gram, then the determinant phase fix.
template <class T> GC_HD SU3<T> ns_finish(const SU3<T> &A, const cx<T> H[3][3]) {
  SU3<T> B;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      cx<T> s = {T(1.5) * A.e[i][j].re, T(1.5) * A.e[i][j].im};
#pragma unroll
      for (int k = 0; k < 3; k++) {
        if (i == k) { // H_ii is real
          s.re = GC_FMA(H[i][i].re, A.e[k][j].re, s.re);
          s.im = GC_FMA(H[i][i].re, A.e[k][j].im, s.im);
        } else {
          s = cmadd(s, H[i][k], A.e[k][j]);
        }
      }
      B.e[i][j] = s;
    }
  cx<T> dt = det(B);
  const T third = T(1) / T(3);
  cx<T> c = {GC_FMA(-third, dt.re - T(1), T(1)), -third * dt.im};
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      B.e[i][j] = cmul(c, B.e[i][j]);
  return B;
}

template <class T> GC_HD SU3<T> ns_step(const SU3<T> &A) {
  cx<T> H[3][3];
  ns_gram(A, H);
  return ns_finish(A, H);
}

template <class T> GC_HD SU3<T> proj(const SU3<T> &A) {
  SU3<T> B = ns_step(A);
#pragma unroll 1
  for (int it = 0; it < 5; it++)
    B = ns_step(B);
  return B;
}

// The same six-step iteration, leaving early once a step changes no element
// by more than tol. The iteration converges quadratically (the error after a
// step of size d is O(d^2)), so the remaining steps would change the result
// by O(tol^2) plus rounding; an input that needs all six steps gets all six.
// The first two steps are always taken (inputs of smearing steps are never
// converged that early), so the check runs only after steps 3, 4 and 5.
template <class T> GC_HD SU3<T> proj(const SU3<T> &A, T tol) {
  SU3<T> B = ns_step(ns_step(A));
#pragma unroll 1
  for (int it = 0; it < 4; it++) {
    SU3<T> N = ns_step(B);
    if (it == 3) { // the sixth and last step
      B = N;
      break;
    }
    T d = T(0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) {
        d = fmax(d, fabs(N.e[i][j].re - B.e[i][j].re));
        d = fmax(d, fabs(N.e[i][j].im - B.e[i][j].im));
      }
    B = N;
    if (d <= tol)
      break;
  }
  return B;
}
template <class T> GC_HD SU2<T> proj(const SU2<T> &A, T) { return proj(A); }

// Newton-Schulz steps from B while its unitarity defect max|A A^dag - 1|
// (read off the step's own Gram matrix) exceeds tol, at most max_steps of
// them; *steps receives the number taken. The mixed-precision projection
// takes these in FP32 and then one step in FP64 (ns_step<double>): a step
// maps a defect d to O(d^2) (A = U(1 + E) becomes U(1 - 3/2 E^2 + ...),
// d = 2|E|), so from d <= 2e-5 the FP64 step lands below 1e-9, under the
// FP32 rounding of the stored link, and removes the FP32 rounding of the
// iterate. Together at most six steps, like the reference's projection.
template <class T> GC_HD SU3<T> ns_until(SU3<T> B, T tol, int max_steps, int *steps) {
  int n = 0;
#pragma unroll 1
  while (n < max_steps) {
    cx<T> H[3][3];
    ns_gram(B, H);
    // A A^dag = -2 H
    T d = T(0);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      d = fmax(d, fabs(T(-2) * H[i][i].re - T(1)));
#pragma unroll
      for (int j = i + 1; j < 3; j++)
        d = fmax(d, fmax(fabs(H[i][j].re), fabs(H[i][j].im)) * T(2));
    }
    if (d <= tol)
      break;
    B = ns_finish(B, H);
    n++;
  }
  *steps = n;
  return B;
}

// Gram-Schmidt reunitarisation: rows 0 and 1 orthonormalised, row 2 =
// conj(row0 x row1). Used by the configuration generator (not on the
// reference path).
template <class T> GC_HD SU3<T> reunitarize_gs(const SU3<T> &A) {
  SU3<T> U;
  T n0 = T(0);
  for (int j = 0; j < 3; j++)
    n0 += A.e[0][j].re * A.e[0][j].re + A.e[0][j].im * A.e[0][j].im;
  n0 = T(1) / sqrt(n0);
  for (int j = 0; j < 3; j++)
    U.e[0][j] = {A.e[0][j].re * n0, A.e[0][j].im * n0};
  // p = <u0, a1> = sum conj(u0_j) a1_j
  cx<T> p = {T(0), T(0)};
  for (int j = 0; j < 3; j++)
    p = cadd(p, cmulc(U.e[0][j], A.e[1][j]));
  cx<T> r[3];
  T n1 = T(0);
  for (int j = 0; j < 3; j++) {
    r[j] = csub(A.e[1][j], cmul(p, U.e[0][j]));
    n1 += r[j].re * r[j].re + r[j].im * r[j].im;
  }
  n1 = T(1) / sqrt(n1);
  for (int j = 0; j < 3; j++)
    U.e[1][j] = {r[j].re * n1, r[j].im * n1};
  // row2 = conj(row0 x row1)
  for (int j = 0; j < 3; j++) {
    int a = (j + 1) % 3, b = (j + 2) % 3;
    cx<T> c = csub(cmul(U.e[0][a], U.e[1][b]), cmul(U.e[0][b], U.e[1][a]));
    U.e[2][j] = {c.re, -c.im};
  }
  return U;
}

} // namespace gc
