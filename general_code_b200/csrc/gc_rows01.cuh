// Two-row SU(3) arithmetic of the mixed form (FP32): an SU(3) matrix is
// determined by its rows 0 and 1 (row 2 = conj(row0 x row1)), and a product
// of SU(3) matrices is again in SU(3), so a product whose third row will be
// rebuilt needs only its first two rows computed (2/3 of the multiply-adds).
// Used by the mixed APE/HYP staples (gc_smear.cu) and the space lines of the
// one-column temporal-gauge W kernel (gc_wilson_gauge.cu).
#pragma once

#include "gc_internal.cuh"

namespace gc {

// row 2 = conj(row0 x row1), as StoreF32SU3::load rebuilds it
__device__ __forceinline__ void rebuild_row2(SU3<float> &u) {
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const int a1 = (j + 1) % 3, b1 = (j + 2) % 3;
    cx<float> t = csub(cmul(u.e[0][a1], u.e[1][b1]), cmul(u.e[0][b1], u.e[1][a1]));
    u.e[2][j] = {t.re, -t.im};
  }
}
// rows 0 and 1 of A B (A: rows 0, 1; B: all rows)
__device__ __forceinline__ SU3<float> mul01(const SU3<float> &A, const SU3<float> &B) {
  SU3<float> C;
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      float re = A.e[i][0].re * B.e[0][j].re;
      float im = A.e[i][0].re * B.e[0][j].im;
      re = fmaf(-A.e[i][0].im, B.e[0][j].im, re);
      im = fmaf(A.e[i][0].im, B.e[0][j].re, im);
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = fmaf(A.e[i][k].re, B.e[k][j].re, re);
        re = fmaf(-A.e[i][k].im, B.e[k][j].im, re);
        im = fmaf(A.e[i][k].re, B.e[k][j].im, im);
        im = fmaf(A.e[i][k].im, B.e[k][j].re, im);
      }
      C.e[i][j] = {re, im};
    }
  return C;
}

} // namespace gc
