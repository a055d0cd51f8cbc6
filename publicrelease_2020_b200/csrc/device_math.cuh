// Device math shared by the Coulomb kernels: Boys-function values with the
// three table variants of fffmtc.F / fffmt4.F / fffmt3.F, the real spherical
// harmonics recursion of harmonics.f, and the Lebedev degree-19 mesh.
#pragma once

#include "common.cuh"

namespace flosic {

// Lebedev degree-19 mesh (set by upload_constants); this header is included by
// one translation unit only.
__constant__ double c_leb_ang[NANG * 3];
__constant__ double c_leb_w[NANG];

// Boys values F_0..F_{maxfmt-1} at x, chgd = exp(-x).  tab: BOYS_NT x BOYS_NC.
// s3/s4/s5 receive the maxfmt=3/4/5 variants (identical when x > 16).
__device__ __forceinline__ void boys_all(const double* __restrict__ tab, double x, double chgd,
                                         double s3[3], double s4[4], double s5[5]) {
  if (x > 16.0) {
    const double ROOTPI = 1.77245385090551602728;
    double pol1 = -chgd;
    double rt = __dmul_rn(sqrt(x), ROOTPI);
    double rect1 = 0.5 / x;
    double f0 = rect1 * (rt + pol1);
    double f1 = rect1 * (f0 + pol1);
    double f2 = rect1 * (3 * f1 + pol1);
    double f3 = rect1 * (5 * f2 + pol1);
    double f4 = rect1 * (7 * f3 + pol1);
    s3[0] = s4[0] = s5[0] = f0;
    s3[1] = s4[1] = s5[1] = f1;
    s3[2] = s4[2] = s5[2] = f2;
    s4[3] = s5[3] = f3;
    s5[4] = f4;
    return;
  }
  int it = (int)(100 * x + 1.5);
  double pol1 = chgd;
  double rect1 = 2 * x;
  double dt = (1.0e-2) * (it - 1) - x;
  const double* f = tab + (size_t)(it - 1) * BOYS_NC;
  const double o7 = 1.0 / 7.0, o5 = 1.0 / 5.0, o3 = 1.0 / 3.0;
  // F2 F3 F4 F5 F4/2 F5/2 F6/2 F5/6 F6/6 F7/6
  s5[4] = f[2] + dt * (f[3] + dt * (f[6] + dt * f[9]));
  s5[3] = (s5[4] * rect1 + pol1) * o7;
  s5[2] = (s5[3] * rect1 + pol1) * o5;
  s5[1] = (s5[2] * rect1 + pol1) * o3;
  s5[0] = (s5[1] * rect1 + pol1);
  s4[3] = f[1] + dt * (f[2] + dt * (f[5] + dt * f[8]));
  s4[2] = (s4[3] * rect1 + pol1) * o5;
  s4[1] = (s4[2] * rect1 + pol1) * o3;
  s4[0] = (s4[1] * rect1 + pol1);
  s3[2] = f[0] + dt * (f[1] + dt * (f[4] + dt * f[7]));
  s3[1] = (s3[2] * rect1 + pol1) * o3;
  s3[0] = (s3[1] * rect1 + pol1);
}

// Pair potential at one point from precomputed per-point quantities.
// mono[35]: monomials of rho = r - C in POLY order; coef[46] the pair's
// coefficients (COEFICIENT order, already scaled by FACTOR).  Mirrors the ERP /
// ADDP assembly of poisson1.f:1000-1087 with the SSCL gates encoded in maxfmt
// and a zeroed constant term when SSCL(3) is false.
__device__ __forceinline__ double pair_potential(const double* __restrict__ coef, const double mono[35],
                                                 int maxfmt, const double s3[3], const double s4[4],
                                                 const double s5[5]) {
  double e0 = coef[0];
  double e1 = coef[1];
  e1 = fma(mono[1], coef[3], e1);
  e1 = fma(mono[2], coef[4], e1);
  e1 = fma(mono[3], coef[5], e1);
  double e2 = coef[2];
#pragma unroll
  for (int i = 1; i < 10; ++i) e2 = fma(mono[i], coef[i + 5], e2);
  double v;
  if (maxfmt == 3) {
    v = e0 * s3[0] + e1 * s3[1] + e2 * s3[2];
    return v;
  }
  double e3 = 0.0;
#pragma unroll
  for (int i = 4; i < 20; ++i) e3 = fma(mono[i], coef[i + 11], e3);
  if (maxfmt == 4) {
    v = e0 * s4[0] + e1 * s4[1] + e2 * s4[2] + e3 * s4[3];
    return v;
  }
  double e4 = 0.0;
#pragma unroll
  for (int i = 20; i < 35; ++i) e4 = fma(mono[i], coef[i + 11], e4);
  v = e0 * s5[0] + e1 * s5[1] + e2 * s5[2] + e3 * s5[3] + e4 * s5[4];
  return v;
}

// Monomials of (x,y,z) up to degree 4 in POLY order (poisson1.f:925-959).
__device__ __forceinline__ void monomials(double x, double y, double z, double p[35]) {
  p[0] = 1.0;
  p[1] = z;
  p[2] = y;
  p[3] = x;
  p[4] = z * z;
  p[5] = y * z;
  p[6] = y * y;
  p[7] = x * z;
  p[8] = x * y;
  p[9] = x * x;
  p[10] = z * p[4];
  p[11] = y * p[4];
  p[12] = z * p[6];
  p[13] = y * p[6];
  p[14] = x * p[4];
  p[15] = x * p[5];
  p[16] = x * p[6];
  p[17] = z * p[9];
  p[18] = y * p[9];
  p[19] = x * p[9];
  p[20] = p[4] * p[4];
  p[21] = p[4] * p[5];
  p[22] = p[6] * p[4];
  p[23] = p[6] * p[5];
  p[24] = p[6] * p[6];
  p[25] = p[4] * p[7];
  p[26] = p[8] * p[4];
  p[27] = p[8] * p[5];
  p[28] = p[6] * p[8];
  p[29] = p[9] * p[4];
  p[30] = p[9] * p[5];
  p[31] = p[9] * p[6];
  p[32] = p[7] * p[9];
  p[33] = p[8] * p[9];
  p[34] = p[9] * p[9];
}

// Real spherical harmonics of harmonics.f for a unit vector, degrees 0..lm
// (lm <= 6), storage order of the reference (l^2 .. (l+1)^2-1 per degree),
// including the normalisation prefactors.
__device__ __forceinline__ void harmonics6(int lm, double x, double y, double z, double Y[NMOM]) {
  Y[0] = 1.0;
  if (lm >= 1) {
    Y[1] = z;
    Y[2] = x;
    Y[3] = y;
  }
#pragma unroll
  for (int l = 2; l <= LM; ++l) {
    if (l > lm) break;
    const int ifc2l1 = 2 * l - 1;
    int now = l * l, il1 = (l - 1) * (l - 1), il2 = (l - 2) * (l - 2);
#pragma unroll
    for (int m = 0; m <= l - 1; ++m) {
      double facrc = 1.0 / (l - m);
      int ifclm1 = (m == l - 1) ? 0 : l + m - 1;
      double aa = facrc * ifc2l1, bb = facrc * ifclm1;
      int nrun = (m == 0) ? 1 : 2;
      for (int r = 0; r < nrun; ++r) {
        now++;
        il1++;
        il2++;
        double t = bb * ((il2 >= 1 && il2 <= (l - 1) * (l - 1)) ? Y[il2 - 1] : 0.0);
        Y[now - 1] = aa * Y[il1 - 1] * Y[1] - t;
      }
    }
    int last = l * l;
    now = (l + 1) * (l + 1);
    double yl = Y[last - 1], ylm1 = Y[last - 2];
    Y[now - 1] = ifc2l1 * (yl * Y[2] + ylm1 * Y[3]);
    Y[now - 2] = ifc2l1 * (ylm1 * Y[2] - yl * Y[3]);
  }
  const double onofpi = 1.0 / (16 * atan(1.0));
#pragma unroll
  for (int l = 0; l <= LM; ++l) {
    if (l > lm) break;
    double facfc = (2 * l + 1) * onofpi;
    int now = l * l;
    for (int m = 0; m <= l; ++m) {
      int nrun = (m == 0) ? 1 : 2;
      double vfac = sqrt(nrun * facfc);
      for (int r = 0; r < nrun; ++r) {
        now++;
        Y[now - 1] = vfac * Y[now - 1];
      }
      facfc = facfc / ((l - m > 1 ? l - m : 1) * (l + m + 1));
    }
  }
}

}  // namespace flosic
