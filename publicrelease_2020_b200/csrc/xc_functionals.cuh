// Exchange-correlation functionals of the SIC path, as device functions.
// Restates pw91ex.f, pbeex.f, pw91lc.f + gcor.f, pw91nc.f, pbecor.f + gcor2.f
// and the point loop of subvlxc_libxc.F90:213-480 (built-in functionals,
// NSPN=2, no core density), with the reference's literal constants.
#pragma once

#include <cuda_runtime.h>

namespace flosic {

struct XCParams {
  int igga[2];
  int idftyp[2];
};

__device__ __forceinline__ void xc_pw91ex(double dkf, double s, double u, double v, double& exl, double& exn,
                                          double& vx) {
  const double A1 = 0.19645, A2 = 0.27430, A3 = 0.15084, A4 = 100.0;
  const double AX = -0.238732414, A = 7.7956, B1 = 0.004;
  const double THRD4 = 1.3333333333333333;
  double fac = AX * dkf;
  double s2 = s * s, s3 = s2 * s, s4 = s2 * s2;
  double as = A * s;
  double pa = sqrt(1.0 + as * as);
  double p0 = as / pa;
  double p1 = A1 * log(as + pa);
  double p2 = A3 * exp(-A4 * s2);
  double p3 = 1.0 / (1.0 + s * p1 + B1 * s4);
  double p4 = 1.0 + s * p1 + (A2 - p2) * s2;
  double f = p3 * p4;
  exl = fac;
  exn = fac * (f - 1.0);
  double p5 = B1 * s2 - (A2 - p2);
  double p6 = s * (p1 + A1 * p0);
  double p7 = 2 * ((A2 - p2) + A4 * s2 * p2 - 2 * B1 * s2 * f);
  double fs = p3 * (p3 * p5 * p6 + p7);
  double p8 = 2 * s * (B1 - A4 * p2);
  double p9 = p1 + A1 * p0 * (3.0 - p0 * p0);
  double p10 = 4 * (A4 * s * p2 * (2.0 - A4 * s2) - 2 * B1 * s * f - B1 * s3 * fs);
  double p11 = p3 * p3 * (p1 + A1 * p0 + 4 * B1 * s3);
  double fss = p3 * p3 * (p5 * p9 + p6 * p8) - 2 * p3 * p5 * p6 * p11 + p3 * p10 - p7 * p11;
  vx = fac * (THRD4 * f - (u - THRD4 * s3) * fss - v * fs);
}

__device__ __forceinline__ void xc_pbeex(int mode, double rho, double s, double u, double v, double& exl,
                                         double& exn, double& vx) {
  const double THRD = 1.0 / 3.0, THRD4 = 4.0 / 3.0;
  const double AX = -0.738558766382022405884230032680836;
  const double UM = 0.2195149727645171;
  double uk = (mode == 2) ? 1.2450 : 0.8040;
  double ul = UM / uk;
  double exunif = AX * pow(rho, THRD);
  double s2 = s * s, p0, fxpbe;
  if (mode == 3) {
    p0 = exp(-ul * s2);
    fxpbe = 1.0 + uk * (1.0 - p0);
  } else {
    p0 = 1.0 + ul * s2;
    fxpbe = 1.0 + uk - uk / p0;
  }
  exl = exunif;
  exn = exunif * (fxpbe - 1.0);
  double fs, fss;
  if (mode == 3) {
    fs = 2.0 * UM * p0;
    fss = -2.0 * ul * s * fs;
  } else {
    fs = 2.0 * uk * ul / (p0 * p0);
    fss = -4.0 * ul * s * fs / p0;
  }
  vx = exunif * (THRD4 * fxpbe - (u - THRD4 * s2 * s) * fss - v * fs);
}

__device__ __forceinline__ void xc_gcor(double A, double A1, double B1, double B2, double B3, double B4,
                                        double rs, double& gg, double& ggrs) {
  double q0 = -2 * A * (1.0 + A1 * rs);
  double rs12 = sqrt(rs);
  double rs32 = rs12 * rs12 * rs12;
  double q1 = 2 * A * (B1 * rs12 + B2 * rs + B3 * rs32 + B4 * rs * rs);
  double q2 = log(1.0 + 1.0 / q1);
  gg = q0 * q2;
  double q3 = A * (B1 / rs12 + 2 * B2 + 3 * B3 * rs12 + 4 * B4 * rs);
  ggrs = -2 * A * A1 * q2 - q0 * q3 / (q1 * q1 + q1);
}

__device__ __forceinline__ void xc_gcor2(double A, double A1, double B1, double B2, double B3, double B4,
                                         double rtrs, double& gg, double& ggrs) {
  double q0 = -2.0 * A * (1.0 + A1 * rtrs * rtrs);
  double q1 = 2.0 * A * rtrs * (B1 + rtrs * (B2 + rtrs * (B3 + B4 * rtrs)));
  double q2 = log(1.0 + 1.0 / q1);
  gg = q0 * q2;
  double q3 = A * (B1 / rtrs + 2.0 * B2 + rtrs * (3.0 * B3 + 4.0 * B4 * rtrs));
  ggrs = -2.0 * A * A1 * q2 - q0 * q3 / (q1 * (1.0 + q1));
}

__device__ __forceinline__ void xc_pw91lc(double rs, double zet, double& ec, double& vcup, double& vcdn,
                                          double& ecrs, double& eczet) {
  const double GAMR = 1.92366105, FZZR = 0.58482234;
  const double THRD = 0.333333333333, THRD4 = 1.333333333333;
  double zetpr = pow(1.0 + zet, THRD);
  double zetmr = pow(1.0 - zet, THRD);
  double f = (pow(zetpr, 4.0) + pow(zetmr, 4.0) - 2.0) * GAMR;
  double eu, eurs, ep, eprs, alfm, alfrsm;
  xc_gcor(0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294, rs, eu, eurs);
  xc_gcor(0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517, rs, ep, eprs);
  xc_gcor(0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671, rs, alfm, alfrsm);
  double z3 = zet * zet * zet, z4 = z3 * zet;
  ec = eu * (1.0 - f * z4) + ep * f * z4 - alfm * f * (1.0 - z4) * FZZR;
  ecrs = eurs * (1.0 - f * z4) + eprs * f * z4 - alfrsm * f * (1.0 - z4) * FZZR;
  double fz = THRD4 * (zetpr - zetmr) * GAMR;
  eczet = 4.0 * z3 * f * (ep - eu + alfm * FZZR) + fz * (z4 * ep - z4 * eu - (1.0 - z4) * alfm * FZZR);
  double comm = ec - rs * ecrs * THRD - zet * eczet;
  vcup = comm + eczet;
  vcdn = comm - eczet;
}

__device__ __forceinline__ void xc_pw91nc(double rs, double zet, double t, double uu, double vv, double ww,
                                          double g, double ec, double ecrs, double eczet, double& h,
                                          double& dvcup, double& dvcdn) {
  const double XNU = 15.75592, CC0 = 0.004235, CX = -0.001667212;
  const double C1 = 0.002568, C2 = 0.023266, C3 = 7.389e-6, C4 = 8.723;
  const double C5 = 0.472, C6 = 7.389e-2, A4 = 100.0;
  const double BET = 0.0667263, BETR = 14.98659;
  const double DELT = 2.697586, DELTR = 0.3707018;
  const double RS2R0 = 0.66343644;
  const double THRD = 0.3333333333333333, THRD2 = 0.6666666666666667;
  const double SIXTH = 0.1666666666666667, THDSEV = 0.4285714285714286;
  double gr = 1.0 / g;
  double g3 = g * g * g, g4 = g3 * g;
  double g3r = gr * gr * gr, g4r = g3r * gr;
  double pon = -DELT * ec * g3r * BETR;
  double bex = exp(pon) - 1.0;
  double b = DELT / bex;
  double b2 = b * b;
  double t2 = t * t, t4 = t2 * t2, t6 = t4 * t2;
  double rs2 = rs * rs, rs3 = rs2 * rs;
  double q4 = 1.0 + b * t2;
  double q5 = 1.0 + b * t2 + b2 * t4;
  double q6 = C1 + C2 * rs + C3 * rs2;
  double q7 = 1.0 + C4 * rs + C5 * rs2 + C6 * rs3;
  double q7r = 1.0 / q7;
  double cc = -CX + q6 * q7r;
  double r0 = RS2R0 * rs;
  double r1 = A4 * r0 * g4;
  double coeff = cc - CC0 - THDSEV * CX;
  double r2 = XNU * coeff * g3;
  double r3 = exp(-r1 * t2);
  double h0 = g3 * BET * DELTR * log(1.0 + DELT * q4 * t2 / q5);
  double h1 = r3 * r2 * t2;
  h = h0 + h1;
  if ((1.0 - fabs(zet)) < 1.0e-10) zet = (1.0 - 1.0e-10) * zet;
  double ccrs = (C2 + 2 * C3 * rs) * q7r - q6 * (C4 + 2 * C5 * rs + 3 * C6 * rs2) * q7r * q7r;
  double rsthrd = rs * THRD;
  double r4 = rsthrd * ccrs / coeff;
  double gz = (pow(1.0 + zet, -THRD) - pow(1.0 - zet, -THRD)) * THRD;
  double fac = bex + 1.0;
  double bg = -3 * b2 * ec * fac * BETR * g4r;
  double bec = b2 * fac * BETR * g3r;
  double q8 = q5 * q5 + DELT * q4 * q5 * t2;
  double q8r = 1.0 / q8;
  double q82r = q8r * q8r;
  double q9 = 1.0 + 2 * b * t2;
  double h0b = -BET * g3 * b * t6 * (2.0 + b * t2) * q8r;
  double h0rs = -rsthrd * h0b * bec * ecrs;
  double fact0 = 2 * DELT - 6 * b;
  double fact1 = q5 * q9 + q4 * q9 * q9;
  double h0bt = 2 * BET * g3 * t4 * (q4 * q5 * fact0 - DELT * fact1) * q82r;
  double h0rst = rsthrd * t2 * h0bt * bec * ecrs;
  double h0z = 3 * gz * h0 * gr + h0b * (bg * gz + bec * eczet);
  double h0t = 2 * BET * g3 * q9 * q8r;
  double h0zt = 3 * gz * h0t * gr + h0bt * (bg * gz + bec * eczet);
  double fact2 = q4 * q5 + b * t2 * (q4 * q9 + q5);
  double fact3 = 2 * b * q5 * q9 + DELT * fact2;
  double h0tt = 4 * BET * g3 * t * (2 * b * q8r - q9 * fact3 * q82r);
  double h1rs = r3 * r2 * t2 * (-r4 + r1 * t2 * THRD);
  double fact4 = 2.0 - r1 * t2;
  double h1rst = r3 * r2 * t2 * (2 * r4 * (1.0 - r1 * t2) - THRD2 * r1 * t2 * fact4);
  double h1z = gz * r3 * r2 * t2 * (3.0 - 4 * r1 * t2) * gr;
  double h1t = 2 * r3 * r2 * (1.0 - r1 * t2);
  double h1zt = 2 * gz * r3 * r2 * (3.0 - 11 * r1 * t2 + 4 * r1 * r1 * t4) * gr;
  double h1tt = 4 * r3 * r2 * r1 * t * (-2.0 + r1 * t2);
  double hrs = h0rs + h1rs, hrst = h0rst + h1rst, ht = h0t + h1t, htt = h0tt + h1tt;
  double hz = h0z + h1z, hzt = h0zt + h1zt;
  double comm = h + hrs + hrst + t2 * ht * SIXTH + 7 * t2 * t * htt * SIXTH;
  double pref = hz - gz * t2 * ht * gr;
  double fact5 = gz * (2 * ht + t * htt) * gr;
  comm = comm - pref * zet - uu * htt - vv * ht - ww * (hzt - fact5);
  dvcup = comm + pref;
  dvcdn = comm - pref;
}

__device__ __forceinline__ void xc_pbecor(double rs, double zet, double t, double uu, double vv, double ww,
                                          double& ec, double& vcup, double& vcdn, double& h, double& dvcup,
                                          double& dvcdn) {
  const double THRD = 1.0 / 3.0, THRDM = -THRD, SIXTHM = THRDM / 2.0;
  const double THRD4 = 4.0 * THRD;
  const double GAM = 0.5198420997897463295344212145565;
  const double FZZ = 8.0 / (9.0 * GAM);
  const double GAMMA = 0.03109069086965489503494086371273;
  const double BET = 0.06672455060314922, DELT = BET / GAMMA;
  const double ETA = 1.0e-12;
  double rtrs = sqrt(rs);
  double eu, eurs, ep, eprs, alfm, alfrsm;
  xc_gcor2(0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294, rtrs, eu, eurs);
  xc_gcor2(0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517, rtrs, ep, eprs);
  xc_gcor2(0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671, rtrs, alfm, alfrsm);
  double z4 = pow(zet, 4.0);
  double f = (pow(1.0 + zet, THRD4) + pow(1.0 - zet, THRD4) - 2.0) / GAM;
  ec = eu * (1.0 - f * z4) + ep * f * z4 - alfm * f * (1.0 - z4) / FZZ;
  double ecrs = eurs * (1.0 - f * z4) + eprs * f * z4 - alfrsm * f * (1.0 - z4) / FZZ;
  double fz = THRD4 * (pow(1.0 + zet, THRD) - pow(1.0 - zet, THRD)) / GAM;
  double eczet = 4.0 * (zet * zet * zet) * f * (ep - eu + alfm / FZZ) + fz * (z4 * ep - z4 * eu - (1.0 - z4) * alfm / FZZ);
  double comm = ec - rs * ecrs / 3.0 - zet * eczet;
  vcup = comm + eczet;
  vcdn = comm - eczet;
  double g = (pow(1.0 + zet, 2.0 * THRD) + pow(1.0 - zet, 2.0 * THRD)) / 2.0;
  double g3 = g * g * g;
  double pon = -ec / (g3 * GAMMA);
  double b = DELT / (exp(pon) - 1.0);
  double b2 = b * b;
  double t2 = t * t, t4 = t2 * t2;
  double q4 = 1.0 + b * t2;
  double q5 = 1.0 + b * t2 + b2 * t4;
  h = g3 * (BET / DELT) * log(1.0 + DELT * q4 * t2 / q5);
  double g4 = g3 * g;
  double t6 = t4 * t2;
  double rsthrd = rs / 3.0;
  double gz = (pow((1.0 + zet) * (1.0 + zet) + ETA, SIXTHM) - pow((1.0 - zet) * (1.0 - zet) + ETA, SIXTHM)) / 3.0;
  double fac = DELT / b + 1.0;
  double bg = -3.0 * b2 * ec * fac / (BET * g4);
  double bec = b2 * fac / (BET * g3);
  double q8 = q5 * q5 + DELT * q4 * q5 * t2;
  double q9 = 1.0 + 2.0 * b * t2;
  double hb = -BET * g3 * b * t6 * (2.0 + b * t2) / q8;
  double hrs = -rsthrd * hb * bec * ecrs;
  double fact0 = 2.0 * DELT - 6.0 * b;
  double fact1 = q5 * q9 + q4 * q9 * q9;
  double hbt = 2.0 * BET * g3 * t4 * ((q4 * q5 * fact0 - DELT * fact1) / q8) / q8;
  double hrst = rsthrd * t2 * hbt * bec * ecrs;
  double hz = 3.0 * gz * h / g + hb * (bg * gz + bec * eczet);
  double ht = 2.0 * BET * g3 * q9 / q8;
  double hzt = 3.0 * gz * ht / g + hbt * (bg * gz + bec * eczet);
  double fact2 = q4 * q5 + b * t2 * (q4 * q9 + q5);
  double fact3 = 2.0 * b * q5 * q9 + DELT * fact2;
  double htt = 4.0 * BET * g3 * t * (2.0 * b / q8 - (q9 * fact3 / q8) / q8);
  comm = h + hrs + hrst + t2 * ht / 6.0 + 7.0 * t2 * t * htt / 6.0;
  double pref = hz - gz * t2 * ht / g;
  double fact5 = gz * (2.0 * ht + t * htt) / g;
  comm = comm - pref * zet - uu * htt - vv * ht - ww * (hzt - fact5);
  dvcup = comm + pref;
  dvcdn = comm - pref;
}

// One mesh point of SUBVLXC with NSPN=2: r[0..9] total-density channels, the
// spin-down density zero (the SIC call of apotnl_sic.F:419-445).  Returns the
// spin-up/down potentials and adds ERGXL,ERGXN,ERGCL,ERGCN contributions.
__device__ __forceinline__ void xc_point_sic(const XCParams& P, const double r[10], double wgt, double& vup,
                                             double& vdn, double e4[4]) {
  const bool isgga = P.igga[0] >= 1 || P.igga[1] >= 1;
  const double THIRD = 0.3333333333333333, THIRD2 = 0.6666666666666667;
  const double TRPI2 = 29.6088132032680759, FRDPI = 1.2732395447351627, DKF2RS = 1.9191582926775128;
  const double EPS = 1.0e-20;
  double rt0 = r[0];
  if (rt0 < 0.0) rt0 = 0.0;
  double den0 = rt0, den2 = 0.0;
  double den1 = den0 - den2;
  double dg2_0 = 0, dg2_1 = 0, dgg_0 = 0, dgg_1 = 0, dlp_0 = 0, dlp_1 = 0;
  if (isgga) {
    dg2_0 = r[1] * r[1] + r[2] * r[2] + r[3] * r[3];
    dgg_0 = r[4] * r[1] * r[1] + r[5] * r[2] * r[2] + r[6] * r[3] * r[3] +
            2 * (r[7] * r[1] * r[2] + r[8] * r[1] * r[3] + r[9] * r[2] * r[3]);
    dlp_0 = r[4] + r[5] + r[6];
    // spin-up channels = total - 0 (subvlxc_libxc.F90:271-286)
    double u1 = r[1] - 0.0, u2 = r[2] - 0.0, u3 = r[3] - 0.0;
    double u4 = r[4] - 0.0, u5 = r[5] - 0.0, u6 = r[6] - 0.0, u7 = r[7] - 0.0, u8 = r[8] - 0.0,
           u9 = r[9] - 0.0;
    dg2_1 = u1 * u1 + u2 * u2 + u3 * u3;
    dgg_1 = u4 * u1 * u1 + u5 * u2 * u2 + u6 * u3 * u3 + 2 * (u7 * u1 * u2 + u8 * u1 * u3 + u9 * u2 * u3);
    dlp_1 = u4 + u5 + u6;
  }
  vup = 0.0;
  vdn = 0.0;
  // exchange, spin up only (spin-down density is zero)
  if (!(P.idftyp[0] == 0 || den0 < EPS)) {
    double D = 2.0 * den1;
    if (D > EPS) {
      double dkf = pow(TRPI2 * D, THIRD);
      double S = 0, U = 0, V = 0;
      if (P.igga[0] != 0) {
        double dgrad = 2.0 * sqrt(dg2_1);
        double dlap = 2.0 * dlp_1;
        double rec2 = 0.5 / (dkf * D);
        double rec1 = rec2 * D;
        double rec22 = rec2 * rec2;
        S = dgrad * rec2;
        V = dlap * rec1 * rec2;
        U = (dgrad > EPS) ? 8.0 * dgg_1 * rec1 * rec22 / dgrad : 0.0;
      }
      double ex = 0, dex = 0, vx = 0;
      if (P.idftyp[0] <= 6) xc_pw91ex(dkf, S, U, V, ex, dex, vx);
      else if (P.idftyp[0] == 7) xc_pbeex(1, D, S, U, V, ex, dex, vx);
      else if (P.idftyp[0] == 8) xc_pbeex(2, D, S, U, V, ex, dex, vx);
      else xc_pbeex(3, D, S, U, V, ex, dex, vx);
      vup += vx;
      e4[0] += 1.0 * 0.5 * ex * D * wgt;
      e4[1] += 1.0 * 0.5 * dex * D * wgt;
    }
  }
  // correlation
  double D = den0;
  if (P.idftyp[1] == 0 || D < EPS) return;
  double drec = 1.0 / D;
  double zet = (den1 - den2) * drec;
  double dkf = pow(TRPI2 * D, THIRD);
  double dks = sqrt(FRDPI * dkf);
  double rs = DKF2RS / dkf;
  double g = 0.5 * (pow(1.0 + zet, THIRD2) + pow(1.0 - zet, THIRD2));
  if (zet == -1.0 || zet == 1.0) g = 0.5 * pow(2.0, THIRD2);
  double T = 0, UU = 0, VV = 0, WW = 0;
  if (P.igga[1] != 0) {
    double dgrad = sqrt(dg2_0);
    double dlap = dlp_0;
    double rec3 = drec;
    double rec1 = 0.5 / (dks * g);
    double rec2 = rec1 * rec3;
    double rec22 = rec2 * rec2;
    T = dgrad * rec2;
    VV = dlap * rec1 * rec2;
    // WW = D*(DG2(2)-DG2(3)) - (DUP-DDN)*DG2(1): DG2(2) is the spin-up |grad|^2
    WW = D * (dg2_1 - 0.0);
    WW = WW - (den1 - den2) * dg2_0;
    WW = WW * rec3 * rec22;
    UU = (dgrad > EPS) ? dgg_0 * rec1 * rec22 / dgrad : 0.0;
  }
  double ec = 0, vcup = 0, vcdn = 0, dec = 0, dvcup = 0, dvcdn = 0;
  if (P.idftyp[1] == 6) {
    double ecrs, eczet;
    xc_pw91lc(rs, zet, ec, vcup, vcdn, ecrs, eczet);
    xc_pw91nc(rs, zet, T, UU, VV, WW, g, ec, ecrs, eczet, dec, dvcup, dvcdn);
  } else {
    xc_pbecor(rs, zet, T, UU, VV, WW, ec, vcup, vcdn, dec, dvcup, dvcdn);
  }
  e4[2] += ec * D * wgt;
  e4[3] += dec * D * wgt;
  vup += vcup + dvcup;
  vdn += vcdn + dvcdn;
}

}  // namespace flosic
