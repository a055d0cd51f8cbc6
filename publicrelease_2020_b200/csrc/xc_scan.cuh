// SCAN meta-GGA exchange and correlation on the device (FP64), the form the
// reference calls for IDFTYP=11 (call_mgga.f90 -> scan.f: VSCANxUNP, VSCANc).
// Energies are per particle; the derivatives are those of rho*e with respect
// to rho, |grad rho| and tau, as scan.f returns them.  The constants and the
// order of the steps follow scan.f, including its exchange pi literal
// 3.1415927 and the clamps of zero gradients to 1e-100.
#pragma once

namespace flosic {

// Exchange enhancement factor Fx(p, alpha) and its first derivatives
// (metaggafx, scan.f:304-470).
__device__ __forceinline__ void scan_fx_dev(double p, double a, double& fx, double& fx_p, double& fx_a) {
  const double K1 = 0.065, C1 = 0.667, C2 = 0.800, D1 = 1.240;
  const double K0 = 0.1740, A1 = 4.9479, MU = 10.0 / 81.0, B1 = 0.156632, B2 = 0.12083, B3 = 0.5;
  const double oma = 1.0 - a, oma2 = oma * oma;
  const double hx0 = 1.0 + K0;
  const double b4 = MU * MU / K1 - 0.112654;  // > 0 for these constants (scan.f keeps both branches)
  double wfac, dwfac;
  if (b4 > 0.0) {
    const double e = exp(-b4 * p / MU);
    wfac = b4 * p * p * e;
    dwfac = b4 * p * e * (2.0 - b4 * p / MU);
  } else {
    const double e = exp(b4 * p / MU);
    wfac = b4 * p * p * e;
    dwfac = b4 * p * e * (2.0 + b4 * p / MU);
  }
  const double ea = exp(-B3 * oma2);
  const double vfac = B1 * p + B2 * oma * ea;
  const double yfac = MU * p + wfac + vfac * vfac;
  const double den = 1.0 + yfac / K1;
  const double hx1 = 1.0 + K1 - K1 / den;
  double fa = 0.0, dfa = 0.0;
  if (a < 1.0) {
    const double e = exp(-C1 * a / oma);
    fa = e;
    dfa = -C1 * e / (oma * oma);
  } else if (a > 1.0) {
    const double e = exp(C2 / oma);
    fa = -D1 * e;
    dfa = -C2 * D1 * e / (oma * oma);
  }
  double gx = 1.0, dgx = 0.0;
  if (p > 0.0) {
    const double p14 = pow(p, 0.25);
    const double e = exp(-A1 / p14);
    gx = 1.0 - e;
    dgx = -A1 / 4.0 / p / p14 * e;
  }
  const double fx1 = hx1 + fa * (hx0 - hx1);
  fx = fx1 * gx;
  const double dhx1_dp = (MU + dwfac + 2.0 * vfac * B1) / (den * den);
  const double dvfac_da = -B2 * (1.0 - 2.0 * B3 * oma2) * ea;
  const double dhx1_da = 2.0 * vfac * dvfac_da / (den * den);
  const double dfx1_dp = dhx1_dp + fa * (0.0 - dhx1_dp);
  const double dfx1_da = (1.0 - fa) * dhx1_da + dfa * (hx0 - hx1);
  fx_p = dfx1_dp * gx + fx1 * dgx;
  fx_a = dfx1_da * gx;
}

// Spin-unpolarised SCAN exchange at density rho, |grad rho| = drho, kinetic
// energy density tau (VSCANxUNP, scan.f:172-287).
__device__ __forceinline__ void scan_x_dev(double rho, double drho, double tau, double& ex, double& vx,
                                           double& vxdd, double& amux) {
  const double PI = 3.1415927, PISQ = PI * PI;
  const double AX = -0.7385587663820224058842300326808360;
  const double TH = 1.0 / 3.0, TH2 = 2.0 * TH, TH4 = 4.0 * TH, TH5 = 1.0 + TH2, TH8 = 1.0 + TH5;
  const double tauw = drho * drho / rho / 8.0;
  const double exunif = AX * pow(rho, TH);
  const double exlda = exunif * rho;
  const double exdlda = exunif * TH4;
  const double c3p = pow(3.0 * PISQ, TH2);
  const double p = drho * drho / (4.0 * c3p * pow(rho, TH8));
  const double tunif = 3.0 / 10.0 * c3p * pow(rho, TH5);
  const double alpha = (tau - tauw) / tunif;
  const double dpd = -TH8 * p / rho;
  const double dpdd = 2.0 * p / drho;
  const double dad = -tau * pow(3.0 * PISQ * rho, TH2) / (2.0 * tunif * tunif) +
                     drho * drho / pow(rho, 11.0 / 3.0) * (10.0 / 9.0 / c3p);
  const double dadd = -drho / (4.0 * rho * tunif);
  const double dadt = 1.0 / tunif;
  double fx, fxp, fxa;
  scan_fx_dev(p, alpha, fx, fxp, fxa);
  vx = exdlda * fx + exlda * (fxp * dpd + fxa * dad);
  vxdd = exlda * (fxp * dpdd + fxa * dadd);
  amux = exlda * (fxa * dadt);
  ex = exunif * fx;
}

// PW92 interpolation G(rs) and dG/drs (GCOR22, scan.f:1155-1166).
__device__ __forceinline__ void scan_gcor_dev(double A, double A1, double B1, double B2, double B3, double B4,
                                              double rtrs, double& gg, double& ggrs) {
  const double q0 = -2.0 * A * (1.0 + A1 * rtrs * rtrs);
  const double q1 = 2.0 * A * rtrs * (B1 + rtrs * (B2 + rtrs * (B3 + B4 * rtrs)));
  const double q2 = log(1.0 + 1.0 / q1);
  gg = q0 * q2;
  const double q3 = A * (B1 / rtrs + 2.0 * B2 + rtrs * (3.0 * B3 + 4.0 * B4 * rtrs));
  ggrs = -2.0 * A * A1 * q2 - q0 * q3 / (q1 * (1.0 + q1));
}

// PW92 LSD correlation energy and spin potentials (the LSD part of
// CORPBE_revtpss, scan.f:700-790).
__device__ __forceinline__ void scan_lsd_dev(double rs, double zet, double& ec, double& vcup, double& vcdn) {
  const double TH = 1.0 / 3.0, TH4 = 4.0 * TH;
  const double GAM = 0.51984209978974632953442121455650, FZZ = 8.0 / (9.0 * GAM);
  const double rtrs = sqrt(rs);
  double eu, eurs, ep, eprs, alfm, alfrsm;
  scan_gcor_dev(0.03109070, 0.213700, 7.59570, 3.58760, 1.63820, 0.492940, rtrs, eu, eurs);
  scan_gcor_dev(0.015545350, 0.205480, 14.11890, 6.19770, 3.36620, 0.625170, rtrs, ep, eprs);
  scan_gcor_dev(0.01688690, 0.111250, 10.3570, 3.62310, 0.880260, 0.496710, rtrs, alfm, alfrsm);
  const double z4 = zet * zet * zet * zet;
  const double f = (pow(1.0 + zet, TH4) + pow(1.0 - zet, TH4) - 2.0) / GAM;
  ec = eu * (1.0 - f * z4) + ep * f * z4 - alfm * f * (1.0 - z4) / FZZ;
  const double ecrs = eurs * (1.0 - f * z4) + eprs * f * z4 - alfrsm * f * (1.0 - z4) / FZZ;
  const double fz = TH4 * (pow(1.0 + zet, TH) - pow(1.0 - zet, TH)) / GAM;
  const double eczet =
      4.0 * (zet * zet * zet) * f * (ep - eu + alfm / FZZ) + fz * (z4 * ep - z4 * eu - (1.0 - z4) * alfm / FZZ);
  const double comm = ec - rs * ecrs / 3.0 - zet * eczet;
  vcup = comm + eczet;
  vcdn = comm - eczet;
}

// Density, spin and reduced-gradient variables shared by CORGGA_0 and CORGGA_1.
struct ScanSpinDev {
  double rt, yc, zeta, dz1, dz2, rs, drs, s, ds;
};

__device__ __forceinline__ ScanSpinDev scan_spin_dev(double ru, double rd, double dru, double drd, double drt) {
  const double PI = 3.141592653589793238, PISQ = PI * PI, TH = 1.0 / 3.0, TH4 = 4.0 * TH;
  ScanSpinDev v;
  v.rt = ru + rd;
  v.yc = (drt * drt - dru * dru - drd * drd) / 2.0;
  v.zeta = fmin(fmax((ru - rd) / v.rt, -0.99999999999990), 0.99999999999990);
  v.dz1 = 2.0 * rd / (v.rt * v.rt);
  v.dz2 = -2.0 * ru / (v.rt * v.rt);
  const double dthrd = exp(log(v.rt) * TH);
  v.rs = pow(0.750 / PI, TH) / dthrd;
  v.drs = -TH / v.rt * v.rs;
  v.s = drt / (2.0 * pow(3.0 * PISQ, TH) * pow(v.rt, TH4));
  v.ds = -TH4 * v.s / v.rt;
  return v;
}

// epsilon_c^1 (CORGGA_1, scan.f:841-1000); out: e, d/drho_up, d/drho_dn,
// d/d|grad rho_up|, d/d|grad rho_dn|.
__device__ __forceinline__ void scan_c1_dev(double ru, double rd, double dru, double drd, double drt,
                                            double out[5]) {
  const double PI = 3.141592653589793238, TH = 1.0 / 3.0;
  const double GAMMA = 0.031090690869654895034940863712730, BETA_MB = 0.066724550603149220;
  const ScanSpinDev v = scan_spin_dev(ru, rd, dru, drd, drt);
  const double zeta = v.zeta, rs = v.rs;
  const double phi = (exp((2.0 * TH) * log(1.0 + zeta)) + exp((2.0 * TH) * log(1.0 - zeta))) / 2.0;
  const double dphi = TH * (pow(1.0 + zeta, -TH) - pow(1.0 - zeta, -TH));
  const double afix = sqrt(PI / 4.0) * pow(9.0 * PI / 4.0, 1.0 / 6.0);
  const double gngnu = 1.0 / (2.0 * drt) * (2.0 * dru + 2.0 * v.yc / dru);
  const double gngnd = 1.0 / (2.0 * drt) * (2.0 * drd + 2.0 * v.yc / drd);
  const double dsdd1 = v.s / drt * gngnu, dsdd2 = v.s / drt * gngnd;
  const double srs = sqrt(rs);
  const double t = afix * v.s / srs / phi;
  const double t2 = t * t;
  const double den_t = phi * phi * pow(rs, 1.5);
  const double dtd1 = afix * (phi * rs * v.ds - 0.5 * v.s * phi * v.drs - v.s * rs * dphi * v.dz1) / den_t;
  const double dtd2 = afix * (phi * rs * v.ds - 0.5 * v.s * phi * v.drs - v.s * rs * dphi * v.dz2) / den_t;
  const double dtdd1 = afix * dsdd1 / (srs * phi), dtdd2 = afix * dsdd2 / (srs * phi);
  double ec, vu, vd;
  scan_lsd_dev(rs, zeta, ec, vu, vd);
  const double dec_dz = (vu - vd) / 2.0;
  const double dec_drs = (ec - zeta * dec_dz - (vu + vd) / 2.0) * 3.0 / rs;
  const double bnum = 1.0 + 0.10 * rs, bden = 1.0 + 0.17780 * rs;
  const double beta = BETA_MB * bnum / bden;
  const double dbeta = BETA_MB * (bden * 0.10 - bnum * 0.17780) / (bden * bden);
  const double phi3 = phi * phi * phi;
  const double w = exp(-ec / (phi3 * GAMMA)) - 1.0;
  const double dw_drs = -(w + 1.0) * dec_drs / (GAMMA * phi3);
  const double dw_dz = -(w + 1.0) / (GAMMA * phi3) * (dec_dz - 3.0 * ec * dphi / phi);
  const double A = beta / (GAMMA * w);
  const double dA_drs = (w * dbeta - beta * dw_drs) / (GAMMA * w * w);
  const double dA_dz = -beta * dw_dz / (GAMMA * w * w);
  const double V = A * t2;
  const double dV_drs = t2 * dA_drs, dV_dz = t2 * dA_dz, dV_dt = 2.0 * A * t;
  const double g = 1.0 / pow(1.0 + 4.0 * V, 0.250);
  const double dg_dv = -1.0 / pow(1.0 + 4.0 * V, 1.250);
  const double hcore = 1.0 + w * (1.0 - g);
  const double ah = GAMMA * phi3;
  const double h = ah * log(hcore);
  const double dh1 = 1.0 - g, dh2 = w * dg_dv;
  const double dh_drs = (dh1 * dw_drs - dh2 * dV_drs) * ah / hcore;
  const double dh_dz = 3.0 * h * dphi / phi + (dh1 * dw_dz - dh2 * dV_dz) * ah / hcore;
  const double dh_dt = (dh1 * 0.0 - dh2 * dV_dt) * ah / hcore;
  out[0] = ec + h;
  out[1] = dec_drs * v.drs + dec_dz * v.dz1 + dh_drs * v.drs + dh_dz * v.dz1 + dh_dt * dtd1;
  out[2] = dec_drs * v.drs + dec_dz * v.dz2 + dh_drs * v.drs + dh_dz * v.dz2 + dh_dt * dtd2;
  out[3] = dh_dt * dtdd1;
  out[4] = dh_dt * dtdd2;
}

// epsilon_c^0 (CORGGA_0, scan.f:1008-1150); clamps drt to 1e-100 and hands the
// clamped value back, as the reference passes it on to CORGGA_1.
__device__ __forceinline__ void scan_c0_dev(double ru, double rd, double dru, double drd, double& drt,
                                            double out[5]) {
  const double B1 = 0.0285764, B2 = 0.0889, B3 = 0.125541, KAI = 0.12802585262625815;
  const double TH = 1.0 / 3.0, TH4 = 4.0 * TH;
  const ScanSpinDev v = scan_spin_dev(ru, rd, dru, drd, drt);
  const double zeta = v.zeta, rs = v.rs;
  if (fabs(drt) < 1.0e-100) drt = 1.0e-100;
  const double gngnu = 1.0 / (2.0 * drt) * (2.0 * dru + 2.0 * v.yc / dru);
  const double gngnd = 1.0 / (2.0 * drt) * (2.0 * drd + 2.0 * v.yc / drd);
  const double dsdd1 = v.s / drt * gngnu, dsdd2 = v.s / drt * gngnd;
  const double rsh = sqrt(rs);
  const double ec0 = -B1 / (1.0 + B2 * rsh + B3 * rs);
  const double dec0 = (B3 + B2 / rsh / 2.0) * ec0 * ec0 / B1;
  const double dx = (pow(1.0 + zeta, TH4) + pow(1.0 - zeta, TH4)) / 2.0;
  const double ddx = 2.0 * (pow(1.0 + zeta, TH) - pow(1.0 - zeta, TH)) / 3.0;
  const double z12 = pow(zeta, 12.0);
  const double gc = (1.0 - 2.363 * (dx - 1.0)) * (1.0 - z12);
  const double dgc = -(1.0 - 2.363 * (dx - 1.0)) * 12.0 * pow(zeta, 11.0) - 2.363 * ddx * (1.0 - z12);
  const double w0 = exp(-ec0 / B1) - 1.0;
  const double dw0 = -(w0 + 1.0) * dec0 / B1;
  const double ginf = 1.0 / pow(1.0 + 4.0 * KAI * v.s * v.s, 0.25);
  const double dginf = -2.0 * KAI * v.s * pow(ginf, 5.0);
  const double hcore = 1.0 + w0 * (1.0 - ginf);
  const double h0 = B1 * log(hcore);
  const double dh0_drs = B1 * dw0 * (1.0 - ginf) / hcore;
  const double dh0_ds = -B1 * w0 * dginf / hcore;
  const double de_dz = (ec0 + h0) * dgc, de_drs = (dec0 + dh0_drs) * gc, de_ds = dh0_ds * gc;
  out[0] = (ec0 + h0) * gc;
  out[1] = de_dz * v.dz1 + de_drs * v.drs + de_ds * v.ds;
  out[2] = de_dz * v.dz2 + de_drs * v.drs + de_ds * v.ds;
  out[3] = de_ds * dsdd1;
  out[4] = de_ds * dsdd2;
}

// SCAN correlation (VSCANc -> Vmetaggac, scan.f:486-697).
__device__ __forceinline__ void scan_c_dev(double ru, double rd, double dru, double drd, double drt, double tauu,
                                           double taud, double& ec, double vc[2], double vcdd[2], double& amu) {
  const double PI = 3.141592653589793238, PISQ = PI * PI, TH = 1.0 / 3.0, TH2 = 2.0 * TH, TH5 = 1.0 + TH2;
  const double C1 = 0.640, C2 = 1.500, D1 = 0.700;
  if (dru == 0.0) dru = 1.0e-100;
  if (drd == 0.0) drd = 1.0e-100;
  const double rt = ru + rd;
  const double yc = (drt * drt - dru * dru - drd * drd) / 2.0;
  const double tauw = 1.0 / 8.0 * (drt * drt / rt);
  const double tau = tauu + taud;
  const double zeta = fmin(fmax((ru - rd) / rt, -0.99999999999990), 0.99999999999990);
  const double dsz = (pow(1.0 + zeta, TH5) + pow(1.0 - zeta, TH5)) / 2.0;
  const double tau0 = 0.30 * pow(3.0 * PISQ, TH2) * pow(rt, TH5) * dsz;
  const double alpha = (tau - tauw) / tau0;
  const double dz1 = 2.0 * rd / (rt * rt), dz2 = -2.0 * ru / (rt * rt);
  const double ddsz = TH5 * (pow(1.0 + zeta, TH2) - pow(1.0 - zeta, TH2)) / 2.0;
  const double dtau0_1 = TH5 * tau0 / rt + tau0 * (ddsz * dz1) / dsz;
  const double dtau0_2 = TH5 * tau0 / rt + tau0 * (ddsz * dz2) / dsz;
  const double dtauw = -tauw / rt;
  const double da1 = (-dtauw - alpha * dtau0_1) / tau0, da2 = (-dtauw - alpha * dtau0_2) / tau0;
  const double dtauw_dd1 = 1.0 / 4.0 / rt * (dru + yc / dru);
  const double dtauw_dd2 = 1.0 / 4.0 / rt * (drd + yc / drd);
  const double dadd1 = -dtauw_dd1 / tau0, dadd2 = -dtauw_dd2 / tau0;
  const double dat = 1.0 / tau0;
  double f = 0.0, df = 0.0;
  if (alpha < 1.0) {
    f = exp(C1 * alpha / (alpha - 1.0));
    df = -C1 * f / ((alpha - 1.0) * (alpha - 1.0));
  } else if (alpha > 1.0) {
    f = -D1 * exp(-C2 / (alpha - 1.0));
    df = C2 * f / ((alpha - 1.0) * (alpha - 1.0));
  }
  double e0[5], e1[5];
  scan_c0_dev(ru, rd, dru, drd, drt, e0);
  scan_c1_dev(ru, rd, dru, drd, drt, e1);
  const double dE = e0[0] - e1[0];
  const double epp = e1[0] + f * dE;
  const double d1 = e1[1] + dE * df * da1 + f * (e0[1] - e1[1]);
  const double d2 = e1[2] + dE * df * da2 + f * (e0[2] - e1[2]);
  const double dd1 = e1[3] + dE * df * dadd1 + f * (e0[3] - e1[3]);
  const double dd2 = e1[4] + dE * df * dadd2 + f * (e0[4] - e1[4]);
  vc[0] = epp + rt * d1;
  vc[1] = epp + rt * d2;
  vcdd[0] = rt * dd1;
  vcdd[1] = rt * dd2;
  amu = rt * (dE * df * dat);
  ec = epp;
}

// One mesh point of SUBVLXC for SCAN with NSPN=2 and the spin-down density
// zero (the SIC call, apotnl_sic.F:419-445): r[0..3] density and gradient of
// the FO density, tau = |grad phi|^2/2 of the FO (spin down zero,
// gettau_par.f90 with unravel2.f:242-246).  Returns the local spin potentials,
// adds ERGXL and ERGCL to e4[0], e4[2] (ERGXN, ERGCN stay zero), and returns
// the spin-up Hamiltonian ingredients z[0..3] (MIXINS of call_mgga.f90).
__device__ __forceinline__ void xc_point_sic_scan(const double r[4], double tau, double wgt, double& vup,
                                                  double& vdn, double e4[4], double z[4]) {
  const double EPS = 1.0e-20;
  const double den0 = r[0] < 0.0 ? 0.0 : r[0];
  const double dg2_0 = r[1] * r[1] + r[2] * r[2] + r[3] * r[3];
  // spin-up gradient = total - spin down (zero): the same channels
  const double dg2_1 = (r[1] - 0.0) * (r[1] - 0.0) + (r[2] - 0.0) * (r[2] - 0.0) + (r[3] - 0.0) * (r[3] - 0.0);
  vup = 0.0;
  vdn = 0.0;
  z[0] = z[1] = z[2] = z[3] = 0.0;
  if (!(den0 < EPS)) {
    const double D = 2.0 * den0;
    if (D > EPS) {
      const double dgrad = 2.0 * sqrt(dg2_1);
      double ex, vx, vxdd, amux;
      scan_x_dev(D, dgrad, 2.0 * tau, ex, vx, vxdd, amux);
      double div = dgrad;
      if (fabs(div) < 1.0e-100) div = 1.0e-100;
#pragma unroll
      for (int d = 0; d < 3; ++d) z[d] = 2.0 * vxdd * r[1 + d] / div;
      z[3] = amux * 0.5;
      vup += vx;
      e4[0] += 1.0 * 0.5 * ex * D * wgt;
    }
  }
  const double D = den0;
  if (D < EPS) return;
  double ec, vc[2], vcdd[2], amu;
  scan_c_dev(den0, 0.0, sqrt(dg2_1), 0.0, sqrt(dg2_0), tau, 0.0, ec, vc, vcdd, amu);
  double div1 = dg2_1;
  if (fabs(div1) < 1.0e-100) div1 = 1.0e-100;
  const double sdiv = sqrt(div1);
#pragma unroll
  for (int d = 0; d < 3; ++d) z[d] = z[d] + vcdd[0] * r[1 + d] / sdiv;
  z[3] = z[3] + amu * 0.5;
  e4[2] += ec * D * wgt;
  vup += vc[0];
  vdn += vc[1];
}

}  // namespace flosic
