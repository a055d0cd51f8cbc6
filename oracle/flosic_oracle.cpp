// FP64 CPU oracle for the FLO-SIC per-Fermi-orbital hot path.
//
// TEST INFRASTRUCTURE ONLY: a routine-by-routine restatement of the
// reference Fortran (FLOSIC/PublicRelease_2020, files under flosic/), used
// by tests/ and by bench.py's CPU-baseline legs to check and time the CUDA
// product path.  The product library never links this file.
//
// Each function cites the reference file:line whose semantics it follows.
// Loop orders that decide floating-point summation order are kept where the
// reference fixes them (per-point accumulation over atoms and functions,
// batch composition of the Poisson solver, block-wise energy sums).

#include "flosic_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <atomic>
#include <thread>

namespace {

constexpr int MAX_BARE = 25;   // PARAMA2
constexpr int MAX_CON = 15;    // PARAMA2
constexpr int NSPEED = 25;     // PARAMA2
constexpr int MPBLOCK = 100;   // PARAMA2
constexpr int MPBLOCKXC = 1000;
constexpr int MXPR = 100;      // MXPOISS
constexpr double CUTEXP = 40.0;
constexpr int LM = 6;                       // poisson1.f:75
constexpr int NMOM = (LM + 1) * (LM + 1);   // 49
constexpr int MPX = 190;                    // MAX_ANG for LMX=18 (poisson1.f:77-79)
constexpr int NANG = 146;                   // Lebedev degree 19 chosen by ANGMSH(LMAX=18)
constexpr double PI = 3.141592653589793;
constexpr double PI2 = 6.283185307179586;
constexpr double PI4 = 12.566370614359172;

thread_local std::string g_err;

int fail(const std::string& msg, int code = 1) {
  g_err = msg;
  return code;
}

// Cartesian component tables (gorbdrv.f PANG index; coupot_sic.F IBEG/IEND).
// comp 0:s 1:x 2:y 3:z 4:xx 5:yy 6:zz 7:xy 8:xz 9:yz
const int kPow[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                         {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
const int kNcomp[3] = {1, 3, 6};
const int kShift[3] = {0, 1, 4};

// Monomial index in the POLY ordering of poisson1.f:925-959 (0-based):
// by degree, then x-power ascending, then y-power ascending.
int mono_index(int px, int py, int pz);
struct MonoTable {
  int p[35][3];
  MonoTable() {
    for (int d = 0; d <= 4; ++d)
      for (int x = 0; x <= d; ++x)
        for (int y = 0; y <= d - x; ++y) {
          int z = d - x - y;
          int i = mono_index(x, y, z);
          p[i][0] = x;
          p[i][1] = y;
          p[i][2] = z;
        }
  }
};
int mono_index(int px, int py, int pz) {
  int d = px + py + pz;
  int base = 0;
  for (int k = 0; k < d; ++k) base += (k + 1) * (k + 2) / 2;
  int off = 0;
  for (int x = 0; x < px; ++x) off += (d - x + 1);
  off += py;
  return base + off;
}

// ---------------------------------------------------------------------------
// Problem description
// ---------------------------------------------------------------------------
struct Problem {
  int natoms = 0, ntypes = 0, nmsh = 0, nspn = 1;
  std::vector<int> atype;
  std::vector<double> rat;       // 3*natoms
  std::vector<int> nbare;        // ntypes
  std::vector<double> bfalp;     // MAX_BARE*ntypes
  std::vector<int> ncon;         // 3*ntypes
  std::vector<double> bfcon;     // MAX_BARE*MAX_CON*3*ntypes
  std::vector<int> lmax;         // per type
  std::vector<int> nloc;         // per type
  std::vector<int> aoff;         // per atom: basis offset
  int nbasis = 0;
  std::vector<double> rmsh, wmsh;
  // Weight of each mesh point in the POISSON1 cost model (poisson1.f:569-583):
  // 1 for the real mesh; m when the mesh is every m-th point of a larger one,
  // so that a timing sample makes the near/far choices of the full mesh.
  double count_scale = 1.0;
  int igga[2] = {0, 0}, idftyp[2] = {6, 6};
  // orbitals
  int nwfs[2] = {0, 0};
  std::vector<double> psi;       // nbasis * (nwfs0+nwfs1)
  int nfrm[2] = {0, 0};
  std::vector<double> fod[2];    // 3*nfrm
  bool have_orbitals = false;
  // derived per spin
  std::vector<double> tmat[2];   // TMAT(k, jwf) row-major [k*nwfs+jwf]
  std::vector<double> lowev[2];
  std::vector<double> fmat[2];   // FMAT(jwf, jfm, K): [(K*nfrm + jfm)*nwfs + jwf]
  bool have_tmat = false, have_fmat = false;

  double bcon(int t, int l, int icon, int ib) const {
    return bfcon[((size_t)(t * 3 + l) * MAX_CON + icon) * MAX_BARE + ib];
  }
  double alp(int t, int ib) const { return bfalp[(size_t)t * MAX_BARE + ib]; }
  bool gga() const { return igga[0] > 0 || igga[1] > 0; }
  bool mgga() const { return igga[0] >= 3 || igga[1] >= 3; }
  // Test knob: evaluate XC on the untruncated pair-route density (every point
  // near, as phi^2) while the Coulomb potential keeps the reference's near/far
  // split.  Isolates the reference's density truncation at far points, which a
  // meta-GGA amplifies in the density tails through alpha.
  bool xc_exact_density = false;
};

// ---------------------------------------------------------------------------
// GORBDRV (gorbdrv.f:18-316): contracted Cartesian Gaussians of one atom
// type at <= NSPEED points given relative to the atom.
// grad layout follows GRAD(NSPEED,10,6,MAX_CON,3).
// ---------------------------------------------------------------------------
inline size_t gidx(int ipt, int igr, int iang, int nb, int l) {
  return (((size_t)l * MAX_CON + nb) * 6 + iang) * 10 * NSPEED + (size_t)igr * NSPEED + ipt;
}

bool gorbdrv(const Problem& P, int nderv, int npts, const double* pts /*PTS(NSPEED,3)*/,
             int t, double* grad, bool* iallctr /*[3*MAX_CON]*/) {
  const int lmax = P.lmax[t];
  const int lmax1 = lmax + 1;
  const double geps = std::exp(-CUTEXP);
  double pang[10][10][NSPEED];
  double rsqr[NSPEED], gaus[NSPEED], alp2r[3][NSPEED];
  const int iend[3] = {1, 4, 10};
  for (int i = 0; i < npts; ++i) {
    double x = pts[i], y = pts[NSPEED + i], z = pts[2 * NSPEED + i];
    pang[0][0][i] = 1.0;
    pang[0][4][i] = x * x;
    pang[0][5][i] = y * y;
    pang[0][6][i] = z * z;
    rsqr[i] = pang[0][4][i] + pang[0][5][i] + pang[0][6][i];
    if (lmax > 0) {
      pang[0][1][i] = x;
      pang[0][2][i] = y;
      pang[0][3][i] = z;
      if (lmax > 1) {
        pang[0][7][i] = x * y;
        pang[0][8][i] = x * z;
        pang[0][9][i] = y * z;
      }
    }
  }
  int ngrad = 1;
  if (nderv == 1) ngrad = 4;
  if (nderv == 2) ngrad = 10;
  if (nderv > 0) {
    for (int ia = 0; ia < iend[lmax]; ++ia)
      for (int ig = 1; ig < ngrad; ++ig)
        for (int i = 0; i < npts; ++i) pang[ig][ia][i] = 0.0;
    if (lmax > 0) {
      for (int i = 0; i < npts; ++i) {
        pang[1][1][i] = 1.0;
        pang[2][2][i] = 1.0;
        pang[3][3][i] = 1.0;
      }
      if (lmax > 1) {
        for (int i = 0; i < npts; ++i) {
          double x = pts[i], y = pts[NSPEED + i], z = pts[2 * NSPEED + i];
          pang[1][4][i] = 2 * x;
          pang[1][7][i] = y;
          pang[1][8][i] = z;
          pang[2][5][i] = 2 * y;
          pang[2][7][i] = x;
          pang[2][9][i] = z;
          pang[3][6][i] = 2 * z;
          pang[3][8][i] = x;
          pang[3][9][i] = y;
        }
        if (nderv == 2) {
          for (int i = 0; i < npts; ++i) {
            pang[4][4][i] = 2.0;
            pang[5][5][i] = 2.0;
            pang[6][6][i] = 2.0;
            pang[7][7][i] = 1.0;
            pang[8][8][i] = 1.0;
            pang[9][9][i] = 1.0;
          }
        }
      }
    }
  }
  for (int l = 0; l < lmax1; ++l)
    for (int nb = 0; nb < P.ncon[t * 3 + l]; ++nb) {
      for (int ia = 0; ia < kNcomp[l]; ++ia)
        for (int ig = 0; ig < ngrad; ++ig)
          for (int i = 0; i < npts; ++i) grad[gidx(i, ig, ia, nb, l)] = 0.0;
      iallctr[l * MAX_CON + nb] = false;
    }
  bool iupdat = false;
  for (int ib = 0; ib < P.nbare[t]; ++ib) {
    const double alp = P.alp(t, ib);
    const double alp2 = 2 * alp;
    bool icount = false;
    for (int i = 0; i < npts; ++i) {
      double rexp = alp * rsqr[i];
      if (rexp < CUTEXP) {
        icount = true;
        gaus[i] = std::exp(-rexp);
      } else {
        gaus[i] = 0.0;
      }
    }
    if (!icount) continue;
    iupdat = true;
    if (nderv >= 1)
      for (int d = 0; d < 3; ++d)
        for (int i = 0; i < npts; ++i) alp2r[d][i] = alp2 * pts[d * NSPEED + i];
    bool ibarctr[3][MAX_CON];
    for (int l = 0; l < lmax1; ++l)
      for (int nb = 0; nb < P.ncon[t * 3 + l]; ++nb) {
        double c = std::fabs(P.bcon(t, l, nb, ib));
        bool on = false;
        for (int i = 0; i < npts; ++i)
          if (c * gaus[i] > geps) on = true;
        ibarctr[l][nb] = on;
        if (on) iallctr[l * MAX_CON + nb] = true;
      }
    for (int l = 0; l < lmax1; ++l)
      for (int nb = 0; nb < P.ncon[t * 3 + l]; ++nb) {
        if (!ibarctr[l][nb]) continue;
        const double contr = P.bcon(t, l, nb, ib);
        for (int ia = 0; ia < kNcomp[l]; ++ia) {
          const int ifc = ia + kShift[l];
          for (int i = 0; i < npts; ++i)
            grad[gidx(i, 0, ia, nb, l)] += pang[0][ifc][i] * gaus[i] * contr;
        }
      }
    if (nderv == 0) continue;
    for (int l = 0; l < lmax1; ++l)
      for (int nb = 0; nb < P.ncon[t * 3 + l]; ++nb) {
        if (!ibarctr[l][nb]) continue;
        const double contr = P.bcon(t, l, nb, ib);
        for (int ia = 0; ia < kNcomp[l]; ++ia) {
          const int ifc = ia + kShift[l];
          for (int d = 0; d < 3; ++d) {
            const int I = d + 1;
            for (int i = 0; i < npts; ++i)
              grad[gidx(i, I, ia, nb, l)] +=
                  (pang[I][ifc][i] - pang[0][ifc][i] * alp2r[d][i]) * gaus[i] * contr;
          }
        }
      }
    if (nderv <= 1) continue;
    for (int l = 0; l < lmax1; ++l)
      for (int nb = 0; nb < P.ncon[t * 3 + l]; ++nb) {
        if (!ibarctr[l][nb]) continue;
        const double contr = P.bcon(t, l, nb, ib);
        for (int ia = 0; ia < kNcomp[l]; ++ia) {
          const int ifc = ia + kShift[l];
          for (int d = 0; d < 3; ++d) {
            const int I = d + 1, J = d + 4;
            for (int i = 0; i < npts; ++i)
              grad[gidx(i, J, ia, nb, l)] +=
                  (pang[J][ifc][i] - pang[I][ifc][i] * alp2r[d][i] * 2 +
                   pang[0][ifc][i] * (alp2r[d][i] * alp2r[d][i] - alp2)) *
                  gaus[i] * contr;
          }
        }
      }
    for (int l = 0; l < lmax1; ++l)
      for (int nb = 0; nb < P.ncon[t * 3 + l]; ++nb) {
        if (!ibarctr[l][nb]) continue;
        const double contr = P.bcon(t, l, nb, ib);
        for (int ia = 0; ia < kNcomp[l]; ++ia) {
          const int ifc = ia + kShift[l];
          for (int ig = 0; ig < 2; ++ig) {
            const int I = ig + 1;
            for (int jg = ig + 1; jg < 3; ++jg) {
              const int J = jg + 1;
              const int K0 = (I + 1) + (J + 1) + 3 - 1;  // K=I+J+3 of gorbdrv.f, 0-based
              for (int i = 0; i < npts; ++i)
                grad[gidx(i, K0, ia, nb, l)] +=
                    (pang[K0][ifc][i] - pang[J][ifc][i] * alp2r[ig][i] -
                     pang[I][ifc][i] * alp2r[jg][i] +
                     pang[0][ifc][i] * alp2r[ig][i] * alp2r[jg][i]) *
                    contr * gaus[i];
            }
          }
        }
      }
  }
  return iupdat;
}

// ---------------------------------------------------------------------------
// Orbital values at a list of points.  mode 0: PSIG accumulation of
// frmiorb.f:270-296 / frmorb2.F:266-292 (coefficients below 1e-10 skipped);
// mode 1: DGEMM accumulation of frmorb_mpi.F:365-397 (no threshold).
// out[(iwf*ngrad + igr)*npts + ipt]
// ---------------------------------------------------------------------------
void orbital_values(const Problem& P, const double* pts3 /*3*npts*/, int npts, int nderv,
                    int ngrad, const double* coef, int ldc, int nwf, int mode,
                    std::vector<double>& out, int only_atom = -1) {
  out.assign((size_t)nwf * ngrad * npts, 0.0);
  std::vector<double> grad((size_t)NSPEED * 10 * 6 * MAX_CON * 3);
  double pts[3 * NSPEED];
  bool iallctr[3 * MAX_CON];
  for (int a = 0; a < P.natoms; ++a) {
    if (only_atom >= 0 && a != only_atom) continue;  // one atom's share (SICLAG_DER's site derivatives)
    const int t = P.atype[a];
    const double* R = &P.rat[3 * a];
    for (int j0 = 0; j0 < npts; j0 += NSPEED) {
      const int npv = std::min(NSPEED, npts - j0);
      for (int i = 0; i < npv; ++i)
        for (int d = 0; d < 3; ++d) pts[d * NSPEED + i] = pts3[3 * (j0 + i) + d] - R[d];
      bool up = gorbdrv(P, nderv, npv, pts, t, grad.data(), iallctr);
      if (!up) continue;
      int iloc = 0;
      for (int l = 0; l <= P.lmax[t]; ++l)
        for (int mu = 0; mu < kNcomp[l]; ++mu)
          for (int ic = 0; ic < P.ncon[t * 3 + l]; ++ic, ++iloc) {
            if (mode == 0 && !iallctr[l * MAX_CON + ic]) continue;
            for (int iwf = 0; iwf < nwf; ++iwf) {
              const double f = coef[(size_t)iwf * ldc + P.aoff[a] + iloc];
              if (mode == 0 && !(std::fabs(f) > 1.0e-10)) continue;
              for (int ig = 0; ig < ngrad; ++ig) {
                double* o = &out[((size_t)iwf * ngrad + ig) * npts + j0];
                for (int i = 0; i < npv; ++i) o[i] += f * grad[gidx(i, ig, mu, ic, l)];
              }
            }
          }
    }
  }
}

// ---------------------------------------------------------------------------
// Symmetric eigen-solver (cyclic Jacobi).  Stands in for DIAGGE_FO
// (diagon_sic.f:45); only the eigen-pairs are used downstream.
// a: n*n row-major symmetric (destroyed), v: eigenvectors in columns v[i*n+k].
// ---------------------------------------------------------------------------
void jacobi_eigen(int n, std::vector<double>& a, std::vector<double>& w, std::vector<double>& v) {
  v.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double x = a[(size_t)i * n + j] * a[(size_t)i * n + j];
        tot += x;
        if (i != j) off += x;
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = a[(size_t)p * n + q];
        if (apq == 0.0) continue;
        double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
        double theta = (aqq - app) / (2.0 * apq);
        double tt = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(tt * tt + 1.0), s = tt * c;
        for (int k = 0; k < n; ++k) {
          double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
          a[(size_t)k * n + p] = c * akp - s * akq;
          a[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
          a[(size_t)p * n + k] = c * apk - s * aqk;
          a[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
          v[(size_t)k * n + p] = c * vkp - s * vkq;
          v[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = a[(size_t)i * n + i];
  // ascending order
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int x, int y) { return w[x] < w[y]; });
  std::vector<double> w2(n), v2((size_t)n * n);
  for (int k = 0; k < n; ++k) {
    w2[k] = w[idx[k]];
    for (int i = 0; i < n; ++i) v2[(size_t)i * n + k] = v[(size_t)i * n + idx[k]];
  }
  w = w2;
  v = v2;
}

// LOWSIC (lowden_files.f:2-172): S^{-1/2} of the FO overlap.
// over: n*n (OVER(i,j) as over[i*n+j]); returns ham = S^{-1/2} (ham[i*n+j]),
// filo eigenvectors (filo[i*n+k] = FILO(i,k)), eval = lambda^{-1/2}.
int lowsic(int n, const std::vector<double>& over, std::vector<double>& ham,
           std::vector<double>& filo, std::vector<double>& eval) {
  std::vector<double> a = over, w, v;
  jacobi_eigen(n, a, w, v);
  for (int i = 0; i < n; ++i)
    if (w[i] < 1.0e-8) return fail("LOWSIC: LOWDEN EIGENVALUES TOO SMALL (< 1e-8): BAD POSITIONS IN FRMORB", 3);
  eval.resize(n);
  for (int i = 0; i < n; ++i) eval[i] = 1.0 / std::sqrt(w[i]);
  filo = v;
  ham.assign((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int m = 0; m < n; ++m) s += v[(size_t)j * n + m] * v[(size_t)i * n + m] * eval[m];
      ham[(size_t)i * n + j] = s;
    }
  return 0;
}

// ---------------------------------------------------------------------------
// Boys-function values, fffmtc.F / fffmt4.F / fffmt3.F.
// ---------------------------------------------------------------------------
struct BoysTable {
  double F[1601][10];
  BoysTable() {
    const double eps = 1.0e-12;
    for (int i = 0; i < 10; ++i) F[0][i] = 1.0 / (2 * (i + 1) - 1);
    for (int L = 2; L <= 1601; ++L) {
      double T = (1.0e-2) * (L - 1);
      double X = 2 * T;
      double den = 39.0, term = 1.0 / den, sum = term;
      for (int i = 2; i <= 100; ++i) {
        den = den + 2.0;
        term = term * X / den;
        sum = sum + term;
        double q = term / sum;
        if (q - eps <= 0) break;
      }
      double ex = std::exp(-T);
      double G[21];
      G[20] = ex * sum;
      for (int i = 1; i <= 19; ++i) {
        int K = 21 - i, KK = K - 1;
        G[KK] = (X * G[K] + ex) / (2 * KK - 1);
      }
      for (int i = 0; i < 10; ++i) F[L - 1][i] = G[i + 1];
    }
  }
};
const BoysTable& boys_table() {
  static BoysTable t;
  return t;
}

void boys(int maxfmt, double xx, double chgd, double* s) {
  const double ROOTPI = 1.77245385090551602728;
  if (xx > 16.0) {
    double pol1 = -chgd;
    double rt = std::sqrt(xx) * ROOTPI;
    double rect1 = 0.5 / xx;
    s[0] = rect1 * (rt + pol1);
    s[1] = rect1 * (s[0] + pol1);
    s[2] = rect1 * (3 * s[1] + pol1);
    if (maxfmt >= 4) s[3] = rect1 * (5 * s[2] + pol1);
    if (maxfmt >= 5) s[4] = rect1 * (7 * s[3] + pol1);
    return;
  }
  const BoysTable& T = boys_table();
  int it = (int)(100 * xx + 1.5);
  double pol1 = chgd;
  double rect1 = 2 * xx;
  double dt = (1.0e-2) * (it - 1) - xx;
  const double* f = T.F[it - 1];
  const double o7 = 1.0 / 7.0, o5 = 1.0 / 5.0, o3 = 1.0 / 3.0;
  if (maxfmt == 5) {
    s[4] = f[4] + dt * (f[5] + dt * (f[6] / 2.0 + dt * (f[7] / 6.0)));
    s[3] = (s[4] * rect1 + pol1) * o7;
    s[2] = (s[3] * rect1 + pol1) * o5;
    s[1] = (s[2] * rect1 + pol1) * o3;
    s[0] = (s[1] * rect1 + pol1);
  } else if (maxfmt == 4) {
    s[3] = f[3] + dt * (f[4] + dt * (f[5] / 2.0 + dt * (f[6] / 6.0)));
    s[2] = (s[3] * rect1 + pol1) * o5;
    s[1] = (s[2] * rect1 + pol1) * o3;
    s[0] = (s[1] * rect1 + pol1);
  } else {
    s[2] = f[2] + dt * (f[3] + dt * (f[4] / 2.0 + dt * (f[5] / 6.0)));
    s[1] = (s[2] * rect1 + pol1) * o3;
    s[0] = (s[1] * rect1 + pol1);
  }
}

// ---------------------------------------------------------------------------
// HARMONICS (harmonics.f:5-118): real spherical harmonics up to lm for
// normalized points; y[(lm+1)^2] in the reference's storage order.
// ---------------------------------------------------------------------------
void harmonics(int lm, double x, double y, double z, double* Y) {
  Y[0] = 1.0;
  if (lm >= 1) {
    Y[1] = z;
    Y[2] = x;
    Y[3] = y;
  }
  for (int l = 2; l <= lm; ++l) {
    const int ifc2l1 = 2 * l - 1;
    int now = l * l, il1 = (l - 1) * (l - 1), il2 = (l - 2) * (l - 2);
    for (int m = 0; m <= l - 1; ++m) {
      double facrc = 1.0 / (l - m);
      int ifclm1 = l + m - 1;
      if (m == l - 1) ifclm1 = 0;
      double aa = facrc * ifc2l1, bb = facrc * ifclm1;
      int nrun = (m == 0) ? 1 : 2;
      for (int r = 0; r < nrun; ++r) {
        now++;
        il1++;
        il2++;
        Y[now - 1] = aa * Y[il1 - 1] * Y[1] - bb * Y[il2 - 1];
      }
    }
    int last = l * l;
    now = (l + 1) * (l + 1);
    double yl = Y[last - 1], ylm1 = Y[last - 2];
    Y[now - 1] = ifc2l1 * (yl * Y[2] + ylm1 * Y[3]);
    Y[now - 2] = ifc2l1 * (ylm1 * Y[2] - yl * Y[3]);
  }
  const double fourpi = 16 * std::atan(1.0);
  const double onofpi = 1.0 / fourpi;
  for (int l = 0; l <= lm; ++l) {
    double facfc = (2 * l + 1) * onofpi;
    int now = l * l;
    for (int m = 0; m <= l; ++m) {
      int nrun = (m == 0) ? 1 : 2;
      double vfac = std::sqrt(nrun * facfc);
      for (int r = 0; r < nrun; ++r) {
        now++;
        Y[now - 1] = vfac * Y[now - 1];
      }
      facfc = facfc / (std::max(l - m, 1) * (l + m + 1));
    }
  }
}

// LEBEDEV degree 19 (lebedev.F:165-190 parameters, 727-905 generation order).
struct Lebedev19 {
  double ang[NANG][3], w[NANG];
  Lebedev19() {
    const double RT2RC = 0.70710678118654752440, RT3RC = 0.57735026918962576451;
    const double A1 = 0.00753519001311713812, A2 = 0.09265184700375432421,
                 A3 = 0.09061000833610514010;
    const double B[3] = {0.09518264418191036893, 0.08487112439121475736, 0.08942676055004592969};
    const double AL[3] = {0.15746766720390817632, 0.41749612279654533594, 0.67644104001142636987};
    const double AM[3] = {0.97488864367717323548, 0.80708981835958250163, 0.29129888220952674629};
    const double D1 = 0.08785259467896816188, AR1 = 0.14035538117131832857,
                 AU1 = 0.44933283232695573488, AW1 = 0.88227001126032263192;
    int n = 0;
    double sg[3];
    for (int i = 0; i < 3; ++i) {
      sg[0] = 1.0;
      for (int j = 0; j < 2; ++j) {
        ang[n][0] = ang[n][1] = ang[n][2] = 0.0;
        ang[n][i] = sg[0];
        w[n] = A1;
        ++n;
        sg[0] = -sg[0];
      }
    }
    for (int i = 0; i < 3; ++i) {
      int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
      sg[0] = RT2RC;
      for (int j = 0; j < 2; ++j) {
        sg[1] = RT2RC;
        for (int k = 0; k < 2; ++k) {
          ang[n][i] = 0.0;
          ang[n][i1] = sg[0];
          ang[n][i2] = sg[1];
          w[n] = A2;
          ++n;
          sg[1] = -sg[1];
        }
        sg[0] = -sg[0];
      }
    }
    sg[0] = RT3RC;
    for (int i = 0; i < 2; ++i) {
      sg[1] = RT3RC;
      for (int j = 0; j < 2; ++j) {
        sg[2] = RT3RC;
        for (int k = 0; k < 2; ++k) {
          for (int l = 0; l < 3; ++l) ang[n][l] = sg[l];
          w[n] = A3;
          ++n;
          sg[2] = -sg[2];
        }
        sg[1] = -sg[1];
      }
      sg[0] = -sg[0];
    }
    for (int g = 0; g < 3; ++g) {
      double z1 = AM[g], z2 = AL[g], ds = B[g];
      for (int i = 0; i < 3; ++i) {
        int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
        sg[i] = z1;
        for (int j = 0; j < 2; ++j) {
          sg[i1] = z2;
          for (int k = 0; k < 2; ++k) {
            sg[i2] = z2;
            for (int l = 0; l < 2; ++l) {
              for (int m = 0; m < 3; ++m) ang[n][m] = sg[m];
              w[n] = ds;
              ++n;
              sg[i2] = -sg[i2];
            }
            sg[i1] = -sg[i1];
          }
          sg[i] = -sg[i];
        }
      }
    }
    {
      double z1 = AR1, z2 = AU1, z3 = AW1, ds = D1;
      for (int i = 0; i < 3; ++i) {
        sg[i] = z1;
        for (int j = 0; j < 2; ++j) {
          int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
          for (int k = 0; k < 2; ++k) {
            sg[i1] = z2;
            for (int l = 0; l < 2; ++l) {
              sg[i2] = z3;
              for (int m = 0; m < 2; ++m) {
                for (int q = 0; q < 3; ++q) ang[n][q] = sg[q];
                w[n] = ds;
                ++n;
                sg[i2] = -sg[i2];
              }
              sg[i1] = -sg[i1];
            }
            int tmp = i1;
            i1 = i2;
            i2 = tmp;
          }
          sg[i] = -sg[i];
        }
      }
    }
  }
};
const Lebedev19& lebedev19() {
  static Lebedev19 L;
  return L;
}

// ---------------------------------------------------------------------------
// Gaussian-pair polynomial expansions.
// Potential (polyx.F + poisson1.f:346-488): the Coulomb potential of
//   prod_d (x_d-A_d)^n_d (x_d-B_d)^m_d exp(-a(r-A)^2 - b(r-B)^2)
// is FACTOR * sum_M sum_mono BB[M][mono] rho^mono F_M(delta rho^2), where
// rho = r' - C.  Each 1-D factor is E[(Y+rho s-a0)^n (Y+rho s-b0)^m] with
// Y ~ N(0,(1-s)/(2 delta)), s = u^2 (the t-substitution of polyx.F:13-33).
// poly1d[n][m][N][M]: coefficient of rho^N s^M.
// ---------------------------------------------------------------------------
struct Poly1D {
  double c[3][3][5][5];
};

void poly1d_coulomb(double a0, double b0, double delta, Poly1D& P) {
  // (h - a0)^k as polynomial in h (h = rho s): coefficients
  std::memset(&P, 0, sizeof(P));
  const double tdi = 0.5 / delta;  // 1/(2 delta)
  static const double binom[3][3] = {{1, 0, 0}, {1, 1, 0}, {1, 2, 1}};
  static const double dfact[5] = {1, 0, 1, 0, 3};  // E[Y^j]/sigma^j
  for (int n = 0; n <= 2; ++n)
    for (int m = 0; m <= 2; ++m) {
      for (int k = 0; k <= n; ++k)
        for (int l = 0; l <= m; ++l) {
          int j = k + l;
          if (j & 1) continue;
          double pre = binom[n][k] * binom[m][l] * dfact[j];
          // (h-a0)^(n-k) (h-b0)^(m-l) in powers of h
          double pa[3] = {0, 0, 0}, pb[3] = {0, 0, 0};
          int na = n - k, nb = m - l;
          // (h - a0)^na
          if (na == 0) pa[0] = 1;
          else if (na == 1) { pa[0] = -a0; pa[1] = 1; }
          else { pa[0] = a0 * a0; pa[1] = -2 * a0; pa[2] = 1; }
          if (nb == 0) pb[0] = 1;
          else if (nb == 1) { pb[0] = -b0; pb[1] = 1; }
          else { pb[0] = b0 * b0; pb[1] = -2 * b0; pb[2] = 1; }
          double ph[5] = {0, 0, 0, 0, 0};
          for (int x = 0; x <= na; ++x)
            for (int y = 0; y <= nb; ++y) ph[x + y] += pa[x] * pb[y];
          // sigma^j = ((1-s) tdi)^(j/2)
          int hj = j / 2;
          double sig[3] = {0, 0, 0};  // coefficients in s
          if (hj == 0) sig[0] = 1;
          else if (hj == 1) { sig[0] = tdi; sig[1] = -tdi; }
          else { sig[0] = tdi * tdi; sig[1] = -2 * tdi * tdi; sig[2] = tdi * tdi; }
          for (int e = 0; e <= na + nb; ++e) {
            if (ph[e] == 0.0) continue;
            for (int q = 0; q <= hj; ++q) {
              if (sig[q] == 0.0) continue;
              P.c[n][m][e][e + q] += pre * ph[e] * sig[q];
            }
          }
        }
    }
}

// coef[46] in the COEFICIENT ordering of poisson1.f:402-482 (0-based), not yet
// multiplied by FACTOR.  rho[mu][nu] is the 10x10 pair density matrix.
int coef_slot(int M, int px, int py, int pz) {
  int d = px + py + pz;
  int mi = mono_index(px, py, pz);  // 0..34
  switch (M) {
    case 0: return d == 0 ? 0 : -1;
    case 1: if (d == 0) return 1; if (d == 1) return 3 + (mi - 1); return -1;     // 4..6 -> z,y,x
    case 2: if (d == 0) return 2; if (d == 1) return 6 + (mi - 1); if (d == 2) return 9 + (mi - 4); return -1;
    case 3: if (d == 2) return 15 + (mi - 4); if (d == 3) return 21 + (mi - 10); return -1;
    case 4: if (d == 4) return 31 + (mi - 20); return -1;
  }
  return -1;
}

void pair_potential_coefs(const double (*rho)[10], double a0[3], double b0[3], double delta,
                          double* coef) {
  Poly1D P[3];
  for (int d = 0; d < 3; ++d) poly1d_coulomb(a0[d], b0[d], delta, P[d]);
  double bb[5][5][5][5];  // [M][nx][ny][nz]
  std::memset(bb, 0, sizeof(bb));
  for (int mu = 0; mu < 10; ++mu)
    for (int nu = 0; nu < 10; ++nu) {
      const double r = rho[mu][nu];
      if (r == 0.0) continue;
      const Poly1D& X = P[0];
      const Poly1D& Yp = P[1];
      const Poly1D& Z = P[2];
      int nx = kPow[mu][0], ny = kPow[mu][1], nz = kPow[mu][2];
      int mx = kPow[nu][0], my = kPow[nu][1], mz = kPow[nu][2];
      for (int ex = 0; ex < 5; ++ex)
        for (int sx = 0; sx < 5; ++sx) {
          double cx = X.c[nx][mx][ex][sx];
          if (cx == 0.0) continue;
          for (int ey = 0; ey < 5; ++ey)
            for (int sy = 0; sy < 5; ++sy) {
              double cy = Yp.c[ny][my][ey][sy];
              if (cy == 0.0) continue;
              double pxy = r * cx * cy;
              for (int ez = 0; ez < 5; ++ez)
                for (int sz = 0; sz < 5; ++sz) {
                  double cz = Z.c[nz][mz][ez][sz];
                  if (cz == 0.0) continue;
                  int M = sx + sy + sz;
                  if (M > 4 || ex + ey + ez > 4) continue;
                  bb[M][ex][ey][ez] += pxy * cz;
                }
            }
        }
    }
  for (int i = 0; i < 46; ++i) coef[i] = 0.0;
  for (int M = 0; M < 5; ++M)
    for (int ex = 0; ex < 5; ++ex)
      for (int ey = 0; ey < 5; ++ey)
        for (int ez = 0; ez < 5; ++ez) {
          double v = bb[M][ex][ey][ez];
          if (v == 0.0) continue;
          int s = coef_slot(M, ex, ey, ez);
          if (s >= 0) coef[s] += v;
        }
}

const MonoTable kMonoTable;
const int (*const kMono)[3] = kMonoTable.p;

// Density polynomial (gtdncf.F:5-1113): rho_pair(r) = exp(-ARG) P(r-C)
// exp(-delta (r-C)^2).  rhoc[35] in POLY order; rhod[20][10]: derivative
// polynomials (columns 1..3: d/dx,d/dy,d/dz on monomials of degree <= 3;
// columns 4..9: xx,yy,zz,xy,xz,yz on degree <= 2).
void pair_density_coefs(const double (*gam)[10], double alp, const double* A, double bet,
                        const double* B, double* rhoc, double (*rhod)[10], double& dlt,
                        double* C) {
  dlt = alp + bet;
  double arg = 0.0;
  for (int i = 0; i < 3; ++i) {
    C[i] = (alp * A[i] + bet * B[i]) / dlt;
    arg = arg + (A[i] - B[i]) * (A[i] - B[i]);
  }
  arg = arg * alp * bet / dlt;
  double ca[3], cb[3];
  for (int d = 0; d < 3; ++d) {
    ca[d] = C[d] - A[d];
    cb[d] = C[d] - B[d];
  }
  for (int i = 0; i < 35; ++i) rhoc[i] = 0.0;
  for (int mu = 0; mu < 10; ++mu)
    for (int nu = 0; nu < 10; ++nu) {
      double g = gam[mu][nu];
      if (g == 0.0) continue;
      double p1[3][5];
      for (int d = 0; d < 3; ++d) {
        // (rho + ca)^na (rho + cb)^nb
        int na = kPow[mu][d], nb = kPow[nu][d];
        double pa[3] = {0, 0, 0}, pb[3] = {0, 0, 0};
        if (na == 0) pa[0] = 1; else if (na == 1) { pa[0] = ca[d]; pa[1] = 1; } else { pa[0] = ca[d] * ca[d]; pa[1] = 2 * ca[d]; pa[2] = 1; }
        if (nb == 0) pb[0] = 1; else if (nb == 1) { pb[0] = cb[d]; pb[1] = 1; } else { pb[0] = cb[d] * cb[d]; pb[1] = 2 * cb[d]; pb[2] = 1; }
        for (int e = 0; e < 5; ++e) p1[d][e] = 0.0;
        for (int x = 0; x <= na; ++x)
          for (int y = 0; y <= nb; ++y) p1[d][x + y] += pa[x] * pb[y];
      }
      for (int ex = 0; ex < 5; ++ex) {
        if (p1[0][ex] == 0.0) continue;
        for (int ey = 0; ey + ex < 5; ++ey) {
          if (p1[1][ey] == 0.0) continue;
          for (int ez = 0; ez + ey + ex < 5; ++ez) {
            if (p1[2][ez] == 0.0) continue;
            rhoc[mono_index(ex, ey, ez)] += g * p1[0][ex] * p1[1][ey] * p1[2][ez];
          }
        }
      }
    }
  double e = std::exp(-arg);
  for (int i = 0; i < 35; ++i) rhoc[i] = rhoc[i] * e;
  // derivative polynomials
  for (int i = 0; i < 20; ++i)
    for (int j = 0; j < 10; ++j) rhod[i][j] = 0.0;
  for (int i = 0; i < 35; ++i) {
    if (rhoc[i] == 0.0) continue;
    const int px = kMono[i][0], py = kMono[i][1], pz = kMono[i][2];
    const int p[3] = {px, py, pz};
    for (int d = 0; d < 3; ++d)
      if (p[d] > 0) {
        int q[3] = {px, py, pz};
        q[d] -= 1;
        rhod[mono_index(q[0], q[1], q[2])][1 + d] += p[d] * rhoc[i];
      }
    // second derivatives: xx yy zz xy xz yz
    const int pairs[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    for (int k = 0; k < 6; ++k) {
      int d1 = pairs[k][0], d2 = pairs[k][1];
      int q[3] = {px, py, pz};
      double f = q[d1];
      q[d1] -= 1;
      if (f <= 0) continue;
      f *= q[d2];
      q[d2] -= 1;
      if (f <= 0) continue;
      rhod[mono_index(q[0], q[1], q[2])][4 + k] += f * rhoc[i];
    }
  }
}

// GINTED (ginted.F:3-77): W(i,j,k) = integral of g_i^A g_j^B {x,y,z,1}.
void ginted(double a1, double a2, const double* A, const double* B, double W[4][10][10]) {
  double at = 1.0 / (a1 + a2);
  double q1 = 0.5 * at;  // variance of Y
  double xs = 0.0;
  double V[3][3][3][2];  // [d][n][m][k]: E[(x-A)^n (x-B)^m x^k]
  for (int d = 0; d < 3; ++d) {
    xs = xs + (a1 * a2 * ((A[d] - B[d]) * (A[d] - B[d]))) * at;
    double D = (a1 * A[d] + a2 * B[d]) * at;
    double f1 = D - A[d], f2 = D - B[d], f3 = D;
    // moments of Y: E[Y^0]=1, E[Y^2]=q1, E[Y^4]=3 q1^2
    const double mom[5] = {1.0, 0.0, q1, 0.0, 3 * q1 * q1};
    for (int n = 0; n < 3; ++n)
      for (int m = 0; m < 3; ++m)
        for (int k = 0; k < 2; ++k) {
          // expand (Y+f1)^n (Y+f2)^m (Y+f3)^k
          double c[6] = {0, 0, 0, 0, 0, 0};
          double pa[3] = {1, 0, 0};
          if (n == 1) { pa[0] = f1; pa[1] = 1; } else if (n == 2) { pa[0] = f1 * f1; pa[1] = 2 * f1; pa[2] = 1; }
          double pb[3] = {1, 0, 0};
          if (m == 1) { pb[0] = f2; pb[1] = 1; } else if (m == 2) { pb[0] = f2 * f2; pb[1] = 2 * f2; pb[2] = 1; }
          double pc[2] = {1, 0};
          if (k == 1) { pc[0] = f3; pc[1] = 1; }
          for (int x = 0; x <= n; ++x)
            for (int y = 0; y <= m; ++y)
              for (int z = 0; z <= k; ++z) c[x + y + z] += pa[x] * pb[y] * pc[z];
          double s = 0.0;
          for (int e = 0; e <= 4; ++e) s += c[e] * mom[e];
          V[d][n][m][k] = s;
        }
  }
  double D = std::exp(-xs) * std::pow(std::sqrt(3.14159265358979324 * at), 3);
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 10; ++j)
      for (int i = 0; i < 10; ++i) {
        double w = 1.0;
        for (int d = 0; d < 3; ++d) {
          int kk = (k == d) ? 1 : 0;
          w *= V[d][kPow[i][d]][kPow[j][d]][kk];
        }
        W[k][i][j] = w * D;
      }
}

// ---------------------------------------------------------------------------
// POISSON1 (poisson1.f:15-1650) for one call: the unique pairs of a batch
// (each pair occupies NSPN slots in the reference's arrays, spin-2 density
// matrix zero as in the SIC path, coupot_sic.F:414-430).
// ---------------------------------------------------------------------------
struct PairRec {
  double a, b, A[3], B[3];
  double dmat[10][10];
};

struct Stats {
  long long pairs = 0, batches = 0, weird = 0, near = 0, far = 0;
  long long near_multi = 0, far_multi = 0;  // the part from calls of more than one pair
  long long npot1_multi = 0, calls_multi = 0;
  // optional record of every POISSON1 call: (CG x3, RCUT, NPOT, pairs) per
  // call, (call, -C x3, delta, COEFICIENT(1:46)) per pair
  std::vector<double>* calls = nullptr;
  std::vector<double>* pairs_out = nullptr;
};

void poisson1(const Problem& P, const std::vector<PairRec>& prs, int nspn, bool gga, bool exact,
              double* coulomb, double* rhog /* [10][nmsh] */, Stats* st) {
  const int n = (int)prs.size();
  const int nslots = nspn * n;
  const double thirtysomething = exact ? 1.0e30 : 30.0;
  const double epsmulti = 1.0e-6;
  const double EPSILON = 0.0;
  double TF[5], TB[5];
  TF[0] = 0.5 * std::sqrt(PI);
  TF[1] = TF[0] * 0.5;
  TF[2] = TF[1] * 1.5;
  TF[3] = TF[2] * 2.5;
  TF[4] = TF[3] * 3.5;
  for (int i = 0; i < 5; ++i) TB[i] = std::pow(TF[i] * (2 * i + 1), 1.0 / (i + 0.5));

  std::vector<std::array<double, 46>> coef(n);
  std::vector<std::array<double, 35>> rhoc(n);
  std::vector<std::array<std::array<double, 10>, 20>> rhod(n);
  std::vector<double> delt(n), dlt(n);
  std::vector<std::array<double, 3>> Cn(n);
  double delta_min = 1.0e30;
  double cg[4] = {0, 0, 0, 0};
  for (int ip = 0; ip < n; ++ip) {
    const PairRec& pr = prs[ip];
    double ccc[3];
    double rd[20][10];
    pair_density_coefs(pr.dmat, pr.a, pr.A, pr.b, pr.B, rhoc[ip].data(), rd, dlt[ip], ccc);
    for (int i = 0; i < 20; ++i)
      for (int j = 0; j < 10; ++j) rhod[ip][i][j] = rd[i][j];
    double rho[10][10];
    for (int i = 0; i < 10; ++i)
      for (int j = 0; j < 10; ++j)
        rho[i][j] = (nspn == 1) ? pr.dmat[i][j] + pr.dmat[i][j] : pr.dmat[i][j] + 0.0;
    if (nslots != 1) {
      double W[4][10][10];
      ginted(pr.a, pr.b, pr.A, pr.B, W);
      for (int ic = 0; ic < 4; ++ic) {
        double t = 0.0;
        for (int j = 0; j < 10; ++j)
          for (int i = 0; i < 10; ++i) t += W[ic][i][j] * rho[i][j];
        cg[ic] += t;
      }
    }
    const double delta = pr.a + pr.b;
    if (delta < delta_min) delta_min = delta;
    const double rcdelt = 1.0 / delta;
    const double arg = pr.a * pr.b * rcdelt *
                       ((pr.A[0] - pr.B[0]) * (pr.A[0] - pr.B[0]) + (pr.A[1] - pr.B[1]) * (pr.A[1] - pr.B[1]) +
                        (pr.A[2] - pr.B[2]) * (pr.A[2] - pr.B[2]));
    const double factor = PI2 * std::exp(-arg) * rcdelt;
    double C[3], a0[3], b0[3];
    for (int i = 0; i < 3; ++i) {
      C[i] = (pr.a * pr.A[i] + pr.b * pr.B[i]) * rcdelt;
      a0[i] = pr.A[i] - C[i];
      b0[i] = pr.B[i] - C[i];
    }
    pair_potential_coefs(rho, a0, b0, delta, coef[ip].data());
    for (int i = 0; i < 46; ++i) coef[ip][i] = factor * coef[ip][i];
    delt[ip] = delta;
    for (int i = 0; i < 3; ++i) Cn[ip][i] = -C[i];
  }
  if (cg[3] != 0.0 && nslots > 1) {
    cg[0] /= cg[3];
    cg[1] /= cg[3];
    cg[2] /= cg[3];
  } else {
    for (int d = 0; d < 3; ++d) cg[d] = 0.0;
    for (int ip = 0; ip < n; ++ip)
      for (int d = 0; d < 3; ++d) cg[d] = cg[d] - Cn[ip][d];
    for (int d = 0; d < 3; ++d) cg[d] = (nspn * cg[d]) / nslots;
  }
  double dmax = 0.0;
  for (int ip = 0; ip < n; ++ip) {
    double dist = std::sqrt((cg[0] + Cn[ip][0]) * (cg[0] + Cn[ip][0]) + (cg[1] + Cn[ip][1]) * (cg[1] + Cn[ip][1]) +
                            (cg[2] + Cn[ip][2]) * (cg[2] + Cn[ip][2]));
    if (dist > dmax) dmax = dist;
  }
  double rcut = std::sqrt(thirtysomething / delta_min) + dmax;
  {
    double pirc = 1.0 / (4 * std::atan(1.0));
    double fact = std::sqrt(pirc / (pirc + LM + 1));
    double dist = 2 * dmax / std::pow(epsmulti / fact, 1.0 / (LM + 1));
    rcut = std::max(rcut, dist);
  }
  const Lebedev19& L = lebedev19();
  double Q[NANG][3];
  for (int ia = 0; ia < NANG; ++ia)
    for (int d = 0; d < 3; ++d) Q[ia][d] = cg[d] + L.ang[ia][d] * rcut;
  const double cgn[3] = {-cg[0], -cg[1], -cg[2]};
  const double rcutsq = rcut * rcut;
  const int nmsh = P.nmsh;
  std::vector<int> iptr, jptr;
  iptr.reserve(nmsh);
  jptr.reserve(nmsh);
  for (int ip = 0; ip < nmsh; ++ip) {
    const double* r = &P.rmsh[3 * ip];
    double rsqr = (r[0] + cgn[0]) * (r[0] + cgn[0]) + (r[1] + cgn[1]) * (r[1] + cgn[1]) +
                  (r[2] + cgn[2]) * (r[2] + cgn[2]);
    if (rsqr > rcutsq) iptr.push_back(ip);
    else jptr.push_back(ip);
  }
  int npot = 2;
  {
    const double cs = P.count_scale;
    double cost1 = 1.36 * ((double)jptr.size() * cs + NANG) * nslots + 0.99 * (double)iptr.size() * cs;
    double cost2 = 1.36 * ((double)iptr.size() + (double)jptr.size()) * cs * nslots;
    if (cost2 < cost1) {
      npot = 1;
      iptr.clear();
      jptr.resize(nmsh);
      for (int ip = 0; ip < nmsh; ++ip) jptr[ip] = ip;
    }
  }
  if (st && st->calls && st->pairs_out) {
    const double cid = (double)(st->calls->size() / 6);
    for (int ip = 0; ip < n; ++ip) {
      st->pairs_out->insert(st->pairs_out->end(), {cid, Cn[ip][0], Cn[ip][1], Cn[ip][2], delt[ip]});
      st->pairs_out->insert(st->pairs_out->end(), coef[ip].begin(), coef[ip].end());
    }
    st->calls->insert(st->calls->end(), {cg[0], cg[1], cg[2], rcut, (double)npot, (double)n});
  }
  if (st) {
    st->near += (long long)jptr.size() * n;
    st->far += (long long)iptr.size();
    if (n > 1) {
      st->near_multi += (long long)jptr.size() * n;
      st->far_multi += (long long)iptr.size();
      st->calls_multi += 1;
      if (npot == 1) st->npot1_multi += 1;
    }
  }
  std::vector<double> potnl(jptr.size(), 0.0);
  double asymptot[NANG];
  for (int i = 0; i < NANG; ++i) asymptot[i] = 0.0;

  static thread_local double poly[MPX][35];
  double xx[MPX], chgd[MPX], sss[MPX][5], addp[MPX], erp[MPX][5], addr[MPX][10];
  for (int ipot = 1; ipot <= npot; ++ipot) {
    const int npts = (ipot == 1) ? (int)jptr.size() : NANG;
    for (int lbeg = 0; lbeg < npts; lbeg += MPX) {
      const int npx = std::min(MPX, npts - lbeg);
      for (int ip = 0; ip < n; ++ip) {
        const double* C = Cn[ip].data();
        for (int i = 0; i < npx; ++i) {
          const double* r = (ipot == 1) ? &P.rmsh[3 * jptr[lbeg + i]] : Q[lbeg + i];
          poly[i][3] = r[0] + C[0];
          poly[i][2] = r[1] + C[1];
          poly[i][1] = r[2] + C[2];
          poly[i][0] = 1.0;
          poly[i][4] = poly[i][1] * poly[i][1];
          poly[i][6] = poly[i][2] * poly[i][2];
          poly[i][9] = poly[i][3] * poly[i][3];
        }
        double tmax = 0.0;
        for (int i = 0; i < npx; ++i) {
          xx[i] = delt[ip] * (poly[i][4] + poly[i][6] + poly[i][9]);
          tmax = std::max(tmax, xx[i]);
        }
        for (int i = 0; i < npx; ++i) chgd[i] = std::exp(-xx[i]);
        const double rmax1 = tmax / delt[ip];
        const double rmax2 = rmax1 * rmax1, rmax3 = rmax1 * rmax2, rmax4 = rmax2 * rmax2;
        double fmb[5];
        fmb[0] = std::sqrt(tmax);
        fmb[1] = fmb[0] * tmax;
        fmb[2] = fmb[1] * tmax;
        fmb[3] = fmb[2] * tmax;
        fmb[4] = fmb[3] * tmax;
        for (int m = 0; m <= 4; ++m) {
          if (tmax > TB[m]) fmb[m] = TF[m] / fmb[m];
          else fmb[m] = 1.0 / (2.0 * m + 1.0);
        }
        const double* cf = coef[ip].data();  // cf[k] = COEFICIENT(k+1)
        bool sscl[5] = {true, true, false, false, false};
        for (int I = 2; I <= 4; ++I)
          if (std::fabs(cf[I + 5 - 1] * rmax1 * fmb[2]) > EPSILON) sscl[2] = true;
        for (int I = 5; I <= 10; ++I)
          if (std::fabs(cf[I + 5 - 1] * rmax2 * fmb[2]) > EPSILON) sscl[2] = true;
        for (int I = 5; I <= 10; ++I)
          if (std::fabs(cf[I + 11 - 1] * rmax2 * fmb[3]) > EPSILON) sscl[3] = true;
        for (int I = 11; I <= 20; ++I)
          if (std::fabs(cf[I + 11 - 1] * rmax3 * fmb[3]) > EPSILON) sscl[3] = true;
        for (int I = 21; I <= 35; ++I)
          if (std::fabs(cf[I + 11 - 1] * rmax4 * fmb[4]) > EPSILON) sscl[4] = true;
        int maxfmt = 3;
        if (sscl[3]) maxfmt = 4;
        if (sscl[4]) maxfmt = 5;
        for (int i = 0; i < npx; ++i) {
          double* p = poly[i];
          p[5] = p[2] * p[1];
          p[7] = p[3] * p[1];
          p[8] = p[3] * p[2];
          p[10] = p[1] * p[4];
          p[11] = p[2] * p[4];
          p[12] = p[1] * p[6];
          p[13] = p[2] * p[6];
          p[14] = p[3] * p[4];
          p[15] = p[3] * p[5];
          p[16] = p[3] * p[6];
          p[17] = p[1] * p[9];
          p[18] = p[2] * p[9];
          p[19] = p[3] * p[9];
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
        if (ipot == 1) {
          // density, spin 1 only (spin-2 pair densities are zero in the SIC path)
          const int ngga = gga ? 10 : 1;
          for (int ii = 0; ii < ngga; ++ii)
            for (int i = 0; i < npx; ++i) addr[i][ii] = 0.0;
          for (int mpm = 0; mpm < 35; ++mpm) {
            double c = rhoc[ip][mpm];
            if (std::fabs(c) > 1.0e-14)
              for (int i = 0; i < npx; ++i) addr[i][0] = addr[i][0] + poly[i][mpm] * c;
          }
          if (gga) {
            for (int mpm = 0; mpm < 20; ++mpm)
              for (int ix = 1; ix <= 3; ++ix) {
                double c = rhod[ip][mpm][ix];
                if (std::fabs(c) > 1.0e-14)
                  for (int i = 0; i < npx; ++i) addr[i][ix] = addr[i][ix] + poly[i][mpm] * c;
              }
            for (int mpm = 0; mpm < 10; ++mpm)
              for (int ix = 4; ix <= 9; ++ix) {
                double c = rhod[ip][mpm][ix];
                if (std::fabs(c) > 1.0e-14)
                  for (int i = 0; i < npx; ++i) addr[i][ix] = addr[i][ix] + poly[i][mpm] * c;
              }
            const double d1x4 = dlt[ip] * 4.0, d2x4 = dlt[ip] * dlt[ip] * 4.0, d1x2 = dlt[ip] * 2.0;
            for (int i = 0; i < npx; ++i) {
              double* a = addr[i];
              const double* p = poly[i];
              a[4] = a[4] - d1x4 * p[3] * a[1] + (d2x4 * p[9] - d1x2) * a[0];
              a[5] = a[5] - d1x4 * p[2] * a[2] + (d2x4 * p[6] - d1x2) * a[0];
              a[6] = a[6] - d1x4 * p[1] * a[3] + (d2x4 * p[4] - d1x2) * a[0];
              a[7] = a[7] - d1x2 * p[2] * a[1] - d1x2 * p[3] * a[2] + d2x4 * p[8] * a[0];
              a[8] = a[8] - d1x2 * p[1] * a[1] - d1x2 * p[3] * a[3] + d2x4 * p[7] * a[0];
              a[9] = a[9] - d1x2 * p[2] * a[3] - d1x2 * p[1] * a[2] + d2x4 * p[5] * a[0];
              a[1] = a[1] - d1x2 * p[3] * a[0];
              a[2] = a[2] - d1x2 * p[2] * a[0];
              a[3] = a[3] - d1x2 * p[1] * a[0];
            }
          }
          for (int ii = 0; ii < ngga; ++ii)
            for (int i = 0; i < npx; ++i) addr[i][ii] = chgd[i] * addr[i][ii];
          for (int ii = 0; ii < ngga; ++ii)
            for (int i = 0; i < npx; ++i) {
              double& g = rhog[(size_t)ii * nmsh + jptr[lbeg + i]];
              g = g + addr[i][ii];
            }
        }
        for (int i = 0; i < npx; ++i) boys(maxfmt, xx[i], chgd[i], sss[i]);
        for (int i = 0; i < npx; ++i) {
          erp[i][0] = cf[0];
          erp[i][1] = cf[1];
          erp[i][2] = cf[2];
          erp[i][3] = 0.0;
          erp[i][4] = 0.0;
        }
        for (int I = 2; I <= 4; ++I) {
          double ct = cf[I + 2 - 1];
          for (int i = 0; i < npx; ++i) erp[i][1] = erp[i][1] + poly[i][I - 1] * ct;
        }
        if (sscl[2]) {
          for (int I = 2; I <= 4; ++I) {
            double ct = cf[I + 5 - 1];
            for (int i = 0; i < npx; ++i) erp[i][2] = erp[i][2] + poly[i][I - 1] * ct;
          }
          for (int I = 5; I <= 10; ++I) {
            double ct = cf[I + 5 - 1];
            for (int i = 0; i < npx; ++i) erp[i][2] = erp[i][2] + poly[i][I - 1] * ct;
          }
        }
        if (sscl[3]) {
          for (int I = 5; I <= 10; ++I) {
            double ct = cf[I + 11 - 1];
            for (int i = 0; i < npx; ++i) erp[i][3] = erp[i][3] + poly[i][I - 1] * ct;
          }
          for (int I = 11; I <= 20; ++I) {
            double ct = cf[I + 11 - 1];
            for (int i = 0; i < npx; ++i) erp[i][3] = erp[i][3] + poly[i][I - 1] * ct;
          }
        }
        if (sscl[4]) {
          for (int I = 21; I <= 35; ++I) {
            double ct = cf[I + 11 - 1];
            for (int i = 0; i < npx; ++i) erp[i][4] = erp[i][4] + poly[i][I - 1] * ct;
          }
        }
        for (int i = 0; i < npx; ++i) addp[i] = 0.0;
        for (int f = 0; f < 5; ++f)
          if (sscl[f])
            for (int i = 0; i < npx; ++i) addp[i] = addp[i] + erp[i][f] * sss[i][f];
        if (ipot == 1)
          for (int i = 0; i < npx; ++i) potnl[lbeg + i] = potnl[lbeg + i] + addp[i];
        else
          for (int i = 0; i < npx; ++i) asymptot[lbeg + i] = asymptot[lbeg + i] + addp[i];
      }
    }
  }
  for (size_t i = 0; i < jptr.size(); ++i) coulomb[jptr[i]] = coulomb[jptr[i]] + potnl[i];
  if (iptr.empty()) return;

  // multipole moments from the potential on the sphere of radius RCUT
  double qn[NANG][3];
  for (int ia = 0; ia < NANG; ++ia)
    for (int d = 0; d < 3; ++d) qn[ia][d] = L.ang[ia][d] * rcut;
  double hnorm = std::sqrt(qn[0][0] * qn[0][0] + qn[0][1] * qn[0][1] + qn[0][2] * qn[0][2]);
  double recipr[LM + 1];
  recipr[0] = hnorm;
  hnorm = 1.0 / hnorm;
  double rmoment[NMOM];
  for (int m = 0; m < NMOM; ++m) rmoment[m] = 0.0;
  for (int ia = 0; ia < NANG; ++ia) {
    double Y[NMOM];
    harmonics(LM, hnorm * qn[ia][0], hnorm * qn[ia][1], hnorm * qn[ia][2], Y);
    for (int m = 0; m < NMOM; ++m) rmoment[m] = rmoment[m] + L.w[ia] * Y[m] * asymptot[ia];
  }
  for (int l = 1; l <= LM; ++l) recipr[l] = recipr[0] * recipr[l - 1];
  {
    int mom = 0;
    for (int l = 0; l <= LM; ++l)
      for (int m = -l; m <= l; ++m, ++mom) rmoment[mom] = rmoment[mom] * recipr[l];
  }
  const int npts = (int)iptr.size();
  for (int lbeg = 0; lbeg < npts; lbeg += MPX) {
    const int npx = std::min(MPX, npts - lbeg);
    double q[MPX][3], recip[MPX][LM + 1];
    double ri1 = 0.0;
    for (int i = 0; i < npx; ++i) {
      const double* r = &P.rmsh[3 * iptr[lbeg + i]];
      for (int d = 0; d < 3; ++d) q[i][d] = r[d] + cgn[d];
      double h = q[i][0] * q[i][0] + q[i][1] * q[i][1] + q[i][2] * q[i][2];
      h = 1.0 / std::sqrt(h);
      recip[i][0] = h;
      if (h > ri1) ri1 = h;
      for (int d = 0; d < 3; ++d) q[i][d] = h * q[i][d];
    }
    double rtest[LM + 1];
    for (int l = 0; l <= LM; ++l) rtest[l] = std::pow(ri1, l + 1);
    bool skip[NMOM];
    int lm_max = 0;
    {
      int mom = 0;
      for (int l = 0; l <= LM; ++l)
        for (int m = -l; m <= l; ++m, ++mom) {
          double t = std::fabs((2 * l + 1) * rmoment[mom] * rtest[l]);
          if (t < 1.0e-12) skip[mom] = true;
          else {
            skip[mom] = false;
            lm_max = l;
          }
        }
    }
    for (int l = 1; l <= lm_max; ++l)
      for (int i = 0; i < npx; ++i) recip[i][l] = recip[i][0] * recip[i][l - 1];
    for (int i = 0; i < npx; ++i) {
      double Y[NMOM];
      harmonics(lm_max, q[i][0], q[i][1], q[i][2], Y);
      double potlr = 0.0;
      int mom = 0;
      for (int l = 0; l <= lm_max; ++l)
        for (int m = -l; m <= l; ++m, ++mom)
          if (!skip[mom]) potlr = potlr + rmoment[mom] * Y[mom] * recip[i][l];
      coulomb[iptr[lbeg + i]] = coulomb[iptr[lbeg + i]] + potlr;
    }
  }
}

// ---------------------------------------------------------------------------
// COUPOT_SIC (coupot_sic.F:9-856), serial branch, MXXD=0 (one FO).
// cfo: local FO coefficients (nbasis) of the orbital.
// ---------------------------------------------------------------------------
struct BatchPlan {
  // enumerate pairs and batches in the reference order; callback per flush
};

template <class Flush>
void coupot_pairs(const Problem& P, const double* cfo, int nspn, Flush&& flush, Stats* st,
                  const double* dmfull = nullptr) {
  const double ZED = 1.0e-30;
  // centres: atoms (C1 symmetry: one site per atom) plus origin if far from atoms
  std::vector<std::array<double, 3>> center;
  double dmin = 1.0e30;
  for (int a = 0; a < P.natoms; ++a) {
    std::array<double, 3> c = {P.rat[3 * a], P.rat[3 * a + 1], P.rat[3 * a + 2]};
    center.push_back(c);
    double dist = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    if (dist < dmin) dmin = dist;
  }
  int mcnt = (int)center.size();
  if (std::sqrt(dmin) > 0.7) {
    center.push_back({0.0, 0.0, 0.0});
    mcnt++;
  }
  const int nclass = mcnt + 1;  // index mcnt == weird (MCNT+1)
  std::vector<std::vector<PairRec>> buf((size_t)nclass * 3);
  const int mxsiz = MXPR;
  for (int ia = 0; ia < P.natoms; ++ia) {
    const int ti = P.atype[ia];
    const double* AI = &P.rat[3 * ia];
    for (int ja = ia; ja < P.natoms; ++ja) {
      const int tj = P.atype[ja];
      const double* AJ = &P.rat[3 * ja];
      const double times_sites = (ja > ia) ? 2.0 : 1.0;
      const double rarg = (AI[0] - AJ[0]) * (AI[0] - AJ[0]) + (AI[1] - AJ[1]) * (AI[1] - AJ[1]) +
                          (AI[2] - AJ[2]) * (AI[2] - AJ[2]);
      for (int ialp = 0; ialp < P.nbare[ti]; ++ialp) {
        const double ai = P.alp(ti, ialp);
        const int jbeg = (ia == ja) ? ialp : 0;
        for (int jalp = jbeg; jalp < P.nbare[tj]; ++jalp) {
          const double times_alpha = (ia == ja && jalp > ialp) ? 2.0 : 1.0;
          const double aj = P.alp(tj, jalp);
          const double rcalp = 1.0 / (ai + aj);
          const double arg = ai * aj * rcalp * rarg;
          if (arg > CUTEXP) continue;
          double C[3];
          for (int d = 0; d < 3; ++d) C[d] = (ai * AI[d] + aj * AJ[d]) * rcalp;
          double dm = 1.0e30;
          int minc = 0;
          for (int ic = 0; ic < mcnt; ++ic) {
            double dist = std::sqrt((C[0] - center[ic][0]) * (C[0] - center[ic][0]) +
                                    (C[1] - center[ic][1]) * (C[1] - center[ic][1]) +
                                    (C[2] - center[ic][2]) * (C[2] - center[ic][2]));
            if (dist < dm) {
              dm = dist;
              minc = ic;
            }
          }
          const double rlen = (ai + aj) * dm * dm;
          if (rlen > 0.5) minc = mcnt;
          if (ai + aj < 3.0) minc = mcnt;
          int lng = 0;
          if (ai + aj > 10.0) lng = 1;
          if (ai + aj > 40.0) lng = 2;
          // density matrix (coupot_sic.F:366-482)
          int muimax = 0, mujmax = 0;
          for (int l = 0; l <= P.lmax[ti]; ++l)
            for (int mu = kShift[l]; mu < kShift[l] + kNcomp[l]; ++mu)
              for (int ib = 0; ib < P.ncon[ti * 3 + l]; ++ib)
                if (std::fabs(P.bcon(ti, l, ib, ialp)) > ZED && mu + 1 > muimax) muimax = mu + 1;
          for (int l = 0; l <= P.lmax[tj]; ++l)
            for (int mu = kShift[l]; mu < kShift[l] + kNcomp[l]; ++mu)
              for (int ib = 0; ib < P.ncon[tj * 3 + l]; ++ib)
                if (std::fabs(P.bcon(tj, l, ib, jalp)) > ZED && mu + 1 > mujmax) mujmax = mu + 1;
          PairRec pr;
          pr.a = ai;
          pr.b = aj;
          for (int d = 0; d < 3; ++d) {
            pr.A[d] = AI[d];
            pr.B[d] = AJ[d];
          }
          for (int i = 0; i < 10; ++i)
            for (int j = 0; j < 10; ++j) pr.dmat[i][j] = 0.0;
          int iloc = 0;
          for (int li = 0; li <= P.lmax[ti]; ++li)
            for (int mui = kShift[li]; mui < kShift[li] + kNcomp[li]; ++mui)
              for (int ib = 0; ib < P.ncon[ti * 3 + li]; ++ib, ++iloc) {
                int jloc = 0;
                // ADD: the FO's rank-1 block (coupot_sic.F:262-281) or, for the
                // DFT density, the occupied orbitals' density matrix (coupot1.F:380-395)
                const double ci = dmfull ? 0.0 : cfo[P.aoff[ia] + iloc];
                for (int lj = 0; lj <= P.lmax[tj]; ++lj)
                  for (int muj = kShift[lj]; muj < kShift[lj] + kNcomp[lj]; ++muj)
                    for (int jb = 0; jb < P.ncon[tj * 3 + lj]; ++jb, ++jloc) {
                      const double add = dmfull ? dmfull[(size_t)(P.aoff[ia] + iloc) * P.nbasis + P.aoff[ja] + jloc]
                                                : ci * cfo[P.aoff[ja] + jloc];
                      const double prod = P.bcon(ti, li, ib, ialp) * P.bcon(tj, lj, jb, jalp);
                      pr.dmat[mui][muj] = pr.dmat[mui][muj] + prod * add;
                    }
              }
          for (int j = 0; j < mujmax; ++j)
            for (int i = 0; i < muimax; ++i) pr.dmat[i][j] = pr.dmat[i][j] * times_sites * times_alpha;
          if (st) st->pairs++;
          if (minc == mcnt && st) st->weird++;
          auto& b = buf[(size_t)minc * 3 + lng];
          b.push_back(pr);
          if ((int)b.size() * nspn == mxsiz) {
            flush(b, minc == mcnt);
            b.clear();
          }
        }
      }
    }
  }
  for (int lng = 0; lng < 3; ++lng)
    for (int minc = 0; minc < nclass; ++minc) {
      auto& b = buf[(size_t)minc * 3 + lng];
      if (!b.empty()) {
        flush(b, minc == mcnt);
        b.clear();
      }
    }
}

int coupot_sic(const Problem& P, const double* cfo, bool exact, double* coulomb,
               double* rhog /*[10][nmsh]*/, Stats* st) {
  const int nspn = P.nspn;
  const bool gga = P.gga();
  for (int i = 0; i < P.nmsh; ++i) coulomb[i] = 0.0;
  for (size_t i = 0; i < (size_t)10 * P.nmsh; ++i) rhog[i] = 0.0;
  auto flush = [&](const std::vector<PairRec>& b, bool weird) {
    if (st) st->batches++;
    if (weird) {
      for (const auto& pr : b) {
        std::vector<PairRec> one(1, pr);
        poisson1(P, one, nspn, gga, exact, coulomb, rhog, st);
      }
    } else {
      poisson1(P, b, nspn, gga, exact, coulomb, rhog, st);
    }
  };
  coupot_pairs(P, cfo, nspn, flush, st);
  return 0;
}

// ---------------------------------------------------------------------------
// Exchange-correlation functionals (pw91ex.f, pbeex.f, pw91lc.f+gcor.f,
// pw91nc.f, pbecor.f+gcor2.f).
// ---------------------------------------------------------------------------
void pw91ex(double dkf, double s, double u, double v, double& exl, double& exn, double& vx) {
  const double A1 = 0.19645, A2 = 0.27430, A3 = 0.15084, A4 = 100.0;
  const double AX = -0.238732414, A = 7.7956, B1 = 0.004;
  const double THRD4 = 1.3333333333333333;
  double fac = AX * dkf;
  double s2 = s * s, s3 = s2 * s, s4 = s2 * s2;
  double as = A * s;
  double pa = std::sqrt(1.0 + as * as);
  double p0 = as / pa;
  double p1 = A1 * std::log(as + pa);
  double p2 = A3 * std::exp(-A4 * s2);
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

void pbeex(int mode, double rho, double s, double u, double v, double& exl, double& exn, double& vx) {
  const double THRD = 1.0 / 3.0, THRD4 = 4.0 / 3.0;
  const double AX = -0.738558766382022405884230032680836;
  const double UM = 0.2195149727645171;
  double uk = (mode == 2) ? 1.2450 : 0.8040;
  double ul = UM / uk;
  double exunif = AX * std::pow(rho, THRD);
  double s2 = s * s, p0, fxpbe;
  if (mode == 3) {
    p0 = std::exp(-ul * s2);
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

void gcor(double A, double A1, double B1, double B2, double B3, double B4, double rs, double& gg,
          double& ggrs) {
  double q0 = -2 * A * (1.0 + A1 * rs);
  double rs12 = std::sqrt(rs);
  double rs32 = rs12 * rs12 * rs12;
  double q1 = 2 * A * (B1 * rs12 + B2 * rs + B3 * rs32 + B4 * rs * rs);
  double q2 = std::log(1.0 + 1.0 / q1);
  gg = q0 * q2;
  double q3 = A * (B1 / rs12 + 2 * B2 + 3 * B3 * rs12 + 4 * B4 * rs);
  ggrs = -2 * A * A1 * q2 - q0 * q3 / (q1 * q1 + q1);
}

void gcor2(double A, double A1, double B1, double B2, double B3, double B4, double rtrs, double& gg,
           double& ggrs) {
  double q0 = -2.0 * A * (1.0 + A1 * rtrs * rtrs);
  double q1 = 2.0 * A * rtrs * (B1 + rtrs * (B2 + rtrs * (B3 + B4 * rtrs)));
  double q2 = std::log(1.0 + 1.0 / q1);
  gg = q0 * q2;
  double q3 = A * (B1 / rtrs + 2.0 * B2 + rtrs * (3.0 * B3 + 4.0 * B4 * rtrs));
  ggrs = -2.0 * A * A1 * q2 - q0 * q3 / (q1 * (1.0 + q1));
}

struct PW91Gas {
  double g, ec, ecrs, eczet;
};

void pw91lc(double rs, double zet, double& ec, double& vcup, double& vcdn, double& ecrs, double& eczet,
            double& alfc) {
  const double GAMR = 1.92366105, FZZR = 0.58482234;
  const double THRD = 0.333333333333, THRD4 = 1.333333333333;
  double zetpr = std::pow(1.0 + zet, THRD);
  double zetmr = std::pow(1.0 - zet, THRD);
  double f = (std::pow(zetpr, 4) + std::pow(zetmr, 4) - 2.0) * GAMR;
  double eu, eurs, ep, eprs, alfm, alfrsm;
  gcor(0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294, rs, eu, eurs);
  gcor(0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517, rs, ep, eprs);
  gcor(0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671, rs, alfm, alfrsm);
  alfc = -alfm;
  double z3 = zet * zet * zet, z4 = z3 * zet;
  ec = eu * (1.0 - f * z4) + ep * f * z4 - alfm * f * (1.0 - z4) * FZZR;
  ecrs = eurs * (1.0 - f * z4) + eprs * f * z4 - alfrsm * f * (1.0 - z4) * FZZR;
  double fz = THRD4 * (zetpr - zetmr) * GAMR;
  eczet = 4.0 * z3 * f * (ep - eu + alfm * FZZR) + fz * (z4 * ep - z4 * eu - (1.0 - z4) * alfm * FZZR);
  double comm = ec - rs * ecrs * THRD - zet * eczet;
  vcup = comm + eczet;
  vcdn = comm - eczet;
}

void pw91nc(double rs, double zet, double t, double uu, double vv, double ww, const PW91Gas& gas,
            double& h, double& dvcup, double& dvcdn) {
  const double XNU = 15.75592, CC0 = 0.004235, CX = -0.001667212;
  const double C1 = 0.002568, C2 = 0.023266, C3 = 7.389e-6, C4 = 8.723;
  const double C5 = 0.472, C6 = 7.389e-2, A4 = 100.0;
  const double BET = 0.0667263, BETR = 14.98659;
  const double DELT = 2.697586, DELTR = 0.3707018;
  const double RS2R0 = 0.66343644;
  const double THRD = 0.3333333333333333, THRD2 = 0.6666666666666667;
  const double SIXTH = 0.1666666666666667, THDSEV = 0.4285714285714286;
  const double g = gas.g, ec = gas.ec, ecrs = gas.ecrs, eczet = gas.eczet;
  double gr = 1.0 / g;
  double g3 = g * g * g, g4 = g3 * g;
  double g3r = gr * gr * gr, g4r = g3r * gr;
  double pon = -DELT * ec * g3r * BETR;
  double bex = std::exp(pon) - 1.0;
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
  double r3 = std::exp(-r1 * t2);
  double h0 = g3 * BET * DELTR * std::log(1.0 + DELT * q4 * t2 / q5);
  double h1 = r3 * r2 * t2;
  h = h0 + h1;
  if ((1.0 - std::fabs(zet)) < 1.0e-10) zet = (1.0 - 1.0e-10) * zet;
  double ccrs = (C2 + 2 * C3 * rs) * q7r - q6 * (C4 + 2 * C5 * rs + 3 * C6 * rs2) * q7r * q7r;
  double rsthrd = rs * THRD;
  double r4 = rsthrd * ccrs / coeff;
  double gz = (std::pow(1.0 + zet, -THRD) - std::pow(1.0 - zet, -THRD)) * THRD;
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

void pbecor(double rs, double zet, double t, double uu, double vv, double ww, double& ec, double& vcup,
            double& vcdn, double& h, double& dvcup, double& dvcdn) {
  const double THRD = 1.0 / 3.0, THRDM = -THRD, THRD2 = 2.0 * THRD, SIXTHM = THRDM / 2.0;
  const double THRD4 = 4.0 * THRD;
  const double GAM = 0.5198420997897463295344212145565;
  const double FZZ = 8.0 / (9.0 * GAM);
  const double GAMMA = 0.03109069086965489503494086371273;
  const double BET = 0.06672455060314922, DELT = BET / GAMMA;
  const double ETA = 1.0e-12;
  (void)THRD2;
  double rtrs = std::sqrt(rs);
  double eu, eurs, ep, eprs, alfm, alfrsm;
  gcor2(0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294, rtrs, eu, eurs);
  gcor2(0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517, rtrs, ep, eprs);
  gcor2(0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671, rtrs, alfm, alfrsm);
  double z4 = std::pow(zet, 4);
  double f = (std::pow(1.0 + zet, THRD4) + std::pow(1.0 - zet, THRD4) - 2.0) / GAM;
  ec = eu * (1.0 - f * z4) + ep * f * z4 - alfm * f * (1.0 - z4) / FZZ;
  double ecrs = eurs * (1.0 - f * z4) + eprs * f * z4 - alfrsm * f * (1.0 - z4) / FZZ;
  double fz = THRD4 * (std::pow(1.0 + zet, THRD) - std::pow(1.0 - zet, THRD)) / GAM;
  double eczet = 4.0 * (zet * zet * zet) * f * (ep - eu + alfm / FZZ) + fz * (z4 * ep - z4 * eu - (1.0 - z4) * alfm / FZZ);
  double comm = ec - rs * ecrs / 3.0 - zet * eczet;
  vcup = comm + eczet;
  vcdn = comm - eczet;
  double g = (std::pow(1.0 + zet, 2.0 * THRD) + std::pow(1.0 - zet, 2.0 * THRD)) / 2.0;
  double g3 = g * g * g;
  double pon = -ec / (g3 * GAMMA);
  double b = DELT / (std::exp(pon) - 1.0);
  double b2 = b * b;
  double t2 = t * t, t4 = t2 * t2;
  double q4 = 1.0 + b * t2;
  double q5 = 1.0 + b * t2 + b2 * t4;
  h = g3 * (BET / DELT) * std::log(1.0 + DELT * q4 * t2 / q5);
  double g4 = g3 * g;
  double t6 = t4 * t2;
  double rsthrd = rs / 3.0;
  double gz = (std::pow((1.0 + zet) * (1.0 + zet) + ETA, SIXTHM) - std::pow((1.0 - zet) * (1.0 - zet) + ETA, SIXTHM)) / 3.0;
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

// ---------------------------------------------------------------------------
// SCAN meta-GGA (scan.f, the form called by call_mgga.f90 for IDFTYP=11).
// Energies are per particle; the derivatives are those of rho*e with respect
// to rho, |grad rho| and tau, as the reference returns them.
// ---------------------------------------------------------------------------
// Exchange enhancement factor Fx(p, alpha) and its first derivatives
// (metaggafx, scan.f:304-470; the second derivatives there are unused).
void scan_fx(double p, double a, double& fx, double& fx_p, double& fx_a) {
  const double K1 = 0.065, C1 = 0.667, C2 = 0.800, D1 = 1.240;
  const double K0 = 0.1740, A1 = 4.9479, MU = 10.0 / 81.0, B1 = 0.156632, B2 = 0.12083, B3 = 0.5;
  const double oma = 1.0 - a, oma2 = oma * oma;
  const double hx0 = 1.0 + K0;
  const double b4 = MU * MU / K1 - 0.112654;
  double wfac, dwfac;
  if (b4 > 0.0) {
    const double e = std::exp(-b4 * p / MU);
    wfac = b4 * p * p * e;
    dwfac = b4 * p * e * (2.0 - b4 * p / MU);
  } else {
    const double e = std::exp(b4 * p / MU);
    wfac = b4 * p * p * e;
    dwfac = b4 * p * e * (2.0 + b4 * p / MU);
  }
  const double ea = std::exp(-B3 * oma2);
  const double vfac = B1 * p + B2 * oma * ea;
  const double yfac = MU * p + wfac + vfac * vfac;
  const double den = 1.0 + yfac / K1;
  const double hx1 = 1.0 + K1 - K1 / den;
  double fa = 0.0, dfa = 0.0;
  if (a < 1.0) {
    fa = std::exp(-C1 * a / oma);
    dfa = -C1 * std::exp(-C1 * a / oma) / (oma * oma);
  } else if (a > 1.0) {
    fa = -D1 * std::exp(C2 / oma);
    dfa = -C2 * D1 * std::exp(C2 / oma) / (oma * oma);
  }
  double gx = 1.0, dgx = 0.0;
  if (p > 0.0) {
    const double p14 = std::pow(p, 0.25);
    gx = 1.0 - std::exp(-A1 / p14);
    dgx = -A1 / 4.0 / p / p14 * std::exp(-A1 / p14);
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

// Spin-unpolarised SCAN exchange (VSCANxUNP, scan.f:172-287) at density rho,
// |grad rho| = drho, kinetic energy density tau.  The reference's pi here is
// the literal 3.1415927.
void scan_x_unp(double rho, double drho, double tau, double& ex, double& vx, double& vxdd, double& amux) {
  const double PI = 3.1415927, PISQ = PI * PI;
  const double AX = -0.7385587663820224058842300326808360;
  const double TH = 1.0 / 3.0, TH2 = 2.0 * TH, TH4 = 4.0 * TH, TH5 = 1.0 + TH2, TH8 = 1.0 + TH5;
  const double tauw = drho * drho / rho / 8.0;
  const double exunif = AX * std::pow(rho, TH);
  const double exlda = exunif * rho;
  const double exdlda = exunif * TH4;
  const double c3p = std::pow(3.0 * PISQ, TH2);
  const double p = drho * drho / (4.0 * c3p * std::pow(rho, TH8));
  const double tunif = 3.0 / 10.0 * std::pow(3.0 * PI * PI, TH2) * std::pow(rho, TH5);
  const double alpha = (tau - tauw) / tunif;
  const double dpd = -TH8 * p / rho;
  const double dpdd = 2.0 * p / drho;
  const double dad = -tau * std::pow(3.0 * PI * PI * rho, TH2) / (2.0 * tunif * tunif) +
                     drho * drho / std::pow(rho, 11.0 / 3.0) * (10.0 / 9.0 / std::pow(3.0 * PI * PI, TH2));
  const double dadd = -drho / (4.0 * rho * tunif);
  const double dadt = 1.0 / tunif;
  double fx, fxp, fxa;
  scan_fx(p, alpha, fx, fxp, fxa);
  vx = exdlda * fx + exlda * (fxp * dpd + fxa * dad);
  vxdd = exlda * (fxp * dpdd + fxa * dadd);
  amux = exlda * (fxa * dadt);
  ex = exunif * fx;
}

// GCOR22 (scan.f:1155-1166): PW92 interpolation and its rs derivative.
void scan_gcor(double A, double A1, double B1, double B2, double B3, double B4, double rtrs, double& gg,
               double& ggrs) {
  const double q0 = -2.0 * A * (1.0 + A1 * rtrs * rtrs);
  const double q1 = 2.0 * A * rtrs * (B1 + rtrs * (B2 + rtrs * (B3 + B4 * rtrs)));
  const double q2 = std::log(1.0 + 1.0 / q1);
  gg = q0 * q2;
  const double q3 = A * (B1 / rtrs + 2.0 * B2 + rtrs * (3.0 * B3 + 4.0 * B4 * rtrs));
  ggrs = -2.0 * A * A1 * q2 - q0 * q3 / (q1 * (1.0 + q1));
}

// PW92 LSD correlation and its spin potentials (the LSD part of
// CORPBE_revtpss, scan.f:700-790).
void scan_lsd(double rs, double zet, double& ec, double& vcup, double& vcdn) {
  const double TH = 1.0 / 3.0, TH4 = 4.0 * TH;
  const double GAM = 0.51984209978974632953442121455650, FZZ = 8.0 / (9.0 * GAM);
  const double rtrs = std::sqrt(rs);
  double eu, eurs, ep, eprs, alfm, alfrsm;
  scan_gcor(0.03109070, 0.213700, 7.59570, 3.58760, 1.63820, 0.492940, rtrs, eu, eurs);
  scan_gcor(0.015545350, 0.205480, 14.11890, 6.19770, 3.36620, 0.625170, rtrs, ep, eprs);
  scan_gcor(0.01688690, 0.111250, 10.3570, 3.62310, 0.880260, 0.496710, rtrs, alfm, alfrsm);
  const double z4 = zet * zet * zet * zet;
  const double f = (std::pow(1.0 + zet, TH4) + std::pow(1.0 - zet, TH4) - 2.0) / GAM;
  ec = eu * (1.0 - f * z4) + ep * f * z4 - alfm * f * (1.0 - z4) / FZZ;
  const double ecrs = eurs * (1.0 - f * z4) + eprs * f * z4 - alfrsm * f * (1.0 - z4) / FZZ;
  const double fz = TH4 * (std::pow(1.0 + zet, TH) - std::pow(1.0 - zet, TH)) / GAM;
  const double eczet =
      4.0 * (zet * zet * zet) * f * (ep - eu + alfm / FZZ) + fz * (z4 * ep - z4 * eu - (1.0 - z4) * alfm / FZZ);
  const double comm = ec - rs * ecrs / 3.0 - zet * eczet;
  vcup = comm + eczet;
  vcdn = comm - eczet;
}

// Common spin/density variables of CORGGA_0 and CORGGA_1.
struct ScanSpin {
  double rt, yc, zeta, dz1, dz2, rs, drs, s, ds;
};
ScanSpin scan_spin(double ru, double rd, double dru, double drd, double drt) {
  const double PI = 3.141592653589793238, PISQ = PI * PI, TH = 1.0 / 3.0, TH4 = 4.0 * TH;
  ScanSpin v;
  v.rt = ru + rd;
  v.yc = (drt * drt - dru * dru - drd * drd) / 2.0;
  v.zeta = std::min(std::max((ru - rd) / v.rt, -0.99999999999990), 0.99999999999990);
  v.dz1 = 2.0 * rd / (v.rt * v.rt);
  v.dz2 = -2.0 * ru / (v.rt * v.rt);
  const double dthrd = std::exp(std::log(v.rt) * TH);
  v.rs = std::pow(0.750 / PI, TH) / dthrd;
  v.drs = -TH / v.rt * v.rs;
  v.s = drt / (2.0 * std::pow(3.0 * PISQ, TH) * std::pow(v.rt, TH4));
  v.ds = -TH4 * v.s / v.rt;
  return v;
}

// epsilon_c^1: the PBE-like correlation of SCAN (CORGGA_1, scan.f:841-1000).
// out[0] energy per particle, out[1..2] d/d rho_up,dn, out[3..4] d/d |grad rho_up,dn|.
void scan_c1(double ru, double rd, double dru, double drd, double drt, double out[5]) {
  const double PI = 3.141592653589793238, TH = 1.0 / 3.0;
  const double GAMMA = 0.031090690869654895034940863712730, BETA_MB = 0.066724550603149220;
  const ScanSpin v = scan_spin(ru, rd, dru, drd, drt);
  const double zeta = v.zeta, rs = v.rs;
  const double phi = (std::exp((2.0 * TH) * std::log(1.0 + zeta)) + std::exp((2.0 * TH) * std::log(1.0 - zeta))) / 2.0;
  const double dphi = TH * (std::pow(1.0 + zeta, -TH) - std::pow(1.0 - zeta, -TH));
  const double afix = std::sqrt(PI / 4.0) * std::pow(9.0 * PI / 4.0, 1.0 / 6.0);
  const double gngnu = 1.0 / (2.0 * drt) * (2.0 * dru + 2.0 * v.yc / dru);
  const double gngnd = 1.0 / (2.0 * drt) * (2.0 * drd + 2.0 * v.yc / drd);
  const double dsdd1 = v.s / drt * gngnu, dsdd2 = v.s / drt * gngnd;
  const double t = afix * v.s / std::sqrt(rs) / phi;
  const double t2 = t * t;
  const double den_t = phi * phi * std::pow(rs, 1.5);
  const double dtd1 = afix * (phi * rs * v.ds - 0.5 * v.s * phi * v.drs - v.s * rs * dphi * v.dz1) / den_t;
  const double dtd2 = afix * (phi * rs * v.ds - 0.5 * v.s * phi * v.drs - v.s * rs * dphi * v.dz2) / den_t;
  const double dtdd1 = afix * dsdd1 / (std::sqrt(rs) * phi), dtdd2 = afix * dsdd2 / (std::sqrt(rs) * phi);
  double ec, vu, vd;
  scan_lsd(rs, zeta, ec, vu, vd);
  const double dec_dz = (vu - vd) / 2.0;
  const double dec_drs = (ec - zeta * dec_dz - (vu + vd) / 2.0) * 3.0 / rs;
  const double bnum = 1.0 + 0.10 * rs, bden = 1.0 + 0.17780 * rs;
  const double beta = BETA_MB * bnum / bden;
  const double dbeta = BETA_MB * (bden * 0.10 - bnum * 0.17780) / (bden * bden);
  const double phi3 = phi * phi * phi;
  const double w = std::exp(-ec / (phi3 * GAMMA)) - 1.0;
  const double dw_drs = -(w + 1.0) * dec_drs / (GAMMA * phi3);
  const double dw_dz = -(w + 1.0) / (GAMMA * phi3) * (dec_dz - 3.0 * ec * dphi / phi);
  const double A = beta / (GAMMA * w);
  const double dA_drs = (w * dbeta - beta * dw_drs) / (GAMMA * w * w);
  const double dA_dz = -beta * dw_dz / (GAMMA * w * w);
  const double V = A * t2;
  const double dV_drs = t2 * dA_drs, dV_dz = t2 * dA_dz, dV_dt = 2.0 * A * t;
  const double g = 1.0 / std::pow(1.0 + 4.0 * V, 0.250);
  const double dg_dv = -1.0 / std::pow(1.0 + 4.0 * V, 1.250);
  const double hcore = 1.0 + w * (1.0 - g);
  const double ah = GAMMA * phi3;
  const double h = ah * std::log(hcore);
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

// epsilon_c^0: the single-orbital correlation of SCAN (CORGGA_0,
// scan.f:1008-1150).  Clamps drt to 1e-100 like the reference, which passes the
// clamped value on to CORGGA_1 (the returned drt).  Same outputs as scan_c1.
void scan_c0(double ru, double rd, double dru, double drd, double& drt, double out[5]) {
  const double B1 = 0.0285764, B2 = 0.0889, B3 = 0.125541, KAI = 0.12802585262625815;
  const double TH = 1.0 / 3.0, TH4 = 4.0 * TH;
  const ScanSpin v = scan_spin(ru, rd, dru, drd, drt);
  const double zeta = v.zeta, rs = v.rs;
  if (std::fabs(drt) < 1.0e-100) drt = 1.0e-100;
  const double gngnu = 1.0 / (2.0 * drt) * (2.0 * dru + 2.0 * v.yc / dru);
  const double gngnd = 1.0 / (2.0 * drt) * (2.0 * drd + 2.0 * v.yc / drd);
  const double dsdd1 = v.s / drt * gngnu, dsdd2 = v.s / drt * gngnd;
  const double rsh = std::sqrt(rs);
  const double ec0 = -B1 / (1.0 + B2 * rsh + B3 * rs);
  const double dec0 = (B3 + B2 / rsh / 2.0) * ec0 * ec0 / B1;
  const double dx = (std::pow(1.0 + zeta, TH4) + std::pow(1.0 - zeta, TH4)) / 2.0;
  const double ddx = 2.0 * (std::pow(1.0 + zeta, TH) - std::pow(1.0 - zeta, TH)) / 3.0;
  const double z12 = std::pow(zeta, 12.0);
  const double gc = (1.0 - 2.363 * (dx - 1.0)) * (1.0 - z12);
  const double dgc = -(1.0 - 2.363 * (dx - 1.0)) * 12.0 * std::pow(zeta, 11.0) - 2.363 * ddx * (1.0 - z12);
  const double w0 = std::exp(-ec0 / B1) - 1.0;
  const double dw0 = -(w0 + 1.0) * dec0 / B1;
  const double ginf = 1.0 / std::pow(1.0 + 4.0 * KAI * v.s * v.s, 0.25);
  const double dginf = -2.0 * KAI * v.s * std::pow(ginf, 5.0);
  const double hcore = 1.0 + w0 * (1.0 - ginf);
  const double h0 = B1 * std::log(hcore);
  const double dh0_drs = B1 * dw0 * (1.0 - ginf) / hcore;
  const double dh0_ds = -B1 * w0 * dginf / hcore;
  const double de_dz = (ec0 + h0) * dgc, de_drs = (dec0 + dh0_drs) * gc, de_ds = dh0_ds * gc;
  out[0] = (ec0 + h0) * gc;
  out[1] = de_dz * v.dz1 + de_drs * v.drs + de_ds * v.ds;
  out[2] = de_dz * v.dz2 + de_drs * v.drs + de_ds * v.ds;
  out[3] = de_ds * dsdd1;
  out[4] = de_ds * dsdd2;
}

// SCAN correlation (VSCANc -> Vmetaggac, scan.f:486-697): ec per particle,
// vc[0..1] d(rho ec)/d rho_up,dn, vcdd[0..1] d(rho ec)/d|grad rho_up,dn|,
// amu d(rho ec)/d tau (the same for both spins).
void scan_c(double ru, double rd, double dru, double drd, double drt, double tauu, double taud, double& ec,
            double vc[2], double vcdd[2], double& amu) {
  const double PI = 3.141592653589793238, PISQ = PI * PI, TH = 1.0 / 3.0, TH2 = 2.0 * TH, TH5 = 1.0 + TH2;
  const double C1 = 0.640, C2 = 1.500, D1 = 0.700;
  if (dru == 0.0) dru = 1.0e-100;
  if (drd == 0.0) drd = 1.0e-100;
  const double rt = ru + rd;
  const double yc = (drt * drt - dru * dru - drd * drd) / 2.0;
  const double tauw = 1.0 / 8.0 * (drt * drt / rt);
  const double tau = tauu + taud;
  const double zeta = std::min(std::max((ru - rd) / rt, -0.99999999999990), 0.99999999999990);
  const double dsz = (std::pow(1.0 + zeta, TH5) + std::pow(1.0 - zeta, TH5)) / 2.0;
  const double tau0 = 0.30 * std::pow(3.0 * PISQ, TH2) * std::pow(rt, TH5) * dsz;
  const double alpha = (tau - tauw) / tau0;
  const double dz1 = 2.0 * rd / (rt * rt), dz2 = -2.0 * ru / (rt * rt);
  const double ddsz = TH5 * (std::pow(1.0 + zeta, TH2) - std::pow(1.0 - zeta, TH2)) / 2.0;
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
    f = std::exp(C1 * alpha / (alpha - 1.0));
    df = -C1 * f / ((alpha - 1.0) * (alpha - 1.0));
  } else if (alpha > 1.0) {
    f = -D1 * std::exp(-C2 / (alpha - 1.0));
    df = C2 * f / ((alpha - 1.0) * (alpha - 1.0));
  }
  double e0[5], e1[5];
  scan_c0(ru, rd, dru, drd, drt, e0);
  scan_c1(ru, rd, dru, drd, drt, e1);
  const double dE = e0[0] - e1[0];
  const double epp = e1[0] + f * dE;
  const double d1 = e1[1] + dE * df * da1 + f * (e0[1] - e1[1]);
  const double d2 = e1[2] + dE * df * da2 + f * (e0[2] - e1[2]);
  const double dd1 = e1[3] + dE * df * dadd1 + f * (e0[3] - e1[3]);
  const double dd2 = e1[4] + dE * df * dadd2 + f * (e0[4] - e1[4]);
  const double dt = dE * df * dat;
  vc[0] = epp + rt * d1;
  vc[1] = epp + rt * d2;
  vcdd[0] = rt * dd1;
  vcdd[1] = rt * dd2;
  amu = rt * dt;
  ec = epp;
}

// SUBVLXC (subvlxc_libxc.F90:23-508, built-in functionals) for one point,
// NSPN=2 layout: rht[ispn][10] with rht[0] the total and rht[1] the spin-down
// density channels.  Adds to vxc[0..1] and the energy accumulators.  SCAN
// (IDFTYP 11) also takes the spin kinetic energy densities tau[0..1] and adds
// the spin-up Hamiltonian ingredients MIXINS(1..4) (call_mgga.f90) to mixin.
void subvlxc_point(const Problem& P, double rht[2][10], double wgt, double* vxc, double* ex4,
                   const double* tau = nullptr, double* mixin = nullptr) {
  const int nspn = 2;
  const bool isgga = P.igga[0] >= 1 || P.igga[1] >= 1;
  const int ngrad = isgga ? 10 : 1;
  const double THIRD = 0.3333333333333333, THIRD2 = 0.6666666666666667;
  const double TRPI2 = 29.6088132032680759, FRDPI = 1.2732395447351627, DKF2RS = 1.9191582926775128;
  const double EPS = 1.0e-20;
  const double ispfac = 2.0 / nspn;
  double dg2[3] = {0, 0, 0}, dgg[3] = {0, 0, 0}, dlp[3] = {0, 0, 0}, den[3];
  for (int s = 0; s < nspn; ++s) {
    if (rht[s][0] < 0.0) rht[s][0] = 0.0;
    if (rht[s][0] > rht[0][0]) rht[s][0] = rht[0][0];
  }
  (void)ngrad;
  den[0] = rht[0][0];
  den[2] = den[0] * 0.5;
  den[2] = rht[nspn - 1][0];
  den[1] = den[0] - den[2];
  if (isgga) {
    dg2[0] = rht[0][1] * rht[0][1] + rht[0][2] * rht[0][2] + rht[0][3] * rht[0][3];
    dg2[1] = dg2[0] * 0.25;
    dg2[2] = dg2[1];
    dgg[0] = rht[0][4] * rht[0][1] * rht[0][1] + rht[0][5] * rht[0][2] * rht[0][2] +
             rht[0][6] * rht[0][3] * rht[0][3] +
             2 * (rht[0][7] * rht[0][1] * rht[0][2] + rht[0][8] * rht[0][1] * rht[0][3] +
                  rht[0][9] * rht[0][2] * rht[0][3]);
    dgg[1] = dgg[0] * 0.125;
    dgg[2] = dgg[1];
    dlp[0] = rht[0][4] + rht[0][5] + rht[0][6];
    dlp[1] = dlp[0] * 0.5;
    dlp[2] = dlp[1];
    for (int i = 0; i < 10; ++i) rht[0][i] = rht[0][i] - rht[nspn - 1][i];
    for (int s = 0; s < nspn; ++s) {
      double* R = rht[s];
      dg2[s + 1] = R[1] * R[1] + R[2] * R[2] + R[3] * R[3];
      dgg[s + 1] = R[4] * R[1] * R[1] + R[5] * R[2] * R[2] + R[6] * R[3] * R[3] +
                   2 * (R[7] * R[1] * R[2] + R[8] * R[1] * R[3] + R[9] * R[2] * R[3]);
      dlp[s + 1] = R[4] + R[5] + R[6];
    }
    for (int i = 0; i < 10; ++i) rht[0][i] = rht[0][i] + rht[nspn - 1][i];
  }
  // exchange
  double D = den[0];
  if (!(P.idftyp[0] == 0 || D < EPS)) {
    for (int s = 0; s < nspn; ++s) {
      D = 2.0 * den[s + 1];
      if (D > EPS) {
        double dkf = std::pow(TRPI2 * D, THIRD);
        double S = 0, U = 0, V = 0;
        if (P.igga[0] != 0) {
          double dgrad = 2.0 * std::sqrt(dg2[s + 1]);
          double dlap = 2.0 * dlp[s + 1];
          double rec2 = 0.5 / (dkf * D);
          double rec1 = rec2 * D;
          double rec22 = rec2 * rec2;
          S = dgrad * rec2;
          V = dlap * rec1 * rec2;
          if (dgrad > EPS) U = 8.0 * dgg[s + 1] * rec1 * rec22 / dgrad;
          else U = 0.0;
        }
        double ex = 0, dex = 0, vx = 0;
        if (P.idftyp[0] >= 11) {
          // call_mgga_ex (call_mgga.f90:8-95) with NSPN=2; DEX is zero
          const double dgrad = 2.0 * std::sqrt(dg2[s + 1]);
          double vxdd, amux;
          scan_x_unp(D, dgrad, 2.0 * tau[s], ex, vx, vxdd, amux);
          double div = dgrad;
          if (std::fabs(div) < 1.0e-100) div = 1.0e-100;
          if (s == 0 && mixin) {
            for (int d = 0; d < 3; ++d) mixin[d] = 2.0 * vxdd * (rht[0][1 + d] - rht[1][1 + d]) / div;
            mixin[3] = amux * 0.5;
          }
        } else if (P.idftyp[0] <= 6) pw91ex(dkf, S, U, V, ex, dex, vx);
        else if (P.idftyp[0] == 7) pbeex(1, D, S, U, V, ex, dex, vx);
        else if (P.idftyp[0] == 8) pbeex(2, D, S, U, V, ex, dex, vx);
        else if (P.idftyp[0] == 9) pbeex(3, D, S, U, V, ex, dex, vx);
        vxc[s] = vxc[s] + vx;
        ex4[0] = ex4[0] + ispfac * 0.5 * ex * D * wgt;
        ex4[1] = ex4[1] + ispfac * 0.5 * dex * D * wgt;
      }
    }
  }
  // correlation
  D = den[0];
  double dup = den[1], ddn = den[2];
  if (P.idftyp[1] == 0 || D < EPS) return;
  double drec = 1.0 / D;
  double zet = (dup - ddn) * drec;
  double dkf = std::pow(TRPI2 * D, THIRD);
  double dks = std::sqrt(FRDPI * dkf);
  double rs = DKF2RS / dkf;
  double g = 0.5 * (std::pow(1.0 + zet, THIRD2) + std::pow(1.0 - zet, THIRD2));
  if (zet == -1.0) g = 0.5 * std::pow(2.0, THIRD2);
  if (zet == 1.0) g = 0.5 * std::pow(2.0, THIRD2);
  double T = 0, UU = 0, VV = 0, WW = 0;
  if (P.igga[1] != 0) {
    double dgrad = std::sqrt(dg2[0]);
    double dlap = dlp[0];
    double rec3 = drec;
    double rec1 = 0.5 / (dks * g);
    double rec2 = rec1 * rec3;
    double rec22 = rec2 * rec2;
    T = dgrad * rec2;
    VV = dlap * rec1 * rec2;
    WW = D * (dg2[1] - dg2[2]);
    WW = WW - (dup - ddn) * dg2[0];
    WW = WW * rec3 * rec22;
    if (dgrad > EPS) UU = dgg[0] * rec1 * rec22 / dgrad;
    else UU = 0.0;
  }
  double ec = 0, vcup = 0, vcdn = 0, dec = 0, dvcup = 0, dvcdn = 0;
  if (P.idftyp[1] >= 11) {
    // call_mgga_cor (call_mgga.f90:100-232), gradient branch, NSPN=2
    double vc[2], vcdd[2], amu;
    scan_c(dup, ddn, std::sqrt(dg2[1]), std::sqrt(dg2[2]), std::sqrt(dg2[0]), tau[0], tau[1], ec, vc, vcdd, amu);
    vcup = vc[0];
    vcdn = vc[1];
    if (mixin) {
      double div1 = dg2[1];
      if (std::fabs(div1) < 1.0e-100) div1 = 1.0e-100;
      for (int d = 0; d < 3; ++d) mixin[d] = mixin[d] + vcdd[0] * (rht[0][1 + d] - rht[1][1 + d]) / std::sqrt(div1);
      mixin[3] = mixin[3] + amu * 0.5;
    }
  } else if (P.idftyp[1] <= 5) {
    return;  // LDACOR variants are outside the supported set (rejected at setup)
  } else if (P.idftyp[1] == 6) {
    PW91Gas gas;
    double alfc;
    gas.g = g;
    pw91lc(rs, zet, gas.ec, vcup, vcdn, gas.ecrs, gas.eczet, alfc);
    ec = gas.ec;
    pw91nc(rs, zet, T, UU, VV, WW, gas, dec, dvcup, dvcdn);
  } else if (P.idftyp[1] == 7) {
    pbecor(rs, zet, T, UU, VV, WW, ec, vcup, vcdn, dec, dvcup, dvcdn);
  }
  ex4[2] = ex4[2] + ec * D * wgt;
  ex4[3] = ex4[3] + dec * D * wgt;
  vxc[0] = vxc[0] + vcup + dvcup;
  vxc[1] = vxc[1] + vcdn + dvcdn;
}

// GETVLXC serial branch (getvlxc.F:125-164) with NSPN=2 and the SIC spin-2
// density zero.  rhog: RHOG(nmsh,10) of the FO; vxc(2*nmsh); ergs[4] =
// ERGXL, ERGXN, ERGCL, ERGCN.
void getvlxc_sic(const Problem& P, const double* rhog, double* vxc, double* ergs, const double* tau = nullptr,
                 double* mixin = nullptr, int sb = 0, int se = INT32_MAX) {
  const int nmsh = P.nmsh;
  const int ng = P.gga() ? 10 : 1;
  for (int i = 0; i < 4; ++i) ergs[i] = 0.0;
  for (int l0 = 0; l0 < nmsh; l0 += MPBLOCKXC) {
    const int mpts = std::min(nmsh - l0, MPBLOCKXC);
    double ex4[4] = {0, 0, 0, 0};
    for (int i = 0; i < mpts; ++i) {
      const int ip = l0 + i;
      double rht[2][10];
      for (int k = 0; k < 10; ++k) {
        rht[0][k] = (k < ng) ? rhog[(size_t)k * nmsh + ip] + 0.0 : 0.0;
        rht[1][k] = 0.0 + 0.5 * 0.0;
      }
      double v[2] = {0.0, 0.0};
      double dump[4] = {0.0, 0.0, 0.0, 0.0};
      double* e4 = (ip >= sb && ip < se) ? ex4 : dump;  // energy sums of the point range only
      if (P.mgga()) {
        // GETTAU_PAR with the SIC FO in spin up (unravel2.f:242-246 zeroes the others)
        const double t2[2] = {tau[ip], 0.0};
        double z[4] = {0.0, 0.0, 0.0, 0.0};
        subvlxc_point(P, rht, P.wmsh[ip], v, e4, t2, z);
        if (mixin)
          for (int d = 0; d < 4; ++d) mixin[(size_t)ip * 4 + d] = z[d];
      } else {
        subvlxc_point(P, rht, P.wmsh[ip], v, e4);
      }
      vxc[ip] = v[0];
      vxc[ip + nmsh] = v[1];
    }
    for (int k = 0; k < 4; ++k) ergs[k] += ex4[k];
  }
}

// ---------------------------------------------------------------------------
// FO construction: FRMORB2(0,0) FMAT and FRMIORB(1,1) TMAT.
// ---------------------------------------------------------------------------
int compute_fmat(Problem& P) {
  const int nwf = P.nwfs[0] + (P.nspn == 2 ? P.nwfs[1] : 0);
  const int nf0 = P.nfrm[0], nf1 = (P.nspn == 2) ? P.nfrm[1] : 0;
  const int mfrm = nf0 + nf1;
  std::vector<double> pts(3 * (size_t)mfrm);
  for (int k = 0; k < nf0; ++k)
    for (int d = 0; d < 3; ++d) pts[3 * k + d] = P.fod[0][3 * k + d];
  for (int k = 0; k < nf1; ++k)
    for (int d = 0; d < 3; ++d) pts[3 * (nf0 + k) + d] = P.fod[1][3 * k + d];
  std::vector<double> psig;
  orbital_values(P, pts.data(), mfrm, 1, 4, P.psi.data(), P.nbasis, nwf, 0, psig);
  for (int s = 0; s < P.nspn; ++s) {
    const int nw = P.nwfs[s], nf = P.nfrm[s];
    P.fmat[s].assign((size_t)4 * nf * nw, 0.0);
    const int jbeg = s * P.nwfs[0];
    for (int jfm = 0; jfm < nf; ++jfm) {
      const int ipt = s * nf0 + jfm;
      double rhi[4] = {0, 0, 0, 0};
      for (int jwf = 0; jwf < nw; ++jwf) {
        const int jl = jwf + jbeg;
        for (int K = 0; K < 4; ++K)
          rhi[K] = rhi[K] + psig[((size_t)jl * 4 + 0) * mfrm + ipt] * psig[((size_t)jl * 4 + K) * mfrm + ipt];
      }
      if (!(rhi[0] > 0.0)) return fail("FRMORB2: zero density at a FOD", 4);
      for (int K = 0; K < 4; ++K)
        for (int jwf = 0; jwf < nw; ++jwf) {
          const int jl = jwf + jbeg;
          double f = psig[((size_t)jl * 4 + K) * mfrm + ipt] / std::sqrt(rhi[0]);
          if (K >= 1) f = f - P.fmat[s][((size_t)0 * nf + jfm) * nw + jwf] * rhi[K] / rhi[0];
          P.fmat[s][((size_t)K * nf + jfm) * nw + jwf] = f;
        }
    }
  }
  P.have_fmat = true;
  return 0;
}

int compute_tmat(Problem& P) {
  const int nwf = P.nwfs[0] + (P.nspn == 2 ? P.nwfs[1] : 0);
  const int nf0 = P.nfrm[0], nf1 = (P.nspn == 2) ? P.nfrm[1] : 0;
  const int norb = nf0 + nf1;
  std::vector<double> pts(3 * (size_t)norb);
  for (int k = 0; k < nf0; ++k)
    for (int d = 0; d < 3; ++d) pts[3 * k + d] = P.fod[0][3 * k + d];
  for (int k = 0; k < nf1; ++k)
    for (int d = 0; d < 3; ++d) pts[3 * (nf0 + k) + d] = P.fod[1][3 * k + d];
  const int nderv = P.gga() ? 2 : 0;
  const int ngrad = P.gga() ? 10 : 1;
  std::vector<double> psig;
  orbital_values(P, pts.data(), norb, nderv, ngrad, P.psi.data(), P.nbasis, nwf, 0, psig);
  for (int s = 0; s < P.nspn; ++s) {
    const int nw = P.nwfs[s], nf = P.nfrm[s];
    if (nw != nf) return fail("FRMIORB: MORB .NE. NFRM", 5);
    const int jbeg = s * P.nwfs[0];
    // T over all FODs, then the rows of this spin's FODs
    std::vector<double> T((size_t)nf * nw);
    for (int k = 0; k < nf; ++k) {
      const int ipt = s * nf0 + k;
      double rho = 0.0;
      for (int jwf = 0; jwf < nw; ++jwf) {
        double v = psig[((size_t)(jwf + jbeg) * ngrad) * norb + ipt];
        rho = rho + v * v;
      }
      if (!(rho > 0.0)) return fail("FRMIORB: zero density at a FOD", 4);
      for (int jwf = 0; jwf < nw; ++jwf)
        T[(size_t)k * nw + jwf] = psig[((size_t)(jwf + jbeg) * ngrad) * norb + ipt] / std::sqrt(rho);
    }
    std::vector<double> over((size_t)nf * nf);
    for (int i = 0; i < nf; ++i)
      for (int j = 0; j < nf; ++j) {
        double s2 = 0.0;
        for (int w = 0; w < nw; ++w) s2 = s2 + T[(size_t)i * nw + w] * T[(size_t)j * nw + w];
        over[(size_t)i * nf + j] = s2;
      }
    std::vector<double> ham, filo, eval;
    int rc = lowsic(nf, over, ham, filo, eval);
    if (rc) return rc;
    P.lowev[s].resize(nf);
    for (int i = 0; i < nf; ++i) P.lowev[s][i] = 1.0 / (eval[i] * eval[i]);
    P.tmat[s].assign((size_t)nf * nw, 0.0);
    for (int i = 0; i < nf; ++i)
      for (int k = 0; k < nf; ++k)
        for (int w = 0; w < nw; ++w)
          P.tmat[s][(size_t)i * nw + w] = P.tmat[s][(size_t)i * nw + w] + ham[(size_t)k * nf + i] * T[(size_t)k * nw + w];
  }
  P.have_tmat = true;
  return 0;
}

// UNRAVEL2 rotation (unravel2.f:200-240): FO k coefficients = sum_j PSI_j TMAT(k,j)
void fo_coefficients(const Problem& P, int s, std::vector<double>& cfo) {
  const int nw = P.nwfs[s], nf = P.nfrm[s], nb = P.nbasis;
  const int jbeg = s * P.nwfs[0];
  cfo.assign((size_t)nb * nf, 0.0);
  for (int ib = 0; ib < nb; ++ib)
    for (int k = 0; k < nf; ++k) {
      double v = 0.0;
      for (int j = 0; j < nw; ++j) v = v + P.psi[(size_t)(j + jbeg) * nb + ib] * P.tmat[s][(size_t)k * nw + j];
      cfo[(size_t)k * nb + ib] = v;
    }
}

// GETTAU_PAR (gettau_par.f90:1-226) for one FO: tau = |grad phi|^2 / 2 from
// the FO coefficients with the |c| <= 1e-10 skip.
void fo_tau(const Problem& P, const double* cfo, std::vector<double>& tau) {
  const int nmsh = P.nmsh;
  tau.assign(nmsh, 0.0);
  std::vector<double> g;
  for (int l0 = 0; l0 < nmsh; l0 += MPBLOCKXC) {
    const int mpts = std::min(MPBLOCKXC, nmsh - l0);
    orbital_values(P, &P.rmsh[3 * (size_t)l0], mpts, 1, 4, cfo, P.nbasis, 1, 0, g);
    for (int i = 0; i < mpts; ++i)
      tau[l0 + i] = tau[l0 + i] + 0.5 * (g[(size_t)1 * mpts + i] * g[(size_t)1 * mpts + i] +
                                         g[(size_t)2 * mpts + i] * g[(size_t)2 * mpts + i] +
                                         g[(size_t)3 * mpts + i] * g[(size_t)3 * mpts + i]);
  }
}

// APOTNL_SIC (apotnl_sic.F:31-668) for one FO.
int apotnl_sic(const Problem& P, int s, int k, const double* cfo, double* results, double* cfrm,
               double* pot, double* coul_out, double* rhog_out, bool exact, double* mixin_out = nullptr) {
  const int nmsh = P.nmsh;
  std::vector<double> coulomb(nmsh), rhog((size_t)10 * nmsh);
  coupot_sic(P, cfo, exact, coulomb.data(), rhog.data(), nullptr);
  if (P.xc_exact_density && !exact) {
    std::vector<double> scratch(nmsh);
    coupot_sic(P, cfo, true, scratch.data(), rhog.data(), nullptr);
  }
  double addit = 0.0;
  for (int i = 0; i < nmsh; ++i) addit += std::fabs(coulomb[i]);
  if (addit < 0.001) return fail("APOTNL_SIC: COUPOT IS ZERO", 6);
  double xcgv = 0, ycgv = 0, zcgv = 0;
  for (int i = 0; i < nmsh; ++i) {
    xcgv = xcgv + P.rmsh[3 * i] * rhog[i] * P.wmsh[i];
    ycgv = ycgv + P.rmsh[3 * i + 1] * rhog[i] * P.wmsh[i];
    zcgv = zcgv + P.rmsh[3 * i + 2] * rhog[i] * P.wmsh[i];
  }
  cfrm[0] = xcgv;
  cfrm[1] = ycgv;
  cfrm[2] = zcgv;
  double rmx = 0.0, asy = 0.0;
  const double fnspn = (double)(float)P.nspn;
  for (int i = 0; i < nmsh; ++i) {
    double rad = std::sqrt(P.rmsh[3 * i] * P.rmsh[3 * i] + P.rmsh[3 * i + 1] * P.rmsh[3 * i + 1] +
                           P.rmsh[3 * i + 2] * P.rmsh[3 * i + 2]);
    coulomb[i] = coulomb[i] * fnspn / 2.0;
    if (rad > rmx) {
      rmx = rad;
      asy = coulomb[i] * rmx;
    }
  }
  std::vector<double> vxc(2 * (size_t)nmsh);
  double ergs[4];
  if (P.mgga()) {
    std::vector<double> tau, mix((size_t)4 * nmsh);
    fo_tau(P, cfo, tau);
    getvlxc_sic(P, rhog.data(), vxc.data(), ergs, tau.data(), mix.data());
    if (mixin_out) std::memcpy(mixin_out, mix.data(), sizeof(double) * 4 * nmsh);
  } else {
    getvlxc_sic(P, rhog.data(), vxc.data(), ergs);
  }
  double xch1 = 0, xch2 = 0, xcou = 0, xexx = 0, xdel = 0;
  const double p43 = (double)(4.0f / 3.0f);
  for (int i = 0; i < nmsh; ++i) pot[i] = vxc[i] + coulomb[i];
  for (int i = 0; i < nmsh; ++i) {
    const double w = P.wmsh[i], r = rhog[i];
    const double vx = pot[i] - coulomb[i];
    xch1 = xch1 + w * r;
    xch2 = xch2 + w * 0.0;
    xcou = xcou + w * r * coulomb[i];
    xexx = xexx + w * std::pow(std::fabs(r), p43);
    xdel = xdel - w * r * vx;
  }
  const double excsic = ergs[0] + ergs[1] + ergs[2] + ergs[3];
  xdel = xdel - xcou;
  const double xeng = -excsic - xcou / 2.0;
  const double pi = 4.0 * std::atan(1.0);
  xexx = xexx * 0.75 * std::pow(6 / pi, (double)(1.0f / 3.0f));
  const double sic_eng = xeng * (2.0 / P.nspn);
  results[0] = k + 1;
  results[1] = xch1;
  results[2] = xch2;
  results[3] = asy;
  results[4] = xexx;
  results[5] = -xcou / 2.0;
  results[6] = xdel;
  results[7] = xeng;
  results[8] = sic_eng;
  results[9] = ergs[0];
  results[10] = ergs[2];
  results[11] = ergs[1];
  results[12] = ergs[3];
  if (coul_out) std::memcpy(coul_out, coulomb.data(), sizeof(double) * nmsh);
  if (rhog_out) std::memcpy(rhog_out, rhog.data(), sizeof(double) * 10 * nmsh);
  (void)s;
  return 0;
}

// SICLAGM / SICLMSLV (frmorb_mpi.F:2-572).  LDA/GGA: NGRAD=1 and the local
// potential only.  Meta-GGA (frmorb_mpi.F:440-509): NGRAD=4 and, with the FOs'
// Hamiltonian ingredients zm [nf][nmsh][4], the gradient terms
// grad phi_j . (phi_l w Z) + phi_j w (grad phi_l . Z) + Z4 w grad phi_j . grad phi_l.
void siclagm(const Problem& P, int s, const double* pots /*[nf][nmsh]*/, const double* cfo,
             double* sic, int ld, const double* zm = nullptr, int pb = 0, int pe = INT32_MAX) {
  const int nf = P.nfrm[s], nmsh = std::min(P.nmsh, pe), nb = P.nbasis;
  for (int l = 0; l < nf; ++l)
    for (int j = 0; j < nf; ++j) sic[(size_t)l * ld + j] = 0.0;
  std::vector<double> pts, phi;
  const int nall = P.nmsh;  // row stride of pots and zm
  if (P.mgga()) {
    for (int l0 = pb; l0 < nmsh; l0 += MPBLOCK) {
      const int mpts = std::min(MPBLOCK, nmsh - l0);
      orbital_values(P, &P.rmsh[3 * (size_t)l0], mpts, 1, 4, cfo, nb, nf, 1, phi);
      auto G = [&](int f, int ig, int i) { return phi[((size_t)f * 4 + ig) * mpts + i]; };
      for (int ll = 0; ll < nf; ++ll) {
        std::vector<double> pl((size_t)8 * mpts);
        for (int i = 0; i < mpts; ++i) {
          const double w = P.wmsh[l0 + i];
          const double* z = &zm[((size_t)ll * nall + l0 + i) * 4];
          pl[i] = G(ll, 0, i) * (pots[(size_t)ll * nall + l0 + i] * w);
          for (int c = 0; c < 3; ++c) pl[(size_t)(1 + c) * mpts + i] = G(ll, 0, i) * w * z[c];
          pl[(size_t)4 * mpts + i] = w * (G(ll, 1, i) * z[0] + G(ll, 2, i) * z[1] + G(ll, 3, i) * z[2]);
          for (int c = 0; c < 3; ++c) pl[(size_t)(5 + c) * mpts + i] = G(ll, 1 + c, i) * w * z[3];
        }
        auto dot = [&](int jf, int ig, int t) {
          double a = 0.0;
          for (int i = 0; i < mpts; ++i) a += G(jf, ig, i) * pl[(size_t)t * mpts + i];
          return a;
        };
        for (int jf = 0; jf < nf; ++jf) {
          double add = dot(jf, 0, 0);
          add = add + dot(jf, 1, 1) + dot(jf, 2, 2) + dot(jf, 3, 3) + dot(jf, 0, 4);
          add = add + dot(jf, 1, 5) + dot(jf, 2, 6) + dot(jf, 3, 7);
          sic[(size_t)ll * ld + jf] = sic[(size_t)ll * ld + jf] - add;
        }
      }
    }
    return;
  }
  for (int l0 = pb; l0 < nmsh; l0 += MPBLOCK) {
    const int mpts = std::min(MPBLOCK, nmsh - l0);
    orbital_values(P, &P.rmsh[3 * (size_t)l0], mpts, 0, 1, cfo, nb, nf, 1, phi);
    for (int ll = 0; ll < nf; ++ll) {
      std::vector<double> pl(mpts);
      for (int i = 0; i < mpts; ++i)
        pl[i] = phi[(size_t)ll * mpts + i] * (pots[(size_t)ll * nall + l0 + i] * P.wmsh[l0 + i]);
      for (int jf = 0; jf < nf; ++jf) {
        double add = 0.0;
        for (int i = 0; i < mpts; ++i) add += phi[(size_t)jf * mpts + i] * pl[i];
        sic[(size_t)ll * ld + jf] = sic[(size_t)ll * ld + jf] - add;
      }
    }
  }
}

// FRMORB2(-s,-1) force branch (frmorb2.F:460-717).
int frmorb2_force(const Problem& P, int s, const double* sic, int ld, double* debdax) {
  const int nf = P.nfrm[s], nw = P.nwfs[s];
  const std::vector<double>& F = P.fmat[s];
  auto fm = [&](int kwf, int ifm, int K) { return F[((size_t)K * nf + ifm) * nw + kwf]; };
  std::vector<double> over((size_t)nf * nf);
  for (int ifm = 0; ifm < nf; ++ifm)
    for (int jfm = 0; jfm < nf; ++jfm) {
      double v = 0.0;
      for (int kwf = 0; kwf < nw; ++kwf) v = v + fm(kwf, ifm, 0) * fm(kwf, jfm, 0);
      over[(size_t)jfm * nf + ifm] = v;
    }
  std::vector<double> ham, filo, eval;
  int rc = lowsic(nf, over, ham, filo, eval);
  if (rc) return rc;
  // FILO(i,a) = filo[i*nf+a]; EVAL restored = lambda^{-1/2}; Q = 1/EVAL^2
  std::vector<double> Q(nf);
  for (int a = 0; a < nf; ++a) Q[a] = 1.0 / (eval[a] * eval[a]);
  auto FI = [&](int i, int a) { return filo[(size_t)i * nf + a]; };
  auto S = [&](int k, int l) { return sic[(size_t)l * ld + k]; };  // SIC(k,l)
  std::vector<double> H((size_t)nf * nf);  // H[ia*nf+ib] = HAM(ib,ia)
  for (int ia = 0; ia < nf; ++ia)
    for (int ib = 0; ib < nf; ++ib) {
      double h = 0.0;
      for (int kf = 0; kf < nf; ++kf)
        for (int lf = 0; lf < nf; ++lf)
          h = h + (FI(kf, ia) * FI(lf, ib) - FI(lf, ia) * FI(kf, ib)) * S(kf, lf);
      h = h / (std::sqrt(Q[ib]) * std::sqrt(Q[ia]));
      H[(size_t)ia * nf + ib] = h;
    }
  for (int i = 0; i < 3 * nf; ++i) debdax[i] = 0.0;
  std::vector<double> X((size_t)3 * nf * nf);  // X[kx][n][m] = sum_kwf F(kwf,n,1) F(kwf,m,kx+1)
  for (int kx = 0; kx < 3; ++kx)
    for (int n = 0; n < nf; ++n)
      for (int m = 0; m < nf; ++m) {
        double v = 0.0;
        for (int kwf = 0; kwf < nw; ++kwf) v = v + fm(kwf, n, 0) * fm(kwf, m, kx + 1);
        X[((size_t)kx * nf + n) * nf + m] = v;
      }
  std::vector<double> sc1(nf);
  for (int ia = 0; ia < nf; ++ia) {
    for (int nn = 0; nn < nf; ++nn) sc1[nn] = 0.0;
    for (int ib = 0; ib < nf; ++ib)
      for (int nn = 0; nn < nf; ++nn) sc1[nn] = H[(size_t)ia * nf + ib] * FI(nn, ib) + sc1[nn];
    for (int kx = 0; kx < 3; ++kx)
      for (int mf = 0; mf < nf; ++mf)
        for (int nn = 0; nn < nf; ++nn)
          debdax[3 * mf + kx] = debdax[3 * mf + kx] - FI(mf, ia) * sc1[nn] * X[((size_t)kx * nf + nn) * nf + mf];
  }
  for (int ia = 0; ia < nf; ++ia)
    for (int ib = 0; ib < nf; ++ib) {
      double& h = H[(size_t)ia * nf + ib];
      h = h * (std::sqrt(Q[ib]) - std::sqrt(Q[ia]));
      h = h / (std::sqrt(Q[ib]) + std::sqrt(Q[ia]));
    }
  for (int kx = 0; kx < 3; ++kx)
    for (int ia = 0; ia < nf; ++ia)
      for (int ib = 0; ib < nf; ++ib) {
        for (int mf = 0; mf < nf; ++mf) {
          double v = 0.0;
          for (int iff = 0; iff < nf; ++iff)
            v = v - (FI(iff, ib) * FI(mf, ia) + FI(mf, ib) * FI(iff, ia)) *
                        (2.0 * X[((size_t)kx * nf + iff) * nf + mf]) * 0.5;
          sc1[mf] = v;
        }
        for (int mf = 0; mf < nf; ++mf)
          debdax[3 * mf + kx] = debdax[3 * mf + kx] - 0.5 * sc1[mf] * H[(size_t)ia * nf + ib];
      }
  return 0;
}

}  // namespace

// ===========================================================================
// C API
// ===========================================================================
struct orc_problem {
  Problem P;
};

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

orc_problem* orc_create(int natoms, const int* atom_type, const double* rat, int ntypes, const int* n_bare,
                        const double* bfalp, const int* n_con, const double* bfcon, int nmsh,
                        const double* rmsh, const double* wmsh, int nspn, int igga_x, int idftyp_x,
                        int igga_c, int idftyp_c) {
  if (natoms <= 0 || ntypes <= 0 || nmsh <= 0 || (nspn != 1 && nspn != 2)) {
    fail("orc_create: bad sizes");
    return nullptr;
  }
  const bool scan = igga_x == 3 && idftyp_x == 11 && igga_c == 3 && idftyp_c == 11;
  if (!scan && (!(idftyp_x >= 6 && idftyp_x <= 9) || !(idftyp_c == 6 || idftyp_c == 7) || igga_x < 0 ||
                igga_x > 1 || igga_c < 0 || igga_c > 1)) {
    fail("orc_create: functional outside the supported set (PW91/PBE exchange, PW91/PBE correlation, SCAN)");
    return nullptr;
  }
  auto* o = new orc_problem;
  Problem& P = o->P;
  P.natoms = natoms;
  P.ntypes = ntypes;
  P.nmsh = nmsh;
  P.nspn = nspn;
  P.igga[0] = igga_x;
  P.igga[1] = igga_c;
  P.idftyp[0] = idftyp_x;
  P.idftyp[1] = idftyp_c;
  P.atype.assign(atom_type, atom_type + natoms);
  P.rat.assign(rat, rat + 3 * (size_t)natoms);
  P.nbare.assign(n_bare, n_bare + ntypes);
  P.bfalp.assign(bfalp, bfalp + (size_t)MAX_BARE * ntypes);
  P.ncon.assign(n_con, n_con + 3 * (size_t)ntypes);
  P.bfcon.assign(bfcon, bfcon + (size_t)MAX_BARE * MAX_CON * 3 * ntypes);
  P.lmax.resize(ntypes);
  P.nloc.resize(ntypes);
  for (int t = 0; t < ntypes; ++t) {
    int lm = 0, nl = 0;
    for (int l = 0; l < 3; ++l) {
      if (P.ncon[t * 3 + l] > 0) lm = l;
      nl += kNcomp[l] * P.ncon[t * 3 + l];
    }
    P.lmax[t] = lm;
    P.nloc[t] = nl;
  }
  P.aoff.resize(natoms);
  int off = 0;
  for (int a = 0; a < natoms; ++a) {
    P.aoff[a] = off;
    off += P.nloc[P.atype[a]];
  }
  P.nbasis = off;
  P.rmsh.assign(rmsh, rmsh + 3 * (size_t)nmsh);
  P.wmsh.assign(wmsh, wmsh + nmsh);
  return o;
}

void orc_destroy(orc_problem* p) { delete p; }
int orc_nbasis(const orc_problem* p) { return p->P.nbasis; }

int orc_set_orbitals(orc_problem* p, const int* nwfs, const double* psi, int ldpsi, const int* nfrm,
                     const double* bfrm, int ldfrm) {
  Problem& P = p->P;
  P.nwfs[0] = nwfs[0];
  P.nwfs[1] = (P.nspn == 2) ? nwfs[1] : 0;
  P.nfrm[0] = nfrm[0];
  P.nfrm[1] = (P.nspn == 2) ? nfrm[1] : 0;
  const int nwf = P.nwfs[0] + P.nwfs[1];
  P.psi.assign((size_t)P.nbasis * nwf, 0.0);
  for (int j = 0; j < nwf; ++j)
    for (int i = 0; i < P.nbasis; ++i) P.psi[(size_t)j * P.nbasis + i] = psi[(size_t)j * ldpsi + i];
  for (int s = 0; s < P.nspn; ++s) {
    P.fod[s].resize(3 * (size_t)P.nfrm[s]);
    for (int k = 0; k < P.nfrm[s]; ++k)
      for (int d = 0; d < 3; ++d) P.fod[s][3 * k + d] = bfrm[((size_t)s * ldfrm + k) * 3 + d];
  }
  P.have_orbitals = true;
  P.have_fmat = P.have_tmat = false;
  return 0;
}

int orc_gorbdrv(orc_problem* p, int nderv, int npts, const double* pts, int ifnct, double* grad, int* iupdat,
                int* iallctr) {
  if (npts > NSPEED || nderv < 0 || nderv > 2) return fail("GORBDRV: bad arguments");
  bool ia[3 * MAX_CON];
  bool up = gorbdrv(p->P, nderv, npts, pts, ifnct - 1, grad, ia);
  *iupdat = up ? 1 : 0;
  for (int l = 0; l < 3; ++l)
    for (int c = 0; c < MAX_CON; ++c) iallctr[l * MAX_CON + c] = (c < p->P.ncon[(ifnct - 1) * 3 + l]) ? ia[l * MAX_CON + c] : 0;
  return 0;
}

int orc_frmorb2_fmat(orc_problem* p, double* fmat, int ld) {
  Problem& P = p->P;
  int rc = compute_fmat(P);
  if (rc) return rc;
  for (int s = 0; s < P.nspn; ++s)
    for (int K = 0; K < 4; ++K)
      for (int j = 0; j < P.nfrm[s]; ++j)
        for (int w = 0; w < P.nwfs[s]; ++w)
          fmat[(((size_t)s * 4 + K) * ld + j) * ld + w] = P.fmat[s][((size_t)K * P.nfrm[s] + j) * P.nwfs[s] + w];
  return 0;
}

int orc_frmiorb(orc_problem* p, double* tmat, double* lowden_eval, int ld) {
  Problem& P = p->P;
  int rc = compute_tmat(P);
  if (rc) return rc;
  for (int s = 0; s < P.nspn; ++s) {
    for (int k = 0; k < P.nfrm[s]; ++k)
      for (int w = 0; w < P.nwfs[s]; ++w)
        tmat[((size_t)s * ld + w) * ld + k] = P.tmat[s][(size_t)k * P.nwfs[s] + w];
    for (int k = 0; k < P.nfrm[s]; ++k) lowden_eval[(size_t)s * ld + k] = P.lowev[s][k];
  }
  return 0;
}

int orc_fo_coefficients(orc_problem* p, int spin, double* cfo) {
  Problem& P = p->P;
  if (!P.have_tmat) {
    int rc = compute_tmat(P);
    if (rc) return rc;
  }
  std::vector<double> c;
  fo_coefficients(P, spin - 1, c);
  std::memcpy(cfo, c.data(), sizeof(double) * c.size());
  return 0;
}

int orc_coupot_sic(orc_problem* p, int spin, int iorb, int exact, double* coulomb, double* rhog, long long* stats) {
  Problem& P = p->P;
  if (!P.have_tmat) {
    int rc = compute_tmat(P);
    if (rc) return rc;
  }
  std::vector<double> c;
  fo_coefficients(P, spin - 1, c);
  Stats st;
  coupot_sic(P, &c[(size_t)(iorb - 1) * P.nbasis], exact != 0, coulomb, rhog, &st);
  if (stats) {
    stats[0] = st.pairs;
    stats[1] = st.batches;
    stats[2] = st.weird;
    stats[3] = st.near;
    stats[4] = st.far;
    stats[5] = st.near_multi;
    stats[6] = st.far_multi;
    stats[7] = st.npot1_multi;
    stats[8] = st.calls_multi;
  }
  return 0;
}

int orc_pair_dump(orc_problem* p, int spin, int iorb, double* calls, long long maxc, long long* ncalls,
                  double* pairs, long long maxp, long long* npairs) {
  Problem& P = p->P;
  if (!P.have_tmat) {
    int rc = compute_tmat(P);
    if (rc) return rc;
  }
  std::vector<double> c;
  fo_coefficients(P, spin - 1, c);
  std::vector<double> coul(P.nmsh), rhog((size_t)10 * P.nmsh), cv, pv;
  Stats st;
  st.calls = &cv;
  st.pairs_out = &pv;
  coupot_sic(P, &c[(size_t)(iorb - 1) * P.nbasis], false, coul.data(), rhog.data(), &st);
  *ncalls = (long long)cv.size() / 6;
  *npairs = (long long)pv.size() / 51;
  if (*ncalls > maxc || *npairs > maxp) return fail("orc_pair_dump: output arrays too small");
  std::memcpy(calls, cv.data(), sizeof(double) * cv.size());
  std::memcpy(pairs, pv.data(), sizeof(double) * pv.size());
  return 0;
}

int orc_pair_stats(orc_problem* p, int spin, int iorb, long long* stats) {
  std::vector<double> coul(p->P.nmsh), rhog((size_t)10 * p->P.nmsh);
  return orc_coupot_sic(p, spin, iorb, 0, coul.data(), rhog.data(), stats);
}

int orc_getvlxc_sic(orc_problem* p, const double* rhog, double* vxc, double* ergs) {
  if (p->P.mgga()) return fail("GETVLXC: a meta-GGA needs tau (orc_getvlxc_mgga)");
  getvlxc_sic(p->P, rhog, vxc, ergs);
  return 0;
}

int orc_getvlxc_mgga(orc_problem* p, const double* rhog, const double* tau, double* vxc, double* mixin,
                     double* ergs) {
  if (!p->P.mgga()) return fail("GETVLXC: tau and MIXIN belong to meta-GGA functionals");
  getvlxc_sic(p->P, rhog, vxc, ergs, tau, mixin);
  return 0;
}

// Mesh-shard decomposition of one SIC cycle, packed like the library's
// flosic_sic_cycle_partial: per spin SIC(nf,nf) at [l*nf + j], the mesh sums
// (XCH1, XCOU, XEXX, XDEL, ERGXL, ERGXN, ERGCL, ERGCN, CFRM x3) per FO, the
// scaled Coulomb potential at the farthest mesh point per FO (zero off the
// range); then three work counters (zero here).  The sums of APOTNL_SIC
// (apotnl_sic.F:381-408, 564-623) and SICLMSLV run over mesh points [b, e) only.
constexpr int ORC_NPART = 11;
static size_t orc_partial_doubles(const Problem& P) {
  size_t n = 3;
  for (int s = 0; s < P.nspn; ++s) n += (size_t)P.nfrm[s] * P.nfrm[s] + (size_t)P.nfrm[s] * (ORC_NPART + 1);
  return n;
}

static void farthest_point(const Problem& P, int& ifar, double& rmx) {
  ifar = 0;
  rmx = 0.0;
  for (int i = 0; i < P.nmsh; ++i) {
    const double* r = &P.rmsh[3 * (size_t)i];
    const double rad = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (rad > rmx) {
      rmx = rad;
      ifar = i;
    }
  }
}

int orc_partial_size(orc_problem* p, long long* n) {
  *n = (long long)orc_partial_doubles(p->P);
  return 0;
}

int orc_cycle_partial(orc_problem* p, int b, int e, double* out) {
  Problem& P = p->P;
  if (b < 0 || e > P.nmsh || b > e) return fail("orc_cycle_partial: bad point range");
  int rc = compute_fmat(P);
  if (rc) return rc;
  rc = compute_tmat(P);
  if (rc) return rc;
  const int nmsh = P.nmsh;
  int ifar;
  double rmx;
  farthest_point(P, ifar, rmx);
  size_t o = 0;
  std::fill(out, out + orc_partial_doubles(P), 0.0);
  for (int s = 0; s < P.nspn; ++s) {
    const int nf = P.nfrm[s];
    if (nf == 0) continue;
    std::vector<double> c;
    fo_coefficients(P, s, c);
    std::vector<double> pots((size_t)nf * nmsh), zm(P.mgga() ? (size_t)nf * nmsh * 4 : 0);
    double* parts = out + o + (size_t)nf * nf;
    double* asy = parts + (size_t)nf * ORC_NPART;
    for (int k = 0; k < nf; ++k) {
      const double* cf = &c[(size_t)k * P.nbasis];
      std::vector<double> coulomb(nmsh), rhog((size_t)10 * nmsh), vxc(2 * (size_t)nmsh);
      coupot_sic(P, cf, false, coulomb.data(), rhog.data(), nullptr);
      if (P.xc_exact_density) {
        std::vector<double> scratch(nmsh);
        coupot_sic(P, cf, true, scratch.data(), rhog.data(), nullptr);
      }
      const double fnspn = (double)(float)P.nspn;
      for (int i = 0; i < nmsh; ++i) coulomb[i] = coulomb[i] * fnspn / 2.0;
      double ergs[4];
      if (P.mgga()) {
        std::vector<double> tau;
        fo_tau(P, cf, tau);
        getvlxc_sic(P, rhog.data(), vxc.data(), ergs, tau.data(), &zm[(size_t)k * nmsh * 4], b, e);
      } else {
        getvlxc_sic(P, rhog.data(), vxc.data(), ergs, nullptr, nullptr, b, e);
      }
      double* q = &parts[(size_t)k * ORC_NPART];
      const double p43 = (double)(4.0f / 3.0f);
      for (int i = 0; i < nmsh; ++i) pots[(size_t)k * nmsh + i] = vxc[i] + coulomb[i];
      for (int i = b; i < e; ++i) {
        const double w = P.wmsh[i], r = rhog[i];
        const double vx = pots[(size_t)k * nmsh + i] - coulomb[i];
        q[0] = q[0] + w * r;
        q[1] = q[1] + w * r * coulomb[i];
        q[2] = q[2] + w * std::pow(std::fabs(r), p43);
        q[3] = q[3] - w * r * vx;
        for (int d = 0; d < 3; ++d) q[8 + d] = q[8 + d] + P.rmsh[3 * (size_t)i + d] * r * w;
      }
      for (int j = 0; j < 4; ++j) q[4 + j] = ergs[j];
      asy[k] = (ifar >= b && ifar < e) ? coulomb[ifar] : 0.0;
    }
    siclagm(P, s, pots.data(), c.data(), out + o, nf, P.mgga() ? zm.data() : nullptr, b, e);
    o += (size_t)nf * nf + (size_t)nf * (ORC_NPART + 1);
  }
  return 0;
}

int orc_cycle_combine(orc_problem* p, const double* in, int ld, double* results, double* sic, double* debdax,
                      double* cfrm, double* esic) {
  Problem& P = p->P;
  int ifar;
  double rmx;
  farthest_point(P, ifar, rmx);
  size_t o = 0;
  double zsic = 0.0;
  for (int s = 0; s < P.nspn; ++s) {
    const int nf = P.nfrm[s];
    if (nf == 0) continue;
    const double* lam = in + o;
    const double* parts = lam + (size_t)nf * nf;
    const double* asy = parts + (size_t)nf * ORC_NPART;
    for (int k = 0; k < nf; ++k) {
      const double* q = &parts[(size_t)k * ORC_NPART];
      double* r = &results[((size_t)s * ld + k) * 13];
      const double xch1 = q[0], xcou = q[1];
      const double excsic = q[4] + q[5] + q[6] + q[7];
      const double xdel = q[3] - xcou;
      const double xeng = -excsic - xcou / 2.0;
      const double pi = 4.0 * std::atan(1.0);
      r[0] = k + 1;
      r[1] = xch1;
      r[2] = 0.0;
      r[3] = asy[k] * rmx;
      r[4] = q[2] * 0.75 * std::pow(6 / pi, (double)(1.0f / 3.0f));
      r[5] = -xcou / 2.0;
      r[6] = xdel;
      r[7] = xeng;
      r[8] = xeng * (2.0 / P.nspn);
      r[9] = q[4];
      r[10] = q[6];
      r[11] = q[5];
      r[12] = q[7];
      for (int d = 0; d < 3; ++d) cfrm[((size_t)s * ld + k) * 3 + d] = q[8 + d];
      zsic += r[8];
    }
    double* ps = sic + (size_t)s * ld * ld;
    for (int l = 0; l < nf; ++l)
      for (int j = 0; j < nf; ++j) ps[(size_t)l * ld + j] = lam[(size_t)l * nf + j];
    int rc = frmorb2_force(P, s, ps, ld, debdax + (size_t)s * ld * 3);
    if (rc) return rc;
    o += (size_t)nf * nf + (size_t)nf * (ORC_NPART + 1);
  }
  *esic = zsic;
  return 0;
}

// SICLAG_DER / SICLM_DERSLV (siclag_der.F:2-688), C1 symmetry:
//   DERSIC(ix, lfn, A) = sum_p w V_l phi_l d_ix phi_l^(A)
// with phi_l^(A) the part of FO l carried by the basis functions of atom A
// (PSID), lfn = l + s*NFRM(1), plus for a meta-GGA the terms of
// siclag_der.F:576-640 with the FO's Hamiltonian ingredients Z:
//   + sum_p w [(grad phi . Z) d_ix phi^(A) + phi sum_c Z_c d_ix d_c phi^(A)
//              + Z_4 sum_c d_c phi d_ix d_c phi^(A)];
// doubled for NSPN=1 (siclag_der.F:153-161).  dersic[(A*ldo + lfn)*3 + ix].
int orc_siclag_der(orc_problem* p, double* dersic, int ldo) {
  Problem& P = p->P;
  int rc = compute_fmat(P);
  if (rc) return rc;
  rc = compute_tmat(P);
  if (rc) return rc;
  const int nmsh = P.nmsh, nb = P.nbasis;
  const bool mg = P.mgga();
  std::fill(dersic, dersic + (size_t)P.natoms * ldo * 3, 0.0);
  // Hessian channel of (d_ix, d_c): value 0, gradient 1-3, xx yy zz 4-6, xy xz yz 7-9
  const int hch[3][3] = {{4, 7, 8}, {7, 5, 9}, {8, 9, 6}};
  for (int s = 0; s < P.nspn; ++s) {
    const int nf = P.nfrm[s];
    if (nf == 0) continue;
    std::vector<double> c;
    fo_coefficients(P, s, c);
    std::vector<double> pots((size_t)nf * nmsh), zm(mg ? (size_t)nf * nmsh * 4 : 0);
    for (int k = 0; k < nf; ++k) {
      double res[13], cf[3];
      rc = apotnl_sic(P, s, k, &c[(size_t)k * nb], res, cf, &pots[(size_t)k * nmsh], nullptr, nullptr, false,
                      mg ? &zm[(size_t)k * nmsh * 4] : nullptr);
      if (rc) return rc;
    }
    std::vector<double> phi, pa;
    for (int l0 = 0; l0 < nmsh; l0 += MPBLOCK) {
      const int mpts = std::min(MPBLOCK, nmsh - l0);
      orbital_values(P, &P.rmsh[3 * (size_t)l0], mpts, 1, 4, c.data(), nb, nf, 1, phi);
      for (int a = 0; a < P.natoms; ++a) {
        orbital_values(P, &P.rmsh[3 * (size_t)l0], mpts, mg ? 2 : 1, mg ? 10 : 4, c.data(), nb, nf, 1, pa, a);
        const int ng = mg ? 10 : 4;
        for (int k = 0; k < nf; ++k) {
          double* d = &dersic[((size_t)a * ldo + k + (size_t)s * P.nfrm[0]) * 3];
          auto F = [&](int ig, int i) { return phi[((size_t)k * 4 + ig) * mpts + i]; };
          auto A = [&](int ig, int i) { return pa[((size_t)k * ng + ig) * mpts + i]; };
          for (int i = 0; i < mpts; ++i) {
            const double w = P.wmsh[l0 + i];
            const double v = pots[(size_t)k * nmsh + l0 + i];
            double y0 = w * v * F(0, i);
            double yc[3] = {0.0, 0.0, 0.0};
            if (mg) {
              const double* z = &zm[((size_t)k * nmsh + l0 + i) * 4];
              y0 = y0 + w * (F(1, i) * z[0] + F(2, i) * z[1] + F(3, i) * z[2]);
              for (int cc = 0; cc < 3; ++cc) yc[cc] = w * z[cc] * F(0, i) + w * z[3] * F(1 + cc, i);
            }
            for (int ix = 0; ix < 3; ++ix) {
              double add = A(1 + ix, i) * y0;
              if (mg)
                for (int cc = 0; cc < 3; ++cc) add = add + A(hch[ix][cc], i) * yc[cc];
              d[ix] = d[ix] + add;
            }
          }
        }
      }
    }
  }
  if (P.nspn == 1)
    for (size_t i = 0; i < (size_t)P.natoms * ldo * 3; ++i) dersic[i] = 2.0 * dersic[i];
  return 0;
}

// COUPOT1 (coupot1.F:5-762): the Coulomb potential of the occupied orbitals'
// total density, ADD(i,j,s) = sum_{iwf in s} PSI(i) PSI(j) summed over the
// spins in POISSON1 (doubled for NSPN=1), with COUPOT_SIC's pair batches.
int orc_coupot1(orc_problem* p, double* coulomb) {
  Problem& P = p->P;
  if (!P.have_orbitals) return fail("COUPOT1: no orbitals");
  const int nb = P.nbasis, nwf = P.nwfs[0] + P.nwfs[1];
  std::vector<double> dm((size_t)nb * nb, 0.0);
  for (int w = 0; w < nwf; ++w)
    for (int i = 0; i < nb; ++i) {
      const double a = P.psi[(size_t)w * nb + i];
      for (int j = 0; j < nb; ++j) dm[(size_t)i * nb + j] += a * P.psi[(size_t)w * nb + j];
    }
  std::vector<double> rhog((size_t)10 * P.nmsh);
  for (int i = 0; i < P.nmsh; ++i) coulomb[i] = 0.0;
  const bool gga = P.gga();
  auto flush = [&](const std::vector<PairRec>& b, bool weird) {
    if (weird) {
      for (const auto& pr : b) {
        std::vector<PairRec> one(1, pr);
        poisson1(P, one, P.nspn, gga, false, coulomb, rhog.data(), nullptr);
      }
    } else {
      poisson1(P, b, P.nspn, gga, false, coulomb, rhog.data(), nullptr);
    }
  };
  coupot_pairs(P, nullptr, P.nspn, flush, nullptr, dm.data());
  return 0;
}

// DENSOLD (densold.F:5-277): rhog[(s*ngrad + ch)*nmsh + i], phig[s*nmsh + i]
// from the orbital values of frmiorb.f's PSIG accumulation (coefficients at or
// below 1e-10 skipped, as densold.F:160-185).
int orc_densold(orc_problem* p, int ngrad, double* rhog, double* phig) {
  Problem& P = p->P;
  if (!P.have_orbitals) return fail("DENSOLD: no orbitals");
  if (ngrad != 1 && ngrad != 10) return fail("DENSOLD: NGRAD must be 1 or 10");
  const int nb = P.nbasis, nmsh = P.nmsh, ns = P.nspn;
  const int nwf = P.nwfs[0] + P.nwfs[1];
  std::fill(rhog, rhog + (size_t)ns * ngrad * nmsh, 0.0);
  if (phig) std::fill(phig, phig + (size_t)ns * nmsh, 0.0);
  std::vector<double> psig;
  for (int l0 = 0; l0 < nmsh; l0 += MPBLOCK) {
    const int mpts = std::min(MPBLOCK, nmsh - l0);
    orbital_values(P, &P.rmsh[3 * (size_t)l0], mpts, ngrad == 10 ? 2 : 0, ngrad, P.psi.data(), nb, nwf, 0, psig);
    auto F = [&](int w, int ig, int i) { return psig[((size_t)w * ngrad + ig) * mpts + i]; };
    for (int s = 0; s < ns; ++s) {
      const int jbeg = s * P.nwfs[0];
      double* r = rhog + (size_t)s * ngrad * nmsh + l0;
      for (int jwf = 0; jwf < P.nwfs[s]; ++jwf) {
        const int w = jwf + jbeg;
        for (int i = 0; i < mpts; ++i) r[i] = r[i] + F(w, 0, i) * F(w, 0, i);
        if (ngrad == 1) continue;
        for (int ig = 1; ig <= 3; ++ig)
          for (int i = 0; i < mpts; ++i) {
            r[(size_t)ig * nmsh + i] = r[(size_t)ig * nmsh + i] + 2 * F(w, 0, i) * F(w, ig, i);
            if (phig) phig[(size_t)s * nmsh + l0 + i] = phig[(size_t)s * nmsh + l0 + i] + F(w, ig, i) * F(w, ig, i);
          }
        for (int ig = 4; ig <= 6; ++ig)
          for (int i = 0; i < mpts; ++i)
            r[(size_t)ig * nmsh + i] =
                r[(size_t)ig * nmsh + i] + 2 * (F(w, ig - 3, i) * F(w, ig - 3, i) + F(w, ig, i) * F(w, 0, i));
        // (x,y) -> 7, (x,z) -> 8, (y,z) -> 9 as densold.F:232-243 (KGR = IGR+JGR+3)
        for (int ig = 1; ig <= 2; ++ig)
          for (int jg = ig + 1; jg <= 3; ++jg) {
            const int kg = ig + jg + 4;
            for (int i = 0; i < mpts; ++i)
              r[(size_t)kg * nmsh + i] =
                  r[(size_t)kg * nmsh + i] + 2 * (F(w, ig, i) * F(w, jg, i) + F(w, kg, i) * F(w, 0, i));
          }
      }
    }
  }
  return 0;
}

// SICHAM / APATCH / NEWWAY (sicham.F:922-944, sicmat.F:146-318) in C1
// symmetry, MM=2: per FO, BASPHI(mu,1) = sum_p w phi chi_mu and BASPHI(mu,2) =
// -sum_p w V phi chi_mu (for a meta-GGA the weak form of the FO's Hamiltonian:
// + w (grad phi . Z) chi_mu + w phi Z . grad chi_mu + w Z4 grad phi . grad chi_mu),
// HAM(j,i) = BASPHI(i,2) BASPHI(j,1), HSTOR += (HAM + HAM^T)/2.  Adds into
// ham[mu*ldh + nu].
int orc_sicham(orc_problem* p, int spin, double* ham, int ldh) {
  Problem& P = p->P;
  int rc = compute_fmat(P);
  if (rc) return rc;
  rc = compute_tmat(P);
  if (rc) return rc;
  const int s = spin - 1, nf = P.nfrm[s], nb = P.nbasis, nmsh = P.nmsh;
  const bool mg = P.mgga();
  if (nf == 0) return 0;
  std::vector<double> c;
  fo_coefficients(P, s, c);
  std::vector<double> eye((size_t)nb * nb, 0.0);
  for (int m = 0; m < nb; ++m) eye[(size_t)m * nb + m] = 1.0;
  std::vector<double> pots((size_t)nf * nmsh), zm(mg ? (size_t)nf * nmsh * 4 : 0);
  for (int k = 0; k < nf; ++k) {
    double res[13], cf[3];
    rc = apotnl_sic(P, s, k, &c[(size_t)k * nb], res, cf, &pots[(size_t)k * nmsh], nullptr, nullptr, false,
                    mg ? &zm[(size_t)k * nmsh * 4] : nullptr);
    if (rc) return rc;
  }
  std::vector<double> b1((size_t)nf * nb, 0.0), b2((size_t)nf * nb, 0.0), phi, chi;
  for (int l0 = 0; l0 < nmsh; l0 += MPBLOCK) {
    const int mpts = std::min(MPBLOCK, nmsh - l0);
    orbital_values(P, &P.rmsh[3 * (size_t)l0], mpts, 1, 4, c.data(), nb, nf, 1, phi);
    orbital_values(P, &P.rmsh[3 * (size_t)l0], mpts, 1, 4, eye.data(), nb, nb, 1, chi);
    for (int k = 0; k < nf; ++k)
      for (int m = 0; m < nb; ++m) {
        double s1 = 0.0, s2 = 0.0;
        for (int i = 0; i < mpts; ++i) {
          const double w = P.wmsh[l0 + i];
          const double f = phi[((size_t)k * 4) * mpts + i];
          const double x = chi[((size_t)m * 4) * mpts + i];
          s1 = s1 + w * f * x;
          double h = w * pots[(size_t)k * nmsh + l0 + i] * f * x;
          if (mg) {
            const double* z = &zm[((size_t)k * nmsh + l0 + i) * 4];
            for (int cc = 0; cc < 3; ++cc) {
              const double gf = phi[((size_t)k * 4 + 1 + cc) * mpts + i];
              const double gx = chi[((size_t)m * 4 + 1 + cc) * mpts + i];
              h = h + w * (gf * z[cc] * x + f * z[cc] * gx + z[3] * gf * gx);
            }
          }
          s2 = s2 - h;
        }
        b1[(size_t)k * nb + m] += s1;
        b2[(size_t)k * nb + m] += s2;
      }
  }
  for (int k = 0; k < nf; ++k)
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j) {
        // HAM(j,i) = BASPHI(i,2) BASPHI(j,1); symmetrised
        const double hji = b2[(size_t)k * nb + i] * b1[(size_t)k * nb + j];
        const double hij = b2[(size_t)k * nb + j] * b1[(size_t)k * nb + i];
        ham[(size_t)i * ldh + j] += (hji + hij) / 2.0;
      }
  return 0;
}

// APOTNL_SIC of one orbital given by its basis coefficients (no FODs needed):
// RESULTS(1:13) as apotnl_sic.F:564-623 writes them.
int orc_fo_energy(orc_problem* p, int spin, const double* cfo, double* results) {
  Problem& P = p->P;
  std::vector<double> pot(P.nmsh);
  double cfrm[3];
  return apotnl_sic(P, spin - 1, 0, cfo, results, cfrm, pot.data(), nullptr, nullptr, false, nullptr);
}

int orc_set_xc_exact_density(orc_problem* p, int on) {
  p->P.xc_exact_density = on != 0;
  return 0;
}

int orc_set_count_scale(orc_problem* p, double scale) {
  p->P.count_scale = scale > 0.0 ? scale : 1.0;
  return 0;
}

int orc_fo_tau(orc_problem* p, int spin, int iorb, double* tau) {
  Problem& P = p->P;
  if (!P.have_tmat) {
    int rc = compute_tmat(P);
    if (rc) return rc;
  }
  std::vector<double> c, t;
  fo_coefficients(P, spin - 1, c);
  fo_tau(P, &c[(size_t)(iorb - 1) * P.nbasis], t);
  std::memcpy(tau, t.data(), sizeof(double) * P.nmsh);
  return 0;
}

int orc_apotnl_sic(orc_problem* p, int spin, int iorb, double* results, double* cfrm, double* pot,
                   double* coulomb, double* rhog, double* mixin) {
  Problem& P = p->P;
  if (!P.have_tmat) {
    int rc = compute_tmat(P);
    if (rc) return rc;
  }
  std::vector<double> c;
  fo_coefficients(P, spin - 1, c);
  return apotnl_sic(P, spin - 1, iorb - 1, &c[(size_t)(iorb - 1) * P.nbasis], results, cfrm, pot, coulomb, rhog,
                    false, P.mgga() ? mixin : nullptr);
}

int orc_siclagm(orc_problem* p, int spin, const double* pots, const double* zm, double* sic, int ld) {
  Problem& P = p->P;
  if (!P.have_tmat) {
    int rc = compute_tmat(P);
    if (rc) return rc;
  }
  std::vector<double> c;
  fo_coefficients(P, spin - 1, c);
  if (P.mgga() && !zm) return fail("SICLAGM: a meta-GGA needs the FOs' MIXIN arrays");
  siclagm(P, spin - 1, pots, c.data(), sic, ld, zm);
  return 0;
}

int orc_frmorb2_force(orc_problem* p, int spin, const double* sic, int ld, double* debdax) {
  Problem& P = p->P;
  if (!P.have_fmat) {
    int rc = compute_fmat(P);
    if (rc) return rc;
  }
  return frmorb2_force(P, spin - 1, sic, ld, debdax);
}

int orc_sic_cycle(orc_problem* p, int ld, double* results, double* sic, double* debdax, double* cfrm,
                  double* esic, int nthreads, int fo_limit) {
  Problem& P = p->P;
  int rc = compute_fmat(P);
  if (rc) return rc;
  rc = compute_tmat(P);
  if (rc) return rc;
  double zsic = 0.0;
  for (int s = 0; s < P.nspn; ++s) {
    std::vector<double> c;
    fo_coefficients(P, s, c);
    int nf = P.nfrm[s];
    int nrun = (fo_limit > 0) ? std::min(fo_limit, nf) : nf;
    std::vector<double> pots((size_t)nf * P.nmsh, 0.0);
    std::vector<double> zm(P.mgga() ? (size_t)nf * P.nmsh * 4 : 0, 0.0);
    std::vector<int> rcs(nf, 0);
    {
      std::atomic<int> next(0);
      auto work = [&]() {
        for (;;) {
          int k = next.fetch_add(1);
          if (k >= nrun) break;
          double res[13], cf[3];
          rcs[k] = apotnl_sic(P, s, k, &c[(size_t)k * P.nbasis], res, cf, &pots[(size_t)k * P.nmsh], nullptr,
                              nullptr, false, P.mgga() ? &zm[(size_t)k * P.nmsh * 4] : nullptr);
          for (int i = 0; i < 13; ++i) results[((size_t)s * ld + k) * 13 + i] = res[i];
          for (int i = 0; i < 3; ++i) cfrm[((size_t)s * ld + k) * 3 + i] = cf[i];
        }
      };
      int nt = std::max(1, std::min(nthreads, nrun));
      std::vector<std::thread> th;
      for (int t = 1; t < nt; ++t) th.emplace_back(work);
      work();
      for (auto& x : th) x.join();
    }
    for (int k = 0; k < nrun; ++k)
      if (rcs[k]) return rcs[k];
    if (fo_limit > 0 && nrun < nf) continue;  // sampled timing run: no SIC matrix / forces
    siclagm(P, s, pots.data(), c.data(), &sic[(size_t)s * ld * ld], ld, P.mgga() ? zm.data() : nullptr);
    rc = frmorb2_force(P, s, &sic[(size_t)s * ld * ld], ld, &debdax[(size_t)s * ld * 3]);
    if (rc) return rc;
    for (int k = 0; k < nf; ++k) zsic += results[((size_t)s * ld + k) * 13 + 8];
  }
  *esic = zsic;
  return 0;
}

int orc_xc_point(int igga_x, int idftyp_x, int igga_c, int idftyp_c, const double* r10, double w, double* v2,
                 double* e4) {
  Problem P;
  P.igga[0] = igga_x;
  P.igga[1] = igga_c;
  P.idftyp[0] = idftyp_x;
  P.idftyp[1] = idftyp_c;
  double rht[2][10];
  for (int k = 0; k < 10; ++k) {
    rht[0][k] = r10[k];
    rht[1][k] = 0.0;
  }
  v2[0] = v2[1] = 0.0;
  for (int i = 0; i < 4; ++i) e4[i] = 0.0;
  subvlxc_point(P, rht, w, v2, e4);
  return 0;
}

void orc_scan_x(double rho, double drho, double tau, double* out) {
  scan_x_unp(rho, drho, tau, out[0], out[1], out[2], out[3]);
}
void orc_scan_c(double ru, double rd, double dru, double drd, double drt, double tauu, double taud, double* out) {
  double vc[2], vcdd[2];
  scan_c(ru, rd, dru, drd, drt, tauu, taud, out[0], vc, vcdd, out[5]);
  out[1] = vc[0];
  out[2] = vc[1];
  out[3] = vcdd[0];
  out[4] = vcdd[1];
  out[6] = 0.0;
}

void orc_boys(int maxfmt, double x, double* s) { boys(maxfmt, x, std::exp(-x), s); }
void orc_harmonics(int lm, const double* xyz, double* y) { harmonics(lm, xyz[0], xyz[1], xyz[2], y); }
int orc_lebedev19(double* ang, double* w) {
  const Lebedev19& L = lebedev19();
  for (int i = 0; i < NANG; ++i) {
    for (int d = 0; d < 3; ++d) ang[3 * i + d] = L.ang[i][d];
    w[i] = L.w[i];
  }
  return NANG;
}

}  // extern "C"
