// Host runtime and C ABI of libflosic_sic_b200.
//
// The context keeps the module state of the reference SIC routines resident
// on one GPU: basis tables, the mesh (sorted into spatial tiles), the
// Gaussian-pair plan of COUPOT_SIC (coupot_sic.F:228-640, built once per
// geometry in the reference's serial batching order), KS orbitals and FODs.
// A spin's FO potentials are computed for all FOs in batched launches and
// cached in GPU memory; APOTNL_SIC / SICLAGM / FRMORB2 entry points read from
// that cache instead of the ZPOT#### files.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/flosic_sic.h"
#include "common.cuh"
#include "kernels.cuh"

using namespace flosic;

namespace {

thread_local std::string g_err;

struct Fail {
  int code;
};

[[noreturn]] void fail(int code, const std::string& msg) {
  g_err = msg;
  throw Fail{code};
}

#define CUDA_CHECK(x)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess) fail(FLOSIC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

const int kNcomp[3] = {1, 3, 6};
const int kShift[3] = {0, 1, 4};
const int kPow[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                         {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  void ensure(size_t m) {
    if (m <= n && p) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    if (m == 0) return;
    CUDA_CHECK(cudaMalloc(&p, sizeof(T) * m));
    n = m;
  }
  void upload(const T* h, size_t m, cudaStream_t st) {
    ensure(m);
    if (m) CUDA_CHECK(cudaMemcpyAsync(p, h, sizeof(T) * m, cudaMemcpyHostToDevice, st));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// ---------------------------------------------------------------------------
// LOWSIC (lowden_files.f:2-172): S^{-1/2} of the FO overlap from its
// eigen-decomposition (the role of DIAGGE_FO, diagon_sic.f:45); sym_eigen(n, a,
// w, v) returns the eigenvalues w and v[k*n + m] = component k of eigenvector m.
// ---------------------------------------------------------------------------
template <class Eig>
void lowsic(Eig&& sym_eigen, int n, const std::vector<double>& over, std::vector<double>& sm12,
            std::vector<double>& filo, std::vector<double>& lam) {
  std::vector<double> w;
  sym_eigen(n, over, w, filo);
  for (int i = 0; i < n; ++i)
    if (w[i] < 1.0e-8)
      fail(FLOSIC_ERR_LOWDEN, "LOWSIC: LOWDEN EIGENVALUES TOO SMALL (< 1e-8): BAD POSITIONS IN FRMORB");
  std::vector<double> e(n);
  for (int i = 0; i < n; ++i) e[i] = 1.0 / std::sqrt(w[i]);
  lam.resize(n);
  for (int i = 0; i < n; ++i) lam[i] = 1.0 / (e[i] * e[i]);
  sm12.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int m = 0; m < n; ++m) s += filo[(size_t)j * n + m] * filo[(size_t)i * n + m] * e[m];
      sm12[(size_t)i * n + j] = s;
    }
}

// Boys-function table of fffmtc.F:25-97 (series for F_19, downward recursion),
// columns F2 F3 F4 F5 F4/2 F5/2 F6/2 F5/6 F6/6 F7/6.
std::vector<double> boys_table() {
  std::vector<double> T((size_t)BOYS_NT * BOYS_NC);
  for (int L = 1; L <= BOYS_NT; ++L) {
    double F[10];
    if (L == 1) {
      for (int i = 0; i < 10; ++i) F[i] = 1.0 / (2 * (i + 1) - 1);
    } else {
      const double t = (1.0e-2) * (L - 1);
      const double x = 2 * t;
      double den = 39.0, term = 1.0 / den, sum = term;
      for (int i = 2; i <= 100; ++i) {
        den = den + 2.0;
        term = term * x / den;
        sum = sum + term;
        if (term / sum - 1.0e-12 <= 0) break;
      }
      const double ex = std::exp(-t);
      double G[21];
      G[20] = ex * sum;
      for (int i = 1; i <= 19; ++i) {
        const int K = 21 - i, KK = K - 1;
        G[KK] = (x * G[K] + ex) / (2 * KK - 1);
      }
      for (int i = 0; i < 10; ++i) F[i] = G[i + 1];
    }
    double* r = &T[(size_t)(L - 1) * BOYS_NC];
    r[0] = F[2];
    r[1] = F[3];
    r[2] = F[4];
    r[3] = F[5];
    r[4] = F[4] / 2.0;
    r[5] = F[5] / 2.0;
    r[6] = F[6] / 2.0;
    r[7] = F[5] / 6.0;
    r[8] = F[6] / 6.0;
    r[9] = F[7] / 6.0;
  }
  return T;
}

// Lebedev degree-19 mesh in the generation order of lebedev.F:741-905.
void lebedev19(std::vector<double>& ang, std::vector<double>& w) {
  const double RT2RC = 0.70710678118654752440, RT3RC = 0.57735026918962576451;
  const double A1 = 0.00753519001311713812, A2 = 0.09265184700375432421, A3 = 0.09061000833610514010;
  const double B[3] = {0.09518264418191036893, 0.08487112439121475736, 0.08942676055004592969};
  const double AL[3] = {0.15746766720390817632, 0.41749612279654533594, 0.67644104001142636987};
  const double AM[3] = {0.97488864367717323548, 0.80708981835958250163, 0.29129888220952674629};
  const double D1 = 0.08785259467896816188, AR1 = 0.14035538117131832857, AU1 = 0.44933283232695573488,
               AW1 = 0.88227001126032263192;
  ang.clear();
  w.clear();
  auto push = [&](double x, double y, double z, double wt) {
    ang.push_back(x);
    ang.push_back(y);
    ang.push_back(z);
    w.push_back(wt);
  };
  double sg[3];
  for (int i = 0; i < 3; ++i) {
    sg[0] = 1.0;
    for (int j = 0; j < 2; ++j) {
      double p[3] = {0, 0, 0};
      p[i] = sg[0];
      push(p[0], p[1], p[2], A1);
      sg[0] = -sg[0];
    }
  }
  for (int i = 0; i < 3; ++i) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    sg[0] = RT2RC;
    for (int j = 0; j < 2; ++j) {
      sg[1] = RT2RC;
      for (int k = 0; k < 2; ++k) {
        double p[3];
        p[i] = 0.0;
        p[i1] = sg[0];
        p[i2] = sg[1];
        push(p[0], p[1], p[2], A2);
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
        push(sg[0], sg[1], sg[2], A3);
        sg[2] = -sg[2];
      }
      sg[1] = -sg[1];
    }
    sg[0] = -sg[0];
  }
  for (int g = 0; g < 3; ++g) {
    for (int i = 0; i < 3; ++i) {
      const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
      sg[i] = AM[g];
      for (int j = 0; j < 2; ++j) {
        sg[i1] = AL[g];
        for (int k = 0; k < 2; ++k) {
          sg[i2] = AL[g];
          for (int l = 0; l < 2; ++l) {
            push(sg[0], sg[1], sg[2], B[g]);
            sg[i2] = -sg[i2];
          }
          sg[i1] = -sg[i1];
        }
        sg[i] = -sg[i];
      }
    }
  }
  for (int i = 0; i < 3; ++i) {
    sg[i] = AR1;
    for (int j = 0; j < 2; ++j) {
      int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
      for (int k = 0; k < 2; ++k) {
        sg[i1] = AU1;
        for (int l = 0; l < 2; ++l) {
          sg[i2] = AW1;
          for (int m = 0; m < 2; ++m) {
            push(sg[0], sg[1], sg[2], D1);
            sg[i2] = -sg[i2];
          }
          sg[i1] = -sg[i1];
        }
        std::swap(i1, i2);
      }
      sg[i] = -sg[i];
    }
  }
}

struct TypeInfo {
  int nbare, lmax, nloc;
  int ncon[3];
  double alp[MAX_BARE];
  double con[3][MAX_CON][MAX_BARE];
};

// Coulomb inputs of one spin for a batched launch over many molecules (the
// per-molecule path keeps them in the context and reuses them per spin).
struct CoulBufs {
  DevBuf<double> coef, cgp, mom;
  DevBuf<int8_t> maxfmt, pairfmt;
  DevBuf<CallFO> callfo;
  DevBuf<CallShare> share;
  DevBuf<int> lists;
  DevBuf<unsigned long long> cnt;
  void release() {
    coef.release();
    cgp.release();
    mom.release();
    maxfmt.release();
    pairfmt.release();
    callfo.release();
    share.release();
    lists.release();
    cnt.release();
  }
};

struct SpinCache {
  bool fo_valid = false;       // FMAT/TMAT/CFO
  bool pot_valid = false;      // potentials, RESULTS
  int nf = 0, nw = 0;
  std::vector<double> fmat;    // [(K*nf + jfm)*nw + jwf]
  std::vector<double> tmat;    // [k*nw + jwf]
  std::vector<double> lam;     // Lowdin eigenvalues
  std::vector<double> filo;    // Lowdin eigenvectors [k*nf + a]: component k of eigenvector a
  std::vector<double> results; // [k*13 + i]
  std::vector<double> parts;   // [k*NPART + j] mesh sums of this context's shard
  std::vector<double> asy;     // [k] scaled Coulomb potential at the farthest point (0 off this shard)
  std::vector<double> cfrm;    // [k*3 + d]
  std::vector<double> sic;     // [l*nf + j] = SIC(j,l)
  bool sic_valid = false;
  DevBuf<double> cfo;          // nb x nf
  DevBuf<double> phi;          // [ch][k][P]
  DevBuf<double> vh;           // raw Coulomb [k][P]
  DevBuf<double> vpot;         // SIC potential [k][P]
  DevBuf<double> y;            // w V phi [k][P]
  DevBuf<double> rhog;         // pair-route density channels [ch][k][P] (FLOSIC_DENSITY_PAIRS)
  CoulBufs bc;                 // batched Coulomb launch only
  void release() {
    bc.release();
    rhog.release();
    cfo.release();
    phi.release();
    vh.release();
    vpot.release();
    y.release();
  }
};

}  // namespace

struct flosic_ctx {
  int device = 0;
  cudaStream_t st = nullptr;
  DevBuf<double> d_gemm_ws;  // split-K partial products of dgemm
  DevBuf<CoulombJob> d_jobs;  // batched Coulomb launch led by this context
  DevBuf<int4> d_items;
  DevBuf<int> d_batch_counters;
  DevBuf<double> d_eig_a, d_eig_w, d_eig_v, d_eig_work;
  DevBuf<int> d_eig_info;
  bool have_geom = false, have_orb = false;
  // geometry
  int natoms = 0, ntypes = 0, nbasis = 0, nprim = 0, nmsh = 0, nspn = 1, gga = 0;
  int mgga = 0;  // SCAN: FO values and gradients only, tau and the meta-GGA SIC-matrix terms
  // FO value channels kept on the mesh: value (LDA), + gradient (meta-GGA),
  // + second derivatives (GGA, whose potential uses the Laplacian terms)
  int nch() const { return mgga ? 4 : (gga ? 10 : 1); }
  int nderv() const { return mgga ? 1 : (gga ? 2 : 0); }
  int xc[4] = {0, 6, 0, 6};
  std::vector<TypeInfo> types;
  std::vector<int> atype, aoff, apoff;
  std::vector<double> rat;
  std::vector<int> perm;       // sorted index -> original index
  int ntiles = 0;
  int ifar_sorted = 0;         // farthest point from the origin (apotnl_sic.F:410-418)
  double rmx = 0.0;
  // Mesh shard this context evaluates: tiles [eval_t0, eval_t0 + eval_nt) of
  // the sorted mesh = sorted points [eval_p0, eval_p0 + eval_n).  One shard
  // (the default) is the whole mesh.
  int shard = 0, nshards = 1;
  int eval_t0 = 0, eval_nt = 0, eval_p0 = 0, eval_n = 0;
  std::vector<PairGeo> pairs;
  std::vector<CallInfo> calls;
  // device geometry
  DevBuf<double> d_atom_pos, d_type_alpha, d_type_amin, d_type_bfcon;
  DevBuf<int> d_atom_type, d_atom_boff, d_atom_poff, d_type_nbare, d_type_lmax, d_type_ncon, d_prim_atom,
      d_prim_ib;
  DevBuf<double> d_x, d_y, d_z, d_w, d_tlo, d_thi, d_boys;
  DevBuf<PairGeo> d_pairs;
  DevBuf<CallInfo> d_calls;
  // orbitals
  int nwfs[2] = {0, 0}, nfrm[2] = {0, 0};
  std::vector<double> psi;     // nb x nwf (column-major)
  std::vector<double> fods[2];
  DevBuf<double> d_psi, d_psi_thr;
  SpinCache spin[2];
  // scratch
  DevBuf<double> d_basis, d_fodpts, d_psig, d_tmat, d_u, d_coef, d_cgp, d_mom, d_part, d_sums, d_sic, d_tmp;
  DevBuf<int8_t> d_maxfmt, d_pairfmt;
  DevBuf<CallShare> d_share;
  DevBuf<int> d_lists, d_tc_err;
  DevBuf<int> d_setup_list;  // one-slot calls first (nsingle), then the others
  int nsingle = 0;
  DevBuf<float> d_coef_hl, d_momv_hl;
  CoulombConfig coulomb_cfg;     // FLOSIC_COULOMB=perfo, FLOSIC_SHARED=mma, FLOSIC_PERFO_WM=1|2|4 (A/B checks)
  int precision = FLOSIC_PRECISION_FP64;
  int density = FLOSIC_DENSITY_PHI2;
  DevBuf<double> d_dens_coef;    // pair-route density polynomials of one spin (FLOSIC_DENSITY_PAIRS)
  DevBuf<unsigned long long> d_cnt;
  unsigned long long work_near = 0, work_far = 0, work_terms = 0;
  DevBuf<CallFO> d_callfo;
  // stats
  long long launches = 0;
  double stage_ms[7] = {0, 0, 0, 0, 0, 0, 0};
  double kernel_ms[2] = {0, 0};  // Coulomb evaluation: shared-geometry kernel (with call set-up), per-FO kernel
  unsigned long long kernel_work[6] = {0, 0, 0, 0, 0, 0};  // near/far/terms of each
  cudaEvent_t ev[10] = {};

  BasisDev basis_dev() const {
    BasisDev B;
    B.natoms = natoms;
    B.ntypes = ntypes;
    B.nbasis = nbasis;
    B.nprim = nprim;
    B.atom_pos = d_atom_pos.p;
    B.atom_type = d_atom_type.p;
    B.atom_boff = d_atom_boff.p;
    B.atom_poff = d_atom_poff.p;
    B.type_nbare = d_type_nbare.p;
    B.type_lmax = d_type_lmax.p;
    B.type_ncon = d_type_ncon.p;
    B.type_alpha = d_type_alpha.p;
    B.type_amin = d_type_amin.p;
    B.type_bfcon = d_type_bfcon.p;
    B.prim_atom = d_prim_atom.p;
    B.prim_ib = d_prim_ib.p;
    return B;
  }
  MeshDev mesh_dev() const {
    MeshDev M;
    M.n = nmsh;
    M.ntiles = ntiles;
    M.x = d_x.p;
    M.y = d_y.p;
    M.z = d_z.p;
    M.w = d_w.p;
    M.tile_lo = d_tlo.p;
    M.tile_hi = d_thi.p;
    return M;
  }
  // The shard's tiles as a mesh of their own (tile-aligned, so every per-tile
  // kernel runs on it unchanged).
  MeshDev eval_mesh() const {
    MeshDev M = mesh_dev();
    M.n = eval_n;
    M.ntiles = eval_nt;
    M.x += eval_p0;
    M.y += eval_p0;
    M.z += eval_p0;
    M.w += eval_p0;
    M.tile_lo += 3 * (size_t)eval_t0;
    M.tile_hi += 3 * (size_t)eval_t0;
    return M;
  }
};

namespace {

// ---------------------------------------------------------------------------
// Pair plan of COUPOT_SIC (coupot_sic.F:149-790), geometry only.
// ---------------------------------------------------------------------------
void build_pair_plan(flosic_ctx* c) {
  std::vector<std::array<double, 3>> center;
  double dmin = 1.0e30;
  for (int a = 0; a < c->natoms; ++a) {
    std::array<double, 3> p = {c->rat[3 * a], c->rat[3 * a + 1], c->rat[3 * a + 2]};
    center.push_back(p);
    const double d = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
    if (d < dmin) dmin = d;
  }
  int mcnt = (int)center.size();
  if (std::sqrt(dmin) > 0.7) {
    center.push_back({0.0, 0.0, 0.0});
    ++mcnt;
  }
  const int nclass = mcnt + 1;
  std::vector<std::vector<PairGeo>> buf((size_t)nclass * 3);
  std::vector<PairGeo> pairs;
  std::vector<CallInfo> calls;
  const int nspn = c->nspn;
  auto flush = [&](std::vector<PairGeo>& b, bool weird) {
    auto emit = [&](const PairGeo* first, int n) {
      // the per-FO Coulomb kernel stages a call's pairs in MXPR shared slots
      if (n > MXPR) fail(FLOSIC_ERR_CAPACITY, "Poisson call with more than MXPR pairs");
      CallInfo ci;
      ci.p0 = (int)pairs.size();
      ci.np = n;
      ci.slots = n * nspn;
      ci.pad = 0;
      ci.delta_min = 1.0e30;
      for (int i = 0; i < n; ++i) {
        PairGeo g = first[i];
        g.call = (int)calls.size();
        ci.delta_min = std::min(ci.delta_min, g.delta);
        pairs.push_back(g);
      }
      calls.push_back(ci);
    };
    if (weird)
      for (auto& g : b) emit(&g, 1);
    else
      emit(b.data(), (int)b.size());
    b.clear();
  };
  for (int ia = 0; ia < c->natoms; ++ia) {
    const TypeInfo& ti = c->types[c->atype[ia]];
    const double* AI = &c->rat[3 * ia];
    for (int ja = ia; ja < c->natoms; ++ja) {
      const TypeInfo& tj = c->types[c->atype[ja]];
      const double* AJ = &c->rat[3 * ja];
      const double times_sites = (ja > ia) ? 2.0 : 1.0;
      const double rarg = (AI[0] - AJ[0]) * (AI[0] - AJ[0]) + (AI[1] - AJ[1]) * (AI[1] - AJ[1]) +
                          (AI[2] - AJ[2]) * (AI[2] - AJ[2]);
      for (int ialp = 0; ialp < ti.nbare; ++ialp) {
        const double ai = ti.alp[ialp];
        for (int jalp = (ia == ja) ? ialp : 0; jalp < tj.nbare; ++jalp) {
          const double times_alpha = (ia == ja && jalp > ialp) ? 2.0 : 1.0;
          const double aj = tj.alp[jalp];
          const double rcalp = 1.0 / (ai + aj);
          const double arg = ai * aj * rcalp * rarg;
          if (arg > CUTEXP) continue;
          double C[3];
          for (int d = 0; d < 3; ++d) C[d] = (ai * AI[d] + aj * AJ[d]) * rcalp;
          double dm = 1.0e30;
          int minc = 0;
          for (int ic = 0; ic < mcnt; ++ic) {
            const double dist = std::sqrt((C[0] - center[ic][0]) * (C[0] - center[ic][0]) +
                                          (C[1] - center[ic][1]) * (C[1] - center[ic][1]) +
                                          (C[2] - center[ic][2]) * (C[2] - center[ic][2]));
            if (dist < dm) {
              dm = dist;
              minc = ic;
            }
          }
          if ((ai + aj) * dm * dm > 0.5) minc = mcnt;
          if (ai + aj < 3.0) minc = mcnt;
          int lng = 0;
          if (ai + aj > 10.0) lng = 1;
          if (ai + aj > 40.0) lng = 2;
          PairGeo g;
          std::memset(&g, 0, sizeof(g));
          g.a = ai;
          g.b = aj;
          for (int d = 0; d < 3; ++d) {
            g.A[d] = AI[d];
            g.B[d] = AJ[d];
          }
          // poisson1.f:299-325
          const double delta = ai + aj;
          const double rcdelt = 1.0 / delta;
          const double parg = ai * aj * rcdelt *
                              ((AI[0] - AJ[0]) * (AI[0] - AJ[0]) + (AI[1] - AJ[1]) * (AI[1] - AJ[1]) +
                               (AI[2] - AJ[2]) * (AI[2] - AJ[2]));
          g.factor = 6.283185307179586 * std::exp(-parg) * rcdelt;
          for (int d = 0; d < 3; ++d) g.C[d] = (ai * AI[d] + aj * AJ[d]) * rcdelt;
          g.delta = delta;
          g.times = times_sites * times_alpha;
          g.pi = c->apoff[ia] + ialp;
          g.pj = c->apoff[ja] + jalp;
          auto& b = buf[(size_t)minc * 3 + lng];
          b.push_back(g);
          if ((int)b.size() * nspn == MXPR) flush(b, minc == mcnt);
        }
      }
    }
  }
  for (int lng = 0; lng < 3; ++lng)
    for (int minc = 0; minc < nclass; ++minc) {
      auto& b = buf[(size_t)minc * 3 + lng];
      if (!b.empty()) flush(b, minc == mcnt);
    }
  c->pairs.swap(pairs);
  c->calls.swap(calls);
}

// Spatial sort of the mesh into tiles of TILE points (Morton order).
void sort_mesh(flosic_ctx* c, const double* rmsh, const double* wmsh) {
  const int n = c->nmsh;
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], rmsh[3 * i + d]);
      hi[d] = std::max(hi[d], rmsh[3 * i + d]);
    }
  auto spread = [](uint64_t v) {
    uint64_t x = v & 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
  };
  std::vector<std::pair<uint64_t, int>> key(n);
  for (int i = 0; i < n; ++i) {
    uint64_t q[3];
    for (int d = 0; d < 3; ++d) {
      const double ext = hi[d] - lo[d];
      double f = ext > 0 ? (rmsh[3 * i + d] - lo[d]) / ext : 0.0;
      q[d] = (uint64_t)std::min(2097151.0, std::max(0.0, f * 2097151.0));
    }
    key[i] = {spread(q[0]) | (spread(q[1]) << 1) | (spread(q[2]) << 2), i};
  }
  std::sort(key.begin(), key.end());
  c->perm.resize(n);
  std::vector<double> x(n), y(n), z(n), w(n);
  for (int i = 0; i < n; ++i) {
    const int o = key[i].second;
    c->perm[i] = o;
    x[i] = rmsh[3 * o];
    y[i] = rmsh[3 * o + 1];
    z[i] = rmsh[3 * o + 2];
    w[i] = wmsh[o];
  }
  c->ntiles = (n + TILE - 1) / TILE;
  std::vector<double> tlo(3 * (size_t)c->ntiles), thi(3 * (size_t)c->ntiles);
  for (int t = 0; t < c->ntiles; ++t) {
    double l[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, h[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int i = t * TILE; i < std::min(n, (t + 1) * TILE); ++i) {
      const double p[3] = {x[i], y[i], z[i]};
      for (int d = 0; d < 3; ++d) {
        l[d] = std::min(l[d], p[d]);
        h[d] = std::max(h[d], p[d]);
      }
    }
    for (int d = 0; d < 3; ++d) {
      tlo[3 * t + d] = l[d];
      thi[3 * t + d] = h[d];
    }
  }
  // farthest point from the origin, first in the original order on ties
  double rmx = 0.0;
  int ifar = 0;
  for (int i = 0; i < n; ++i) {
    const double rad = std::sqrt(rmsh[3 * i] * rmsh[3 * i] + rmsh[3 * i + 1] * rmsh[3 * i + 1] +
                                 rmsh[3 * i + 2] * rmsh[3 * i + 2]);
    if (rad > rmx) {
      rmx = rad;
      ifar = i;
    }
  }
  c->rmx = rmx;
  for (int i = 0; i < n; ++i)
    if (c->perm[i] == ifar) c->ifar_sorted = i;
  cudaStream_t st = c->st;
  c->d_x.upload(x.data(), n, st);
  c->d_y.upload(y.data(), n, st);
  c->d_z.upload(z.data(), n, st);
  c->d_w.upload(w.data(), n, st);
  c->d_tlo.upload(tlo.data(), tlo.size(), st);
  c->d_thi.upload(thi.data(), thi.size(), st);
}

void invalidate(flosic_ctx* c) {
  for (auto& s : c->spin) {
    s.fo_valid = s.pot_valid = s.sic_valid = false;
  }
}

// Tiles of shard `shard` of `nshards`: an even split of the sorted tiles.
void set_eval_range(flosic_ctx* c) {
  const long long nt = c->ntiles;
  const int t0 = (int)(nt * c->shard / c->nshards), t1 = (int)(nt * (c->shard + 1) / c->nshards);
  c->eval_t0 = t0;
  c->eval_nt = t1 - t0;
  c->eval_p0 = t0 * TILE;
  c->eval_n = std::min(t1 * TILE, c->nmsh) - c->eval_p0;
}

// ---------------------------------------------------------------------------
// FO construction (FRMORB2(0,0) and FRMIORB(1,1)) for one spin
// ---------------------------------------------------------------------------
// C = alpha op(A) op(B) + beta C on the context stream (column-major, as BLAS
// DGEMM), on the FP64 tensor cores (csrc/contract.cu).
void gemm(flosic_ctx* c, bool ta, bool tb, int M, int N, int K, double alpha, const double* A, int lda,
          const double* B, int ldb, double beta, double* C, int ldc) {
  const size_t w = dgemm_work(M, N, K);
  if (w) c->d_gemm_ws.ensure(w);
  dgemm(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, c->d_gemm_ws.p, c->st);
  c->launches += w ? 2 : 1;
}

// Symmetric eigen-decomposition on the GPU (k_sym_eigen, cyclic Jacobi,
// FP64, ascending eigenvalues) in the convention lowsic expects.
auto device_eigen(flosic_ctx* c) {
  return [c](int n, const std::vector<double>& a, std::vector<double>& w, std::vector<double>& v) {
    cudaStream_t st = c->st;
    c->d_eig_a.upload(a.data(), (size_t)n * n, st);
    c->d_eig_w.ensure(n);
    c->d_eig_v.ensure((size_t)n * n);
    c->d_eig_work.ensure(sym_eigen_work(n));
    c->d_eig_info.ensure(1);
    if (!launch_sym_eigen(n, c->d_eig_a.p, c->d_eig_work.p, c->d_eig_w.p, c->d_eig_v.p, c->d_eig_info.p, st))
      fail(FLOSIC_ERR_CAPACITY, "LOWSIC: more FOs per spin than the eigen-solver holds");
    c->launches++;
    CUDA_CHECK(cudaGetLastError());
    v.resize((size_t)n * n);
    w.resize(n);
    int info = 0;
    CUDA_CHECK(cudaMemcpyAsync(v.data(), c->d_eig_v.p, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, st));
    CUDA_CHECK(cudaMemcpyAsync(w.data(), c->d_eig_w.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CUDA_CHECK(cudaMemcpyAsync(&info, c->d_eig_info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_CHECK(cudaStreamSynchronize(st));
    if (info != 0) fail(FLOSIC_ERR_LOWDEN, "LOWSIC: eigen-decomposition of the FO overlap did not converge");
  };
}

void fo_setup(flosic_ctx* c, int s) {
  SpinCache& S = c->spin[s];
  if (S.fo_valid) return;
  const int nw = c->nwfs[s], nf = c->nfrm[s], nb = c->nbasis;
  if (nw != nf) fail(FLOSIC_ERR_NFRM, "FRMIORB: MORB .NE. NFRM");
  if (nf <= 0) fail(FLOSIC_ERR_ARG, "no FODs for this spin");
  S.nf = nf;
  S.nw = nw;
  cudaStream_t st = c->st;
  // orbital values and gradients at the FODs (basis values -> PSIG by DGEMM with
  // the KS coefficients whose magnitude exceeds 1e-10, frmorb2.F:270-286)
  std::vector<double> pts(3 * (size_t)nf);
  for (int k = 0; k < nf; ++k)
    for (int d = 0; d < 3; ++d) pts[(size_t)d * nf + k] = c->fods[s][3 * k + d];
  c->d_fodpts.upload(pts.data(), pts.size(), st);
  c->d_psig.ensure((size_t)4 * nf * nw);
  const double* cthr = c->d_psi_thr.p + (size_t)s * c->nwfs[0] * nb;
  // PSIG_ch (nf x nw) = B_ch (FODs x nb) * C (nb x nw), basis values formed in the kernel
  launch_fo_values(c->basis_dev(), 1, nf, c->d_fodpts.p, c->d_fodpts.p + nf, c->d_fodpts.p + 2 * nf, cthr, nb, nw,
                   c->d_psig.p, nf, c->coulomb_cfg.fo_values_bn, st);
  c->launches++;
  std::vector<double> psig((size_t)4 * nf * nw);
  CUDA_CHECK(cudaMemcpyAsync(psig.data(), c->d_psig.p, sizeof(double) * psig.size(), cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  auto PS = [&](int ch, int k, int j) { return psig[((size_t)ch * nw + j) * nf + k]; };
  // FMAT (frmorb2.F:296-346)
  S.fmat.assign((size_t)4 * nf * nw, 0.0);
  for (int k = 0; k < nf; ++k) {
    double rhi[4] = {0, 0, 0, 0};
    for (int j = 0; j < nw; ++j)
      for (int K = 0; K < 4; ++K) rhi[K] = rhi[K] + PS(0, k, j) * PS(K, k, j);
    if (!(rhi[0] > 0.0)) fail(FLOSIC_ERR_ZERO_DENSITY, "FRMORB2: zero density at an FOD");
    for (int K = 0; K < 4; ++K)
      for (int j = 0; j < nw; ++j) {
        double f = PS(K, k, j) / std::sqrt(rhi[0]);
        if (K >= 1) f = f - S.fmat[((size_t)0 * nf + k) * nw + j] * rhi[K] / rhi[0];
        S.fmat[((size_t)K * nf + k) * nw + j] = f;
      }
  }
  // TMAT (frmiorb.f:351-480)
  std::vector<double> T((size_t)nf * nw), over((size_t)nf * nf);
  for (int k = 0; k < nf; ++k) {
    double rho = 0.0;
    for (int j = 0; j < nw; ++j) rho = rho + PS(0, k, j) * PS(0, k, j);
    if (!(rho > 0.0)) fail(FLOSIC_ERR_ZERO_DENSITY, "FRMIORB: zero density at an FOD");
    for (int j = 0; j < nw; ++j) T[(size_t)k * nw + j] = PS(0, k, j) / std::sqrt(rho);
  }
  for (int i = 0; i < nf; ++i)
    for (int j = 0; j < nf; ++j) {
      double v = 0.0;
      for (int w = 0; w < nw; ++w) v = v + T[(size_t)i * nw + w] * T[(size_t)j * nw + w];
      over[(size_t)i * nf + j] = v;
    }
  std::vector<double> sm12;
  lowsic(device_eigen(c), nf, over, sm12, S.filo, S.lam);
  S.tmat.assign((size_t)nf * nw, 0.0);
  for (int i = 0; i < nf; ++i)
    for (int k = 0; k < nf; ++k) {
      const double h = sm12[(size_t)k * nf + i];
      for (int w = 0; w < nw; ++w) S.tmat[(size_t)i * nw + w] += h * T[(size_t)k * nw + w];
    }
  // FO coefficients C_FO(nb x nf) = C_KS(nb x nw) * TMAT^T (unravel2.f:200-240)
  c->d_tmat.upload(S.tmat.data(), S.tmat.size(), st);
  S.cfo.ensure((size_t)nb * nf);
  const double* cks = c->d_psi.p + (size_t)s * c->nwfs[0] * nb;
  gemm(c, false, false, nb, nf, nw, 1.0, cks, nb, c->d_tmat.p, nw, 0.0, S.cfo.p, nb);
  S.fo_valid = true;
}

// FO values (+ derivatives for GGA) on the mesh: phi[(ch*nf + k)*P + p]
void fo_values(flosic_ctx* c, int s) {
  SpinCache& S = c->spin[s];
  const int nf = S.nf, nb = c->nbasis, P = c->eval_n;
  const int nch = c->nch();
  const int nderv = c->nderv();
  S.phi.ensure((size_t)nch * nf * P);
  // Phi_ch (P x nf) = B_ch (P x nb) C_FO, basis values formed in shared memory
  const size_t q0 = (size_t)c->eval_p0;
  launch_fo_values(c->basis_dev(), nderv, P, c->d_x.p + q0, c->d_y.p + q0, c->d_z.p + q0, S.cfo.p, nb, nf, S.phi.p,
                   P, c->coulomb_cfg.fo_values_bn, c->st);
  c->launches++;
}

// Pair coefficients, POISSON1 call set-up and the Coulomb kernels for nf
// densities whose primitive projections are in d_u (dm == nullptr: FO k is
// the rank-1 density of u_k), or for the one density given by its pair
// blocks dm (nf = 1).  vh[k*P + p] over the evaluated mesh.
float elapsed(cudaEvent_t a, cudaEvent_t b);

void coulomb_eval(flosic_ctx* c, int nf, const double* dm, double* vh) {
  const int P = c->eval_n;
  const int npairs = (int)c->pairs.size(), ncalls = (int)c->calls.size();
  cudaStream_t st = c->st;
  c->d_coef.ensure((size_t)std::max(npairs, 1) * nf * COEF_LD);
  c->d_maxfmt.ensure((size_t)std::max(npairs, 1) * nf);
  c->d_cgp.ensure((size_t)std::max(npairs, 1) * nf * 4);
  c->d_callfo.ensure((size_t)std::max(ncalls, 1) * nf);
  c->d_mom.ensure((size_t)std::max(ncalls, 1) * nf * MOM_LD);
  CUDA_CHECK(cudaEventRecord(c->ev[2], st));
  launch_pair_coef(npairs, c->d_pairs.p, c->d_calls.p, nf, c->nprim, c->d_u.p, dm, c->nspn, c->d_coef.p,
                   c->d_maxfmt.p, c->d_cgp.p, st);
  c->launches++;
  launch_call_setup(ncalls, c->d_setup_list.p, c->nsingle, c->d_calls.p, c->d_pairs.p, nf, c->nspn, c->d_coef.p,
                    c->d_maxfmt.p, c->d_cgp.p, c->mesh_dev(), c->d_boys.p, c->d_callfo.p, c->d_mom.p, st);
  c->launches++;
  CUDA_CHECK(cudaEventRecord(c->ev[3], st));
  c->d_pairfmt.ensure((size_t)std::max(npairs, 1));
  c->d_share.ensure((size_t)std::max(ncalls, 1));
  c->d_lists.ensure((size_t)2 * ncalls + 2);
  c->d_cnt.ensure(6);
  CUDA_CHECK(cudaMemsetAsync(c->d_cnt.p, 0, 6 * sizeof(unsigned long long), st));
  const bool mixed = c->precision == FLOSIC_PRECISION_MIXED;
  if (mixed) {
    c->d_coef_hl.ensure((size_t)2 * std::max(npairs, 1) * nf * COEF_LD);
    c->d_momv_hl.ensure((size_t)2 * std::max(ncalls, 1) * nf * MOM_LD);
    c->d_tc_err.ensure(1);
    CUDA_CHECK(cudaMemsetAsync(c->d_tc_err.p, 0, sizeof(int), st));
  }
  CoulombScratch scr{c->d_pairfmt.p, c->d_share.p, c->d_lists.p, c->d_coef_hl.p, c->d_momv_hl.p, c->d_tc_err.p};
  CUDA_CHECK(launch_coulomb_mma(ncalls, c->d_calls.p, c->d_pairs.p, npairs, nf, c->d_coef.p, c->d_maxfmt.p,
                                c->d_callfo.p, c->d_mom.p, c->eval_mesh(), c->d_boys.p, vh, P, c->coulomb_cfg, mixed,
                                scr, c->d_cnt.p, c->ev[8], st));
  CUDA_CHECK(cudaEventRecord(c->ev[9], st));
  c->launches += c->coulomb_cfg.per_fo_only ? 4 : 5;
  unsigned long long cnt[6];
  int tc_err = 0;
  CUDA_CHECK(cudaMemcpyAsync(cnt, c->d_cnt.p, sizeof(cnt), cudaMemcpyDeviceToHost, st));
  if (mixed) CUDA_CHECK(cudaMemcpyAsync(&tc_err, c->d_tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  if (tc_err) fail(FLOSIC_ERR_CUDA, "mixed-precision Coulomb kernel: a pipeline wait reached its limit");
  c->work_near += cnt[0] + cnt[3];
  c->work_far += cnt[1] + cnt[4];
  c->work_terms += cnt[2] + cnt[5];
  for (int j = 0; j < 6; ++j) c->kernel_work[j] += cnt[j];
  c->kernel_ms[0] += elapsed(c->ev[3], c->ev[8]);
  c->kernel_ms[1] += elapsed(c->ev[8], c->ev[9]);
  CUDA_CHECK(cudaGetLastError());
}

// FLOSIC_DENSITY_PAIRS: the FO densities of spin s by the reference's route,
// from the Gaussian pairs of every POISSON1 call at the points inside its RCUT
// sphere (poisson1.f:849-948), into S.rhog; the primitive projections in d_u
// and the calls' per-FO geometry cfo must be those of spin s.
void pair_density(flosic_ctx* c, int s, const CallFO* cfo) {
  if (c->density != FLOSIC_DENSITY_PAIRS) return;
  SpinCache& S = c->spin[s];
  const int nf = S.nf, P = c->eval_n, nch = c->nch();
  const int npairs = (int)c->pairs.size(), ncalls = (int)c->calls.size();
  c->d_dens_coef.ensure((size_t)std::max(npairs, 1) * nf * pair_density_ld(nch));
  S.rhog.ensure((size_t)nch * nf * P);
  launch_pair_density(npairs, c->d_pairs.p, ncalls, c->d_calls.p, cfo, nf, c->nprim, c->d_u.p, nch, c->eval_mesh(),
                      c->d_dens_coef.p, S.rhog.p, (size_t)P, c->st);
  CUDA_CHECK(cudaGetLastError());
  c->launches += 2;
}

// COUPOT_SIC's Coulomb part for the FOs of spin s.
void coulomb(flosic_ctx* c, int s) {
  SpinCache& S = c->spin[s];
  const int nf = S.nf;
  c->d_u.ensure((size_t)nf * c->nprim * 10);
  launch_prim_u(c->basis_dev(), nf, S.cfo.p, c->nbasis, c->d_u.p, c->st);
  c->launches++;
  S.vh.ensure((size_t)nf * c->eval_n);
  coulomb_eval(c, nf, nullptr, S.vh.p);
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

void results_from_parts(const flosic_ctx* c, int nf, const double* parts, const double* asy,
                        std::vector<double>& results, std::vector<double>& cfrm);

void spin_xc(flosic_ctx* c, int s);

// Everything of APOTNL_SIC for all FOs of spin s (apotnl_sic.F:232-623).
void spin_potentials(flosic_ctx* c, int s) {
  SpinCache& S = c->spin[s];
  if (S.pot_valid) return;
  cudaStream_t st = c->st;
  CUDA_CHECK(cudaEventRecord(c->ev[0], st));
  fo_setup(c, s);
  CUDA_CHECK(cudaEventRecord(c->ev[1], st));
  fo_values(c, s);
  CUDA_CHECK(cudaEventRecord(c->ev[7], st));
  coulomb(c, s);
  CUDA_CHECK(cudaEventRecord(c->ev[4], st));
  pair_density(c, s, c->d_callfo.p);  // FLOSIC_DENSITY_PAIRS only; timed with XC
  spin_xc(c, s);
  c->stage_ms[0] += elapsed(c->ev[0], c->ev[1]);
  c->stage_ms[1] += elapsed(c->ev[1], c->ev[7]);
  c->stage_ms[2] += elapsed(c->ev[7], c->ev[3]);
  c->stage_ms[3] += elapsed(c->ev[3], c->ev[4]);
  c->stage_ms[4] += elapsed(c->ev[4], c->ev[5]);
}

// XC and the APOTNL_SIC mesh sums of spin s from its FO values and raw
// Coulomb potentials (S.phi, S.vh), then RESULTS; marks the potentials valid.
void spin_xc(flosic_ctx* c, int s) {
  SpinCache& S = c->spin[s];
  cudaStream_t st = c->st;
  const int nf = S.nf, P = c->eval_n;
  S.vpot.ensure((size_t)nf * P);
  S.y.ensure((size_t)(c->mgga ? 4 : 1) * nf * P);
  S.vh.ensure((size_t)nf * P);
  const int nblk = std::min(1024, (P + 255) / 256);
  c->d_part.ensure((size_t)nf * nblk * NPART);
  c->d_sums.ensure((size_t)nf * NPART);
  // XC reads the raw Coulomb potential; keep a scaled copy out of place
  c->d_tmp.ensure((size_t)nf * P);
  CUDA_CHECK(cudaMemcpyAsync(c->d_tmp.p, S.vh.p, sizeof(double) * nf * P, cudaMemcpyDeviceToDevice, st));
  const double* rhog = c->density == FLOSIC_DENSITY_PAIRS ? S.rhog.p : nullptr;
  launch_xc(c->eval_mesh(), nf, c->gga, c->mgga, c->nspn, c->xc, S.phi.p, P, rhog, c->d_tmp.p, S.vpot.p, S.y.p,
            c->d_part.p, nblk, st);
  launch_reduce_parts(nf, nblk, c->d_part.p, c->d_sums.p, st);
  c->launches += 2;
  std::vector<double>& sums = S.parts;
  sums.assign((size_t)nf * NPART, 0.0);
  S.asy.assign(nf, 0.0);
  CUDA_CHECK(cudaMemcpyAsync(sums.data(), c->d_sums.p, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, st));
  // the farthest point's scaled Coulomb potential, from the shard that holds it
  const int ifar = c->ifar_sorted - c->eval_p0;
  if (ifar >= 0 && ifar < P)
    CUDA_CHECK(cudaMemcpy2DAsync(S.asy.data(), sizeof(double), c->d_tmp.p + ifar, sizeof(double) * P,
                                 sizeof(double), nf, cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaEventRecord(c->ev[5], st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  results_from_parts(c, nf, sums.data(), S.asy.data(), S.results, S.cfrm);
  S.pot_valid = true;
}

// RESULTS(1:13) and CFRM of nf FOs (apotnl_sic.F:564-623) from the mesh sums
// parts[k*NPART + j] (j: XCH1, XCOU, XEXX, XDEL, ERGXL, ERGXN, ERGCL, ERGCN,
// CFRM x3) and the farthest point's scaled Coulomb potential asy[k] -- of one
// context, or summed over the mesh shards.
void results_from_parts(const flosic_ctx* c, int nf, const double* parts, const double* asy,
                        std::vector<double>& results, std::vector<double>& cfrm) {
  results.assign((size_t)nf * 13, 0.0);
  cfrm.assign((size_t)nf * 3, 0.0);
  for (int k = 0; k < nf; ++k) {
    const double* q = &parts[(size_t)k * NPART];
    double* r = &results[(size_t)k * 13];
    const double xch1 = q[0], xcou = q[1];
    double xexx = q[2];
    double xdel = q[3];
    const double ergxl = q[4], ergxn = q[5], ergcl = q[6], ergcn = q[7];
    const double excsic = ergxl + ergxn + ergcl + ergcn;
    xdel = xdel - xcou;
    const double xeng = -excsic - xcou / 2.0;
    const double pi = 4.0 * std::atan(1.0);
    xexx = xexx * 0.75 * std::pow(6 / pi, (double)(1.0f / 3.0f));
    r[0] = k + 1;
    r[1] = xch1;
    r[2] = 0.0;
    r[3] = asy[k] * c->rmx;
    r[4] = xexx;
    r[5] = -xcou / 2.0;
    r[6] = xdel;
    r[7] = xeng;
    r[8] = xeng * (2.0 / c->nspn);
    r[9] = ergxl;
    r[10] = ergcl;
    r[11] = ergxn;
    r[12] = ergcn;
    for (int d = 0; d < 3; ++d) cfrm[(size_t)k * 3 + d] = q[8 + d];
  }
}

// SICLAGM (frmorb_mpi.F:456-517): SIC(j,l) = -sum_p phi_j w V_l phi_l; for a
// meta-GGA -sum_c sum_p d_c phi_j Y_c,l over the four channels of Y (k_xc).
void spin_sic(flosic_ctx* c, int s) {
  SpinCache& S = c->spin[s];
  if (S.sic_valid) return;
  spin_potentials(c, s);
  const int nf = S.nf, P = c->eval_n;
  cudaStream_t st = c->st;
  CUDA_CHECK(cudaEventRecord(c->ev[0], st));
  c->d_sic.ensure((size_t)nf * nf);
  const int nyc = c->mgga ? 4 : 1;
  for (int ch = 0; ch < nyc; ++ch)
    gemm(c, true, false, nf, nf, P, -1.0, S.phi.p + (size_t)ch * nf * P, P, S.y.p + (size_t)ch * nf * P, P,
         ch == 0 ? 0.0 : 1.0, c->d_sic.p, nf);
  S.sic.resize((size_t)nf * nf);
  CUDA_CHECK(cudaMemcpyAsync(S.sic.data(), c->d_sic.p, sizeof(double) * nf * nf, cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaEventRecord(c->ev[1], st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  c->stage_ms[5] += elapsed(c->ev[0], c->ev[1]);
  S.sic_valid = true;
}

// FRMORB2(-s,-1) force branch (frmorb2.F:586-717), with the O(n^4) loops of
// the second term regrouped into O(n^3) products.
// C = A B, row-major A (n x k), B (k x m), C (n x m).
void mat_mul(const double* A, const double* B, double* C, int n, int k, int m) {
  for (size_t i = 0; i < (size_t)n * m; ++i) C[i] = 0.0;
  for (int i = 0; i < n; ++i) {
    double* ci = C + (size_t)i * m;
    for (int p = 0; p < k; ++p) {
      const double a = A[(size_t)i * k + p];
      if (a == 0.0) continue;
      const double* bp = B + (size_t)p * m;
      for (int j = 0; j < m; ++j) ci[j] += a * bp[j];
    }
  }
}

void spin_force(flosic_ctx* c, int s, const double* sic /* SIC(j,l) at [l*ld + j] */, int ld, double* deb) {
  fo_setup(c, s);
  SpinCache& S = c->spin[s];
  const int nf = S.nf, nw = S.nw;
  auto t0 = std::chrono::steady_clock::now();
  // the Lowdin eigenpairs of the overlap sum_w F(w,i,0) F(w,j,0) (frmorb2.F:460-583)
  // are those fo_setup computed for TMAT: the same overlap of the same FMAT.
  // Fm[i][a] = FILO(i,a): component i of eigenvector a.
  const std::vector<double>& Fm = S.filo;
  const std::vector<double>& Q = S.lam;
  const size_t n2 = (size_t)nf * nf;
  std::vector<double> FmT(n2), sicm(n2), tmp(n2), G(n2);
  for (int i = 0; i < nf; ++i)
    for (int a = 0; a < nf; ++a) {
      FmT[(size_t)a * nf + i] = Fm[(size_t)i * nf + a];
      sicm[(size_t)i * nf + a] = sic[(size_t)a * ld + i];  // SIC(i,a)
    }
  // G = FILO^T SIC FILO  ->  HAM(b,a) = (G[a][b] - G[b][a]) / sqrt(Qa Qb)
  mat_mul(FmT.data(), sicm.data(), tmp.data(), nf, nf, nf);
  mat_mul(tmp.data(), Fm.data(), G.data(), nf, nf, nf);
  // Both terms of frmorb2.F:612-717 in one matrix:
  //   term 1: -sum_a FILO(m,a) (HAM^T FILO^T X_kx)[a][m]           (frmorb2.F:616-667)
  //   term 2: +1/4 sum_ab HAM'(b,a) [FILO(m,a) Y_b(m) + FILO(m,b) Y_a(m)],
  //           HAM' = HAM (sqrtQb - sqrtQa)/(sqrtQb + sqrtQa), Y = 2 FILO^T X_kx (:673-717)
  // with X_kx[n][m] = sum_w F(w,n,1) F(w,m,kx+1), so that
  //   DEBDAX(kx,m) = sum_n L[m][n] X_kx[n][m],  L = FILO (HAM'^T/2 + HAM'/2 - HAM^T) FILO^T
  // (H[a][b] = HAM(b,a)), i.e. sum_w M[m][w] F(w,m,kx+1) with M = L F_0.
  std::vector<double> A1(n2);
  for (int a = 0; a < nf; ++a)
    for (int b = 0; b < nf; ++b) {
      const double sa = std::sqrt(Q[a]), sb = std::sqrt(Q[b]);
      const double hab = (G[(size_t)a * nf + b] - G[(size_t)b * nf + a]) / (sb * sa);
      const double hba = (G[(size_t)b * nf + a] - G[(size_t)a * nf + b]) / (sa * sb);
      const double hpab = hab * (sb - sa) / (sb + sa);
      const double hpba = hba * (sa - sb) / (sa + sb);
      A1[(size_t)a * nf + b] = 0.5 * (hpab + hpba) - hab;
    }
  std::vector<double> T(n2), L(n2), M((size_t)nf * nw);
  mat_mul(Fm.data(), A1.data(), T.data(), nf, nf, nf);
  mat_mul(T.data(), FmT.data(), L.data(), nf, nf, nf);
  mat_mul(L.data(), &S.fmat[0], M.data(), nf, nf, nw);  // F_0[n][w] = F(w,n,1)
  for (int m = 0; m < nf; ++m)
    for (int kx = 0; kx < 3; ++kx) {
      const double* fk = &S.fmat[((size_t)(kx + 1) * nf + m) * nw];
      const double* mr = &M[(size_t)m * nw];
      double v = 0.0;
      for (int w = 0; w < nw; ++w) v += mr[w] * fk[w];
      deb[3 * m + kx] = v;
    }
  auto t1 = std::chrono::steady_clock::now();
  c->stage_ms[6] += std::chrono::duration<double, std::milli>(t1 - t0).count();
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return FLOSIC_OK;
  } catch (const Fail& e) {
    return e.code;
  } catch (const std::exception& e) {
    g_err = e.what();
    return FLOSIC_ERR_CUDA;
  }
}

void require(flosic_ctx* c, bool orb) {
  if (!c) fail(FLOSIC_ERR_ARG, "null context");
  if (!c->have_geom) fail(FLOSIC_ERR_STATE, "flosic_sic_set_geometry has not been called");
  if (orb && !c->have_orb) fail(FLOSIC_ERR_STATE, "flosic_sic_set_orbitals has not been called");
  CUDA_CHECK(cudaSetDevice(c->device));
}

// Entry points whose outputs cover the whole mesh need an unsharded context.
void require_whole_mesh(flosic_ctx* c) {
  if (c->nshards != 1)
    fail(FLOSIC_ERR_STATE, "this context evaluates one mesh shard: use flosic_sic_cycle_partial / _combine");
}

// ---------------------------------------------------------------------------
// Allocation-free GETVLXC scratch
// ---------------------------------------------------------------------------
// flosic_sic_getvlxc_device keeps its per-block energy partial sums in this
// file-scope device array instead of allocating: XC_SCRATCH_BLOCKS blocks of
// 256 points (4,194,304 points at most) times NPART partials, then the NPART
// final sums.  Every call overwrites the partials of its nblk blocks and the
// sums before reading them, so no part of the array has to start at zero.  All
// calls on one device share it: calls that overlap in time (other host threads,
// other contexts or streams on the same device) race on it.
constexpr int XC_SCRATCH_BLOCKS = 16384;
constexpr int XC_SCRATCH_POINTS = XC_SCRATCH_BLOCKS * 256;
static __device__ __align__(256) double g_xc_scratch[(XC_SCRATCH_BLOCKS + 1) * NPART];

// Device address of g_xc_scratch for the current device, looked up once per
// device with that device current.  flosic_sic_create calls it, so the module
// that holds the array is loaded (and the array placed in device memory) when
// the first context on a device is made, not inside the entry point.
double* xc_scratch_address(int device) {
  static std::mutex mu;
  static double* addr[64] = {};
  if (device < 0 || device >= 64) fail(FLOSIC_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    double* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_xc_scratch);
    if (e != cudaSuccess)
      fail(FLOSIC_ERR_CUDA, std::string("cudaGetSymbolAddress(g_xc_scratch): ") + cudaGetErrorString(e));
    addr[device] = ptr;
  }
  return addr[device];
}

// dE_SIC/dC_FO (nb x nf, column k = FO k) of spin s on the device, summed over
// this context's points: -(4/NSPN) sum_c sum_p chi_c,mu(p) Y_c,k(p).  E_SIC =
// (2/NSPN) sum_k XENG_k and dXENG_k/dphi_k(p) = -2 w V_k phi_k (+ the meta-GGA
// gradient terms, carried by Y_1..3).  The basis values are recomputed in mesh
// chunks, so no per-FO array beyond the cycle's is kept.
void adjoint_device(flosic_ctx* c, int s, DevBuf<double>& dg) {
  spin_potentials(c, s);
  SpinCache& S = c->spin[s];
  const int nf = S.nf, nb = c->nbasis, P = c->eval_n;
  const int nyc = c->mgga ? 4 : 1;
  const int nderv = c->mgga ? 1 : 0;
  const size_t budget = (size_t)3 << 30;
  int chunk = (int)std::min<size_t>(P, std::max<size_t>(TILE, budget / (sizeof(double) * nyc * nb)));
  chunk = std::max(TILE, chunk / TILE * TILE);
  c->d_basis.ensure((size_t)nyc * nb * chunk);
  dg.ensure((size_t)nb * nf);
  const double alpha = -4.0 / c->nspn;
  bool first = true;
  for (int p0 = 0; p0 < P; p0 += chunk) {
    const int np = std::min(chunk, P - p0);
    const size_t q0 = (size_t)c->eval_p0 + p0;
    launch_basis_values(c->basis_dev(), nderv, np, c->d_x.p + q0, c->d_y.p + q0, c->d_z.p + q0, c->d_basis.p, np,
                        c->st);
    c->launches++;
    for (int ch = 0; ch < nyc; ++ch) {
      gemm(c, true, false, nb, nf, np, alpha, c->d_basis.p + (size_t)ch * nb * np, np,
           S.y.p + (size_t)ch * nf * P + p0, P, first ? 0.0 : 1.0, dg.p, nb);
      first = false;
    }
  }
}

// dE_SIC/dFOD of spin s, grad[k*3 + d], from the adjoint G by the chain rule
// through the FO construction.  C_FO = U C_KS with U = S^-1/2 T the
// Lowdin-orthonormalised Fermi transformation (frmiorb.f:351-480), T_kj =
// psi_j(a_k)/sqrt(rho(a_k)) = FMAT(j,k,1), S = T T^T = V diag(q) V^T (the
// eigenpairs LOWSIC kept); row k of T depends on FOD a_k only, with
// derivatives FMAT(.,k,2:4) (frmorb2.F:296-346).  With M = C_KS G and A = T M:
//   W = V ((V^T A V) o F) V^T,  F_ab = -1 / (sqrt q_a sqrt q_b (sqrt q_a + sqrt q_b)),
//   dE/dT = (W + W^T) T + (M S^-1/2)^T,  dE/da_m = sum_j (dE/dT)_mj dT_mj/da_m.
// This is the reference's FOD force (frmorb2.F:586-717, times 2/NSPN) reached
// through the basis-space adjoint instead of the SIC matrix.
// Batch of molecules: everything of spin s before its Coulomb evaluation --
// FO construction, FO values, pair coefficients, POISSON1 call set-up and
// call classification -- into the spin's own buffers, on the context's stream.
// Returns the spin's job for the batched Coulomb launch.
CoulombJob batch_prepare(flosic_ctx* c, int s) {
  SpinCache& S = c->spin[s];
  fo_setup(c, s);
  fo_values(c, s);
  const int nf = S.nf, P = c->eval_n;
  const int npairs = (int)c->pairs.size(), ncalls = (int)c->calls.size();
  cudaStream_t st = c->st;
  c->d_u.ensure((size_t)nf * c->nprim * 10);
  launch_prim_u(c->basis_dev(), nf, S.cfo.p, c->nbasis, c->d_u.p, st);
  CoulBufs& B = S.bc;
  B.coef.ensure((size_t)std::max(npairs, 1) * nf * COEF_LD);
  B.maxfmt.ensure((size_t)std::max(npairs, 1) * nf);
  B.cgp.ensure((size_t)std::max(npairs, 1) * nf * 4);
  B.callfo.ensure((size_t)std::max(ncalls, 1) * nf);
  B.mom.ensure((size_t)std::max(ncalls, 1) * nf * MOM_LD);
  B.pairfmt.ensure((size_t)std::max(npairs, 1));
  B.share.ensure((size_t)std::max(ncalls, 1));
  B.lists.ensure((size_t)2 * ncalls + 2);
  B.cnt.ensure(3);
  launch_pair_coef(npairs, c->d_pairs.p, c->d_calls.p, nf, c->nprim, c->d_u.p, nullptr, c->nspn, B.coef.p,
                   B.maxfmt.p, B.cgp.p, st);
  launch_call_setup(ncalls, c->d_setup_list.p, c->nsingle, c->d_calls.p, c->d_pairs.p, nf, c->nspn, B.coef.p,
                    B.maxfmt.p, B.cgp.p, c->mesh_dev(), c->d_boys.p, B.callfo.p, B.mom.p, st);
  CUDA_CHECK(cudaMemsetAsync(B.cnt.p, 0, 3 * sizeof(unsigned long long), st));
  CoulombScratch scr{B.pairfmt.p, B.share.p, B.lists.p, nullptr, nullptr, nullptr};
  launch_coulomb_classify(ncalls, npairs, nf, B.maxfmt.p, B.callfo.p, scr, false, st);
  c->launches += 6;
  pair_density(c, s, B.callfo.p);
  S.vh.ensure((size_t)nf * P);
  CoulombJob J{};
  J.ncalls = ncalls;
  J.nfo = nf;
  J.ldv = P;
  J.lists = B.lists.p;
  J.share = B.share.p;
  J.calls = c->d_calls.p;
  J.pairs = c->d_pairs.p;
  J.coef = B.coef.p;
  J.pair_fmt = B.pairfmt.p;
  J.cfo = B.callfo.p;
  J.momv = B.mom.p;
  J.M = c->eval_mesh();
  J.vh = S.vh.p;
  J.cnt = B.cnt.p;
  return J;
}

void fod_gradient(flosic_ctx* c, int s, double* grad) {
  DevBuf<double> dg, dm;
  adjoint_device(c, s, dg);
  SpinCache& S = c->spin[s];
  const int n = S.nf, nw = S.nw, nb = c->nbasis;
  if (n != nw) fail(FLOSIC_ERR_NFRM, "FRMIORB: MORB .NE. NFRM");
  const double* cks = c->d_psi.p + (size_t)s * c->nwfs[0] * nb;
  dm.ensure((size_t)nw * n);
  gemm(c, true, false, nw, n, nb, 1.0, cks, nb, dg.p, nb, 0.0, dm.p, nw);  // M(j,k) = sum_mu C_KS(mu,j) G(mu,k)
  std::vector<double> mh((size_t)nw * n);
  CUDA_CHECK(cudaMemcpyAsync(mh.data(), dm.p, sizeof(double) * mh.size(), cudaMemcpyDeviceToHost, c->st));
  CUDA_CHECK(cudaStreamSynchronize(c->st));
  const size_t nn = (size_t)n * n;
  std::vector<double> T(nn), M(nn), V(nn), Vt(nn), rq(n), A(nn), B(nn), X(nn), W(nn), Sm(nn), MS(nn), D(nn);
  for (int a = 0; a < n; ++a)
    for (int j = 0; j < n; ++j) {
      T[(size_t)a * n + j] = S.fmat[(size_t)a * nw + j];
      M[(size_t)j * n + a] = mh[(size_t)a * nw + j];
      V[(size_t)a * n + j] = S.filo[(size_t)a * n + j];
      Vt[(size_t)j * n + a] = S.filo[(size_t)a * n + j];
    }
  for (int a = 0; a < n; ++a) rq[a] = std::sqrt(S.lam[a]);
  mat_mul(T.data(), M.data(), A.data(), n, n, n);    // A = T M
  mat_mul(Vt.data(), A.data(), X.data(), n, n, n);   // V^T A
  mat_mul(X.data(), V.data(), B.data(), n, n, n);    // V^T A V
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) B[(size_t)a * n + b] *= -1.0 / (rq[a] * rq[b] * (rq[a] + rq[b]));
  mat_mul(V.data(), B.data(), X.data(), n, n, n);
  mat_mul(X.data(), Vt.data(), W.data(), n, n, n);   // W = V (B o F) V^T
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) X[(size_t)a * n + b] = V[(size_t)a * n + b] / rq[b];
  mat_mul(X.data(), Vt.data(), Sm.data(), n, n, n);  // S^-1/2
  mat_mul(M.data(), Sm.data(), MS.data(), n, n, n);  // M S^-1/2
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) X[(size_t)a * n + b] = W[(size_t)a * n + b] + W[(size_t)b * n + a];
  mat_mul(X.data(), T.data(), D.data(), n, n, n);    // (W + W^T) T
  for (int m = 0; m < n; ++m)
    for (int d = 0; d < 3; ++d) {
      double acc = 0.0;
      for (int j = 0; j < n; ++j)
        acc += (D[(size_t)m * n + j] + MS[(size_t)j * n + m]) * S.fmat[((size_t)(1 + d) * n + m) * nw + j];
      grad[(size_t)m * 3 + d] = acc;
    }
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* flosic_sic_last_error(void) { return g_err.c_str(); }

int flosic_sic_create(int device, flosic_ctx** out) {
  return guarded([&] {
    if (!out) fail(FLOSIC_ERR_ARG, "null output pointer");
    int ndev = 0;
    CUDA_CHECK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) fail(FLOSIC_ERR_ARG, "invalid device");
    CUDA_CHECK(cudaSetDevice(device));
    auto* c = new flosic_ctx;
    c->device = device;
    if (const char* e = std::getenv("FLOSIC_COULOMB")) c->coulomb_cfg.per_fo_only = (std::string(e) == "perfo");
    if (const char* e = std::getenv("FLOSIC_SHARED")) c->coulomb_cfg.shared_tc = (std::string(e) != "mma");
    if (const char* e = std::getenv("FLOSIC_FOV_BN")) c->coulomb_cfg.fo_values_bn = std::atoi(e) == 128 ? 128 : 64;
    if (const char* e = std::getenv("FLOSIC_PERFO_WM")) {
      const int wm = std::atoi(e);
      c->coulomb_cfg.perfo_wm = (wm == 1 || wm == 2 || wm == 4) ? wm : 0;
    }
    CUDA_CHECK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    for (auto& e : c->ev) CUDA_CHECK(cudaEventCreate(&e));
    std::vector<double> ang, w;
    lebedev19(ang, w);
    upload_constants(ang.data(), w.data());
    init_call_setup();
    init_coulomb_mma();
    init_coulomb_tc();
    CUDA_CHECK(init_sym_eigen());
    CUDA_CHECK(init_contract());
    CUDA_CHECK(preload_xc_rhog());
    xc_scratch_address(device);
    std::vector<double> bt = boys_table();
    c->d_boys.upload(bt.data(), bt.size(), c->st);
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    *out = c;
  });
}

int flosic_sic_destroy(flosic_ctx* c) {
  if (!c) return FLOSIC_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->st);
  for (auto& s : c->spin) s.release();
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  c->d_atom_pos.release(); c->d_type_alpha.release(); c->d_type_amin.release(); c->d_type_bfcon.release();
  c->d_atom_type.release(); c->d_atom_boff.release(); c->d_atom_poff.release(); c->d_type_nbare.release();
  c->d_type_lmax.release(); c->d_type_ncon.release(); c->d_prim_atom.release(); c->d_prim_ib.release();
  c->d_x.release(); c->d_y.release(); c->d_z.release(); c->d_w.release(); c->d_tlo.release(); c->d_thi.release();
  c->d_boys.release(); c->d_pairs.release(); c->d_calls.release(); c->d_psi.release(); c->d_psi_thr.release();
  c->d_basis.release(); c->d_fodpts.release(); c->d_psig.release(); c->d_tmat.release(); c->d_u.release();
  c->d_coef.release(); c->d_cgp.release(); c->d_mom.release(); c->d_part.release(); c->d_sums.release();
  c->d_sic.release(); c->d_tmp.release(); c->d_maxfmt.release(); c->d_callfo.release(); c->d_cnt.release(); c->d_pairfmt.release();
  c->d_share.release(); c->d_lists.release(); c->d_setup_list.release();
  c->d_eig_a.release(); c->d_eig_w.release(); c->d_eig_v.release(); c->d_eig_work.release(); c->d_eig_info.release();
  c->d_coef_hl.release(); c->d_momv_hl.release(); c->d_tc_err.release(); c->d_dens_coef.release();
  c->d_gemm_ws.release();
  c->d_jobs.release();
  c->d_items.release();
  c->d_batch_counters.release();
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return FLOSIC_OK;
}

int flosic_sic_set_geometry(flosic_ctx* c, int natoms, const int32_t* atom_type, const double* rat, int ntypes,
                            const int32_t* n_bare, const double* bfalp, const int32_t* n_con, const double* bfcon,
                            int nmsh, const double* rmsh, const double* wmsh, int nspn, const int32_t* igga,
                            const int32_t* idftyp) {
  return guarded([&] {
    if (!c) fail(FLOSIC_ERR_ARG, "null context");
    CUDA_CHECK(cudaSetDevice(c->device));
    if (natoms <= 0 || ntypes <= 0 || nmsh <= 0) fail(FLOSIC_ERR_ARG, "natoms, ntypes and nmsh must be positive");
    if (nspn != 1 && nspn != 2) fail(FLOSIC_ERR_ARG, "nspn must be 1 or 2");
    if (!atom_type || !rat || !n_bare || !bfalp || !n_con || !bfcon || !rmsh || !wmsh || !igga || !idftyp)
      fail(FLOSIC_ERR_ARG, "null array argument");
    const bool scan = igga[0] == 3 && igga[1] == 3 && idftyp[0] == 11 && idftyp[1] == 11;
    if (!scan) {
      for (int i = 0; i < 2; ++i)
        if (igga[i] < 0 || igga[i] > 1)
          fail(FLOSIC_ERR_ARG, "IGGA must be 0 (LDA) or 1 (GGA), or 3 with IDFTYP 11 for both (SCAN)");
      if (idftyp[0] < 6 || idftyp[0] > 9) fail(FLOSIC_ERR_ARG, "exchange IDFTYP must be PW91, PBE, REVPBE or RPBE");
      if (idftyp[1] != 6 && idftyp[1] != 7) fail(FLOSIC_ERR_ARG, "correlation IDFTYP must be PW91 or PBE");
    }
    invalidate(c);
    c->have_geom = c->have_orb = false;
    c->natoms = natoms;
    c->ntypes = ntypes;
    c->nmsh = nmsh;
    c->nspn = nspn;
    c->xc[0] = igga[0];
    c->xc[1] = idftyp[0];
    c->xc[2] = igga[1];
    c->xc[3] = idftyp[1];
    c->gga = (igga[0] > 0 || igga[1] > 0) ? 1 : 0;
    c->mgga = scan ? 1 : 0;
    c->types.assign(ntypes, TypeInfo());
    for (int t = 0; t < ntypes; ++t) {
      TypeInfo& T = c->types[t];
      T.nbare = n_bare[t];
      if (T.nbare < 1 || T.nbare > MAX_BARE) fail(FLOSIC_ERR_CAPACITY, "N_BARE exceeds MAX_BARE=25");
      T.lmax = 0;
      T.nloc = 0;
      for (int l = 0; l < 3; ++l) {
        T.ncon[l] = n_con[t * 3 + l];
        if (T.ncon[l] < 0 || T.ncon[l] > MAX_CON) fail(FLOSIC_ERR_CAPACITY, "N_CON exceeds MAX_CON=15");
        if (T.ncon[l] > 0) T.lmax = l;
        T.nloc += kNcomp[l] * T.ncon[l];
      }
      for (int ib = 0; ib < MAX_BARE; ++ib) T.alp[ib] = bfalp[(size_t)t * MAX_BARE + ib];
      for (int ib = 0; ib < T.nbare; ++ib)
        if (!(T.alp[ib] > 0.0)) fail(FLOSIC_ERR_ARG, "BFALP must be positive");
      for (int l = 0; l < 3; ++l)
        for (int cc = 0; cc < MAX_CON; ++cc)
          for (int ib = 0; ib < MAX_BARE; ++ib)
            T.con[l][cc][ib] = bfcon[(((size_t)t * 3 + l) * MAX_CON + cc) * MAX_BARE + ib];
    }
    c->atype.resize(natoms);
    c->aoff.resize(natoms);
    c->apoff.resize(natoms);
    c->rat.assign(rat, rat + 3 * (size_t)natoms);
    int off = 0, poff = 0;
    std::vector<int> prim_atom, prim_ib;
    for (int a = 0; a < natoms; ++a) {
      const int t = atom_type[a] - 1;
      if (t < 0 || t >= ntypes) fail(FLOSIC_ERR_ARG, "atom_type out of range (1-based IFNCT)");
      if (a > 0 && t < c->atype[a - 1])
        fail(FLOSIC_ERR_ARG, "atoms must be ordered by function set (IFNCT outer, I_POS inner)");
      c->atype[a] = t;
      c->aoff[a] = off;
      c->apoff[a] = poff;
      off += c->types[t].nloc;
      for (int ib = 0; ib < c->types[t].nbare; ++ib) {
        prim_atom.push_back(a);
        prim_ib.push_back(ib);
      }
      poff += c->types[t].nbare;
    }
    c->nbasis = off;
    c->nprim = poff;
    for (int i = 0; i < nmsh; ++i)
      if (!(wmsh[i] > 0.0) && wmsh[i] != 0.0) fail(FLOSIC_ERR_ARG, "WMSH must be finite");
    cudaStream_t st = c->st;
    // device basis tables
    std::vector<double> alpha((size_t)ntypes * MAX_BARE), amin(ntypes), con((size_t)ntypes * 3 * MAX_CON * MAX_BARE);
    std::vector<int> nbarev(ntypes), lmaxv(ntypes), nconv(3 * (size_t)ntypes);
    for (int t = 0; t < ntypes; ++t) {
      const TypeInfo& T = c->types[t];
      nbarev[t] = T.nbare;
      lmaxv[t] = T.lmax;
      double am = DBL_MAX;
      for (int ib = 0; ib < MAX_BARE; ++ib) {
        alpha[(size_t)t * MAX_BARE + ib] = T.alp[ib];
        if (ib < T.nbare) am = std::min(am, T.alp[ib]);
      }
      amin[t] = am;
      for (int l = 0; l < 3; ++l) {
        nconv[3 * t + l] = T.ncon[l];
        for (int cc = 0; cc < MAX_CON; ++cc)
          for (int ib = 0; ib < MAX_BARE; ++ib)
            con[(((size_t)t * 3 + l) * MAX_CON + cc) * MAX_BARE + ib] = T.con[l][cc][ib];
      }
    }
    c->d_atom_pos.upload(c->rat.data(), c->rat.size(), st);
    c->d_atom_type.upload(c->atype.data(), natoms, st);
    c->d_atom_boff.upload(c->aoff.data(), natoms, st);
    c->d_atom_poff.upload(c->apoff.data(), natoms, st);
    c->d_type_nbare.upload(nbarev.data(), ntypes, st);
    c->d_type_lmax.upload(lmaxv.data(), ntypes, st);
    c->d_type_ncon.upload(nconv.data(), nconv.size(), st);
    c->d_type_alpha.upload(alpha.data(), alpha.size(), st);
    c->d_type_amin.upload(amin.data(), ntypes, st);
    c->d_type_bfcon.upload(con.data(), con.size(), st);
    c->d_prim_atom.upload(prim_atom.data(), prim_atom.size(), st);
    c->d_prim_ib.upload(prim_ib.data(), prim_ib.size(), st);
    sort_mesh(c, rmsh, wmsh);
    if (c->nshards > c->ntiles)
      fail(FLOSIC_ERR_ARG, "more mesh shards (" + std::to_string(c->nshards) + ") than mesh tiles of 128 points");
    set_eval_range(c);
    build_pair_plan(c);
    c->d_pairs.upload(c->pairs.data(), c->pairs.size(), st);
    c->d_calls.upload(c->calls.data(), c->calls.size(), st);
    {
      std::vector<int> list;
      for (size_t i = 0; i < c->calls.size(); ++i)
        if (c->calls[i].slots == 1) list.push_back((int)i);
      c->nsingle = (int)list.size();
      for (size_t i = 0; i < c->calls.size(); ++i)
        if (c->calls[i].slots != 1) list.push_back((int)i);
      c->d_setup_list.upload(list.data(), list.size(), st);
    }
    CUDA_CHECK(cudaStreamSynchronize(st));
    c->have_geom = true;
  });
}

int flosic_sic_set_orbitals(flosic_ctx* c, const int32_t* nwfs, const double* psi, int ldpsi, const int32_t* nfrm,
                            const double* bfrm, int ldfrm) {
  return guarded([&] {
    require(c, false);
    if (!nwfs || !psi || !nfrm || !bfrm) fail(FLOSIC_ERR_ARG, "null array argument");
    if (ldpsi < c->nbasis) fail(FLOSIC_ERR_ARG, "ldpsi smaller than the number of basis functions");
    const int ns = c->nspn;
    for (int s = 0; s < ns; ++s) {
      if (nwfs[s] < 0 || nfrm[s] < 0 || nfrm[s] > ldfrm) fail(FLOSIC_ERR_ARG, "bad NWFS/NFRM");
      if (nwfs[s] != nfrm[s]) fail(FLOSIC_ERR_NFRM, "MORB .NE. NFRM (frmiorb.f:418)");
    }
    invalidate(c);
    c->nwfs[0] = nwfs[0];
    c->nwfs[1] = (ns == 2) ? nwfs[1] : 0;
    c->nfrm[0] = nfrm[0];
    c->nfrm[1] = (ns == 2) ? nfrm[1] : 0;
    const int nwf = c->nwfs[0] + c->nwfs[1];
    const int nb = c->nbasis;
    c->psi.assign((size_t)nb * nwf, 0.0);
    std::vector<double> thr((size_t)nb * nwf, 0.0);
    for (int j = 0; j < nwf; ++j)
      for (int i = 0; i < nb; ++i) {
        const double v = psi[(size_t)j * ldpsi + i];
        c->psi[(size_t)j * nb + i] = v;
        thr[(size_t)j * nb + i] = (std::fabs(v) > 1.0e-10) ? v : 0.0;
      }
    for (int s = 0; s < ns; ++s) {
      c->fods[s].resize(3 * (size_t)c->nfrm[s]);
      for (int k = 0; k < c->nfrm[s]; ++k)
        for (int d = 0; d < 3; ++d) c->fods[s][3 * k + d] = bfrm[((size_t)s * ldfrm + k) * 3 + d];
    }
    c->d_psi.upload(c->psi.data(), c->psi.size(), c->st);
    c->d_psi_thr.upload(thr.data(), thr.size(), c->st);
    c->have_orb = true;
  });
}

int flosic_sic_gorbdrv(flosic_ctx* c, int nderv, int32_t* iupdat, int32_t* iallctr, int npts, const double* pts,
                       int ifnct, double* grad) {
  return guarded([&] {
    require(c, false);
    if (nderv < 0 || nderv > 2) fail(FLOSIC_ERR_ARG, "GORBDRV: INVALID VALUE FOR NDERV");
    if (npts < 0 || npts > NSPEED) fail(FLOSIC_ERR_CAPACITY, "GORBDRV: NSPEED MUST BE AT LEAST NPTS");
    if (ifnct < 1 || ifnct > c->ntypes) fail(FLOSIC_ERR_ARG, "GORBDRV: bad IFNCT");
    if (!iupdat || !iallctr || !pts || !grad) fail(FLOSIC_ERR_ARG, "null array argument");
    const int t = ifnct - 1;
    const TypeInfo& T = c->types[t];
    const int nch = nderv == 0 ? 1 : (nderv == 1 ? 4 : 10);
    // one-atom basis at the origin; points are relative to the atom already
    int tz = t, boff = 0, poff = 0;
    double origin[3] = {0, 0, 0};
    DevBuf<double> pos, ptsd, out;
    DevBuf<int> ty, bo, po;
    pos.upload(origin, 3, c->st);
    ty.upload(&tz, 1, c->st);
    bo.upload(&boff, 1, c->st);
    po.upload(&poff, 1, c->st);
    std::vector<double> p(3 * (size_t)std::max(npts, 1));
    for (int i = 0; i < npts; ++i)
      for (int d = 0; d < 3; ++d) p[(size_t)d * npts + i] = pts[(size_t)d * NSPEED + i];
    ptsd.upload(p.data(), p.size(), c->st);
    BasisDev B = c->basis_dev();
    B.natoms = 1;
    B.nbasis = T.nloc;
    B.atom_pos = pos.p;
    B.atom_type = ty.p;
    B.atom_boff = bo.p;
    B.atom_poff = po.p;
    out.ensure((size_t)nch * T.nloc * std::max(npts, 1));
    launch_basis_values(B, nderv, npts, ptsd.p, ptsd.p + npts, ptsd.p + 2 * npts, out.p, npts, c->st);
    std::vector<double> h((size_t)nch * T.nloc * std::max(npts, 1));
    CUDA_CHECK(cudaMemcpyAsync(h.data(), out.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    pos.release(); ptsd.release(); out.release(); ty.release(); bo.release(); po.release();
    // GRAD(NSPEED,10,6,MAX_CON,3)
    auto gi = [](int ipt, int igr, int ia, int nb, int l) {
      return (((size_t)l * MAX_CON + nb) * 6 + ia) * 10 * NSPEED + (size_t)igr * NSPEED + ipt;
    };
    std::memset(grad, 0, sizeof(double) * (size_t)NSPEED * 10 * 6 * MAX_CON * 3);
    int base = 0;
    for (int l = 0; l <= T.lmax; ++l) {
      for (int mu = 0; mu < kNcomp[l]; ++mu)
        for (int cc = 0; cc < T.ncon[l]; ++cc)
          for (int ch = 0; ch < nch; ++ch)
            for (int i = 0; i < npts; ++i)
              grad[gi(i, ch, mu, cc, l)] = h[((size_t)ch * T.nloc + base + mu * T.ncon[l] + cc) * npts + i];
      base += kNcomp[l] * T.ncon[l];
    }
    // IUPDAT / IALLCTR screening flags (gorbdrv.f:183-220)
    const double geps = std::exp(-CUTEXP);
    bool up = false;
    for (int l = 0; l < 3; ++l)
      for (int cc = 0; cc < MAX_CON; ++cc) iallctr[l * MAX_CON + cc] = 0;
    for (int ib = 0; ib < T.nbare; ++ib) {
      bool icount = false;
      std::vector<double> gaus(npts);
      for (int i = 0; i < npts; ++i) {
        const double r2 = pts[i] * pts[i] + pts[NSPEED + i] * pts[NSPEED + i] + pts[2 * NSPEED + i] * pts[2 * NSPEED + i];
        const double rex = T.alp[ib] * r2;
        gaus[i] = rex < CUTEXP ? std::exp(-rex) : 0.0;
        if (rex < CUTEXP) icount = true;
      }
      if (!icount) continue;
      up = true;
      for (int l = 0; l <= T.lmax; ++l)
        for (int cc = 0; cc < T.ncon[l]; ++cc)
          for (int i = 0; i < npts; ++i)
            if (std::fabs(T.con[l][cc][ib]) * gaus[i] > geps) iallctr[l * MAX_CON + cc] = 1;
    }
    *iupdat = up ? 1 : 0;
  });
}

int flosic_sic_frmorb2_fmat(flosic_ctx* c, double* fmat, int ld) {
  return guarded([&] {
    require(c, true);
    if (!fmat) fail(FLOSIC_ERR_ARG, "null array argument");
    for (int s = 0; s < c->nspn; ++s) {
      if (c->nfrm[s] > ld) fail(FLOSIC_ERR_ARG, "ld smaller than NFRM");
      fo_setup(c, s);
      const SpinCache& S = c->spin[s];
      for (int K = 0; K < 4; ++K)
        for (int j = 0; j < S.nf; ++j)
          for (int w = 0; w < S.nw; ++w)
            fmat[(((size_t)s * 4 + K) * ld + j) * ld + w] = S.fmat[((size_t)K * S.nf + j) * S.nw + w];
    }
  });
}

int flosic_sic_frmiorb(flosic_ctx* c, double* tmat, double* eval, int ld) {
  return guarded([&] {
    require(c, true);
    if (!tmat || !eval) fail(FLOSIC_ERR_ARG, "null array argument");
    for (int s = 0; s < c->nspn; ++s) {
      if (c->nfrm[s] > ld) fail(FLOSIC_ERR_ARG, "ld smaller than NFRM");
      fo_setup(c, s);
      const SpinCache& S = c->spin[s];
      for (int k = 0; k < S.nf; ++k) {
        for (int w = 0; w < S.nw; ++w) tmat[((size_t)s * ld + w) * ld + k] = S.tmat[(size_t)k * S.nw + w];
        eval[(size_t)s * ld + k] = S.lam[k];
      }
    }
  });
}

int flosic_sic_coupot_sic(flosic_ctx* c, int kxxs, int kxxo, double* coulomb, double* rhog) {
  return guarded([&] {
    require(c, true);
    require_whole_mesh(c);
    if (kxxs < 1 || kxxs > c->nspn) fail(FLOSIC_ERR_ARG, "KXXS out of range");
    const int s = kxxs - 1;
    if (kxxo < 1 || kxxo > c->nfrm[s]) fail(FLOSIC_ERR_ARG, "KXXO out of range");
    spin_potentials(c, s);
    SpinCache& S = c->spin[s];
    const int P = c->nmsh, k = kxxo - 1;
    std::vector<double> v(P), r((size_t)10 * P, 0.0);
    CUDA_CHECK(cudaMemcpyAsync(v.data(), S.vh.p + (size_t)k * P, sizeof(double) * P, cudaMemcpyDeviceToHost, c->st));
    if (c->density == FLOSIC_DENSITY_PAIRS) {
      // the channels POISSON1 accumulated (meta-GGA: 4, the rest of the 10-channel layout zero)
      CUDA_CHECK(cudaMemcpy2DAsync(r.data(), sizeof(double) * P, S.rhog.p + (size_t)k * P,
                                   sizeof(double) * P * S.nf, sizeof(double) * P, c->nch(), cudaMemcpyDeviceToHost,
                                   c->st));
    } else {
      c->d_tmp.ensure((size_t)10 * P);
      launch_density(P, S.nf, k, c->nch(), S.phi.p, P, c->d_tmp.p, P, c->st);
      const int nch = c->gga ? 10 : 1;  // the meta-GGA layout has 10 channels, 4..9 zero
      CUDA_CHECK(cudaMemcpyAsync(r.data(), c->d_tmp.p, sizeof(double) * nch * P, cudaMemcpyDeviceToHost, c->st));
    }
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    for (int i = 0; i < P; ++i) {
      const int o = c->perm[i];
      if (coulomb) coulomb[o] = v[i];
      if (rhog)
        for (int ch = 0; ch < 10; ++ch) rhog[(size_t)ch * P + o] = r[(size_t)ch * P + i];
    }
  });
}

int flosic_sic_getvlxc(flosic_ctx* c, int ndim, const double* rhog, double* vxc, double* ergs) {
  return guarded([&] {
    require(c, false);
    if (c->mgga) fail(FLOSIC_ERR_ARG, "GETVLXC: a meta-GGA needs tau; use flosic_sic_getvlxc_mgga");
    if (ndim != c->nmsh) fail(FLOSIC_ERR_ARG, "NDIM must equal the mesh size");
    if (!rhog || !vxc || !ergs) fail(FLOSIC_ERR_ARG, "null array argument");
    const int P = c->nmsh;
    std::vector<double> r((size_t)10 * P);
    for (int i = 0; i < P; ++i)
      for (int ch = 0; ch < 10; ++ch) r[(size_t)ch * P + i] = rhog[(size_t)ch * ndim + c->perm[i]];
    DevBuf<double> dr, dv;
    dr.upload(r.data(), r.size(), c->st);
    dv.ensure(2 * (size_t)P);
    const int nblk = std::min(1024, (P + 255) / 256);
    c->d_part.ensure((size_t)nblk * NPART);
    c->d_sums.ensure(NPART);
    launch_xc_rhog(c->mesh_dev(), c->gga, c->xc, dr.p, P, dv.p, c->d_part.p, nblk, c->st);
    launch_reduce_parts(1, nblk, c->d_part.p, c->d_sums.p, c->st);
    std::vector<double> v(2 * (size_t)P), sums(NPART);
    CUDA_CHECK(cudaMemcpyAsync(v.data(), dv.p, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaMemcpyAsync(sums.data(), c->d_sums.p, sizeof(double) * NPART, cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    dr.release();
    dv.release();
    for (int i = 0; i < P; ++i) {
      vxc[c->perm[i]] = v[i];
      vxc[ndim + c->perm[i]] = v[P + i];
    }
    for (int j = 0; j < 4; ++j) ergs[j] = sums[4 + j];
  });
}

int flosic_sic_getvlxc_mgga(flosic_ctx* c, int ndim, const double* rhog, const double* tau, double* vxc,
                            double* mixin, double* ergs) {
  return guarded([&] {
    require(c, false);
    if (!c->mgga) fail(FLOSIC_ERR_ARG, "GETVLXC: tau and MIXIN belong to meta-GGA functionals");
    if (ndim != c->nmsh) fail(FLOSIC_ERR_ARG, "NDIM must equal the mesh size");
    if (!rhog || !tau || !vxc || !mixin || !ergs) fail(FLOSIC_ERR_ARG, "null array argument");
    const int P = c->nmsh;
    std::vector<double> r((size_t)5 * P);  // 4 density channels, then tau
    for (int i = 0; i < P; ++i) {
      for (int ch = 0; ch < 4; ++ch) r[(size_t)ch * P + i] = rhog[(size_t)ch * ndim + c->perm[i]];
      r[(size_t)4 * P + i] = tau[c->perm[i]];
    }
    DevBuf<double> dr, dv, dm;
    dr.upload(r.data(), r.size(), c->st);
    dv.ensure(2 * (size_t)P);
    dm.ensure(4 * (size_t)P);
    const int nblk = std::min(1024, (P + 255) / 256);
    c->d_part.ensure((size_t)nblk * NPART);
    c->d_sums.ensure(NPART);
    launch_xc_mgga_rhog(c->mesh_dev(), dr.p, P, dr.p + (size_t)4 * P, dv.p, dm.p, c->d_part.p, nblk, c->st);
    launch_reduce_parts(1, nblk, c->d_part.p, c->d_sums.p, c->st);
    std::vector<double> v(2 * (size_t)P), m(4 * (size_t)P), sums(NPART);
    CUDA_CHECK(cudaMemcpyAsync(v.data(), dv.p, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaMemcpyAsync(m.data(), dm.p, sizeof(double) * m.size(), cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaMemcpyAsync(sums.data(), c->d_sums.p, sizeof(double) * NPART, cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    dr.release();
    dv.release();
    dm.release();
    for (int i = 0; i < P; ++i) {
      const int o = c->perm[i];
      vxc[o] = v[i];
      vxc[ndim + o] = v[P + i];
      for (int d = 0; d < 4; ++d) {
        mixin[(size_t)4 * o + d] = m[(size_t)4 * i + d];
        mixin[(size_t)4 * (ndim + o) + d] = 0.0;  // spin-down half: no SIC density there
      }
    }
    for (int j = 0; j < 4; ++j) ergs[j] = sums[4 + j];
  });
}

int flosic_sic_set_wait_limit(flosic_ctx* c, int64_t polls) {
  return guarded([&] {
    if (!c) fail(FLOSIC_ERR_ARG, "null context");
    c->coulomb_cfg.wait_limit = polls > 0 ? (long long)polls : 0;
  });
}

int flosic_sic_set_density_mode(flosic_ctx* c, int mode) {
  return guarded([&] {
    if (!c) fail(FLOSIC_ERR_ARG, "null context");
    if (mode != FLOSIC_DENSITY_PHI2 && mode != FLOSIC_DENSITY_PAIRS) fail(FLOSIC_ERR_ARG, "unknown density mode");
    if (mode != c->density) {
      c->density = mode;
      for (auto& s : c->spin) {
        s.pot_valid = false;
        s.sic_valid = false;
        if (mode == FLOSIC_DENSITY_PHI2) s.rhog.release();
      }
      if (mode == FLOSIC_DENSITY_PHI2) c->d_dens_coef.release();
    }
  });
}

int flosic_sic_set_precision(flosic_ctx* c, int mode) {
  return guarded([&] {
    if (!c) fail(FLOSIC_ERR_ARG, "null context");
    if (mode != FLOSIC_PRECISION_FP64 && mode != FLOSIC_PRECISION_MIXED) fail(FLOSIC_ERR_ARG, "unknown precision mode");
    if (mode != c->precision) {
      c->precision = mode;
      for (auto& s : c->spin) {
        s.pot_valid = false;
        s.sic_valid = false;
      }
    }
  });
}

// Tile-shape autotuner of the per-FO Coulomb kernel: its tiles are 128 mesh
// points by 32, 64 or 128 compacted FO slots.  Each width is timed (CUDA
// events on the context's stream, best of reps after one untimed run) on the
// full COUPOT_SIC Coulomb evaluation of the spin with the most FOs, under the
// context's precision mode and mesh shard, and the fastest is kept.  The
// widths only regroup FOs into CTAs; every potential is formed by the same
// operations in the same order, so the choice changes time, not results.
// Work counters and launch counts are left as they were.
int flosic_sic_autotune(flosic_ctx* c, int reps, int* perfo_fos, float* ms) {
  return guarded([&] {
    require(c, true);
    if (reps < 1 || reps > 100) fail(FLOSIC_ERR_ARG, "REPS must be in 1..100");
    if (!perfo_fos) fail(FLOSIC_ERR_ARG, "null output pointer");
    const int s = (c->nspn == 2 && c->nfrm[1] > c->nfrm[0]) ? 1 : 0;
    if (c->nfrm[s] < 1) fail(FLOSIC_ERR_STATE, "no FOs to tune on");
    // The timing runs overwrite this spin's potentials: drop the cached ones
    // first, and put the width and counters back on every way out.
    c->spin[s].pot_valid = false;
    c->spin[s].sic_valid = false;
    struct Restore {
      flosic_ctx* c;
      int wm;
      unsigned long long wn, wf, wt;
      long long nl;
      ~Restore() {
        c->coulomb_cfg.perfo_wm = wm;
        c->work_near = wn;
        c->work_far = wf;
        c->work_terms = wt;
        c->launches = nl;
      }
    } restore{c, c->coulomb_cfg.perfo_wm, c->work_near, c->work_far, c->work_terms, c->launches};
    fo_setup(c, s);
    const int nf = c->spin[s].nf;
    cudaStream_t st = c->st;
    float best = std::numeric_limits<float>::infinity();
    int best_wm = 0;
    for (int i = 0; i < 3; ++i) {
      const int wm = 1 << i;
      if (ms) ms[i] = -1.f;
      if (wm > 1 && 16 * wm >= nf) continue;  // half the block or more would stay empty
      c->coulomb_cfg.perfo_wm = wm;
      coulomb(c, s);
      float t = std::numeric_limits<float>::infinity();
      for (int r = 0; r < reps; ++r) {
        CUDA_CHECK(cudaEventRecord(c->ev[5], st));
        coulomb(c, s);
        CUDA_CHECK(cudaEventRecord(c->ev[6], st));
        CUDA_CHECK(cudaEventSynchronize(c->ev[6]));
        t = std::min(t, elapsed(c->ev[5], c->ev[6]));
      }
      if (ms) ms[i] = t;
      if (t < best) {
        best = t;
        best_wm = wm;
      }
    }
    restore.wm = best_wm;
    *perfo_fos = 32 * best_wm;
  });
}

int flosic_sic_getvlxc_device(flosic_ctx* c, int npts, const double* d_rhog, int ldr, const double* d_wmsh,
                              double* d_vxc, double* ergs) {
  return guarded([&] {
    require(c, false);
    if (c->mgga) fail(FLOSIC_ERR_ARG, "GETVLXC: a meta-GGA needs tau; use flosic_sic_getvlxc_mgga");
    if (npts < 1) fail(FLOSIC_ERR_ARG, "NPTS must be positive");
    if (ldr < npts) fail(FLOSIC_ERR_ARG, "LDR smaller than NPTS");
    if (!d_rhog || !d_wmsh || !d_vxc || !ergs) fail(FLOSIC_ERR_ARG, "null array argument");
    if (npts > XC_SCRATCH_POINTS)
      fail(FLOSIC_ERR_CAPACITY, "NPTS = " + std::to_string(npts) + " exceeds the " +
                                    std::to_string(XC_SCRATCH_POINTS) +
                                    "-point capacity of the allocation-free GETVLXC scratch");
    double* part = xc_scratch_address(c->device);
    double* sums = part + (size_t)XC_SCRATCH_BLOCKS * NPART;
    const int nblk = std::min(1024, (npts + 255) / 256);  // k_xc_rhog strides over the rest
    MeshDev M{};
    M.n = npts;
    M.w = d_wmsh;
    launch_xc_rhog(M, c->gga, c->xc, d_rhog, ldr, d_vxc, part, nblk, c->st);
    launch_reduce_parts(1, nblk, part, sums, c->st);
    CUDA_CHECK(cudaGetLastError());
    double s[NPART];
    CUDA_CHECK(cudaMemcpyAsync(s, sums, sizeof(s), cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    for (int j = 0; j < 4; ++j) ergs[j] = s[4 + j];
  });
}

int flosic_sic_apotnl_sic(flosic_ctx* c, double* totqnum, int lspx, int iorbx, double* results, double* cfrm,
                          double* pot) {
  return guarded([&] {
    require(c, true);
    require_whole_mesh(c);
    if (lspx < 1 || lspx > c->nspn) fail(FLOSIC_ERR_ARG, "LSPX out of range");
    const int s = lspx - 1;
    if (iorbx == 0) fail(FLOSIC_ERR_ARG, "APOTNL_SIC is trying to run DFT calculation");
    const int k = std::abs(iorbx) - 1;
    if (k >= c->nfrm[s]) fail(FLOSIC_ERR_ARG, "IORBX out of range");
    spin_potentials(c, s);
    SpinCache& S = c->spin[s];
    if (results)
      for (int i = 0; i < 13; ++i) results[i] = S.results[(size_t)k * 13 + i];
    if (cfrm)
      for (int d = 0; d < 3; ++d) cfrm[d] = S.cfrm[(size_t)k * 3 + d];
    if (totqnum) *totqnum = S.results[(size_t)k * 13 + 1];
    if (pot) {
      const int P = c->nmsh;
      std::vector<double> v(P);
      CUDA_CHECK(cudaMemcpyAsync(v.data(), S.vpot.p + (size_t)k * P, sizeof(double) * P, cudaMemcpyDeviceToHost, c->st));
      CUDA_CHECK(cudaStreamSynchronize(c->st));
      for (int i = 0; i < P; ++i) pot[c->perm[i]] = v[i];
    }
  });
}

int flosic_sic_siclagm(flosic_ctx* c, int lspn, double* sic, int ld) {
  return guarded([&] {
    require(c, true);
    require_whole_mesh(c);
    if (lspn < 1 || lspn > c->nspn) fail(FLOSIC_ERR_ARG, "LSPN out of range");
    const int s = lspn - 1;
    if (c->nfrm[s] > ld) fail(FLOSIC_ERR_ARG, "ld smaller than NFRM");
    if (!sic) fail(FLOSIC_ERR_ARG, "null array argument");
    spin_sic(c, s);
    const SpinCache& S = c->spin[s];
    for (int l = 0; l < S.nf; ++l)
      for (int j = 0; j < S.nf; ++j) sic[(size_t)l * ld + j] = S.sic[(size_t)l * S.nf + j];
  });
}

int flosic_sic_frmorb2_force(flosic_ctx* c, int lspn, const double* sic, int ld, double* debdax) {
  return guarded([&] {
    require(c, true);
    if (lspn < 1 || lspn > c->nspn) fail(FLOSIC_ERR_ARG, "LSPN out of range");
    const int s = lspn - 1;
    if (c->nfrm[s] > ld) fail(FLOSIC_ERR_ARG, "ld smaller than NFRM");
    if (!sic || !debdax) fail(FLOSIC_ERR_ARG, "null array argument");
    std::vector<double> deb(3 * (size_t)c->nfrm[s]);
    spin_force(c, s, sic, ld, deb.data());
    for (int k = 0; k < c->nfrm[s]; ++k)
      for (int d = 0; d < 3; ++d) debdax[3 * (size_t)k + d] = deb[3 * (size_t)k + d];
  });
}

int flosic_sic_cycle(flosic_ctx* c, int ld, double* results, double* sic, double* debdax, double* cfrm,
                     double* esic) {
  return guarded([&] {
    require(c, true);
    require_whole_mesh(c);
    if (!results || !sic || !debdax || !cfrm || !esic) fail(FLOSIC_ERR_ARG, "null array argument");
    for (int s = 0; s < c->nspn; ++s)
      if (c->nfrm[s] > ld) fail(FLOSIC_ERR_ARG, "ld smaller than NFRM");
    c->launches = 0;
    c->work_near = c->work_far = c->work_terms = 0;
    for (double& m : c->stage_ms) m = 0.0;
    c->kernel_ms[0] = c->kernel_ms[1] = 0.0;
    for (auto& w : c->kernel_work) w = 0;
    invalidate(c);
    double zsic = 0.0;
    for (int s = 0; s < c->nspn; ++s) {
      const int nf = c->nfrm[s];
      if (nf == 0) continue;
      spin_sic(c, s);
      const SpinCache& S = c->spin[s];
      for (int k = 0; k < nf; ++k) {
        for (int i = 0; i < 13; ++i) results[((size_t)s * ld + k) * 13 + i] = S.results[(size_t)k * 13 + i];
        for (int d = 0; d < 3; ++d) cfrm[((size_t)s * ld + k) * 3 + d] = S.cfrm[(size_t)k * 3 + d];
        zsic += S.results[(size_t)k * 13 + 8];
      }
      double* ps = sic + (size_t)s * ld * ld;
      for (int l = 0; l < nf; ++l)
        for (int j = 0; j < nf; ++j) ps[(size_t)l * ld + j] = S.sic[(size_t)l * nf + j];
      spin_force(c, s, ps, ld, debdax + (size_t)s * ld * 3);
    }
    *esic = zsic;
  });
}

int flosic_sic_batch_cycle(flosic_ctx** ctxs, int n, int wm, int ld, double* results, double* sic,
                           double* debdax, double* cfrm, double* esic) {
  return guarded([&] {
    if (!ctxs || n < 1) fail(FLOSIC_ERR_ARG, "empty batch");
    if (!results || !sic || !debdax || !cfrm || !esic) fail(FLOSIC_ERR_ARG, "null array argument");
    if (wm != 0 && wm != 1 && wm != 2 && wm != 4) fail(FLOSIC_ERR_ARG, "FO block width must be 0, 1, 2 or 4 warps");
    flosic_ctx* c0 = ctxs[0];
    for (int m = 0; m < n; ++m) {
      flosic_ctx* c = ctxs[m];
      require(c, true);
      require_whole_mesh(c);
      if (c->device != c0->device) fail(FLOSIC_ERR_ARG, "batch contexts on different devices");
      if (c->precision != c0->precision) fail(FLOSIC_ERR_ARG, "batch contexts in different precisions");
      for (int s = 0; s < c->nspn; ++s)
        if (c->nfrm[s] > ld) fail(FLOSIC_ERR_ARG, "ld smaller than NFRM");
      for (int j = 0; j < m; ++j)
        if (ctxs[j] == c) fail(FLOSIC_ERR_ARG, "a context appears twice in the batch");
    }
    CUDA_CHECK(cudaSetDevice(c0->device));
    if (wm == 0) {  // widest block that the largest FO count fills at least half
      int nfmax = 1;
      for (int m = 0; m < n; ++m)
        for (int s = 0; s < ctxs[m]->nspn; ++s) nfmax = std::max(nfmax, ctxs[m]->nfrm[s]);
      wm = nfmax > 64 ? 4 : (nfmax > 32 ? 2 : 1);
    }
    // 1. every (molecule, spin) up to its Coulomb evaluation, on its own stream
    std::vector<CoulombJob> jobs;
    std::vector<std::pair<int, int>> owner;  // (molecule, spin) of each job
    std::vector<int4> items;
    for (int m = 0; m < n; ++m) {
      flosic_ctx* c = ctxs[m];
      c->launches = 0;
      c->work_near = c->work_far = c->work_terms = 0;
      for (double& x : c->stage_ms) x = 0.0;
      c->kernel_ms[0] = c->kernel_ms[1] = 0.0;
      for (auto& w : c->kernel_work) w = 0;
      invalidate(c);
      CUDA_CHECK(cudaEventRecord(c->ev[0], c->st));
      for (int s = 0; s < c->nspn; ++s) {
        if (c->nfrm[s] == 0) continue;
        jobs.push_back(batch_prepare(c, s));
        owner.push_back({m, s});
      }
      CUDA_CHECK(cudaEventRecord(c->ev[3], c->st));
      if (m > 0) CUDA_CHECK(cudaStreamWaitEvent(c0->st, c->ev[3], 0));
    }
    // work list, costliest jobs first (a tile walks every call of its job; the
    // counter then hands the cheap items to whichever CTA frees up)
    std::vector<int> order(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) order[j] = (int)j;
    auto cost = [&](int j) { return (double)jobs[j].ncalls * std::min(jobs[j].nfo, 32 * wm); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    for (int job : order) {
      const CoulombJob& J = jobs[job];
      const int nfb = (J.nfo + 32 * wm - 1) / (32 * wm);
      for (int t = 0; t < J.M.ntiles; ++t)
        for (int b = 0; b < nfb; ++b) items.push_back(make_int4(job, t, b, 0));
    }
    // 2. all potentials of all molecules: two persistent launches on the first context's stream
    int nsm = 148;
    CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c0->device));
    c0->d_jobs.ensure(std::max<size_t>(jobs.size(), 1));
    c0->d_items.ensure(std::max<size_t>(items.size(), 1));
    if (!jobs.empty()) {
      CUDA_CHECK(cudaMemcpyAsync(c0->d_jobs.p, jobs.data(), sizeof(CoulombJob) * jobs.size(), cudaMemcpyHostToDevice,
                                 c0->st));
      CUDA_CHECK(cudaMemcpyAsync(c0->d_items.p, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice,
                                 c0->st));
      c0->d_batch_counters.ensure(2);
      launch_coulomb_batch(c0->d_jobs.p, c0->d_items.p, (int)items.size(), c0->d_batch_counters.p, wm,
                           c0->precision == FLOSIC_PRECISION_MIXED, c0->d_boys.p, nsm, c0->st);
      CUDA_CHECK(cudaGetLastError());
      c0->launches += 2;
    }
    CUDA_CHECK(cudaEventRecord(c0->ev[4], c0->st));
    for (int m = 1; m < n; ++m) CUDA_CHECK(cudaStreamWaitEvent(ctxs[m]->st, c0->ev[4], 0));
    CUDA_CHECK(cudaStreamSynchronize(c0->st));  // the host job and item arrays may go
    // 3. per molecule: work counts, XC and energies, SIC matrix, forces
    for (size_t j = 0; j < jobs.size(); ++j) {
      flosic_ctx* c = ctxs[owner[j].first];
      unsigned long long cnt[3];
      CUDA_CHECK(cudaMemcpyAsync(cnt, c->spin[owner[j].second].bc.cnt.p, sizeof(cnt), cudaMemcpyDeviceToHost, c->st));
      CUDA_CHECK(cudaStreamSynchronize(c->st));
      c->work_near += cnt[0];
      c->work_far += cnt[1];
      c->work_terms += cnt[2];
      spin_xc(c, owner[j].second);
    }
    for (int m = 0; m < n; ++m) {
      flosic_ctx* c = ctxs[m];
      double zsic = 0.0;
      for (int s = 0; s < c->nspn; ++s) {
        const int nf = c->nfrm[s];
        if (nf == 0) continue;
        spin_sic(c, s);
        const SpinCache& S = c->spin[s];
        const size_t o = (size_t)m * 2 + s;
        for (int k = 0; k < nf; ++k) {
          for (int i = 0; i < 13; ++i) results[(o * ld + k) * 13 + i] = S.results[(size_t)k * 13 + i];
          for (int d = 0; d < 3; ++d) cfrm[(o * ld + k) * 3 + d] = S.cfrm[(size_t)k * 3 + d];
          zsic += S.results[(size_t)k * 13 + 8];
        }
        double* ps = sic + o * ld * ld;
        for (int l = 0; l < nf; ++l)
          for (int jj = 0; jj < nf; ++jj) ps[(size_t)l * ld + jj] = S.sic[(size_t)l * nf + jj];
        spin_force(c, s, ps, ld, debdax + o * ld * 3);
      }
      esic[m] = zsic;
    }
  });
}

int flosic_sic_mgga_mixin(flosic_ctx* c, int lspx, int iorbx, double* mixin) {
  return guarded([&] {
    require(c, true);
    require_whole_mesh(c);
    if (!c->mgga) fail(FLOSIC_ERR_ARG, "MIXIN belongs to meta-GGA functionals");
    if (lspx < 1 || lspx > c->nspn) fail(FLOSIC_ERR_ARG, "LSPX out of range");
    const int s = lspx - 1, k = iorbx - 1;
    if (k < 0 || k >= c->nfrm[s]) fail(FLOSIC_ERR_ARG, "IORBX out of range");
    if (!mixin) fail(FLOSIC_ERR_ARG, "null array argument");
    spin_potentials(c, s);
    SpinCache& S = c->spin[s];
    const int P = c->nmsh;
    // the FO's density channels (those k_xc used: phi^2, or the pair route's)
    // and tau, then SUBVLXC's SCAN branch
    DevBuf<double> dr, dv, dm;
    dr.ensure((size_t)11 * P);
    dv.ensure(2 * (size_t)P);
    dm.ensure(4 * (size_t)P);
    if (c->density == FLOSIC_DENSITY_PAIRS)
      CUDA_CHECK(cudaMemcpy2DAsync(dr.p, sizeof(double) * P, S.rhog.p + (size_t)k * P, sizeof(double) * P * S.nf,
                                   sizeof(double) * P, 4, cudaMemcpyDeviceToDevice, c->st));
    else
      launch_density(P, S.nf, k, 4, S.phi.p, P, dr.p, P, c->st);
    launch_fo_tau(P, S.nf, k, S.phi.p, P, dr.p + (size_t)10 * P, c->st);
    const int nblk = std::min(1024, (P + 255) / 256);
    c->d_part.ensure((size_t)nblk * NPART);
    launch_xc_mgga_rhog(c->mesh_dev(), dr.p, P, dr.p + (size_t)10 * P, dv.p, dm.p, c->d_part.p, nblk, c->st);
    std::vector<double> m(4 * (size_t)P);
    CUDA_CHECK(cudaMemcpyAsync(m.data(), dm.p, sizeof(double) * m.size(), cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    dr.release();
    dv.release();
    dm.release();
    for (int i = 0; i < P; ++i) {
      const int o = c->perm[i];
      for (int d = 0; d < 4; ++d) {
        mixin[(size_t)4 * o + d] = m[(size_t)4 * i + d];
        mixin[(size_t)4 * (P + o) + d] = 0.0;
      }
    }
  });
}

int flosic_sic_adjoint(flosic_ctx* c, int lspn, double* g, int ldg) {
  return guarded([&] {
    require(c, true);  // on a mesh shard: the shard's partial sum
    if (lspn < 1 || lspn > c->nspn) fail(FLOSIC_ERR_ARG, "LSPN out of range");
    if (!g) fail(FLOSIC_ERR_ARG, "null array argument");
    if (ldg < c->nbasis) fail(FLOSIC_ERR_ARG, "ldg smaller than the number of basis functions");
    const int s = lspn - 1;
    DevBuf<double> dg;
    adjoint_device(c, s, dg);
    const int nf = c->spin[s].nf, nb = c->nbasis;
    std::vector<double> h((size_t)nb * nf);
    CUDA_CHECK(cudaMemcpyAsync(h.data(), dg.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    dg.release();
    for (int k = 0; k < nf; ++k)
      for (int mu = 0; mu < nb; ++mu) g[(size_t)k * ldg + mu] = h[(size_t)k * nb + mu];
  });
}

int flosic_sic_adjoint_fod(flosic_ctx* c, int lspn, double* grad, int ld) {
  return guarded([&] {
    require(c, true);
    require_whole_mesh(c);
    if (lspn < 1 || lspn > c->nspn) fail(FLOSIC_ERR_ARG, "LSPN out of range");
    if (!grad) fail(FLOSIC_ERR_ARG, "null array argument");
    const int s = lspn - 1;
    if (ld < std::max(1, c->nfrm[s])) fail(FLOSIC_ERR_ARG, "ld smaller than NFRM");
    std::fill(grad, grad + (size_t)3 * ld, 0.0);
    if (c->nfrm[s] == 0) return;
    fod_gradient(c, s, grad);
  });
}

int flosic_sic_siclag_der(flosic_ctx* c, double* dersic, int ldo) {
  return guarded([&] {
    require(c, true);  // on a mesh shard: the shard's partial sum
    if (!dersic) fail(FLOSIC_ERR_ARG, "null array argument");
    const int nwft = c->nfrm[0] + (c->nspn == 2 ? c->nfrm[1] : 0);
    if (ldo < std::max(1, nwft)) fail(FLOSIC_ERR_ARG, "ldo smaller than NFRM(1)+NFRM(2)");
    const int nb = c->nbasis, P = c->eval_n;
    std::fill(dersic, dersic + (size_t)c->natoms * ldo * 3, 0.0);
    // Hessian channel of (d_ix, d_c) in the basis layout: xx yy zz 4-6, xy xz yz 7-9
    const int hch[3][3] = {{4, 7, 8}, {7, 5, 9}, {8, 9, 6}};
    const int nderv = c->mgga ? 2 : 1, nbch = c->mgga ? 10 : 4;
    const size_t budget = (size_t)3 << 30;
    int chunk = (int)std::min<size_t>(P, std::max<size_t>(TILE, budget / (sizeof(double) * nbch * nb)));
    chunk = std::max(TILE, chunk / TILE * TILE);
    for (int s = 0; s < c->nspn; ++s) {
      const int nf = c->nfrm[s];
      if (nf == 0) continue;
      spin_potentials(c, s);
      SpinCache& S = c->spin[s];
      c->d_basis.ensure((size_t)nbch * nb * chunk);
      // H_ix = B_{1+ix}^T Y_0 (+ sum_c B_{h(ix,c)}^T Y_{1+c}), nb x nf each
      DevBuf<double> dh;
      dh.ensure((size_t)3 * nb * nf);
      bool first = true;
      for (int p0 = 0; p0 < P; p0 += chunk) {
        const int np = std::min(chunk, P - p0);
        const size_t q0 = (size_t)c->eval_p0 + p0;
        launch_basis_values(c->basis_dev(), nderv, np, c->d_x.p + q0, c->d_y.p + q0, c->d_z.p + q0, c->d_basis.p, np,
                            c->st);
        c->launches++;
        for (int ix = 0; ix < 3; ++ix) {
          const int nterm = c->mgga ? 4 : 1;
          for (int t = 0; t < nterm; ++t) {
            const int bch = t == 0 ? 1 + ix : hch[ix][t - 1];
            gemm(c, true, false, nb, nf, np, 1.0, c->d_basis.p + (size_t)bch * nb * np, np,
                 S.y.p + (size_t)t * nf * P + p0, P, (first && t == 0) ? 0.0 : 1.0, dh.p + (size_t)ix * nb * nf, nb);
          }
        }
        first = false;
      }
      std::vector<double> h((size_t)3 * nb * nf), cf((size_t)nb * nf);
      CUDA_CHECK(cudaMemcpyAsync(h.data(), dh.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
      CUDA_CHECK(cudaMemcpyAsync(cf.data(), S.cfo.p, sizeof(double) * cf.size(), cudaMemcpyDeviceToHost, c->st));
      CUDA_CHECK(cudaStreamSynchronize(c->st));
      dh.release();
      // DERSIC(ix, lfn, A) = sum_{mu on A} C_mu,k H_ix[mu, k]
      const double fac = c->nspn == 1 ? 2.0 : 1.0;
      for (int a = 0; a < c->natoms; ++a) {
        const int m0 = c->aoff[a], m1 = (a + 1 < c->natoms) ? c->aoff[a + 1] : nb;
        for (int k = 0; k < nf; ++k) {
          double* d = dersic + ((size_t)a * ldo + k + (size_t)s * c->nfrm[0]) * 3;
          for (int ix = 0; ix < 3; ++ix) {
            const double* hk = &h[((size_t)ix * nf + k) * nb];
            double acc = 0.0;
            for (int mu = m0; mu < m1; ++mu) acc += cf[(size_t)k * nb + mu] * hk[mu];
            d[ix] = fac * acc;
          }
        }
      }
    }
  });
}

int flosic_sic_sicham(flosic_ctx* c, int lspn, double* ham, int ldh, int packed) {
  return guarded([&] {
    require(c, true);
    require_whole_mesh(c);
    if (lspn < 1 || lspn > c->nspn) fail(FLOSIC_ERR_ARG, "LSPN out of range");
    if (!ham) fail(FLOSIC_ERR_ARG, "null array argument");
    if (packed != 0 && packed != 1) fail(FLOSIC_ERR_ARG, "packed must be 0 or 1");
    if (!packed && ldh < c->nbasis) fail(FLOSIC_ERR_ARG, "ldh smaller than the number of basis functions");
    const int s = lspn - 1, nb = c->nbasis, P = c->eval_n;
    const int nf = c->nfrm[s];
    if (nf == 0) return;
    spin_potentials(c, s);
    SpinCache& S = c->spin[s];
    // a = sum_c B_c^T Y_c = <chi|V_k|phi_k> (NEWWAY's BASPHI(.,2) up to its sign),
    // b = B_0^T (w phi) = <chi|phi_k> (BASPHI(.,1)), both nb x nf
    const int nyc = c->mgga ? 4 : 1;
    const int nderv = c->mgga ? 1 : 0;
    const size_t budget = (size_t)3 << 30;
    int chunk = (int)std::min<size_t>(P, std::max<size_t>(TILE, budget / (sizeof(double) * nyc * nb)));
    chunk = std::max(TILE, chunk / TILE * TILE);
    c->d_basis.ensure((size_t)nyc * nb * chunk);
    c->d_tmp.ensure((size_t)nf * P);
    launch_scale_rows(P, nf, S.phi.p, P, c->d_w.p + c->eval_p0, c->d_tmp.p, P, c->st);
    c->launches++;
    DevBuf<double> dab, dh;
    dab.ensure((size_t)2 * nb * nf);
    dh.ensure((size_t)nb * nb);
    double* da = dab.p;
    double* db = dab.p + (size_t)nb * nf;
    for (int p0 = 0; p0 < P; p0 += chunk) {
      const int np = std::min(chunk, P - p0);
      const size_t q0 = (size_t)c->eval_p0 + p0;
      launch_basis_values(c->basis_dev(), nderv, np, c->d_x.p + q0, c->d_y.p + q0, c->d_z.p + q0, c->d_basis.p, np,
                          c->st);
      c->launches++;
      const double beta = p0 == 0 ? 0.0 : 1.0;
      for (int ch = 0; ch < nyc; ++ch)
        gemm(c, true, false, nb, nf, np, 1.0, c->d_basis.p + (size_t)ch * nb * np, np,
             S.y.p + (size_t)ch * nf * P + p0, P, ch == 0 ? beta : 1.0, da, nb);
      gemm(c, true, false, nb, nf, np, 1.0, c->d_basis.p, np, c->d_tmp.p + p0, P, beta, db, nb);
    }
    // APATCH: HSTOR += (HAM + HAM^T)/2 with HAM(j,i) = BASPHI(i,2) BASPHI(j,1), summed
    // over the spin's FOs: H = -(a b^T + b a^T)/2
    gemm(c, false, true, nb, nb, nf, -0.5, da, nb, db, nb, 0.0, dh.p, nb);
    gemm(c, false, true, nb, nb, nf, -0.5, db, nb, da, nb, 1.0, dh.p, nb);
    std::vector<double> h((size_t)nb * nb);
    CUDA_CHECK(cudaMemcpyAsync(h.data(), dh.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    dab.release();
    dh.release();
    if (packed) {
      // HSTOR order of a C1 calculation: IBAS = 1..N outer, JBAS = IBAS..N inner
      size_t indx = 0;
      for (int i = 0; i < nb; ++i)
        for (int j = i; j < nb; ++j) ham[indx++] += h[(size_t)i * nb + j];
    } else {
      for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) ham[(size_t)i * ldh + j] += h[(size_t)i * nb + j];
    }
  });
}

int flosic_sic_densold(flosic_ctx* c, int ngrad, double* rhog, double* phig) {
  return guarded([&] {
    require(c, true);
    require_whole_mesh(c);
    if (ngrad != 1 && ngrad != 10) fail(FLOSIC_ERR_ARG, "NGRAD must be 1 or 10");
    if (!rhog) fail(FLOSIC_ERR_ARG, "null array argument");
    const int nb = c->nbasis, P = c->nmsh, ns = c->nspn;
    const int nw0 = c->nwfs[0], nw1 = ns == 2 ? c->nwfs[1] : 0, nwf = nw0 + nw1;
    const int nderv = ngrad == 10 ? 2 : 0;
    const size_t budget = (size_t)3 << 30;
    int chunk = (int)std::min<size_t>(P, std::max<size_t>(TILE, budget / (sizeof(double) * ngrad * (nb + nwf))));
    chunk = std::max(TILE, chunk / TILE * TILE);
    DevBuf<double> dv, dr, dph;
    dv.ensure((size_t)ngrad * std::max(nwf, 1) * chunk);
    dr.ensure((size_t)ns * ngrad * P);
    if (phig) dph.ensure((size_t)ns * P);
    for (int p0 = 0; p0 < P; p0 += chunk) {
      const int np = std::min(chunk, P - p0);
      // PSIG (densold.F:160-185): coefficients at or below 1e-10 are skipped, as in d_psi_thr
      if (nwf > 0) {
        launch_fo_values(c->basis_dev(), nderv, np, c->d_x.p + p0, c->d_y.p + p0, c->d_z.p + p0, c->d_psi_thr.p, nb,
                         nwf, dv.p, np, c->coulomb_cfg.fo_values_bn, c->st);
        c->launches++;
      }
      launch_densold(np, nw0, nw1, ns, ngrad, dv.p, np, dr.p + p0, phig ? dph.p + p0 : nullptr, P, c->st);
      c->launches++;
    }
    std::vector<double> h((size_t)ns * ngrad * P), hp(phig ? (size_t)ns * P : 0);
    CUDA_CHECK(cudaMemcpyAsync(h.data(), dr.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
    if (phig) CUDA_CHECK(cudaMemcpyAsync(hp.data(), dph.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    for (int i = 0; i < P; ++i) {
      const int o = c->perm[i];
      for (int q = 0; q < ns * ngrad; ++q) rhog[(size_t)q * P + o] = h[(size_t)q * P + i];
      if (phig)
        for (int q = 0; q < ns; ++q) phig[(size_t)q * P + o] = hp[(size_t)q * P + i];
    }
  });
}

int flosic_sic_coupot1(flosic_ctx* c, double* coulomb) {
  return guarded([&] {
    require(c, true);
    require_whole_mesh(c);
    if (!coulomb) fail(FLOSIC_ERR_ARG, "null array argument");
    const int P = c->nmsh, nwf = c->nwfs[0] + (c->nspn == 2 ? c->nwfs[1] : 0);
    const int npairs = (int)c->pairs.size();
    c->d_u.ensure((size_t)std::max(nwf, 1) * c->nprim * 10);
    if (nwf > 0) launch_prim_u(c->basis_dev(), nwf, c->d_psi.p, c->nbasis, c->d_u.p, c->st);
    DevBuf<double> ddm, dvh;
    ddm.ensure((size_t)std::max(npairs, 1) * 100);
    dvh.ensure((size_t)P);
    launch_pair_dm(npairs, c->d_pairs.p, nwf, c->nprim, c->d_u.p, ddm.p, c->st);
    c->launches += 2;
    coulomb_eval(c, 1, ddm.p, dvh.p);
    std::vector<double> v(P);
    CUDA_CHECK(cudaMemcpyAsync(v.data(), dvh.p, sizeof(double) * P, cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    for (int i = 0; i < P; ++i) coulomb[c->perm[i]] = v[i];
  });
}

int flosic_sic_set_shard(flosic_ctx* c, int shard, int nshards) {
  return guarded([&] {
    if (!c) fail(FLOSIC_ERR_ARG, "null context");
    if (nshards < 1 || shard < 0 || shard >= nshards) fail(FLOSIC_ERR_ARG, "shard must lie in [0, nshards)");
    if (c->have_geom && nshards > c->ntiles)
      fail(FLOSIC_ERR_ARG, "more mesh shards (" + std::to_string(nshards) + ") than mesh tiles of 128 points");
    c->shard = shard;
    c->nshards = nshards;
    if (c->have_geom) set_eval_range(c);
    invalidate(c);
  });
}

// Packed partial sums of one shard: per spin SIC(nf,nf) | parts(NPART,nf) |
// asy(nf), then the three work counters.
static size_t partial_doubles(const flosic_ctx* c) {
  size_t n = 3;
  for (int s = 0; s < c->nspn; ++s) {
    const size_t nf = (size_t)c->nfrm[s];
    n += nf * nf + nf * NPART + nf;
  }
  return n;
}

int flosic_sic_partial_size(flosic_ctx* c, int64_t* ndoubles) {
  return guarded([&] {
    require(c, true);
    if (!ndoubles) fail(FLOSIC_ERR_ARG, "null argument");
    *ndoubles = (int64_t)partial_doubles(c);
  });
}

int flosic_sic_cycle_partial(flosic_ctx* c, double* d_partial) {
  return guarded([&] {
    require(c, true);
    if (!d_partial) fail(FLOSIC_ERR_ARG, "null partial buffer");
    c->launches = 0;
    c->work_near = c->work_far = c->work_terms = 0;
    for (double& m : c->stage_ms) m = 0.0;
    c->kernel_ms[0] = c->kernel_ms[1] = 0.0;
    for (auto& w : c->kernel_work) w = 0;
    invalidate(c);
    std::vector<double> h(partial_doubles(c), 0.0);
    size_t o = 0;
    for (int s = 0; s < c->nspn; ++s) {
      const int nf = c->nfrm[s];
      if (nf == 0) continue;
      spin_sic(c, s);
      const SpinCache& S = c->spin[s];
      std::copy(S.sic.begin(), S.sic.end(), h.begin() + o);
      o += (size_t)nf * nf;
      std::copy(S.parts.begin(), S.parts.end(), h.begin() + o);
      o += (size_t)nf * NPART;
      std::copy(S.asy.begin(), S.asy.end(), h.begin() + o);
      o += nf;
    }
    h[o] = (double)c->work_near;
    h[o + 1] = (double)c->work_far;
    h[o + 2] = (double)c->work_terms;
    CUDA_CHECK(cudaMemcpyAsync(d_partial, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
  });
}

int flosic_sic_cycle_combine(flosic_ctx* c, const double* d_partial, int ld, double* results, double* sic,
                             double* debdax, double* cfrm, double* esic) {
  return guarded([&] {
    require(c, true);
    if (!d_partial || !results || !sic || !debdax || !cfrm || !esic) fail(FLOSIC_ERR_ARG, "null array argument");
    for (int s = 0; s < c->nspn; ++s)
      if (c->nfrm[s] > ld) fail(FLOSIC_ERR_ARG, "ld smaller than NFRM");
    for (int s = 0; s < c->nspn; ++s)
      if (c->nfrm[s] > 0 && !c->spin[s].fo_valid)
        fail(FLOSIC_ERR_STATE, "flosic_sic_cycle_partial has not run on this context");
    std::vector<double> h(partial_doubles(c));
    CUDA_CHECK(cudaMemcpyAsync(h.data(), d_partial, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
    CUDA_CHECK(cudaStreamSynchronize(c->st));
    size_t o = 0;
    double zsic = 0.0;
    for (int s = 0; s < c->nspn; ++s) {
      const int nf = c->nfrm[s];
      if (nf == 0) continue;
      const double* lam = &h[o];
      const double* parts = &h[o + (size_t)nf * nf];
      const double* asy = &h[o + (size_t)nf * nf + (size_t)nf * NPART];
      o += (size_t)nf * nf + (size_t)nf * NPART + nf;
      std::vector<double> res, cf;
      results_from_parts(c, nf, parts, asy, res, cf);
      for (int k = 0; k < nf; ++k) {
        for (int i = 0; i < 13; ++i) results[((size_t)s * ld + k) * 13 + i] = res[(size_t)k * 13 + i];
        for (int d = 0; d < 3; ++d) cfrm[((size_t)s * ld + k) * 3 + d] = cf[(size_t)k * 3 + d];
        zsic += res[(size_t)k * 13 + 8];
      }
      double* ps = sic + (size_t)s * ld * ld;
      for (int l = 0; l < nf; ++l)
        for (int j = 0; j < nf; ++j) ps[(size_t)l * ld + j] = lam[(size_t)l * nf + j];
      spin_force(c, s, ps, ld, debdax + (size_t)s * ld * 3);
    }
    c->work_near = (unsigned long long)h[o];
    c->work_far = (unsigned long long)h[o + 1];
    c->work_terms = (unsigned long long)h[o + 2];
    *esic = zsic;
  });
}

int flosic_sic_stats(flosic_ctx* c, int64_t* launches, double* stage_ms, int64_t* npairs, int64_t* ncalls,
                     int64_t* work) {
  if (!c) return FLOSIC_ERR_ARG;
  if (work) {
    work[0] = (int64_t)c->work_near;
    work[1] = (int64_t)c->work_far;
    work[2] = (int64_t)c->work_terms;
  }
  if (launches) *launches = c->launches;
  if (stage_ms)
    for (int i = 0; i < 7; ++i) stage_ms[i] = c->stage_ms[i];
  if (npairs) *npairs = (int64_t)c->pairs.size();
  if (ncalls) *ncalls = (int64_t)c->calls.size();
  return FLOSIC_OK;
}

int flosic_sic_kernel_stats(flosic_ctx* c, double* ms, int64_t* work) {
  if (!c) return FLOSIC_ERR_ARG;
  if (ms) {
    ms[0] = c->kernel_ms[0];
    ms[1] = c->kernel_ms[1];
  }
  if (work)
    for (int j = 0; j < 6; ++j) work[j] = (int64_t)c->kernel_work[j];
  return FLOSIC_OK;
}

}  // extern "C"
