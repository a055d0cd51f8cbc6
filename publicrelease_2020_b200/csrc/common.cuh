// Shared device definitions for libflosic_sic_b200 (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace flosic {

constexpr int MAX_BARE = 25;      // PARAMA2
constexpr int MAX_CON = 15;       // PARAMA2
constexpr int NSPEED = 25;        // PARAMA2
constexpr int MXPR = 100;         // MXPOISS: slots per Poisson batch
constexpr double CUTEXP = 40.0;   // PARAMA2
constexpr int LM = 6;             // multipole order of poisson1.f:75
constexpr int NMOM = 49;          // (LM+1)^2
constexpr int NANG = 146;         // Lebedev degree-19 mesh used by ANGMSH(LMAX=18)
constexpr int NCOEF = 46;         // potential polynomial coefficients per pair
constexpr int COEF_LD = 52;       // coefficient row stride (zero padded; 52 = 4 mod 16 doubles)
constexpr int MOM_LD = 52;        // normalised-moment row stride (zero padded)
constexpr int TILE = 128;         // mesh points per spatial tile
constexpr int BOYS_NT = 1601;     // Boys table rows (T = 0..16 step 0.01)
constexpr int BOYS_NC = 10;       // columns: F2 F3 F4 F5 F4/2 F5/2 F6/2 F5/6 F6/6 F7/6

// Pair geometry, FO independent (built on the host in the reference's order).
struct PairGeo {
  double a, b;        // exponents alpha, beta
  double A[3], B[3];  // centres
  double C[3];        // (a A + b B) / (a+b) as computed by poisson1.f:320
  double delta;       // a+b
  double factor;      // 2 pi exp(-ARG) / delta
  double times;       // TIMES_SITES*TIMES_ALPHA (coupot_sic.F:257-262)
  int32_t pi, pj;     // global primitive indices of the two bare Gaussians
  int32_t call;       // owning Poisson call
  int32_t pad;
};

// One POISSON1 invocation (a batch, or one weird pair).
struct CallInfo {
  int32_t p0, np;     // pair range in the pair array
  int32_t slots;      // NPAIR of poisson1.f (NSPN slots per pair)
  int32_t pad;
  double delta_min;   // smallest a+b in the call
};

// Per (call, FO) parameters of the near/far split.
struct CallFO {
  double cg[3];       // centre of gravity (poisson1.f:503-520)
  double rcut;        // RCUT
  double rcut2;       // RCUT^2, or +inf when every point is evaluated exactly (NPOT=1)
  int32_t npot;       // 1 or 2
  int32_t nfar;       // number of far points
  uint64_t keep;      // multipole terms kept by the skip rule of poisson1.f:1252-1270
  int32_t lmax;       // highest kept degree
  int32_t pad;
};

// Near/far geometry of one call when it is the same for every FO (bitwise equal
// CG, RCUT^2 and NPOT), as for a single-pair call with NSPN=1 (poisson1.f:503-520
// then gives CG = the pair centre).
struct CallShare {
  double cg[3];
  double rcut2;
  int32_t npot;
  int32_t kf;         // moment columns of the far segment: (lmax over FOs + 1)^2 rounded up to 4; 0 = none
  int32_t shared;     // 1 when the geometry is FO independent
  int32_t ksum;       // multipole terms kept by the skip rule, summed over the FOs
};

#define FLOSIC_HD __host__ __device__ __forceinline__

// Monomial ordering of poisson1.f:925-959 (POLY(1..35)); index tables.
// mono power triples for indices 0..34: degree, then x power ascending, then y.
FLOSIC_HD int mono_index(int px, int py, int pz) {
  int d = px + py + pz;
  int base = (d == 0) ? 0 : (d == 1) ? 1 : (d == 2) ? 4 : (d == 3) ? 10 : 20;
  int off = 0;
  for (int x = 0; x < px; ++x) off += (d - x + 1);
  return base + off + py;
}

}  // namespace flosic
