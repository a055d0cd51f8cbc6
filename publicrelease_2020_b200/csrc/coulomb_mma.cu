// Coulomb potential of all FOs at all mesh points, FP64 tensor-core form.
//
// For one POISSON1 call (a batch of Gaussian pairs, poisson1.f:611-1098) the
// near-field potential of FO k at point p is
//     T[k][p] = sum_{pair q} sum_{t<46} COEF[q][k][t] * G[q][t][p],
//     G[q][t][p] = F_{m(t)}(delta_q |p-C_q|^2) * mono_t(p - C_q),
// where COEF are the pair's potential-polynomial coefficients of FO k and G is
// FO independent (Boys values times monomials).  A CTA owns 128 spatially
// sorted mesh points and 64 FOs; for each call it builds G for two pairs at a
// time in shared memory and contracts it with the coefficient tile on the FP64
// tensor cores (mma.sync m8n8k4 .f64), then merges per (FO, point): near points
// take T, far points (beyond RCUT of that FO's call, NPOT=2) take the L<=6
// multipole expansion (poisson1.f:1224-1600).  Calls are walked in order, so
// per-point sums are deterministic.
#include <cfloat>

#include "device_math.cuh"
#include "kernels.cuh"

namespace flosic {

constexpr int MMA_PTS = TILE;               // 128 points per CTA
constexpr int MMA_FOS = 64;                 // FOs per CTA
constexpr int MMA_THREADS = 256;            // 8 warps: 2 (FO) x 4 (points), 32x32 warp tiles
constexpr int KPP = 48;                     // coefficients per pair, padded to a multiple of 4
constexpr int PAIRS_PER_STEP = 2;
constexpr int KSTEP = KPP * PAIRS_PER_STEP; // 96
constexpr int A_LD = KSTEP + 4;             // 100: conflict-free A fragment loads
constexpr int G_LD = MMA_PTS + 4;           // 132 (= 4 mod 16 doubles): conflict-free B fragment loads

__constant__ double c_vfac[NMOM];           // harmonics.f prefactors sqrt(NRUN (2l+1)/4pi (l-m)!/(l+m)!)
__constant__ int8_t c_slot_m[NCOEF];        // u^2 power of coefficient slot t (Boys index)
__constant__ int8_t c_slot_mono[NCOEF];     // monomial of slot t (POLY order)

void upload_mma_constants() {
  double vfac[NMOM];
  const double onofpi = 1.0 / (16 * atan(1.0));
  for (int l = 0; l <= LM; ++l) {
    double facfc = (2 * l + 1) * onofpi;
    int now = l * l;
    for (int m = 0; m <= l; ++m) {
      const int nrun = (m == 0) ? 1 : 2;
      const double v = sqrt(nrun * facfc);
      for (int r = 0; r < nrun; ++r) vfac[now++] = v;
      facfc = facfc / ((l - m > 1 ? l - m : 1) * (l + m + 1));
    }
  }
  int8_t sm[NCOEF], sn[NCOEF];
  // COEFICIENT order of poisson1.f:402-482
  sm[0] = 0; sn[0] = 0;
  sm[1] = 1; sn[1] = 0;
  sm[2] = 2; sn[2] = 0;
  for (int i = 0; i < 3; ++i) { sm[3 + i] = 1; sn[3 + i] = (int8_t)(1 + i); }
  for (int i = 0; i < 3; ++i) { sm[6 + i] = 2; sn[6 + i] = (int8_t)(1 + i); }
  for (int i = 0; i < 6; ++i) { sm[9 + i] = 2; sn[9 + i] = (int8_t)(4 + i); }
  for (int i = 0; i < 6; ++i) { sm[15 + i] = 3; sn[15 + i] = (int8_t)(4 + i); }
  for (int i = 0; i < 10; ++i) { sm[21 + i] = 3; sn[21 + i] = (int8_t)(10 + i); }
  for (int i = 0; i < 15; ++i) { sm[31 + i] = 4; sn[31 + i] = (int8_t)(20 + i); }
  cudaMemcpyToSymbol(c_vfac, vfac, sizeof(vfac));
  cudaMemcpyToSymbol(c_slot_m, sm, sizeof(sm));
  cudaMemcpyToSymbol(c_slot_mono, sn, sizeof(sn));
}

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ double sqdist_rn2(double x, double y, double z, double cx, double cy, double cz) {
  const double dx = __dadd_rn(x, -cx), dy = __dadd_rn(y, -cy), dz = __dadd_rn(z, -cz);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// L<=6 multipole potential at unit direction (ux,uy,uz), 1/r = hn, with the
// unnormalised recursion of harmonics.f evaluated level by level.
__device__ __forceinline__ double multipole(const double* __restrict__ mo, int lmx, unsigned long long keep,
                                            double ux, double uy, double uz, double hn) {
  double p2[13], p1[13], cu[13];
  double pot = 0.0, rec = hn;
  // l = 0
  if (keep & 1ull) pot += mo[0] * (c_vfac[0] * 1.0) * rec;
  if (lmx == 0) return pot;
  rec *= hn;
  p2[0] = 1.0;
  p1[0] = uz;
  p1[1] = ux;
  p1[2] = uy;
  for (int j = 0; j < 3; ++j)
    if (keep & (1ull << (1 + j))) pot += mo[1 + j] * (c_vfac[1 + j] * p1[j]) * rec;
#pragma unroll
  for (int l = 2; l <= LM; ++l) {
    if (l > lmx) break;
    rec *= hn;
    const int n = 2 * l + 1;
    const double ifc = (double)(2 * l - 1);
#pragma unroll
    for (int j = 0; j < 2 * l - 1; ++j) {
      const int m = (j + 1) / 2;
      const double facrc = 1.0 / (l - m);
      const double aa = facrc * (2 * l - 1);
      const double bb = (m == l - 1) ? 0.0 : facrc * (l + m - 1);
      const double prev2 = (j < 2 * l - 3) ? p2[j] : 0.0;
      cu[j] = aa * p1[j] * uz - bb * prev2;
    }
    cu[2 * l - 1] = ifc * (p1[2 * l - 3] * ux - p1[2 * l - 2] * uy);
    cu[2 * l] = ifc * (p1[2 * l - 2] * ux + p1[2 * l - 3] * uy);
    const int base = l * l;
#pragma unroll
    for (int j = 0; j < n; ++j)
      if (keep & (1ull << (base + j))) pot += mo[base + j] * (c_vfac[base + j] * cu[j]) * rec;
#pragma unroll
    for (int j = 0; j < 13; ++j) {
      p2[j] = p1[j];
      p1[j] = (j < n) ? cu[j] : 0.0;
    }
  }
  return pot;
}

// G column of one (pair, point) in the COEFICIENT slot order (poisson1.f:402-482):
// slot t holds F_{m(t)} * POLY(mono(t)); monomials are formed in the order of
// poisson1.f:925-959 and stored as soon as they are complete.
__device__ __forceinline__ void write_g(double* g, double x, double y, double z, double F0, double F1, double F2,
                                        double F3, double F4) {
#define GW(t, v) g[(size_t)(t) * G_LD] = (v)
  GW(0, F0);
  GW(1, F1);
  GW(2, F2);
  GW(3, F1 * z);
  GW(4, F1 * y);
  GW(5, F1 * x);
  GW(6, F2 * z);
  GW(7, F2 * y);
  GW(8, F2 * x);
  const double zz = z * z, yz = y * z, yy = y * y, xz = x * z, xy = x * y, xx = x * x;
  GW(9, F2 * zz);
  GW(10, F2 * yz);
  GW(11, F2 * yy);
  GW(12, F2 * xz);
  GW(13, F2 * xy);
  GW(14, F2 * xx);
  GW(15, F3 * zz);
  GW(16, F3 * yz);
  GW(17, F3 * yy);
  GW(18, F3 * xz);
  GW(19, F3 * xy);
  GW(20, F3 * xx);
  GW(21, F3 * (z * zz));
  GW(22, F3 * (y * zz));
  GW(23, F3 * (z * yy));
  GW(24, F3 * (y * yy));
  GW(25, F3 * (x * zz));
  GW(26, F3 * (x * yz));
  GW(27, F3 * (x * yy));
  GW(28, F3 * (z * xx));
  GW(29, F3 * (y * xx));
  GW(30, F3 * (x * xx));
  GW(31, F4 * (zz * zz));
  GW(32, F4 * (zz * yz));
  GW(33, F4 * (yy * zz));
  GW(34, F4 * (yy * yz));
  GW(35, F4 * (yy * yy));
  GW(36, F4 * (zz * xz));
  GW(37, F4 * (xy * zz));
  GW(38, F4 * (xy * yz));
  GW(39, F4 * (yy * xy));
  GW(40, F4 * (xx * zz));
  GW(41, F4 * (xx * yz));
  GW(42, F4 * (xx * yy));
  GW(43, F4 * (xz * xx));
  GW(44, F4 * (xy * xx));
  GW(45, F4 * (xx * xx));
  GW(46, 0.0);
  GW(47, 0.0);
#undef GW
}

struct MmaSmem {
  double A[MMA_FOS * A_LD];
  double G[KSTEP * G_LD];
  double px[MMA_PTS], py[MMA_PTS], pz[MMA_PTS];
  double cg[MMA_FOS][3];
  double rc2[MMA_FOS];
  unsigned long long keep[MMA_FOS];
  int stat[MMA_FOS];
  int npot[MMA_FOS];
  int lmax[MMA_FOS];
  int anynear, anyfar;
};

__global__ void __launch_bounds__(MMA_THREADS, 1)
k_coulomb_mma(int ncalls, const CallInfo* __restrict__ calls, const PairGeo* __restrict__ pairs, int nfo,
              const double* __restrict__ coef, const int8_t* __restrict__ pair_fmt,
              const CallFO* __restrict__ cfo, const double* __restrict__ mom, MeshDev M,
              const double* __restrict__ boys_tab, double* __restrict__ vh, int ldv) {
  extern __shared__ __align__(16) unsigned char smraw[];
  MmaSmem& S = *reinterpret_cast<MmaSmem*>(smraw);
  const int tile = blockIdx.x;
  const int k0 = blockIdx.y * MMA_FOS;
  const int nk = min(MMA_FOS, nfo - k0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int p0 = tile * MMA_PTS;
  const int np = min(MMA_PTS, M.n - p0);
  for (int i = tid; i < MMA_PTS; i += MMA_THREADS) {
    const bool a = i < np;
    S.px[i] = a ? M.x[p0 + i] : 0.0;
    S.py[i] = a ? M.y[p0 + i] : 0.0;
    S.pz[i] = a ? M.z[p0 + i] : 0.0;
  }
  const double lo[3] = {M.tile_lo[3 * tile], M.tile_lo[3 * tile + 1], M.tile_lo[3 * tile + 2]};
  const double hi[3] = {M.tile_hi[3 * tile], M.tile_hi[3 * tile + 1], M.tile_hi[3 * tile + 2]};
  // accumulator ownership: FO k = wm*32 + mt*8 + (lane>>2), point p = wn*32 + nt*8 + 2*(lane&3) + i
  double V[4][4][2], T[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) V[a][b][0] = V[a][b][1] = 0.0;

  for (int c = 0; c < ncalls; ++c) {
    __syncthreads();
    if (tid == 0) {
      S.anynear = 0;
      S.anyfar = 0;
    }
    __syncthreads();
    if (tid < MMA_FOS) {
      int st = 1, npot = 2, lmx = 0;
      unsigned long long keep = 0ull;
      double cgx = 0, cgy = 0, cgz = 0, rc2 = 0;
      if (tid < nk) {
        const CallFO f = cfo[(size_t)c * nfo + k0 + tid];
        cgx = f.cg[0];
        cgy = f.cg[1];
        cgz = f.cg[2];
        rc2 = f.rcut2;
        npot = f.npot;
        double dmin2 = 0.0, dmax2 = 0.0;
        const double cgv[3] = {cgx, cgy, cgz};
        for (int d = 0; d < 3; ++d) {
          const double a = lo[d] - cgv[d], b = cgv[d] - hi[d];
          const double m = fmax(fmax(a, b), 0.0);
          dmin2 += m * m;
          const double e = fmax(fabs(cgv[d] - lo[d]), fabs(hi[d] - cgv[d]));
          dmax2 += e * e;
        }
        if (npot == 1) st = 0;
        else if (dmin2 > rc2 * (1.0 + 1e-9)) st = 1;
        else if (dmax2 < rc2 * (1.0 - 1e-9)) st = 0;
        else st = 2;
        if (st != 1) atomicOr(&S.anynear, 1);
        if (st != 0) {
          atomicOr(&S.anyfar, 1);
          // skip rule of poisson1.f:1252-1270; RI1 bounded by the tile box and RCUT
          const double* mo = mom + ((size_t)c * nfo + k0 + tid) * NMOM;
          const double ri1 = 1.0 / fmax(sqrt(dmin2), f.rcut);
          double rt = ri1;
          int m = 0;
          for (int l = 0; l <= LM; ++l) {
            for (int j = -l; j <= l; ++j, ++m) {
              const double tst = fabs((2 * l + 1) * mo[m] * rt);
              if (!(tst < 1.0e-12)) {
                keep |= (1ull << m);
                lmx = l;
              }
            }
            rt *= ri1;
          }
        }
      }
      S.stat[tid] = st;
      S.npot[tid] = npot;
      S.cg[tid][0] = cgx;
      S.cg[tid][1] = cgy;
      S.cg[tid][2] = cgz;
      S.rc2[tid] = rc2;
      S.keep[tid] = keep;
      S.lmax[tid] = lmx;
    }
    __syncthreads();
    const CallInfo ci = calls[c];
    if (S.anynear) {
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) T[a][b][0] = T[a][b][1] = 0.0;
      for (int q0 = 0; q0 < ci.np; q0 += PAIRS_PER_STEP) {
        const int npc = min(PAIRS_PER_STEP, ci.np - q0);
        __syncthreads();
        // G for (pair ql, point p): Boys values times monomials
        {
          const int ql = tid >> 7, p = tid & 127;
          double* g = &S.G[(size_t)ql * KPP * G_LD + p];
          if (ql < npc && p < np) {
            const int q = ci.p0 + q0 + ql;
            const PairGeo& pg = pairs[q];
            const double rx = S.px[p] - pg.C[0], ry = S.py[p] - pg.C[1], rz = S.pz[p] - pg.C[2];
            const double xx = pg.delta * (rz * rz + ry * ry + rx * rx);
            const double chgd = exp(-xx);
            double s3[3], s4[4], s5[5];
            boys_all(boys_tab, xx, chgd, s3, s4, s5);
            const int fmt = pair_fmt[q];
            double F0, F1, F2, F3, F4;
            if (fmt == 5) {
              F0 = s5[0]; F1 = s5[1]; F2 = s5[2]; F3 = s5[3]; F4 = s5[4];
            } else if (fmt == 4) {
              F0 = s4[0]; F1 = s4[1]; F2 = s4[2]; F3 = s4[3]; F4 = 0.0;
            } else {
              F0 = s3[0]; F1 = s3[1]; F2 = s3[2]; F3 = 0.0; F4 = 0.0;
            }
            write_g(g, rx, ry, rz, F0, F1, F2, F3, F4);
          } else {
#pragma unroll
            for (int t = 0; t < KPP; ++t) g[(size_t)t * G_LD] = 0.0;
          }
        }
        // coefficient tile A[k][ql*48 + t]
        for (int e = tid; e < MMA_FOS * KSTEP; e += MMA_THREADS) {
          const int k = e / KSTEP, col = e - k * KSTEP;
          const int ql = col / KPP, t = col - ql * KPP;
          double v = 0.0;
          if (k < nk && ql < npc && t < NCOEF) v = coef[((size_t)(ci.p0 + q0 + ql) * nfo + k0 + k) * NCOEF + t];
          S.A[k * A_LD + col] = v;
        }
        __syncthreads();
        const int kend = npc * KPP;
        const double* Aw = &S.A[(wm * 32 + (lane >> 2)) * A_LD + (lane & 3)];
        const double* Gw = &S.G[(size_t)(lane & 3) * G_LD + wn * 32 + (lane >> 2)];
        for (int kk = 0; kk < kend; kk += 4) {
          double af[4], bf[4];
#pragma unroll
          for (int mt = 0; mt < 4; ++mt) af[mt] = Aw[mt * 8 * A_LD + kk];
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) bf[nt] = Gw[(size_t)kk * G_LD + nt * 8];
#pragma unroll
          for (int mt = 0; mt < 4; ++mt)
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) dmma884(T[mt][nt][0], T[mt][nt][1], af[mt], bf[nt]);
        }
      }
      // near merge
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int k = wm * 32 + mt * 8 + (lane >> 2);
        const int st = S.stat[k];
        if (k >= nk || st == 1) continue;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int p = wn * 32 + nt * 8 + 2 * (lane & 3) + i;
            bool nr = (st == 0);
            if (st == 2)
              nr = !(sqdist_rn2(S.px[p], S.py[p], S.pz[p], S.cg[k][0], S.cg[k][1], S.cg[k][2]) > S.rc2[k]);
            if (nr) V[mt][nt][i] += T[mt][nt][i];
          }
      }
    }
    if (S.anyfar) {
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int k = wm * 32 + mt * 8 + (lane >> 2);
        if (k >= nk) continue;
        const int st = S.stat[k];
        if (st == 0 || S.npot[k] == 1) continue;
        const double cx = S.cg[k][0], cy = S.cg[k][1], cz = S.cg[k][2], rc2 = S.rc2[k];
        const int lmx = S.lmax[k];
        const unsigned long long keep = S.keep[k];
        const double* mo = mom + ((size_t)c * nfo + k0 + k) * NMOM;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int p = wn * 32 + nt * 8 + 2 * (lane & 3) + i;
            if (p >= np) continue;
            const double r2 = sqdist_rn2(S.px[p], S.py[p], S.pz[p], cx, cy, cz);
            if (!(r2 > rc2)) continue;
            const double hn = 1.0 / sqrt(r2);
            V[mt][nt][i] += multipole(mo, lmx, keep, hn * (S.px[p] - cx), hn * (S.py[p] - cy), hn * (S.pz[p] - cz),
                                      hn);
          }
      }
    }
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const int k = wm * 32 + mt * 8 + (lane >> 2);
    if (k >= nk) continue;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int p = wn * 32 + nt * 8 + 2 * (lane & 3) + i;
        if (p < np) vh[(size_t)(k0 + k) * ldv + p0 + p] = V[mt][nt][i];
      }
  }
}

// Largest Boys variant over the FOs of each pair (the G tile is shared by all FOs).
__global__ void k_pair_fmt(int npairs, int nfo, const int8_t* __restrict__ maxfmt, int8_t* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npairs) return;
  int m = 3;
  for (int k = 0; k < nfo; ++k) m = max(m, (int)maxfmt[(size_t)q * nfo + k]);
  out[q] = (int8_t)m;
}

// Per-device set-up: constant tables and the dynamic shared-memory opt-in.
void init_coulomb_mma() {
  upload_mma_constants();
  cudaFuncSetAttribute(k_coulomb_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MmaSmem));
}

void launch_coulomb_mma(int ncalls, const CallInfo* calls, const PairGeo* pairs, int npairs, int nfo,
                        const double* coef, const int8_t* maxfmt, int8_t* pair_fmt, const CallFO* cfo,
                        const double* mom, const MeshDev& M, const double* boys_tab, double* vh, int ldv,
                        cudaStream_t st) {
  const size_t smem = sizeof(MmaSmem);
  if (npairs > 0) k_pair_fmt<<<(npairs + 127) / 128, 128, 0, st>>>(npairs, nfo, maxfmt, pair_fmt);
  dim3 grid(M.ntiles, (nfo + MMA_FOS - 1) / MMA_FOS);
  k_coulomb_mma<<<grid, MMA_THREADS, smem, st>>>(ncalls, calls, pairs, nfo, coef, pair_fmt, cfo, mom, M, boys_tab,
                                                  vh, ldv);
}

}  // namespace flosic
