// CUDA kernels of the FLO-SIC per-FO hot path (sm_100a, FP64).
//
//   k_basis_values   contracted Cartesian Gaussians and derivatives (gorbdrv.f)
//   k_prim_u         FO coefficients projected on bare primitives (the rank-1
//                    factor of the pair density matrix of coupot_sic.F:366-482)
//   k_pair_coef      Gaussian-pair Coulomb polynomial coefficients (polyx.F,
//                    poisson1.f:259-501) and centre-of-gravity moments (ginted.F)
//   k_call_setup     per POISSON1 call and FO: CG, RCUT, NPOT, sphere potential
//                    and L<=6 multipole moments (poisson1.f:503-1230)
//   k_xc             XC potential of the FO density, SIC potential, energy
//                    partial sums (getvlxc.F, subvlxc_libxc.F90, apotnl_sic.F)
#include <cfloat>
#include <cstdio>

#include "device_math.cuh"
#include "kernels.cuh"
#include "xc_functionals.cuh"
#include "xc_scan.cuh"

namespace flosic {

void upload_constants(const double* leb_ang, const double* leb_w) {
  cudaMemcpyToSymbol(c_leb_ang, leb_ang, sizeof(double) * NANG * 3);
  cudaMemcpyToSymbol(c_leb_w, leb_w, sizeof(double) * NANG);
}

__constant__ int c_pow[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                                 {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};

// ---------------------------------------------------------------------------
// Basis values
// ---------------------------------------------------------------------------
template <int NDERV>
__global__ void __launch_bounds__(128) k_basis_values(BasisDev B, int npts, const double* __restrict__ px,
                                                      const double* __restrict__ py,
                                                      const double* __restrict__ pz, double* __restrict__ out,
                                                      int ldo) {
  constexpr int NCH = NDERV == 0 ? 1 : (NDERV == 1 ? 4 : 10);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const double X = px[i], Y = py[i], Z = pz[i];
  const size_t chs = (size_t)B.nbasis * ldo;
  for (int a = 0; a < B.natoms; ++a) {
    const int t = B.atom_type[a];
    const double x = X - B.atom_pos[3 * a], y = Y - B.atom_pos[3 * a + 1], z = Z - B.atom_pos[3 * a + 2];
    const double r2 = x * x + y * y + z * z;
    const int b0 = B.atom_boff[a];
    const int lmax = B.type_lmax[t];
    const int nbare = B.type_nbare[t];
    const bool any = r2 * B.type_amin[t] < CUTEXP;
    double g[MAX_BARE];
#pragma unroll
    for (int ib = 0; ib < MAX_BARE; ++ib) {
      double v = 0.0;
      if (any && ib < nbare) {
        const double rex = B.type_alpha[t * MAX_BARE + ib] * r2;
        v = (rex < CUTEXP) ? exp(-rex) : 0.0;
      }
      g[ib] = v;
    }
    const double xyz[3] = {x, y, z};
    int base = 0;
    for (int l = 0; l <= lmax; ++l) {
      const int ncon = B.type_ncon[t * 3 + l];
      const int ncomp = (l == 0) ? 1 : (l == 1 ? 3 : 6);
      const int shift = (l == 0) ? 0 : (l == 1 ? 1 : 4);
      for (int c = 0; c < ncon; ++c) {
        double R0 = 0.0, R1 = 0.0, R2 = 0.0;
        if (any) {
          const double* con = B.type_bfcon + ((size_t)(t * 3 + l) * MAX_CON + c) * MAX_BARE;
#pragma unroll
          for (int ib = 0; ib < MAX_BARE; ++ib) {
            if (ib < nbare) {
              const double cg = con[ib] * g[ib];
              R0 += cg;
              if (NDERV > 0) {
                const double a2 = 2.0 * B.type_alpha[t * MAX_BARE + ib];
                R1 += cg * a2;
                if (NDERV > 1) R2 += cg * a2 * a2;
              }
            }
          }
        }
        for (int mu = 0; mu < ncomp; ++mu) {
          const int* pw = c_pow[shift + mu];
          const size_t o = (size_t)(b0 + base + mu * ncon + c) * ldo + i;
          // angular polynomial and its derivatives
          double P = 1.0;
          for (int d = 0; d < 3; ++d)
            for (int k = 0; k < pw[d]; ++k) P *= xyz[d];
          out[o] = P * R0;
          if (NDERV == 0) continue;
          double dP[3];
          for (int d = 0; d < 3; ++d) {
            if (pw[d] == 0) {
              dP[d] = 0.0;
              continue;
            }
            double v = (double)pw[d];
            for (int e = 0; e < 3; ++e) {
              int p = pw[e] - (e == d ? 1 : 0);
              for (int k = 0; k < p; ++k) v *= xyz[e];
            }
            dP[d] = v;
          }
          for (int d = 0; d < 3; ++d) out[o + (size_t)(1 + d) * chs] = dP[d] * R0 - P * xyz[d] * R1;
          if (NDERV == 1) continue;
          // second derivatives: xx yy zz xy xz yz
          const int dd[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
          for (int q = 0; q < 6; ++q) {
            const int d = dd[q][0], e = dd[q][1];
            double d2 = 0.0;
            {
              int p[3] = {pw[0], pw[1], pw[2]};
              double f = p[d];
              p[d] -= 1;
              if (f > 0) {
                f *= p[e];
                p[e] -= 1;
                if (f > 0) {
                  double v = f;
                  for (int m = 0; m < 3; ++m)
                    for (int k = 0; k < p[m]; ++k) v *= xyz[m];
                  d2 = v;
                }
              }
            }
            double v;
            if (d == e)
              v = d2 * R0 - 2.0 * dP[d] * xyz[d] * R1 + P * (xyz[d] * xyz[d] * R2 - R1);
            else
              v = d2 * R0 - dP[e] * xyz[d] * R1 - dP[d] * xyz[e] * R1 + P * xyz[d] * xyz[e] * R2;
            out[o + (size_t)(4 + q) * chs] = v;
          }
        }
      }
      base += ncomp * ncon;
    }
  }
}

void launch_basis_values(const BasisDev& B, int nderv, int npts, const double* px, const double* py,
                         const double* pz, double* out, int ldo, cudaStream_t st) {
  if (npts <= 0) return;
  dim3 grid((npts + 127) / 128);
  if (nderv == 0) k_basis_values<0><<<grid, 128, 0, st>>>(B, npts, px, py, pz, out, ldo);
  else if (nderv == 1) k_basis_values<1><<<grid, 128, 0, st>>>(B, npts, px, py, pz, out, ldo);
  else k_basis_values<2><<<grid, 128, 0, st>>>(B, npts, px, py, pz, out, ldo);
}

// ---------------------------------------------------------------------------
// Primitive projections u
// ---------------------------------------------------------------------------
__global__ void k_prim_u(BasisDev B, int nfo, const double* __restrict__ cfo, int ldc, double* __restrict__ u) {
  const int gp = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (gp >= B.nprim) return;
  const int a = B.prim_atom[gp], ib = B.prim_ib[gp];
  const int t = B.atom_type[a];
  const double* c = cfo + (size_t)k * ldc + B.atom_boff[a];
  double uu[10];
#pragma unroll
  for (int m = 0; m < 10; ++m) uu[m] = 0.0;
  int base = 0;
  for (int l = 0; l <= B.type_lmax[t]; ++l) {
    const int ncon = B.type_ncon[t * 3 + l];
    const int ncomp = (l == 0) ? 1 : (l == 1 ? 3 : 6);
    const int shift = (l == 0) ? 0 : (l == 1 ? 1 : 4);
    for (int mu = 0; mu < ncomp; ++mu) {
      double s = 0.0;
      for (int cc = 0; cc < ncon; ++cc)
        s += B.type_bfcon[((size_t)(t * 3 + l) * MAX_CON + cc) * MAX_BARE + ib] * c[base + mu * ncon + cc];
      uu[shift + mu] = s;
    }
    base += ncomp * ncon;
  }
  double* o = u + ((size_t)k * B.nprim + gp) * 10;
#pragma unroll
  for (int m = 0; m < 10; ++m) o[m] = uu[m];
}

void launch_prim_u(const BasisDev& B, int nfo, const double* cfo, int ldc, double* u, cudaStream_t st) {
  dim3 grid((B.nprim + 127) / 128, nfo);
  k_prim_u<<<grid, 128, 0, st>>>(B, nfo, cfo, ldc, u);
}

// ---------------------------------------------------------------------------
// Pair coefficients
// ---------------------------------------------------------------------------
// slot of (u-power M, monomial) in the COEFICIENT order (poisson1.f:402-482)
__device__ __forceinline__ int coef_slot(int M, int ex, int ey, int ez) {
  int d = ex + ey + ez;
  int mi = mono_index(ex, ey, ez);
  switch (M) {
    case 0: return d == 0 ? 0 : -1;
    case 1: return d == 0 ? 1 : (d == 1 ? 3 + (mi - 1) : -1);
    case 2: return d == 0 ? 2 : (d == 1 ? 6 + (mi - 1) : (d == 2 ? 9 + (mi - 4) : -1));
    case 3: return d == 2 ? 15 + (mi - 4) : (d == 3 ? 21 + (mi - 10) : -1);
    case 4: return d == 4 ? 31 + (mi - 20) : -1;
  }
  return -1;
}

struct Poly1DNZ {
  int8_t cnt[3][3][3];         // [d][n][m]
  int8_t e[3][3][3][16];
  int8_t s[3][3][3][16];
  double v[3][3][3][16];
};

// 1-D factor E[(Y + rho s - a0)^n (Y + rho s - b0)^m], Y ~ N(0,(1-s)/(2 delta)),
// as nonzero (rho power, s power, value) triples in (rho, s) lexicographic order.
__device__ void poly1d_entry(double a0, double b0, double delta, int n, int m, int8_t& cnt, int8_t* eo,
                             int8_t* so, double* vo) {
  double c[5][5];
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) c[i][j] = 0.0;
  const double tdi = 0.5 / delta;
  const double binom[3][3] = {{1, 0, 0}, {1, 1, 0}, {1, 2, 1}};
  const double dfact[5] = {1, 0, 1, 0, 3};
  for (int k = 0; k <= n; ++k)
    for (int l = 0; l <= m; ++l) {
      int j = k + l;
      if (j & 1) continue;
      double pre = binom[n][k] * binom[m][l] * dfact[j];
      int na = n - k, nb = m - l;
      double pa[3] = {0, 0, 0}, pb[3] = {0, 0, 0};
      if (na == 0) pa[0] = 1;
      else if (na == 1) { pa[0] = -a0; pa[1] = 1; }
      else { pa[0] = a0 * a0; pa[1] = -2 * a0; pa[2] = 1; }
      if (nb == 0) pb[0] = 1;
      else if (nb == 1) { pb[0] = -b0; pb[1] = 1; }
      else { pb[0] = b0 * b0; pb[1] = -2 * b0; pb[2] = 1; }
      double ph[5] = {0, 0, 0, 0, 0};
      for (int x = 0; x <= na; ++x)
        for (int y = 0; y <= nb; ++y) ph[x + y] += pa[x] * pb[y];
      int hj = j / 2;
      double sig[3] = {0, 0, 0};
      if (hj == 0) sig[0] = 1;
      else if (hj == 1) { sig[0] = tdi; sig[1] = -tdi; }
      else { sig[0] = tdi * tdi; sig[1] = -2 * tdi * tdi; sig[2] = tdi * tdi; }
      for (int e = 0; e <= na + nb; ++e) {
        if (ph[e] == 0.0) continue;
        for (int q = 0; q <= hj; ++q) {
          if (sig[q] == 0.0) continue;
          c[e][e + q] += pre * ph[e] * sig[q];
        }
      }
    }
  int k = 0;
  for (int e = 0; e < 5; ++e)
    for (int s = 0; s < 5; ++s)
      if (c[e][s] != 0.0 && k < 16) {
        eo[k] = (int8_t)e;
        so[k] = (int8_t)s;
        vo[k] = c[e][s];
        ++k;
      }
  cnt = (int8_t)k;
}

__global__ void __launch_bounds__(128) k_pair_coef(const PairGeo* __restrict__ pairs,
                                                   const CallInfo* __restrict__ calls, int nfo, int nprim,
                                                   const double* __restrict__ u, const double* __restrict__ dm,
                                                   int nspn, double* __restrict__ coef,
                                                   int8_t* __restrict__ maxfmt, double* __restrict__ cgp) {
  __shared__ Poly1DNZ P;
  __shared__ double W[4][10][10];
  __shared__ double V[3][3][3][2];
  const int ip = blockIdx.x;
  const PairGeo g = pairs[ip];
  const int slots = calls[g.call].slots;
  const double a0[3] = {g.A[0] - g.C[0], g.A[1] - g.C[1], g.A[2] - g.C[2]};
  const double b0[3] = {g.B[0] - g.C[0], g.B[1] - g.C[1], g.B[2] - g.C[2]};
  const int tid = threadIdx.x;
  if (tid < 27) {
    const int d = tid / 9, n = (tid / 3) % 3, m = tid % 3;
    poly1d_entry(a0[d], b0[d], g.delta, n, m, P.cnt[d][n][m], P.e[d][n][m], P.s[d][n][m], P.v[d][n][m]);
  }
  // ginted.F moments: V[d][n][m][k] = E[(x-A)^n (x-B)^m x^k], x ~ N(Cg, 1/(2(a+b)))
  const double at = 1.0 / (g.a + g.b);
  if (tid >= 32 && tid < 32 + 54) {
    const int q = tid - 32;
    const int d = q / 18, n = (q / 6) % 3, m = (q / 2) % 3, kk = q % 2;
    const double q1 = 0.5 * at;
    const double D = (g.a * g.A[d] + g.b * g.B[d]) * at;
    const double f1 = D - g.A[d], f2 = D - g.B[d], f3 = D;
    const double mom[5] = {1.0, 0.0, q1, 0.0, 3 * q1 * q1};
    double c[6] = {0, 0, 0, 0, 0, 0};
    double pa[3] = {1, 0, 0};
    if (n == 1) { pa[0] = f1; pa[1] = 1; } else if (n == 2) { pa[0] = f1 * f1; pa[1] = 2 * f1; pa[2] = 1; }
    double pb[3] = {1, 0, 0};
    if (m == 1) { pb[0] = f2; pb[1] = 1; } else if (m == 2) { pb[0] = f2 * f2; pb[1] = 2 * f2; pb[2] = 1; }
    double pc[2] = {1, 0};
    if (kk == 1) { pc[0] = f3; pc[1] = 1; }
    for (int x = 0; x <= n; ++x)
      for (int y = 0; y <= m; ++y)
        for (int z = 0; z <= kk; ++z) c[x + y + z] += pa[x] * pb[y] * pc[z];
    double s = 0.0;
    for (int e = 0; e <= 4; ++e) s += c[e] * mom[e];
    V[d][n][m][kk] = s;
  }
  __syncthreads();
  if (slots != 1) {
    double xs = 0.0;
    for (int d = 0; d < 3; ++d) xs = xs + (g.a * g.b * ((g.A[d] - g.B[d]) * (g.A[d] - g.B[d]))) * at;
    const double sq = sqrt(3.14159265358979324 * at);
    const double Dn = exp(-xs) * (sq * sq * sq);
    for (int q = tid; q < 400; q += blockDim.x) {
      const int kq = q / 100, i = (q / 10) % 10, j = q % 10;
      double w = 1.0;
      for (int d = 0; d < 3; ++d) w *= V[d][c_pow[i][d]][c_pow[j][d]][kq == d ? 1 : 0];
      W[kq][i][j] = w * Dn;
    }
  }
  __syncthreads();
  // dm != nullptr: one density, the pair's block of a general density matrix
  // (COUPOT1's ADD, coupot1.F:380-395); otherwise the rank-1 block u_i u_j^T of FO k
  for (int k = tid; k < nfo; k += blockDim.x) {
    double ui[10], vj[10];
    const double* dmb = dm ? dm + (size_t)ip * 100 : nullptr;
    if (dmb) {
#pragma unroll
      for (int m = 0; m < 10; ++m) ui[m] = vj[m] = 1.0;
    } else {
      const double* pu = u + ((size_t)k * nprim + g.pi) * 10;
      const double* pv = u + ((size_t)k * nprim + g.pj) * 10;
#pragma unroll
      for (int m = 0; m < 10; ++m) {
        ui[m] = pu[m];
        vj[m] = pv[m];
      }
    }
    double cf[NCOEF];
#pragma unroll
    for (int s = 0; s < NCOEF; ++s) cf[s] = 0.0;
    double cg4[4] = {0, 0, 0, 0};
    for (int mu = 0; mu < 10; ++mu) {
      if (ui[mu] == 0.0) continue;
      const int nx = c_pow[mu][0], ny = c_pow[mu][1], nz = c_pow[mu][2];
      for (int nu = 0; nu < 10; ++nu) {
        double d = (dmb ? dmb[mu * 10 + nu] : ui[mu] * vj[nu]) * g.times;
        const double r = (nspn == 1) ? d + d : d;
        if (r == 0.0) continue;
        if (slots != 1)
          for (int kq = 0; kq < 4; ++kq) cg4[kq] += W[kq][mu][nu] * r;
        const int mx = c_pow[nu][0], my = c_pow[nu][1], mz = c_pow[nu][2];
        const int cx = P.cnt[0][nx][mx], cy = P.cnt[1][ny][my], cz = P.cnt[2][nz][mz];
        for (int ix = 0; ix < cx; ++ix) {
          const int ex = P.e[0][nx][mx][ix], sx = P.s[0][nx][mx][ix];
          const double vx = P.v[0][nx][mx][ix];
          for (int iy = 0; iy < cy; ++iy) {
            const int ey = P.e[1][ny][my][iy], sy = P.s[1][ny][my][iy];
            const double pxy = r * vx * P.v[1][ny][my][iy];
            for (int iz = 0; iz < cz; ++iz) {
              const int ez = P.e[2][nz][mz][iz], sz = P.s[2][nz][mz][iz];
              const int M = sx + sy + sz;
              if (M > 4 || ex + ey + ez > 4) continue;
              const int slot = coef_slot(M, ex, ey, ez);
              if (slot >= 0) cf[slot] += pxy * P.v[2][nz][mz][iz];
            }
          }
        }
      }
    }
    bool s3 = false, s4 = false, s5 = false;
#pragma unroll
    for (int s = 0; s < NCOEF; ++s) {
      cf[s] = g.factor * cf[s];
      if (s >= 6 && s <= 14 && cf[s] != 0.0) s3 = true;
      if (s >= 15 && s <= 30 && cf[s] != 0.0) s4 = true;
      if (s >= 31 && cf[s] != 0.0) s5 = true;
    }
    if (!s3) cf[2] = 0.0;
    double* o = coef + ((size_t)ip * nfo + k) * COEF_LD;
#pragma unroll
    for (int s = 0; s < NCOEF; ++s) o[s] = cf[s];
#pragma unroll
    for (int s = NCOEF; s < COEF_LD; ++s) o[s] = 0.0;
    maxfmt[(size_t)ip * nfo + k] = (int8_t)(s5 ? 5 : (s4 ? 4 : 3));
    double* oc = cgp + ((size_t)ip * nfo + k) * 4;
    for (int kq = 0; kq < 4; ++kq) oc[kq] = cg4[kq];
  }
}

void launch_pair_coef(int npairs, const PairGeo* pairs, const CallInfo* calls, int nfo, int nprim,
                      const double* u, const double* dm, int nspn, double* coef, int8_t* maxfmt, double* cgp,
                      cudaStream_t st) {
  if (npairs <= 0) return;
  k_pair_coef<<<npairs, 128, 0, st>>>(pairs, calls, nfo, nprim, u, dm, nspn, coef, maxfmt, cgp);
}

// Pair blocks of the density matrix of norb orbitals (both spins):
// dm[(ip*10 + mu)*10 + nu] = sum_i u_i(pi)[mu] u_i(pj)[nu] (coupot1.F:380-395
// summed with the contraction of coupot1.F:405-430 folded into u).
__global__ void __launch_bounds__(128) k_pair_dm(const PairGeo* __restrict__ pairs, int norb, int nprim,
                                                 const double* __restrict__ u, double* __restrict__ dm) {
  const int ip = blockIdx.x;
  const int t = threadIdx.x;
  if (t >= 100) return;
  const PairGeo g = pairs[ip];
  const int mu = t / 10, nu = t % 10;
  double acc = 0.0;
  for (int i = 0; i < norb; ++i)
    acc += u[((size_t)i * nprim + g.pi) * 10 + mu] * u[((size_t)i * nprim + g.pj) * 10 + nu];
  dm[(size_t)ip * 100 + t] = acc;
}

void launch_pair_dm(int npairs, const PairGeo* pairs, int norb, int nprim, const double* u, double* dm,
                    cudaStream_t st) {
  if (npairs <= 0) return;
  k_pair_dm<<<npairs, 128, 0, st>>>(pairs, norb, nprim, u, dm);
}

// ---------------------------------------------------------------------------
// Per (call, FO) setup
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sqdist_rn(double x, double y, double z, const double c[3]) {
  // (x - cx)^2 + (y - cy)^2 + (z - cz)^2 without FMA contraction (poisson1.f:540-544)
  const double dx = __dadd_rn(x, -c[0]), dy = __dadd_rn(y, -c[1]), dz = __dadd_rn(z, -c[2]);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ __forceinline__ void box_dist2(const double lo[3], const double hi[3], const double c[3],
                                          double& dmin2, double& dmax2) {
  dmin2 = 0.0;
  dmax2 = 0.0;
  for (int d = 0; d < 3; ++d) {
    double a = lo[d] - c[d], b = c[d] - hi[d];
    double m = fmax(fmax(a, b), 0.0);
    dmin2 += m * m;
    double f = fmax(fabs(c[d] - lo[d]), fabs(hi[d] - c[d]));
    dmax2 += f * f;
  }
}

constexpr int SETUP_THREADS = 160;
constexpr int SETUP1_THREADS = 128;
constexpr int GEO_LD = 48;  // per sphere point: 35 monomials, F_0..2 (s3), F_0..3 (s4), F_0..4 (s5)

// RCUT of a call around its centre of gravity (poisson1.f:522-538).
__device__ double call_rcut(const CallInfo& ci, const PairGeo* __restrict__ pairs, const double cgr[3]) {
  double dmax = 0.0;
  for (int q = 0; q < ci.np; ++q) {
    const double* C = pairs[ci.p0 + q].C;
    const double dist = sqrt(sqdist_rn(C[0], C[1], C[2], cgr));
    if (dist > dmax) dmax = dist;
  }
  double rcut = sqrt(30.0 / ci.delta_min) + dmax;
  const double pirc = 1.0 / (4 * atan(1.0));
  const double fact = sqrt(pirc / (pirc + LM + 1));
  const double dist = 2 * dmax / pow(1.0e-6 / fact, 1.0 / (LM + 1));
  return fmax(rcut, dist);
}

// Far-point count of a call (all threads of the block), with early exit once
// NPOT=2 is certain; returns NPOT of the cost model (poisson1.f:548-583) and
// the count in nfar.
__device__ int call_far_count(const CallInfo& ci, const MeshDev& M, const double cg[3], double rcut2, int* s_far,
                              int* s_stop, int& nfar) {
  const int tid = threadIdx.x, nth = blockDim.x;
  if (tid == 0) {
    *s_far = 0;
    *s_stop = 0;
  }
  __syncthreads();
  const double slots = (double)ci.slots;
  const double thr = 1.36 * slots * NANG / (1.36 * slots - 0.99) + 2.0;
  for (int t0 = 0; t0 < M.ntiles; t0 += nth) {
    const int t = t0 + tid;
    int myfar = 0;
    if (t < M.ntiles) {
      double lo[3] = {M.tile_lo[3 * t], M.tile_lo[3 * t + 1], M.tile_lo[3 * t + 2]};
      double hi[3] = {M.tile_hi[3 * t], M.tile_hi[3 * t + 1], M.tile_hi[3 * t + 2]};
      double dmin2, dmax2;
      box_dist2(lo, hi, cg, dmin2, dmax2);
      const int p0 = t * TILE, p1 = min(M.n, p0 + TILE);
      if (dmin2 > rcut2 * (1.0 + 1e-9)) {
        myfar = p1 - p0;
      } else if (dmax2 < rcut2 * (1.0 - 1e-9)) {
        myfar = 0;
      } else {
        for (int p = p0; p < p1; ++p)
          if (sqdist_rn(M.x[p], M.y[p], M.z[p], cg) > rcut2) ++myfar;
      }
    }
    if (myfar) atomicAdd(s_far, myfar);
    __syncthreads();
    if (tid == 0 && (double)*s_far > thr) *s_stop = 1;
    __syncthreads();
    if (*s_stop) break;
  }
  nfar = *s_far;
  int npot = 2;
  if (!*s_stop) {
    const double cls = (double)(M.n - nfar);
    const double cost1 = 1.36 * (cls + NANG) * slots + 0.99 * (double)nfar;
    const double cost2 = 1.36 * ((double)nfar + cls) * slots;
    if (cost2 < cost1) npot = 1;
  }
  return npot;
}

__global__ void __launch_bounds__(SETUP_THREADS) k_call_setup(const int* __restrict__ list,
                                                              const CallInfo* __restrict__ calls,
                                                              const PairGeo* __restrict__ pairs, int nfo,
                                                              int nspn, const double* __restrict__ coef,
                                                              const int8_t* __restrict__ maxfmt,
                                                              const double* __restrict__ cgp, MeshDev M,
                                                              const double* __restrict__ boys_tab,
                                                              CallFO* __restrict__ out,
                                                              double* __restrict__ momv) {
  extern __shared__ double sm[];  // [NANG][NMOM] products, then NANG potentials
  double* prod = sm;
  double* vang = sm + NANG * NMOM;
  __shared__ double s_cg[3], s_rcut;
  __shared__ int s_far, s_stop;
  const int c = list[blockIdx.x], k = blockIdx.y, tid = threadIdx.x;
  const CallInfo ci = calls[c];
  if (tid == 0) {
    double cg[4] = {0, 0, 0, 0};
    for (int q = 0; q < ci.np; ++q) {
      const double* p = cgp + ((size_t)(ci.p0 + q) * nfo + k) * 4;
      for (int i = 0; i < 4; ++i) cg[i] += p[i];
    }
    double cgr[3];
    if (cg[3] != 0.0 && ci.slots > 1) {
      for (int d = 0; d < 3; ++d) cgr[d] = cg[d] / cg[3];
    } else {
      for (int d = 0; d < 3; ++d) {
        double s = 0.0;
        for (int q = 0; q < ci.np; ++q) s = s - (-pairs[ci.p0 + q].C[d]);
        cgr[d] = (nspn * s) / ci.slots;
      }
    }
    const double rcut = call_rcut(ci, pairs, cgr);
    for (int d = 0; d < 3; ++d) s_cg[d] = cgr[d];
    s_rcut = rcut;
  }
  __syncthreads();
  const double cg[3] = {s_cg[0], s_cg[1], s_cg[2]};
  const double rcut = s_rcut;
  const double rcut2 = __dmul_rn(rcut, rcut);
  int nfar = 0;
  const int npot = call_far_count(ci, M, cg, rcut2, &s_far, &s_stop, nfar);
  CallFO* o = out + (size_t)c * nfo + k;
  if (tid == 0) {
    o->cg[0] = cg[0];
    o->cg[1] = cg[1];
    o->cg[2] = cg[2];
    o->rcut = rcut;
    o->rcut2 = (npot == 1) ? DBL_MAX : rcut2;
    o->npot = npot;
    o->nfar = (npot == 1) ? 0 : nfar;
  }
  double* mv = momv + ((size_t)c * nfo + k) * MOM_LD;
  if (npot == 1 || nfar == 0) {
    if (tid < MOM_LD) mv[tid] = 0.0;
    if (tid == 0) {
      o->keep = 0ull;
      o->lmax = 0;
    }
    return;
  }
  // exact potential on the Lebedev sphere of radius RCUT around CG
  if (tid < NANG) {
    const double q[3] = {cg[0] + c_leb_ang[3 * tid] * rcut, cg[1] + c_leb_ang[3 * tid + 1] * rcut,
                         cg[2] + c_leb_ang[3 * tid + 2] * rcut};
    double v = 0.0;
    for (int qq = 0; qq < ci.np; ++qq) {
      const PairGeo& g = pairs[ci.p0 + qq];
      const double rx = q[0] - g.C[0], ry = q[1] - g.C[1], rz = q[2] - g.C[2];
      const double xx = g.delta * (rz * rz + ry * ry + rx * rx);
      const double chgd = exp(-xx);
      double s3[3], s4[4], s5[5], mono[35];
      boys_all(boys_tab, xx, chgd, s3, s4, s5);
      monomials(rx, ry, rz, mono);
      const size_t pk = (size_t)(ci.p0 + qq) * nfo + k;
      v += pair_potential(coef + pk * COEF_LD, mono, maxfmt[pk], s3, s4, s5);
    }
    vang[tid] = v;
    // harmonics at the normalised sphere point
    const double hn = 1.0 / sqrt(rcut * rcut);
    double Y[NMOM];
    harmonics6(LM, hn * (c_leb_ang[3 * tid] * rcut), hn * (c_leb_ang[3 * tid + 1] * rcut),
               hn * (c_leb_ang[3 * tid + 2] * rcut), Y);
    for (int m = 0; m < NMOM; ++m) prod[tid * NMOM + m] = c_leb_w[tid] * Y[m] * v;
  }
  __syncthreads();
  __shared__ double s_mom[NMOM];
  __shared__ unsigned long long s_keep_bits;
  if (tid < NMOM) {
    double s = 0.0;
    for (int i = 0; i < NANG; ++i) s += prod[i * NMOM + tid];
    int l = 0;
    while ((l + 1) * (l + 1) <= tid) ++l;
    const double h = sqrt(rcut * rcut);
    double rl = h;
    for (int j = 1; j <= l; ++j) rl = h * rl;
    s_mom[tid] = s * rl;
  }
  __syncthreads();
  if (tid == 0) {
    // skip rule of poisson1.f:1252-1270 with RI1 = 1/RCUT, an upper bound of
    // 1/r over every far point: keeps every term the reference keeps
    const double ri1 = 1.0 / rcut;
    unsigned long long keep = 0ull;
    int lmx = 0, m = 0;
    double rt = ri1;
    for (int l = 0; l <= LM; ++l) {
      for (int j = -l; j <= l; ++j, ++m)
        if (!(fabs((2 * l + 1) * s_mom[m] * rt) < 1.0e-12)) {
          keep |= (1ull << m);
          lmx = l;
        }
      rt *= ri1;
    }
    o->keep = keep;
    o->lmax = lmx;
    s_keep_bits = keep;
  }
  __syncthreads();
  // normalised moments with the skipped terms zeroed: M_lm * sqrt(NRUN (2l+1)/4pi (l-m)!/(l+m)!)
  if (tid < NMOM) {
    int l = 0;
    while ((l + 1) * (l + 1) <= tid) ++l;
    const int j = tid - l * l;
    const int m = (j + 1) / 2;
    const int nrun = (m == 0) ? 1 : 2;
    double facfc = (2 * l + 1) * (1.0 / (16 * atan(1.0)));
    for (int mm = 0; mm < m; ++mm) facfc = facfc / ((l - mm > 1 ? l - mm : 1) * (l + mm + 1));
    const double vf = sqrt(nrun * facfc);
    const bool kept = (s_keep_bits >> tid) & 1ull;
    mv[tid] = kept ? s_mom[tid] * vf : 0.0;
  } else if (tid < MOM_LD) {
    mv[tid] = 0.0;
  }
}

// The same set-up for a call of one slot (one pair, NSPN=1), all FOs in one
// block: CG is the pair centre (poisson1.f:515-520), so CG, RCUT, the far
// count and NPOT are the same for every FO and are formed once; the sphere
// points' Boys values, monomials and weighted harmonics are formed once and
// each thread (FO) contracts them with its coefficients.  Every FO's numbers
// are bitwise those of k_call_setup: the same expressions, in the same order.
__global__ void __launch_bounds__(SETUP1_THREADS) k_call_setup_single(
    const int* __restrict__ list, const CallInfo* __restrict__ calls, const PairGeo* __restrict__ pairs, int nfo,
    int nspn, const double* __restrict__ coef, const int8_t* __restrict__ maxfmt, MeshDev M,
    const double* __restrict__ boys_tab, CallFO* __restrict__ out, double* __restrict__ momv) {
  extern __shared__ double sm[];  // [NANG][GEO_LD] geometry, then [NANG][NMOM] w Y
  double* geo = sm;
  double* wy = sm + NANG * GEO_LD;
  __shared__ double s_cg[3], s_rcut, s_vf[NMOM];
  __shared__ int s_far, s_stop;
  const int c = list[blockIdx.x], tid = threadIdx.x;
  const CallInfo ci = calls[c];
  if (tid < NMOM) {
    // normalisation sqrt(NRUN (2l+1)/4pi (l-m)!/(l+m)!) of moment tid, as k_call_setup
    int l = 0;
    while ((l + 1) * (l + 1) <= tid) ++l;
    const int j = tid - l * l;
    const int m = (j + 1) / 2;
    const int nrun = (m == 0) ? 1 : 2;
    double facfc = (2 * l + 1) * (1.0 / (16 * atan(1.0)));
    for (int mm = 0; mm < m; ++mm) facfc = facfc / ((l - mm > 1 ? l - mm : 1) * (l + mm + 1));
    s_vf[tid] = sqrt(nrun * facfc);
  }
  if (tid == 0) {
    double cgr[3];
    for (int d = 0; d < 3; ++d) {
      double s = 0.0;
      for (int q = 0; q < ci.np; ++q) s = s - (-pairs[ci.p0 + q].C[d]);
      cgr[d] = (nspn * s) / ci.slots;
    }
    const double rcut = call_rcut(ci, pairs, cgr);
    for (int d = 0; d < 3; ++d) s_cg[d] = cgr[d];
    s_rcut = rcut;
  }
  __syncthreads();
  const double cg[3] = {s_cg[0], s_cg[1], s_cg[2]};
  const double rcut = s_rcut;
  const double rcut2 = __dmul_rn(rcut, rcut);
  int nfar = 0;
  const int npot = call_far_count(ci, M, cg, rcut2, &s_far, &s_stop, nfar);
  for (int k = tid; k < nfo; k += blockDim.x) {
    CallFO* o = out + (size_t)c * nfo + k;
    o->cg[0] = cg[0];
    o->cg[1] = cg[1];
    o->cg[2] = cg[2];
    o->rcut = rcut;
    o->rcut2 = (npot == 1) ? DBL_MAX : rcut2;
    o->npot = npot;
    o->nfar = (npot == 1) ? 0 : nfar;
    if (npot == 1 || nfar == 0) {
      double* mv = momv + ((size_t)c * nfo + k) * MOM_LD;
      for (int m = 0; m < MOM_LD; ++m) mv[m] = 0.0;
      o->keep = 0ull;
      o->lmax = 0;
    }
  }
  if (npot == 1 || nfar == 0) return;
  // the sphere points: Boys values and monomials of the pair, weighted harmonics
  const PairGeo& g = pairs[ci.p0];
  for (int i = tid; i < NANG; i += blockDim.x) {
    const double q[3] = {cg[0] + c_leb_ang[3 * i] * rcut, cg[1] + c_leb_ang[3 * i + 1] * rcut,
                         cg[2] + c_leb_ang[3 * i + 2] * rcut};
    const double rx = q[0] - g.C[0], ry = q[1] - g.C[1], rz = q[2] - g.C[2];
    const double xx = g.delta * (rz * rz + ry * ry + rx * rx);
    const double chgd = exp(-xx);
    double* gi = geo + (size_t)i * GEO_LD;
    double s3[3], s4[4], s5[5], mono[35];
    boys_all(boys_tab, xx, chgd, s3, s4, s5);
    monomials(rx, ry, rz, mono);
    for (int t = 0; t < 35; ++t) gi[t] = mono[t];
    for (int t = 0; t < 3; ++t) gi[35 + t] = s3[t];
    for (int t = 0; t < 4; ++t) gi[38 + t] = s4[t];
    for (int t = 0; t < 5; ++t) gi[42 + t] = s5[t];
    const double hn = 1.0 / sqrt(rcut * rcut);
    double Y[NMOM];
    harmonics6(LM, hn * (c_leb_ang[3 * i] * rcut), hn * (c_leb_ang[3 * i + 1] * rcut),
               hn * (c_leb_ang[3 * i + 2] * rcut), Y);
    for (int m = 0; m < NMOM; ++m) wy[(size_t)i * NMOM + m] = __dmul_rn(c_leb_w[i], Y[m]);
  }
  __syncthreads();
  const double h = sqrt(rcut * rcut);
  const double ri1 = 1.0 / rcut;
  for (int k = tid; k < nfo; k += blockDim.x) {
    const size_t pk = (size_t)ci.p0 * nfo + k;
    const double* cf = coef + pk * COEF_LD;
    const int fmt = maxfmt[pk];
    double acc[NMOM];
#pragma unroll
    for (int m = 0; m < NMOM; ++m) acc[m] = 0.0;
    for (int i = 0; i < NANG; ++i) {
      const double* gi = geo + (size_t)i * GEO_LD;
      double v = 0.0;
      v += pair_potential(cf, gi, fmt, gi + 35, gi + 38, gi + 42);
      const double* wyi = wy + (size_t)i * NMOM;
#pragma unroll
      for (int m = 0; m < NMOM; ++m) acc[m] = __dadd_rn(acc[m], __dmul_rn(wyi[m], v));
    }
    // moments, skip rule and normalisation as k_call_setup
    unsigned long long keep = 0ull;
    int lmx = 0;
    double rt = ri1;
    double rl = h;
#pragma unroll
    for (int l = 0; l <= LM; ++l) {
#pragma unroll
      for (int j = 0; j <= 2 * l; ++j) {
        const int m = l * l + j;
        acc[m] = acc[m] * rl;
        if (!(fabs((2 * l + 1) * acc[m] * rt) < 1.0e-12)) {
          keep |= (1ull << m);
          lmx = l;
        }
      }
      rt *= ri1;
      rl = h * rl;
    }
    CallFO* o = out + (size_t)c * nfo + k;
    o->keep = keep;
    o->lmax = lmx;
    double* mv = momv + ((size_t)c * nfo + k) * MOM_LD;
#pragma unroll
    for (int t = 0; t < NMOM; ++t) mv[t] = ((keep >> t) & 1ull) ? acc[t] * s_vf[t] : 0.0;
#pragma unroll
    for (int t = NMOM; t < MOM_LD; ++t) mv[t] = 0.0;
  }
}

void init_call_setup() {
  cudaFuncSetAttribute(k_call_setup, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(sizeof(double) * (NANG * NMOM + NANG)));
  cudaFuncSetAttribute(k_call_setup_single, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(sizeof(double) * NANG * (GEO_LD + NMOM)));
}

void launch_call_setup(int ncalls, const int* list, int nsingle, const CallInfo* calls, const PairGeo* pairs,
                       int nfo, int nspn, const double* coef, const int8_t* maxfmt, const double* cgp,
                       const MeshDev& M, const double* boys_tab, CallFO* cfo, double* momv, cudaStream_t st) {
  if (ncalls <= 0) return;
  if (nsingle > 0)
    k_call_setup_single<<<nsingle, SETUP1_THREADS, sizeof(double) * NANG * (GEO_LD + NMOM), st>>>(
        list, calls, pairs, nfo, nspn, coef, maxfmt, M, boys_tab, cfo, momv);
  if (ncalls > nsingle) {
    const size_t smem = sizeof(double) * (NANG * NMOM + NANG);
    dim3 grid(ncalls - nsingle, nfo);
    k_call_setup<<<grid, SETUP_THREADS, smem, st>>>(list + nsingle, calls, pairs, nfo, nspn, coef, maxfmt, cgp, M,
                                                     boys_tab, cfo, momv);
  }
}

// ---------------------------------------------------------------------------
// XC, SIC potential and energy partial sums
// ---------------------------------------------------------------------------
// parts: 0 XCH1 1 XCOU 2 XEXX 3 XDEL 4 ERGXL 5 ERGXN 6 ERGCL 7 ERGCN 8..10 CFRM
constexpr int XC_THREADS = 256;

__device__ __forceinline__ void block_reduce_parts(double v[NPART], double* out) {
  __shared__ double red[XC_THREADS / 32][NPART];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NPART; ++j) {
    double x = v[j];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[wid][j] = x;
  }
  __syncthreads();
  if (threadIdx.x < NPART) {
    double s = 0.0;
    for (int w = 0; w < XC_THREADS / 32; ++w) s += red[w][threadIdx.x];
    out[threadIdx.x] = s;
  }
}

// Per (point, FO k): the FO density channels from phi (1, 4 or 10 channels:
// value, gradient, second derivatives) or, when rhog is given, the
// reference-route channels read from it, the XC potential, the SIC potential
// V = V_xc + V_H, Y = w V phi for the SIC matrix and the energy partials.  For
// SCAN (mgga) also tau = |grad phi|^2/2 and the Hamiltonian ingredients Z of
// call_mgga.f90, which enter the SIC matrix through four Y channels
// (frmorb_mpi.F:440-509):
//   Y0 = w V phi + w grad phi . Z,   Yc = w Z_c phi + w Z_4 d_c phi  (c = x, y, z).
// MGGA selects the SCAN instance, so that the LDA/GGA instance keeps its own
// (smaller) register allocation.
template <bool MGGA>
__global__ void __launch_bounds__(XC_THREADS) k_xc(MeshDev M, int nfo, int gga, int nspn, XCParams xp,
                                                   const double* __restrict__ phi, int ldp,
                                                   const double* __restrict__ rhog,
                                                   double* __restrict__ vh, double* __restrict__ vpot,
                                                   double* __restrict__ y, double* __restrict__ part, int nblk) {
  const int k = blockIdx.y;
  double pv[NPART];
#pragma unroll
  for (int j = 0; j < NPART; ++j) pv[j] = 0.0;
  const double fnspn = (double)nspn;
  const double p43 = (double)(4.0f / 3.0f);
  for (int p = blockIdx.x * XC_THREADS + threadIdx.x; p < M.n; p += nblk * XC_THREADS) {
    const double w = M.w[p];
    double r[10];
    const double f0 = phi[(size_t)k * ldp + p];
    r[0] = f0 * f0;
    if constexpr (MGGA) {
      double f[4];
      f[0] = f0;
#pragma unroll
      for (int ch = 1; ch < 4; ++ch) f[ch] = phi[((size_t)ch * nfo + k) * ldp + p];
#pragma unroll
      for (int d = 1; d <= 3; ++d) r[d] = 2 * f[0] * f[d];
      if (rhog) {
#pragma unroll
        for (int d = 0; d < 4; ++d) r[d] = rhog[((size_t)d * nfo + k) * ldp + p];
      }
      const double tau = 0.5 * (f[1] * f[1] + f[2] * f[2] + f[3] * f[3]);
      const size_t kp = (size_t)k * M.n + p;
      const size_t cs = (size_t)nfo * M.n;  // Y channel stride
      const double coul = vh[kp] * fnspn / 2.0;
      vh[kp] = coul;
      double vup, vdn, e4[4] = {0, 0, 0, 0}, z[4];
      xc_point_sic_scan(r, tau, w, vup, vdn, e4, z);
      const double pot = vup + coul;
      vpot[kp] = pot;
      y[kp] = w * pot * f0 + w * (f[1] * z[0] + f[2] * z[1] + f[3] * z[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) y[(c + 1) * cs + kp] = w * z[c] * f0 + w * z[3] * f[1 + c];
      const double vx = pot - coul;
      pv[0] += w * r[0];
      pv[1] += w * r[0] * coul;
      pv[2] += w * pow(fabs(r[0]), p43);
      pv[3] -= w * r[0] * vx;
      pv[4] += e4[0];
      pv[5] += e4[1];
      pv[6] += e4[2];
      pv[7] += e4[3];
      pv[8] += M.x[p] * r[0] * w;
      pv[9] += M.y[p] * r[0] * w;
      pv[10] += M.z[p] * r[0] * w;
      continue;
    }
    if (gga) {
      double f[10];
      f[0] = f0;
#pragma unroll
      for (int ch = 1; ch < 10; ++ch) f[ch] = phi[((size_t)ch * nfo + k) * ldp + p];
      for (int d = 1; d <= 3; ++d) r[d] = 2 * f[0] * f[d];
      for (int d = 4; d <= 6; ++d) r[d] = 2 * (f[d - 3] * f[d - 3] + f[d] * f[0]);
      r[7] = 2 * (f[1] * f[2] + f[7] * f[0]);
      r[8] = 2 * (f[1] * f[3] + f[8] * f[0]);
      r[9] = 2 * (f[2] * f[3] + f[9] * f[0]);
    } else {
      for (int d = 1; d < 10; ++d) r[d] = 0.0;
    }
    if (rhog) {
      for (int d = 0; d < (gga ? 10 : 1); ++d) r[d] = rhog[((size_t)d * nfo + k) * ldp + p];
    }
    const size_t kp = (size_t)k * M.n + p;
    const double coul = vh[kp] * fnspn / 2.0;
    vh[kp] = coul;
    double vup, vdn, e4[4] = {0, 0, 0, 0};
    xc_point_sic(xp, r, w, vup, vdn, e4);
    const double pot = vup + coul;
    vpot[kp] = pot;
    y[kp] = w * pot * f0;
    const double vx = pot - coul;
    pv[0] += w * r[0];
    pv[1] += w * r[0] * coul;
    pv[2] += w * pow(fabs(r[0]), p43);
    pv[3] -= w * r[0] * vx;
    pv[4] += e4[0];
    pv[5] += e4[1];
    pv[6] += e4[2];
    pv[7] += e4[3];
    pv[8] += M.x[p] * r[0] * w;
    pv[9] += M.y[p] * r[0] * w;
    pv[10] += M.z[p] * r[0] * w;
  }
  block_reduce_parts(pv, part + ((size_t)k * nblk + blockIdx.x) * NPART);
}

void launch_xc(const MeshDev& M, int nfo, int gga, int mgga, int nspn, const int* xc, const double* phi, int ldp,
               const double* rhog, double* vh, double* vpot, double* y, double* part, int nblk, cudaStream_t st) {
  XCParams xp;
  xp.igga[0] = xc[0];
  xp.idftyp[0] = xc[1];
  xp.igga[1] = xc[2];
  xp.idftyp[1] = xc[3];
  dim3 grid(nblk, nfo);
  if (mgga) k_xc<true><<<grid, XC_THREADS, 0, st>>>(M, nfo, gga, nspn, xp, phi, ldp, rhog, vh, vpot, y, part, nblk);
  else k_xc<false><<<grid, XC_THREADS, 0, st>>>(M, nfo, gga, nspn, xp, phi, ldp, rhog, vh, vpot, y, part, nblk);
}

// Compensated (Neumaier) sums of the block partials, in block order.
__global__ void k_reduce_parts(int nfo, int nblk, const double* __restrict__ part, double* __restrict__ sums) {
  const int k = blockIdx.x, j = threadIdx.x;
  if (j >= NPART) return;
  double s = 0.0, cmp = 0.0;
  for (int b = 0; b < nblk; ++b) {
    const double x = part[((size_t)k * nblk + b) * NPART + j];
    const double t = s + x;
    if (fabs(s) >= fabs(x)) cmp += (s - t) + x;
    else cmp += (x - t) + s;
    s = t;
  }
  sums[(size_t)k * NPART + j] = s + cmp;
}

void launch_reduce_parts(int nfo, int nblk, const double* part, double* sums, cudaStream_t st) {
  k_reduce_parts<<<nfo, 32, 0, st>>>(nfo, nblk, part, sums);
}

// FO density channels RHOG(ldr, nch) from the phi channels: nch = 1 (LDA),
// 4 (meta-GGA: value and gradient; the second-derivative channels of the
// 10-channel layout are written as zero) or 10 (GGA).
__global__ void k_density(int npts, int nfo, int k, int nch, const double* __restrict__ phi, int ldp,
                          double* __restrict__ rhog, int ldr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const double f0 = phi[(size_t)k * ldp + p];
  rhog[p] = f0 * f0;
  if (nch == 1) return;
  if (nch == 4) {
    for (int d = 1; d <= 3; ++d) rhog[(size_t)d * ldr + p] = 2 * f0 * phi[((size_t)d * nfo + k) * ldp + p];
    for (int d = 4; d < 10; ++d) rhog[(size_t)d * ldr + p] = 0.0;
    return;
  }
  double f[10];
  f[0] = f0;
  for (int ch = 1; ch < 10; ++ch) f[ch] = phi[((size_t)ch * nfo + k) * ldp + p];
  for (int d = 1; d <= 3; ++d) rhog[(size_t)d * ldr + p] = 2 * f[0] * f[d];
  for (int d = 4; d <= 6; ++d) rhog[(size_t)d * ldr + p] = 2 * (f[d - 3] * f[d - 3] + f[d] * f[0]);
  rhog[(size_t)7 * ldr + p] = 2 * (f[1] * f[2] + f[7] * f[0]);
  rhog[(size_t)8 * ldr + p] = 2 * (f[1] * f[3] + f[8] * f[0]);
  rhog[(size_t)9 * ldr + p] = 2 * (f[2] * f[3] + f[9] * f[0]);
}

void launch_density(int npts, int nfo, int k, int nch, const double* phi, int ldp, double* rhog, int ldr,
                    cudaStream_t st) {
  k_density<<<(npts + 255) / 256, 256, 0, st>>>(npts, nfo, k, nch, phi, ldp, rhog, ldr);
}

// DENSOLD (densold.F:190-250): spin densities of the occupied orbitals and,
// for ngrad = 10, their gradients and second derivatives, plus PHIG = sum
// |grad psi|^2, from the orbital values psig[(ch*nwf + i)*ldp + p] (ch < ngrad).
// Orbitals [0, nw0) are spin 1, [nw0, nw0+nw1) spin 2.  rhog[(s*ngrad + ch)*ldr + p],
// phig[s*ldr + p].
__global__ void k_densold(int npts, int nw0, int nw1, int nspn, int ngrad, const double* __restrict__ psig, int ldp,
                          double* __restrict__ rhog, double* __restrict__ phig, int ldr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int nwf = nw0 + nw1;
  for (int s = 0; s < nspn; ++s) {
    const int i0 = s == 0 ? 0 : nw0, i1 = s == 0 ? nw0 : nw0 + nw1;
    double r[10], ph = 0.0;
#pragma unroll
    for (int ch = 0; ch < 10; ++ch) r[ch] = 0.0;
    for (int i = i0; i < i1; ++i) {
      const double f0 = psig[(size_t)i * ldp + p];
      r[0] += f0 * f0;
      if (ngrad == 1) continue;
      double f[10];
      f[0] = f0;
#pragma unroll
      for (int ch = 1; ch < 10; ++ch) f[ch] = psig[((size_t)ch * nwf + i) * ldp + p];
#pragma unroll
      for (int d = 1; d <= 3; ++d) {
        r[d] += 2 * f[0] * f[d];
        ph += f[d] * f[d];
      }
#pragma unroll
      for (int d = 4; d <= 6; ++d) r[d] += 2 * (f[d - 3] * f[d - 3] + f[d] * f[0]);
      r[7] += 2 * (f[1] * f[2] + f[7] * f[0]);
      r[8] += 2 * (f[1] * f[3] + f[8] * f[0]);
      r[9] += 2 * (f[2] * f[3] + f[9] * f[0]);
    }
    for (int ch = 0; ch < ngrad; ++ch) rhog[((size_t)s * ngrad + ch) * ldr + p] = r[ch];
    if (phig) phig[(size_t)s * ldr + p] = ph;
  }
}

void launch_densold(int npts, int nw0, int nw1, int nspn, int ngrad, const double* psig, int ldp, double* rhog,
                    double* phig, int ldr, cudaStream_t st) {
  if (npts <= 0) return;
  k_densold<<<(npts + 255) / 256, 256, 0, st>>>(npts, nw0, nw1, nspn, ngrad, psig, ldp, rhog, phig, ldr);
}

// tau = |grad phi_k|^2 / 2 of FO k (GETTAU_PAR for the SIC FO).
__global__ void k_fo_tau(int npts, int nfo, int k, const double* __restrict__ phi, int ldp, double* __restrict__ tau) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  double t = 0.0;
  for (int d = 1; d <= 3; ++d) {
    const double g = phi[((size_t)d * nfo + k) * ldp + p];
    t += g * g;
  }
  tau[p] = 0.5 * t;
}

void launch_fo_tau(int npts, int nfo, int k, const double* phi, int ldp, double* tau, cudaStream_t st) {
  k_fo_tau<<<(npts + 255) / 256, 256, 0, st>>>(npts, nfo, k, phi, ldp, tau);
}

// Meta-GGA GETVLXC on given density channels RHOG(ldr, 4+) and tau: VXC(2n),
// MIXIN(4, n) of the spin-up half, energy partials.
__global__ void __launch_bounds__(XC_THREADS) k_xc_mgga_rhog(MeshDev M, const double* __restrict__ rhog, int ldr,
                                                             const double* __restrict__ tau,
                                                             double* __restrict__ vxc, double* __restrict__ mixin,
                                                             double* __restrict__ part, int nblk) {
  double pv[NPART];
#pragma unroll
  for (int j = 0; j < NPART; ++j) pv[j] = 0.0;
  for (int p = blockIdx.x * XC_THREADS + threadIdx.x; p < M.n; p += nblk * XC_THREADS) {
    double r[4];
    for (int d = 0; d < 4; ++d) r[d] = rhog[(size_t)d * ldr + p];
    double vup, vdn, e4[4] = {0, 0, 0, 0}, z[4];
    xc_point_sic_scan(r, tau[p], M.w[p], vup, vdn, e4, z);
    vxc[p] = vup;
    vxc[M.n + p] = vdn;
    for (int d = 0; d < 4; ++d) mixin[(size_t)4 * p + d] = z[d];
    for (int j = 0; j < 4; ++j) pv[4 + j] += e4[j];
  }
  block_reduce_parts(pv, part + (size_t)blockIdx.x * NPART);
}

void launch_xc_mgga_rhog(const MeshDev& M, const double* rhog, int ldr, const double* tau, double* vxc,
                         double* mixin, double* part, int nblk, cudaStream_t st) {
  k_xc_mgga_rhog<<<nblk, XC_THREADS, 0, st>>>(M, rhog, ldr, tau, vxc, mixin, part, nblk);
}

__global__ void __launch_bounds__(XC_THREADS) k_xc_rhog(MeshDev M, int gga, XCParams xp,
                                                        const double* __restrict__ rhog, int ldr,
                                                        double* __restrict__ vxc, double* __restrict__ part,
                                                        int nblk) {
  double pv[NPART];
#pragma unroll
  for (int j = 0; j < NPART; ++j) pv[j] = 0.0;
  for (int p = blockIdx.x * XC_THREADS + threadIdx.x; p < M.n; p += nblk * XC_THREADS) {
    double r[10];
    for (int d = 0; d < 10; ++d) r[d] = (d == 0 || gga) ? rhog[(size_t)d * ldr + p] : 0.0;
    double vup, vdn, e4[4] = {0, 0, 0, 0};
    xc_point_sic(xp, r, M.w[p], vup, vdn, e4);
    vxc[p] = vup;
    vxc[M.n + p] = vdn;
    for (int j = 0; j < 4; ++j) pv[4 + j] += e4[j];
  }
  block_reduce_parts(pv, part + (size_t)blockIdx.x * NPART);
}

// Loads the two kernels of the GETVLXC-on-device-buffers path on the current
// device.  With CUDA's lazy loading a kernel's code is placed in device memory
// at its first launch; doing that here, at context creation, keeps that
// allocation out of the allocation-free entry point.
cudaError_t preload_xc_rhog() {
  cudaFuncAttributes a;
  const cudaError_t e = cudaFuncGetAttributes(&a, k_xc_rhog);
  return e != cudaSuccess ? e : cudaFuncGetAttributes(&a, k_reduce_parts);
}

void launch_xc_rhog(const MeshDev& M, int gga, const int* xc, const double* rhog, int ldr, double* vxc,
                    double* part, int nblk, cudaStream_t st) {
  XCParams xp;
  xp.igga[0] = xc[0];
  xp.idftyp[0] = xc[1];
  xp.igga[1] = xc[2];
  xp.idftyp[1] = xc[3];
  k_xc_rhog<<<nblk, XC_THREADS, 0, st>>>(M, gga, xp, rhog, ldr, vxc, part, nblk);
}

}  // namespace flosic
