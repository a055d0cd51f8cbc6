// FO densities by the reference's route (sm_100a, FP64).
//
// POISSON1 builds the density of each FO, for the SIC exchange-correlation,
// from the Gaussian-pair polynomials of the Poisson calls: at the points inside
// a call's RCUT sphere (every point when NPOT = 1) it adds, pair by pair,
//   rho_p(r) = exp(-ARG) POLY(r - C) . RHOC  exp(-delta |r - C|^2)
// and, for gradient corrections, the derivative polynomials RHOD of the
// gradient and second-derivative channels (poisson1.f:849-948, coefficients
// from gtdncf.F:5-1113).  Coefficients of magnitude <= 1e-14 are skipped and
// the points outside RCUT receive nothing from the call's pairs, so this
// density is the reference's truncated one rather than phi^2.
//
//   k_pair_dens_coef   RHOC (35) and the RHOD entries the channels use, per
//                      (pair, FO), thresholded as the reference skips them
//   k_pair_density     all calls of one FO over one mesh tile: near test per
//                      point, pair polynomials, channel sums in call order
#include <cstddef>

#include "coulomb_common.cuh"
#include "kernels.cuh"

namespace flosic {

namespace {

// Cartesian powers of the ten s/p/d components (x, y, z order).
__constant__ int c_dens_pow[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                                      {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};

constexpr double DENS_EPS = 1.0e-14;  // poisson1.f:860,870,880
constexpr int DENS_THREADS = TILE;    // one mesh point per thread

__device__ __forceinline__ double dens_keep(double v) { return fabs(v) > DENS_EPS ? v : 0.0; }

// Powers (px, py, pz) of monomial m in the POLY order (degree, then x power
// ascending, then y power ascending).
__device__ __forceinline__ void mono_powers(int m, int& px, int& py, int& pz) {
  const int d = (m == 0) ? 0 : (m < 4) ? 1 : (m < 10) ? 2 : (m < 20) ? 3 : 4;
  const int base = (d == 0) ? 0 : (d == 1) ? 1 : (d == 2) ? 4 : (d == 3) ? 10 : 20;
  int off = m - base, x = 0;
  while (off >= d - x + 1) {
    off -= d - x + 1;
    ++x;
  }
  px = x;
  py = off;
  pz = d - x - off;
}

__global__ void __launch_bounds__(128) k_pair_dens_coef(const PairGeo* __restrict__ pairs, int nfo, int nprim,
                                                        const double* __restrict__ u, int nch,
                                                        double* __restrict__ dc, int ldc) {
  __shared__ double P1[10][10][3][5];
  const int ip = blockIdx.x, tid = threadIdx.x;
  const PairGeo g = pairs[ip];
  // gtdncf.F:9-16: the product centre and exponent argument of the pair
  const double dlt = g.a + g.b;
  double C[3], arg = 0.0;
  for (int d = 0; d < 3; ++d) {
    C[d] = (g.a * g.A[d] + g.b * g.B[d]) / dlt;
    arg = arg + (g.A[d] - g.B[d]) * (g.A[d] - g.B[d]);
  }
  arg = arg * g.a * g.b / dlt;
  // 1-D factors (rho + C - A)^na (rho + C - B)^nb as polynomials in rho
  for (int q = tid; q < 300; q += blockDim.x) {
    const int mu = q / 30, nu = (q / 3) % 10, d = q % 3;
    const double ca = C[d] - g.A[d], cb = C[d] - g.B[d];
    const int na = c_dens_pow[mu][d], nb = c_dens_pow[nu][d];
    double pa[3] = {0, 0, 0}, pb[3] = {0, 0, 0};
    if (na == 0) pa[0] = 1;
    else if (na == 1) { pa[0] = ca; pa[1] = 1; }
    else { pa[0] = ca * ca; pa[1] = 2 * ca; pa[2] = 1; }
    if (nb == 0) pb[0] = 1;
    else if (nb == 1) { pb[0] = cb; pb[1] = 1; }
    else { pb[0] = cb * cb; pb[1] = 2 * cb; pb[2] = 1; }
    double e[5] = {0, 0, 0, 0, 0};
    for (int x = 0; x <= na; ++x)
      for (int y = 0; y <= nb; ++y) e[x + y] += pa[x] * pb[y];
    for (int j = 0; j < 5; ++j) P1[mu][nu][d][j] = e[j];
  }
  __syncthreads();
  const double ex = exp(-arg);
  for (int q = tid; q < nfo * 35; q += blockDim.x) {
    const int k = q / 35, m = q % 35;
    int px, py, pz;
    mono_powers(m, px, py, pz);
    const double* pu = u + ((size_t)k * nprim + g.pi) * 10;
    const double* pv = u + ((size_t)k * nprim + g.pj) * 10;
    // RHOC(m) = exp(-ARG) sum_{mu,nu} GAM(mu,nu) x-factor y-factor z-factor, with
    // GAM the pair block of the FO's density matrix (coupot_sic.F:366-482)
    double s = 0.0;
    for (int mu = 0; mu < 10; ++mu) {
      const double ui = pu[mu];
      if (ui == 0.0) continue;
      for (int nu = 0; nu < 10; ++nu) {
        const double gm = ui * pv[nu] * g.times;
        if (gm == 0.0) continue;
        const double fx = P1[mu][nu][0][px], fy = P1[mu][nu][1][py], fz = P1[mu][nu][2][pz];
        if (fx == 0.0 || fy == 0.0 || fz == 0.0) continue;
        s += gm * fx * fy * fz;
      }
    }
    const double rc = s * ex;
    double* row = dc + ((size_t)ip * nfo + k) * ldc;
    row[m] = dens_keep(rc);
    if (m == 0) row[35] = 0.0;
    if (nch == 1) continue;
    // RHOD: every entry is one power times one RHOC entry (gtdncf.F), so the
    // thread of monomial m writes the entries that m feeds
    const int p[3] = {px, py, pz};
    for (int d = 0; d < 3; ++d)
      if (p[d] > 0) {
        int r[3] = {px, py, pz};
        r[d] -= 1;
        row[36 + mono_index(r[0], r[1], r[2]) * 3 + d] = dens_keep((double)p[d] * rc);
      }
    if (nch < 10) continue;
    const int dd[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    for (int kk = 0; kk < 6; ++kk) {
      int r[3] = {px, py, pz};
      double f = r[dd[kk][0]];
      r[dd[kk][0]] -= 1;
      if (f <= 0) continue;
      f *= r[dd[kk][1]];
      r[dd[kk][1]] -= 1;
      if (f <= 0) continue;
      row[96 + mono_index(r[0], r[1], r[2]) * 6 + kk] = dens_keep(f * rc);
    }
  }
}

// Monomials POLY(r - C) of poisson1.f:820-847 (formed by the same products)
// and the pair Gaussian exp(-delta |r - C|^2) at one point.
__device__ __forceinline__ double pair_poly(double x, double y, double z, const PairGeo& g, double (&p)[35]) {
  p[0] = 1.0;
  p[3] = x - g.C[0];
  p[2] = y - g.C[1];
  p[1] = z - g.C[2];
  p[4] = p[1] * p[1];
  p[6] = p[2] * p[2];
  p[9] = p[3] * p[3];
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
  return exp(-(g.delta * (p[4] + p[6] + p[9])));
}

// Channel values of one pair and one FO at one point before the Gaussian
// factor (poisson1.f:849-940): the RHOC and RHOD sums in the reference's
// order, then the product-rule terms of the Gaussian's derivatives.  row: the
// pair's coefficient row, staged in shared memory.
template <int NCH>
__device__ __forceinline__ void pair_channels(const double (&p)[35], double delta, const double* row,
                                              double (&a)[NCH]) {
  const double2* r2 = reinterpret_cast<const double2*>(row);
#pragma unroll
  for (int c = 0; c < NCH; ++c) a[c] = 0.0;
#pragma unroll
  for (int j = 0; j < 18; ++j) {
    const double2 v = r2[j];
    a[0] = fma(p[2 * j], v.x, a[0]);
    if (2 * j + 1 < 35) a[0] = fma(p[2 * j + 1], v.y, a[0]);
  }
  if constexpr (NCH > 1) {
    // gradient channels: 20 monomials x 3, row[36 + q*3 + d]
#pragma unroll
    for (int j = 0; j < 30; ++j) {
      const double2 v = r2[18 + j];
      const int e0 = 2 * j, e1 = 2 * j + 1;
      a[1 + e0 % 3] = fma(p[e0 / 3], v.x, a[1 + e0 % 3]);
      a[1 + e1 % 3] = fma(p[e1 / 3], v.y, a[1 + e1 % 3]);
    }
  }
  if constexpr (NCH == 10) {
    // second-derivative channels: 10 monomials x 6, row[96 + q*6 + kk]
#pragma unroll
    for (int j = 0; j < 30; ++j) {
      const double2 v = r2[48 + j];
      const int e0 = 2 * j, e1 = 2 * j + 1;
      a[4 + e0 % 6] = fma(p[e0 / 6], v.x, a[4 + e0 % 6]);
      a[4 + e1 % 6] = fma(p[e1 / 6], v.y, a[4 + e1 % 6]);
    }
    const double d1x4 = delta * 4.0, d2x4 = delta * delta * 4.0, d1x2 = delta * 2.0;
    a[4] = a[4] - d1x4 * p[3] * a[1] + (d2x4 * p[9] - d1x2) * a[0];
    a[5] = a[5] - d1x4 * p[2] * a[2] + (d2x4 * p[6] - d1x2) * a[0];
    a[6] = a[6] - d1x4 * p[1] * a[3] + (d2x4 * p[4] - d1x2) * a[0];
    a[7] = a[7] - d1x2 * p[2] * a[1] - d1x2 * p[3] * a[2] + d2x4 * p[8] * a[0];
    a[8] = a[8] - d1x2 * p[1] * a[1] - d1x2 * p[3] * a[3] + d2x4 * p[7] * a[0];
    a[9] = a[9] - d1x2 * p[2] * a[3] - d1x2 * p[1] * a[2] + d2x4 * p[5] * a[0];
  }
  if constexpr (NCH > 1) {
    const double d1x2 = delta * 2.0;
    a[1] = a[1] - d1x2 * p[3] * a[0];
    a[2] = a[2] - d1x2 * p[2] * a[0];
    a[3] = a[3] - d1x2 * p[1] * a[0];
  }
}

// Block = (mesh tile, FO k).  The calls whose sphere reaches the tile are
// gathered in call order, 128 at a time, with their sphere and pair range in
// shared memory; their pairs then stream through a DENS_NBUF-deep ring of
// shared-memory stages (coefficient row and pair centre/exponent, copied with
// cp.async DENS_NBUF-1 pairs ahead), and each is added at the tile's points
// inside the call's sphere, in pair order, so each point sums its
// contributions in the reference's order.
constexpr int DENS_NBUF = 4;
template <int NCH, int LDC>
__global__ void __launch_bounds__(DENS_THREADS) k_pair_density(MeshDev M, int ncalls, const CallInfo* __restrict__ calls,
                                                               const PairGeo* __restrict__ pairs,
                                                               const CallFO* __restrict__ cfo, int nfo,
                                                               const double* __restrict__ dc,
                                                               double* __restrict__ rhog, size_t ldr) {
  static_assert(LDC % 2 == 0 && LDC / 2 <= DENS_THREADS, "one 16-byte chunk of a row per thread");
  static_assert(sizeof(PairGeo) % 16 == 0 && offsetof(PairGeo, C) == 64 && offsetof(PairGeo, delta) == 88,
                "pair centre and exponent are the 32 bytes at offset 64");
  __shared__ __align__(16) double s_row[DENS_NBUF][LDC];
  __shared__ __align__(16) double s_geo[DENS_NBUF][4];  // C[3], delta
  __shared__ double s_cg[DENS_THREADS][4];              // CG, RCUT^2 of the listed calls
  __shared__ int s_p0[DENS_THREADS], s_np[DENS_THREADS];
  __shared__ int s_cnt[DENS_THREADS / 32];
  const int tile = blockIdx.x, k = blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double lo[3], hi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = M.tile_lo[3 * tile + d];
    hi[d] = M.tile_hi[3 * tile + d];
  }
  const int pt = tile * TILE + tid;
  const bool valid = pt < M.n;
  const double x = valid ? M.x[pt] : 0.0, y = valid ? M.y[pt] : 0.0, z = valid ? M.z[pt] : 0.0;
  double acc[NCH];
#pragma unroll
  for (int c = 0; c < NCH; ++c) acc[c] = 0.0;
  for (int c0 = 0; c0 < ncalls; c0 += DENS_THREADS) {
    const int c = c0 + tid;
    bool hit = false;
    CallFO cf;
    if (c < ncalls) {
      cf = cfo[(size_t)c * nfo + k];
      hit = cf.npot == 1 || tile_class(lo, hi, cf.cg[0], cf.cg[1], cf.cg[2], cf.rcut2) != 1;
    }
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) s_cnt[warp] = __popc(b);
    __syncthreads();
    int before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < DENS_THREADS / 32; ++w) {
      before += (w < warp) ? s_cnt[w] : 0;
      total += s_cnt[w];
    }
    if (hit) {
      const int i = before + __popc(b & ((1u << lane) - 1u));
      const CallInfo ci = calls[c];
      s_cg[i][0] = cf.cg[0];
      s_cg[i][1] = cf.cg[1];
      s_cg[i][2] = cf.cg[2];
      s_cg[i][3] = cf.rcut2;
      s_p0[i] = ci.p0;
      s_np[i] = ci.np;
    }
    __syncthreads();
    // the copy side walks (call, pair) DENS_NBUF-1 stages ahead of the compute side
    int fi = 0, fq = 0;
    while (fi < total && s_np[fi] == 0) ++fi;
    auto issue = [&](int buf) {
      if (fi < total) {
        const int q = s_p0[fi] + fq;
        const double* src = dc + ((size_t)q * nfo + k) * LDC;
        if (tid < LDC / 2) cp_async16(&s_row[buf][2 * tid], src + 2 * tid);
        if (tid >= DENS_THREADS - 2) {
          const int h = tid - (DENS_THREADS - 2);
          cp_async16(&s_geo[buf][2 * h], reinterpret_cast<const char*>(pairs + q) + 64 + 16 * h);
        }
        if (++fq == s_np[fi]) {
          fq = 0;
          ++fi;
          while (fi < total && s_np[fi] == 0) ++fi;
        }
      }
      cp_async_commit();
    };
#pragma unroll
    for (int j = 0; j < DENS_NBUF - 1; ++j) issue(j);
    int ci = 0, cq = 0;
    while (ci < total && s_np[ci] == 0) ++ci;
    bool near = false;
    for (int st = 0; ci < total; ++st) {
      asm volatile("cp.async.wait_group %0;\n" ::"n"(DENS_NBUF - 2) : "memory");
      __syncthreads();  // stage st has landed for every thread; stage st-1's buffer is free
      issue((st + DENS_NBUF - 1) % DENS_NBUF);
      if (cq == 0)
        near = valid && !(sqdist_rn2(x, y, z, s_cg[ci][0], s_cg[ci][1], s_cg[ci][2]) > s_cg[ci][3]);
      if (near) {
        const int buf = st % DENS_NBUF;
        PairGeo g;
        g.C[0] = s_geo[buf][0];
        g.C[1] = s_geo[buf][1];
        g.C[2] = s_geo[buf][2];
        g.delta = s_geo[buf][3];
        double p[35];
        const double chgd = pair_poly(x, y, z, g, p);
        double a[NCH];
        pair_channels<NCH>(p, g.delta, s_row[buf], a);
#pragma unroll
        for (int ch = 0; ch < NCH; ++ch) acc[ch] += chgd * a[ch];
      }
      if (++cq == s_np[ci]) {
        cq = 0;
        ++ci;
        while (ci < total && s_np[ci] == 0) ++ci;
      }
    }
    cp_async_wait_all();
    __syncthreads();  // the lists and stage buffers are rewritten by the next batch of calls
  }
  if (valid) {
#pragma unroll
    for (int c = 0; c < NCH; ++c) rhog[((size_t)c * nfo + k) * ldr + pt] = acc[c];
  }
}

}  // namespace

int pair_density_ld(int nch) { return nch == 1 ? 36 : (nch == 4 ? 96 : 156); }

void launch_pair_density(int npairs, const PairGeo* pairs, int ncalls, const CallInfo* calls, const CallFO* cfo,
                         int nfo, int nprim, const double* u, int nch, const MeshDev& M, double* dc, double* rhog,
                         size_t ldr, cudaStream_t st) {
  if (nfo <= 0 || M.ntiles <= 0) return;
  const int ldc = pair_density_ld(nch);
  if (npairs > 0) k_pair_dens_coef<<<npairs, 128, 0, st>>>(pairs, nfo, nprim, u, nch, dc, ldc);
  dim3 grid(M.ntiles, nfo);
  if (nch == 1)
    k_pair_density<1, 36><<<grid, DENS_THREADS, 0, st>>>(M, ncalls, calls, pairs, cfo, nfo, dc, rhog, ldr);
  else if (nch == 4)
    k_pair_density<4, 96><<<grid, DENS_THREADS, 0, st>>>(M, ncalls, calls, pairs, cfo, nfo, dc, rhog, ldr);
  else
    k_pair_density<10, 156><<<grid, DENS_THREADS, 0, st>>>(M, ncalls, calls, pairs, cfo, nfo, dc, rhog, ldr);
}

}  // namespace flosic
