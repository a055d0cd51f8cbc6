// Dense contractions of the SIC path on the FP64 tensor cores
// (mma.sync.m8n8k4.f64), written for this library in place of library GEMMs:
//
//   k_fo_values  FO values and derivatives on the mesh, Phi_c = B_c C_FO
//                (frmorb_mpi.F:387-397 GORBDRV + DGEMM; FRMIORB/FRMORB2 at the
//                FODs, frmorb2.F:270-286).  The basis values B_c of a block of
//                points are formed in shared memory atom by atom (gorbdrv.f:
//                primitive screen alpha r^2 < CUTEXP, contraction, Cartesian
//                factors and their first and second derivatives) and
//                multiplied into the FO coefficients there, so B never reaches
//                global memory.  Rows of the CTA's product are (channel, point)
//                pairs, columns FOs.
//   k_dgemm      C = alpha op(A) op(B) + beta C for the remaining products:
//                the SIC matrix -Phi^T Y (frmorb_mpi.F:456-517) and the basis-
//                space sums B^T Y with K = mesh points (split over CTAs, the
//                partial products summed in a fixed order by k_dgemm_reduce,
//                so results do not depend on scheduling), and the small
//                products of the FO construction (C_KS TMAT^T, unravel2.f).
//
// Operands are staged in shared memory by 8-byte cp.async with zero fill
// outside the matrices, double buffered; k-major layouts with a row pitch of
// 4 mod 16 doubles keep the fragment loads free of bank conflicts.
#include "kernels.cuh"

namespace flosic {

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// General product
// ---------------------------------------------------------------------------
constexpr int GM = 64, GN = 64, GK = 16;     // CTA tile
constexpr int GLD_M = GM + 4, GLD_N = GN + 4;  // shared pitches (4 mod 16 doubles)
constexpr int G_THREADS = 256;                // 8 warps: 2 along M (32 rows) x 4 along N (16 columns)

template <bool TA, bool TB>
__global__ void __launch_bounds__(G_THREADS) k_dgemm(int M, int N, int K, int kchunk, const double* __restrict__ A,
                                                     int lda, const double* __restrict__ B, int ldb,
                                                     double* __restrict__ out, int ldo, size_t split_stride,
                                                     double alpha, double beta, int direct) {
  __shared__ __align__(16) double As[2][GK][GLD_M];
  __shared__ __align__(16) double Bs[2][GK][GLD_N];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int m0 = blockIdx.x * GM, n0 = blockIdx.y * GN;
  const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  double acc[4][2][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

  auto load = [&](int buf, int k0) {
#pragma unroll
    for (int j = 0; j < (GM * GK) / G_THREADS; ++j) {
      const int e = tid + j * G_THREADS;
      int m, k;
      if (!TA) {
        m = e % GM;
        k = e / GM;
      } else {
        k = e % GK;
        m = e / GK;
      }
      const int gm = m0 + m, gk = k0 + k;
      const bool v = gm < M && gk < ke;
      const double* src = v ? (TA ? A + (size_t)gm * lda + gk : A + (size_t)gk * lda + gm) : A;
      cp_async8(&As[buf][k][m], src, v);
    }
#pragma unroll
    for (int j = 0; j < (GN * GK) / G_THREADS; ++j) {
      const int e = tid + j * G_THREADS;
      int n, k;
      if (TB) {
        n = e % GN;
        k = e / GN;
      } else {
        k = e % GK;
        n = e / GK;
      }
      const int gn = n0 + n, gk = k0 + k;
      const bool v = gn < N && gk < ke;
      const double* src = v ? (TB ? B + (size_t)gk * ldb + gn : B + (size_t)gn * ldb + gk) : B;
      cp_async8(&Bs[buf][k][n], src, v);
    }
    cp_commit();
  };

  const int nk = (ke > kb) ? (ke - kb + GK - 1) / GK : 0;
  if (nk > 0) load(0, kb);
  for (int it = 0; it < nk; ++it) {
    const int buf = it & 1;
    if (it + 1 < nk) {
      load(buf ^ 1, kb + (it + 1) * GK);
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GK; kk += 4) {
      double af[4], bf[2];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) af[mt] = As[buf][kk + (lane & 3)][wm * 32 + mt * 8 + (lane >> 2)];
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) bf[nt] = Bs[buf][kk + (lane & 3)][wn * 16 + nt * 8 + (lane >> 2)];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) dmma(acc[mt][nt][0], acc[mt][nt][1], af[mt], bf[nt]);
    }
    __syncthreads();
  }
  double* o = direct ? out : out + blockIdx.z * split_stride;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int m = m0 + wm * 32 + mt * 8 + (lane >> 2);
        const int n = n0 + wn * 16 + nt * 8 + 2 * (lane & 3) + i;
        if (m >= M || n >= N) continue;
        double* c = o + (size_t)n * ldo + m;
        if (!direct) *c = acc[mt][nt][i];
        else *c = (beta == 0.0) ? alpha * acc[mt][nt][i] : alpha * acc[mt][nt][i] + beta * *c;
      }
}

// C = alpha sum_z W_z + beta C, the partial products summed in split order.
__global__ void k_dgemm_reduce(int M, int N, int nsplit, const double* __restrict__ ws, double alpha, double beta,
                               double* __restrict__ C, int ldc) {
  const size_t MN = (size_t)M * N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < MN; e += (size_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int z = 0; z < nsplit; ++z) s += ws[(size_t)z * MN + e];
    const int n = (int)(e / M), m = (int)(e - (size_t)n * M);
    double* c = C + (size_t)n * ldc + m;
    *c = (beta == 0.0) ? alpha * s : alpha * s + beta * *c;
  }
}

int dgemm_splits(int M, int N, int K) {
  const int tiles = ((M + GM - 1) / GM) * ((N + GN - 1) / GN);
  const int want = (2 * 148 + tiles - 1) / tiles;  // about two CTAs per SM
  const int maxs = (K + 4 * GK - 1) / (4 * GK);    // at least four k-steps per split
  return std::max(1, std::min(want, maxs));
}

size_t dgemm_work(int M, int N, int K) {
  const int s = dgemm_splits(M, N, K);
  return s > 1 ? (size_t)s * M * N : 0;
}

void dgemm(bool ta, bool tb, int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
           double beta, double* C, int ldc, double* work, cudaStream_t st) {
  if (M <= 0 || N <= 0) return;
  const int s = (K > 0) ? dgemm_splits(M, N, K) : 1;
  const int kchunk = (s > 1) ? ((K + s - 1) / s + GK - 1) / GK * GK : std::max(K, 1);
  const int ns = (s > 1) ? (K + kchunk - 1) / kchunk : 1;
  const bool direct = ns == 1;
  dim3 grid((M + GM - 1) / GM, (N + GN - 1) / GN, ns);
  double* out = direct ? C : work;
  const int ldo = direct ? ldc : M;
  const size_t ss = (size_t)M * N;
#define DG(a, b) k_dgemm<a, b><<<grid, G_THREADS, 0, st>>>(M, N, K, kchunk, A, lda, B, ldb, out, ldo, ss, alpha, beta, direct)
  if (!ta && !tb) DG(false, false);
  else if (ta && !tb) DG(true, false);
  else if (!ta && tb) DG(false, true);
  else DG(true, true);
#undef DG
  if (!direct) {
    const int nblk = (int)std::min<size_t>(1024, (ss + 255) / 256);
    k_dgemm_reduce<<<nblk, 256, 0, st>>>(M, N, ns, work, alpha, beta, C, ldc);
  }
}

// out[k * ldo + p] = w[p] a[k * lda + p] (rows scaled by the mesh weights).
__global__ void k_scale_rows(int P, int N, const double* __restrict__ a, int lda, const double* __restrict__ w,
                             double* __restrict__ out, int ldo) {
  const size_t PN = (size_t)P * N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < PN; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / P), p = (int)(e - (size_t)k * P);
    out[(size_t)k * ldo + p] = w[p] * a[(size_t)k * lda + p];
  }
}

void launch_scale_rows(int P, int N, const double* a, int lda, const double* w, double* out, int ldo,
                       cudaStream_t st) {
  const size_t PN = (size_t)P * N;
  if (PN == 0) return;
  k_scale_rows<<<(int)std::min<size_t>(4096, (PN + 255) / 256), 256, 0, st>>>(P, N, a, lda, w, out, ldo);
}

// ---------------------------------------------------------------------------
// Basis values fused with the FO coefficients
// ---------------------------------------------------------------------------
constexpr int FV_BN = 64;                // FOs per CTA
constexpr int FV_KC = 32;                // basis functions per stage (one atom, or a part of one)
constexpr int FV_CONS = 256;             // 8 consumer warps: 4 along the rows x 2 along the FOs (32 columns)
constexpr int FV_PROD = 128;             // 4 producer warps
constexpr int FV_THREADS = FV_CONS + FV_PROD;
constexpr int FV_BAR_FULL = 1, FV_BAR_EMPTY = 3, FV_BAR_PROD = 5;  // named barriers 1-2, 3-4, 5

template <int NDERV>
struct FoValShape {
  static constexpr int NCH = NDERV == 0 ? 1 : (NDERV == 1 ? 4 : 10);
  static constexpr int BP = NDERV == 0 ? 128 : (NDERV == 1 ? 32 : 16);  // points per CTA
  static constexpr int ROWS = NCH * BP;                                 // 128, 128, 160
  static constexpr int MTW = ROWS / 32;                                 // m-tiles per consumer warp
  static constexpr int LDR = ROWS + 4;
};

template <int NDERV>
struct FoValSmem {
  using S = FoValShape<NDERV>;
  double As[2][FV_KC][S::LDR];     // basis values: k = function, row = channel * BP + point
  double Bs[2][FV_KC][FV_BN + 4];  // coefficients: k = function, column = FO
  double g[S::BP][MAX_BARE];       // exp(-alpha r^2) of the atom's bare primitives
  double R[S::BP][3 * MAX_CON][NDERV + 1];  // radial sums per contraction (l, c): sum c g (2 alpha)^d
  double rel[S::BP][3];            // point - atom centre
  double px[S::BP], py[S::BP], pz[S::BP];
  int kpad[2];                     // k rows of the stage in each buffer, -1 = end
  int near[3];                     // per atom (mod 3): some point of the block in range
};

__device__ __forceinline__ void fv_bar_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void fv_bar_arrive(int id, int n) {
  asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "r"(n) : "memory");
}

__constant__ int c_fv_pow[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                                    {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};

// Values (and derivatives) of one contracted Cartesian function at one point
// from its radial sums R0 = sum c g, R1 = sum c g 2 alpha, R2 = sum c g
// (2 alpha)^2 (gorbdrv.f:196-230): the Cartesian factor x^a y^b z^c
// (a, b, c <= 2) and the product rule, written as NCH channels into column k
// of As (channel stride bp).
template <int NDERV>
__device__ __forceinline__ void fv_function(int l, int mu, const double* Rv, const double* xyz, double* col,
                                            int bp) {
  constexpr int NCH = FoValShape<NDERV>::NCH;
  const double R0 = Rv[0], R1 = NDERV > 0 ? Rv[1] : 0.0, R2 = NDERV > 1 ? Rv[2] : 0.0;
  const int shift = (l == 0) ? 0 : (l == 1 ? 1 : 4);
  const int* pw = c_fv_pow[shift + mu];
  const double x = xyz[0], y = xyz[1], z = xyz[2];
  // v^e for e = 0..2, and 0 for e < 0 (derivatives of lower powers)
  auto pw2 = [](double v, int e) -> double { return e < 0 ? 0.0 : (e == 0 ? 1.0 : (e == 1 ? v : v * v)); };
  auto P3 = [&](int a, int b, int cc) -> double { return pw2(x, a) * pw2(y, b) * pw2(z, cc); };
  const int a = pw[0], b = pw[1], cz = pw[2];
  const double P = P3(a, b, cz);
  col[0] = P * R0;
  if (NCH == 1) return;
  const double dP[3] = {a * P3(a - 1, b, cz), b * P3(a, b - 1, cz), cz * P3(a, b, cz - 1)};
#pragma unroll
  for (int d = 0; d < 3; ++d) col[(1 + d) * bp] = dP[d] * R0 - P * xyz[d] * R1;
  if (NCH == 4) return;
  // second derivatives: xx yy zz xy xz yz
  const double d2[6] = {a * (a - 1) * P3(a - 2, b, cz), b * (b - 1) * P3(a, b - 2, cz),
                        cz * (cz - 1) * P3(a, b, cz - 2), a * b * P3(a - 1, b - 1, cz),
                        a * cz * P3(a - 1, b, cz - 1), b * cz * P3(a, b - 1, cz - 1)};
  const int dd[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int d = dd[q][0], e = dd[q][1];
    double v;
    if (d == e) v = d2[q] * R0 - 2.0 * dP[d] * xyz[d] * R1 + P * (xyz[d] * xyz[d] * R2 - R1);
    else v = d2[q] * R0 - dP[e] * xyz[d] * R1 - dP[d] * xyz[e] * R1 + P * xyz[d] * xyz[e] * R2;
    col[(4 + q) * bp] = v;
  }
}

// out[(ch * ncol + k) * ldo + p] = sum_f B_ch(p, f) coef[k * ldc + f] for the
// npts points (px, py, pz) and ncol columns of coef.  Warp specialised: four
// producer warps form the basis values of one atom (or 32 of its functions)
// and its coefficient rows into one of two stage buffers while eight consumer
// warps multiply the other on the FP64 tensor cores.  Stage hand-over by named
// barriers FULL+b (producers arrive, consumers wait) and EMPTY+b (consumers
// arrive, producers wait before refilling); every stage, including the final
// end marker, is waited on exactly once on each side.
template <int NDERV>
__global__ void __launch_bounds__(FV_THREADS, 1)
k_fo_values(BasisDev B, int npts, const double* __restrict__ px, const double* __restrict__ py,
            const double* __restrict__ pz, const double* __restrict__ coef, int ldc, int ncol,
            double* __restrict__ out, size_t ldo) {
  using S = FoValShape<NDERV>;
  extern __shared__ __align__(16) unsigned char fv_raw[];
  FoValSmem<NDERV>& sm = *reinterpret_cast<FoValSmem<NDERV>*>(fv_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p0 = blockIdx.x * S::BP, n0 = blockIdx.y * FV_BN;
  const int np = min(S::BP, npts - p0);
  for (int i = tid; i < S::BP; i += FV_THREADS) {
    const bool v = i < np;
    sm.px[i] = v ? px[p0 + i] : 0.0;
    sm.py[i] = v ? py[p0 + i] : 0.0;
    sm.pz[i] = v ? pz[p0 + i] : 0.0;
  }
  if (tid < 3) sm.near[tid] = 0;
  __syncthreads();

  if (warp >= FV_CONS / 32) {
    // ---------------- producers
    const int pt = tid - FV_CONS;
    int qi = 0;  // stages handed over
    auto begin = [&](int b) {
      if (qi >= 2) fv_bar_sync(FV_BAR_EMPTY + b, FV_THREADS);
    };
    auto finish = [&](int b, int kp) {
      if (pt == 0) sm.kpad[b] = kp;
      fv_bar_arrive(FV_BAR_FULL + b, FV_THREADS);
      ++qi;
    };
    for (int a = 0; a < B.natoms; ++a) {
      const int t = B.atom_type[a];
      const double ax = B.atom_pos[3 * a], ay = B.atom_pos[3 * a + 1], az = B.atom_pos[3 * a + 2];
      const double amin = B.type_amin[t];
      // primitive screen of the whole atom (gorbdrv.f:186-195): skipped when no
      // point of the block is in range (all its values are then zero)
      bool near = false;
      for (int i = pt; i < np; i += FV_PROD) {
        const double x = sm.px[i] - ax, y = sm.py[i] - ay, z = sm.pz[i] - az;
        if ((x * x + y * y + z * z) * amin < CUTEXP) near = true;
      }
      if (near) atomicOr(&sm.near[a % 3], 1);
      if (pt == 0) sm.near[(a + 1) % 3] = 0;
      fv_bar_sync(FV_BAR_PROD, FV_PROD);  // also: every producer is done with g of the previous atom
      if (!sm.near[a % 3]) continue;
      const int nbare = B.type_nbare[t];
      for (int e = pt; e < S::BP * MAX_BARE; e += FV_PROD) {
        const int i = e / MAX_BARE, ib = e - i * MAX_BARE;
        const double x = sm.px[i] - ax, y = sm.py[i] - ay, z = sm.pz[i] - az;
        const double r2 = x * x + y * y + z * z;
        double v = 0.0;
        if (i < np && ib < nbare && r2 * amin < CUTEXP) {
          const double rex = B.type_alpha[t * MAX_BARE + ib] * r2;
          v = (rex < CUTEXP) ? exp(-rex) : 0.0;
        }
        sm.g[i][ib] = v;
        if (ib == 0) {
          sm.rel[i][0] = x;
          sm.rel[i][1] = y;
          sm.rel[i][2] = z;
        }
      }
      fv_bar_sync(FV_BAR_PROD, FV_PROD);
      // radial sums of every contraction (l, c) at every point, once per atom
      const int lmax = B.type_lmax[t];
      const int nc0 = B.type_ncon[t * 3], nc1 = lmax >= 1 ? B.type_ncon[t * 3 + 1] : 0;
      const int nc2 = lmax >= 2 ? B.type_ncon[t * 3 + 2] : 0;
      const int nlc = nc0 + nc1 + nc2;
      const double* alp = B.type_alpha + t * MAX_BARE;
      for (int e = pt; e < S::BP * nlc; e += FV_PROD) {
        const int lc = e / S::BP, i = e - lc * S::BP;
        const int l = lc < nc0 ? 0 : (lc < nc0 + nc1 ? 1 : 2);
        const int c = lc - (l == 0 ? 0 : (l == 1 ? nc0 : nc0 + nc1));
        const double* con = B.type_bfcon + ((size_t)(t * 3 + l) * MAX_CON + c) * MAX_BARE;
        double R0 = 0.0, R1 = 0.0, R2 = 0.0;
        for (int ib = 0; ib < nbare; ++ib) {
          const double cg = con[ib] * sm.g[i][ib];
          R0 += cg;
          if (NDERV > 0) {
            const double a2 = 2.0 * alp[ib];
            R1 += cg * a2;
            if (NDERV > 1) R2 += cg * a2 * a2;
          }
        }
        sm.R[i][lc][0] = R0;
        if (NDERV > 0) sm.R[i][lc][1] = R1;
        if (NDERV > 1) sm.R[i][lc][2] = R2;
      }
      fv_bar_sync(FV_BAR_PROD, FV_PROD);
      // the atom's functions: l-major, then Cartesian component, then contraction
      const int nfa = nc0 + 3 * nc1 + 6 * nc2;
      const int b0 = B.atom_boff[a];
      for (int f0 = 0; f0 < nfa; f0 += FV_KC) {
        const int nfc = min(FV_KC, nfa - f0), kp = (nfc + 3) & ~3;
        const int b = qi & 1;
        begin(b);
        for (int e = pt; e < S::BP * kp; e += FV_PROD) {
          const int fi = e / S::BP, i = e - fi * S::BP;
          double* col = &sm.As[b][fi][i];
          if (fi >= nfc) {
#pragma unroll
            for (int ch = 0; ch < S::NCH; ++ch) col[ch * S::BP] = 0.0;
            continue;
          }
          int f = f0 + fi, l, lc0, ncon;
          if (f < nc0) {
            l = 0;
            lc0 = 0;
            ncon = nc0;
          } else if (f < nc0 + 3 * nc1) {
            f -= nc0;
            l = 1;
            lc0 = nc0;
            ncon = nc1;
          } else {
            f -= nc0 + 3 * nc1;
            l = 2;
            lc0 = nc0 + nc1;
            ncon = nc2;
          }
          const int mu = f / ncon, c = f - mu * ncon;
          fv_function<NDERV>(l, mu, sm.R[i][lc0 + c], sm.rel[i], col, S::BP);
        }
        for (int e = pt; e < kp * FV_BN; e += FV_PROD) {
          const int n = e / kp, fi = e - n * kp;
          const bool v = fi < nfc && n0 + n < ncol;
          sm.Bs[b][fi][n] = v ? coef[(size_t)(n0 + n) * ldc + b0 + f0 + fi] : 0.0;
        }
        finish(b, kp);
      }
    }
    // end marker, then release of the last two stages
    {
      const int b = qi & 1;
      begin(b);
      finish(b, -1);
      for (int j = max(qi - 2, 0); j < qi; ++j) fv_bar_sync(FV_BAR_EMPTY + (j & 1), FV_THREADS);
    }
  } else {
    // ---------------- consumers
    const int wr = warp & 3, wc = warp >> 2;
    double acc[S::MTW][4][2];
#pragma unroll
    for (int x = 0; x < S::MTW; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) acc[x][y][0] = acc[x][y][1] = 0.0;
    for (int qi = 0;; ++qi) {
      const int b = qi & 1;
      fv_bar_sync(FV_BAR_FULL + b, FV_THREADS);
      const int kp = sm.kpad[b];
      for (int kk = 0; kk < kp; kk += 4) {
        double af[S::MTW], bf[4];
#pragma unroll
        for (int mt = 0; mt < S::MTW; ++mt) af[mt] = sm.As[b][kk + (lane & 3)][(wr * S::MTW + mt) * 8 + (lane >> 2)];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) bf[nt] = sm.Bs[b][kk + (lane & 3)][wc * 32 + nt * 8 + (lane >> 2)];
#pragma unroll
        for (int mt = 0; mt < S::MTW; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt][0], acc[mt][nt][1], af[mt], bf[nt]);
      }
      fv_bar_arrive(FV_BAR_EMPTY + b, FV_THREADS);
      if (kp < 0) break;
    }
#pragma unroll
    for (int mt = 0; mt < S::MTW; ++mt) {
      const int row = (wr * S::MTW + mt) * 8 + (lane >> 2);
      const int ch = row / S::BP, i = row - ch * S::BP;
      if (i >= np) continue;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int k = n0 + wc * 32 + nt * 8 + 2 * (lane & 3) + j;
          if (k < ncol) out[((size_t)ch * ncol + k) * ldo + p0 + i] = acc[mt][nt][j];
        }
    }
  }
}

template <int NDERV>
static cudaError_t fo_values_attr() {
  return cudaFuncSetAttribute(k_fo_values<NDERV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sizeof(FoValSmem<NDERV>));
}

cudaError_t init_contract() {
  cudaError_t e = fo_values_attr<0>();
  if (e == cudaSuccess) e = fo_values_attr<1>();
  if (e == cudaSuccess) e = fo_values_attr<2>();
  return e;
}

void launch_fo_values(const BasisDev& B, int nderv, int npts, const double* px, const double* py, const double* pz,
                      const double* coef, int ldc, int ncol, double* out, size_t ldo, cudaStream_t st) {
  if (npts <= 0 || ncol <= 0) return;
#define FV(D)                                                                                           \
  k_fo_values<D><<<dim3((npts + FoValShape<D>::BP - 1) / FoValShape<D>::BP, (ncol + FV_BN - 1) / FV_BN), \
                   FV_THREADS, sizeof(FoValSmem<D>), st>>>(B, npts, px, py, pz, coef, ldc, ncol, out, ldo)
  if (nderv == 0) FV(0);
  else if (nderv == 1) FV(1);
  else FV(2);
#undef FV
}

}  // namespace flosic
