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
constexpr int FV_KC = 32;                // basis functions per stage (one atom, or a part of one)
constexpr int FV_CONS = 256;             // 8 consumer warps, 32 FO columns each
constexpr int FV_PROD = 256;             // 8 producer warps
constexpr int FV_THREADS = FV_CONS + FV_PROD;
constexpr int FV_BAR_FULL = 1, FV_BAR_EMPTY = 3, FV_BAR_PROD = 5;  // named barriers 1-2, 3-4, 5

// A CTA's product: ROWS = NCH x BP rows of (channel, point) by BN FO columns.
// BN = 64: 4 warp rows x 2 warp columns; BN = 128: half the points, 2 x 4, so
// each point's basis values serve 128 FOs (formed once for up to 128 FOs).
template <int NDERV, int BN>
struct FoValShape {
  static constexpr int NCH = NDERV == 0 ? 1 : (NDERV == 1 ? 4 : 10);
  static constexpr int BP0 = NDERV == 0 ? 128 : (NDERV == 1 ? 32 : 16);
  static constexpr int BP = BN == 64 ? BP0 : BP0 / 2;  // points per CTA
  static constexpr int ROWS = NCH * BP;                 // 128/128/160 (BN 64), 64/64/80 (BN 128)
  static constexpr int WR = BN == 64 ? 4 : 2;           // consumer warps along the rows
  static constexpr int MTW = ROWS / 8 / WR;             // m-tiles per consumer warp
  static constexpr int LDR = ROWS + 4;
  static constexpr int GA = BP <= 32 ? 4 : 2;           // atoms per stage at most (their exponentials in smem)
};

template <int NDERV, int BN>
struct FoValSmem {
  using S = FoValShape<NDERV, BN>;
  double As[2][FV_KC][S::LDR];     // basis values: k = function, row = channel * BP + point
  double Bs[3][FV_KC][BN + 4];     // coefficients: k = function, column = FO (stage qi in Bs[qi % 3])
  double g[S::GA][S::BP][MAX_BARE];  // exp(-alpha r^2) of each stage atom's bare primitives
  double rel[S::GA][S::BP][3];       // point - atom centre
  double px[S::BP], py[S::BP], pz[S::BP];
  int kpad[2];                     // k rows of the stage in each buffer, -1 = end
  unsigned near[3];                // per window of atoms (mod 3): bit j set when atom j has a point in range
};

__device__ __forceinline__ void fv_bar_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void fv_bar_arrive(int id, int n) {
  asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "r"(n) : "memory");
}

__constant__ int c_fv_pow[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                                    {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};

// Values (and derivatives) of one contracted Cartesian function x^a y^b z^cz
// (a, b, cz <= 2) at one point from its radial sums R0 = sum c g, R1 = sum
// c g 2 alpha, R2 = sum c g (2 alpha)^2 (gorbdrv.f:196-230), by the product
// rule, written as NCH channels into column col of As (channel stride bp).
// Called with powers known at compile time, so the polynomial code folds.
template <int NDERV>
__device__ __forceinline__ void fv_function(int a, int b, int cz, double R0, double R1, double R2,
                                            const double* xyz, double* col, int bp) {
  constexpr int NCH = NDERV == 0 ? 1 : (NDERV == 1 ? 4 : 10);
  const double x = xyz[0], y = xyz[1], z = xyz[2];
  // v^e for e = 0..2, and 0 for e < 0 (derivatives of lower powers)
  auto pw2 = [](double v, int e) -> double { return e < 0 ? 0.0 : (e == 0 ? 1.0 : (e == 1 ? v : v * v)); };
  auto P3 = [&](int i, int j, int k) -> double { return pw2(x, i) * pw2(y, j) * pw2(z, k); };
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

// The Cartesian components of one contraction of angular momentum L (s; x y z;
// xx yy zz xy xz yz, the order of gorbdrv.f) whose function index lies in the
// stage: component mu is function fbase + mu * ncon of the stage.
template <int NDERV, int L>
__device__ __forceinline__ void fv_contraction(double R0, double R1, double R2, const double* xyz, double* As_b,
                                               int ldr, int bp, int i, int fbase, int ncon, int nfc) {
  constexpr int NCOMP = L == 0 ? 1 : (L == 1 ? 3 : 6);
  constexpr int SHIFT = L == 0 ? 0 : (L == 1 ? 1 : 4);
  constexpr int PW[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                             {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
#pragma unroll
  for (int mu = 0; mu < NCOMP; ++mu) {
    const int fi = fbase + mu * ncon;
    if (fi < 0 || fi >= nfc) continue;
    fv_function<NDERV>(PW[SHIFT + mu][0], PW[SHIFT + mu][1], PW[SHIFT + mu][2], R0, R1, R2, xyz,
                       As_b + (size_t)fi * ldr + i, bp);
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
template <int NDERV, int BN>
__global__ void __launch_bounds__(FV_THREADS, 1)
k_fo_values(BasisDev B, int npts, const double* __restrict__ px, const double* __restrict__ py,
            const double* __restrict__ pz, const double* __restrict__ coef, int ldc, int ncol,
            double* __restrict__ out, size_t ldo) {
  using S = FoValShape<NDERV, BN>;
  extern __shared__ __align__(16) unsigned char fv_raw[];
  FoValSmem<NDERV, BN>& sm = *reinterpret_cast<FoValSmem<NDERV, BN>*>(fv_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p0 = blockIdx.x * S::BP, n0 = blockIdx.y * BN;
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
    // The atoms go to the tensor cores in stages of up to 32 basis functions:
    // consecutive atoms that some point of the block reaches (primitive
    // screen of gorbdrv.f:186-195; the others' values are all zero) are
    // packed into one stage while they fit, at most GA of them; an atom with
    // more than 32 functions takes stages of its own, 32 functions each.
    constexpr int GA = S::GA;
    struct Member {
      int atom, type, nbare, nc0, nc1, nc2, nfa, boff, off;
      double ax, ay, az, amin;
    };
    auto member = [&](int at) {
      Member m;
      m.atom = at;
      m.type = B.atom_type[at];
      const int t = m.type, lmax = B.type_lmax[t];
      m.nbare = B.type_nbare[t];
      m.nc0 = B.type_ncon[t * 3];
      m.nc1 = lmax >= 1 ? B.type_ncon[t * 3 + 1] : 0;
      m.nc2 = lmax >= 2 ? B.type_ncon[t * 3 + 2] : 0;
      m.nfa = m.nc0 + 3 * m.nc1 + 6 * m.nc2;
      m.boff = B.atom_boff[at];
      m.off = 0;
      m.ax = B.atom_pos[3 * at];
      m.ay = B.atom_pos[3 * at + 1];
      m.az = B.atom_pos[3 * at + 2];
      m.amin = B.type_amin[t];
      return m;
    };
    // coefficient rows of the stage (function fi of the stage is row
    // row_of(fi) of coef) into Bs[qi % 3] by cp.async (zero outside the
    // matrix); issued early so their latency overlaps the basis values.
    // Bs[qi % 3] was last read by stage qi - 3, which the consumers released
    // before the producers passed begin() of stage qi - 1.
    auto fetch_coef = [&](int q, int nfc, int kp, auto row_of) {
      for (int e = pt; e < kp * BN; e += FV_PROD) {
        const int n = e / kp, fi = e - n * kp;
        const bool v = fi < nfc && n0 + n < ncol;
        cp_async8(&sm.Bs[q % 3][fi][n], v ? coef + (size_t)(n0 + n) * ldc + row_of(fi) : coef, v);
      }
      cp_commit();
    };
    // exp(-alpha r^2) of member slot ms at the block's points
    auto exps = [&](int ms, const Member& m) {
      for (int e = pt; e < S::BP * m.nbare; e += FV_PROD) {
        const int i = e / m.nbare, ib = e - i * m.nbare;
        const double x = sm.px[i] - m.ax, y = sm.py[i] - m.ay, z = sm.pz[i] - m.az;
        const double r2 = x * x + y * y + z * z;
        double v = 0.0;
        if (i < np && r2 * m.amin < CUTEXP) {
          const double rex = B.type_alpha[m.type * MAX_BARE + ib] * r2;
          v = (rex < CUTEXP) ? exp(-rex) : 0.0;
        }
        sm.g[ms][i][ib] = v;
        if (ib == 0) {
          sm.rel[ms][i][0] = x;
          sm.rel[ms][i][1] = y;
          sm.rel[ms][i][2] = z;
        }
      }
    };
    // one item per (point, contraction of member slot ms): its radial sums,
    // then the components whose stage column fbase + mu * ncon lies in [0, nfc)
    auto item = [&](int ms, const Member& m, int lc, int i, int f0, double* As_b, int nfc) {
      const int l = lc < m.nc0 ? 0 : (lc < m.nc0 + m.nc1 ? 1 : 2);
      const int c = lc - (l == 0 ? 0 : (l == 1 ? m.nc0 : m.nc0 + m.nc1));
      const double* con = B.type_bfcon + ((size_t)(m.type * 3 + l) * MAX_CON + c) * MAX_BARE;
      const double* alp = B.type_alpha + m.type * MAX_BARE;
      double R0 = 0.0, R1 = 0.0, R2 = 0.0;
      for (int ib = 0; ib < m.nbare; ++ib) {
        const double cg = con[ib] * sm.g[ms][i][ib];
        R0 += cg;
        if (NDERV > 0) {
          const double a2 = 2.0 * alp[ib];
          R1 += cg * a2;
          if (NDERV > 1) R2 += cg * a2 * a2;
        }
      }
      const int base = m.off - f0;
      if (l == 0) fv_contraction<NDERV, 0>(R0, R1, R2, sm.rel[ms][i], As_b, S::LDR, S::BP, i, base + c, m.nc0, nfc);
      else if (l == 1)
        fv_contraction<NDERV, 1>(R0, R1, R2, sm.rel[ms][i], As_b, S::LDR, S::BP, i, base + m.nc0 + c, m.nc1, nfc);
      else
        fv_contraction<NDERV, 2>(R0, R1, R2, sm.rel[ms][i], As_b, S::LDR, S::BP, i, base + m.nc0 + 3 * m.nc1 + c,
                                 m.nc2, nfc);
    };
    auto pad_rows = [&](int b, int nfc, int kp) {  // zero rows up to the k-step of 4
      for (int e = pt; e < S::BP * (kp - nfc); e += FV_PROD) {
        const int fi = nfc + e / S::BP, i = e % S::BP;
#pragma unroll
        for (int ch = 0; ch < S::NCH; ++ch) sm.As[b][fi][ch * S::BP + i] = 0.0;
      }
    };
    int win = 0;
    for (int a = 0; a < B.natoms;) {
      // screen the window a .. a + GA - 1; every producer passed the previous
      // stage's items, so g and rel may be rewritten after this barrier
      const int wn = min(GA, B.natoms - a);
      unsigned bits = 0;
      for (int j = 0; j < wn; ++j) {
        const int at = a + j;
        const int t = B.atom_type[at];
        const double ax = B.atom_pos[3 * at], ay = B.atom_pos[3 * at + 1], az = B.atom_pos[3 * at + 2];
        const double amin = B.type_amin[t];
        for (int i = pt; i < np; i += FV_PROD) {
          const double x = sm.px[i] - ax, y = sm.py[i] - ay, z = sm.pz[i] - az;
          if ((x * x + y * y + z * z) * amin < CUTEXP) bits |= 1u << j;
        }
      }
      if (bits) atomicOr(&sm.near[win % 3], bits);
      if (pt == 0) sm.near[(win + 1) % 3] = 0u;
      fv_bar_sync(FV_BAR_PROD, FV_PROD);
      const unsigned mask = sm.near[win % 3];
      ++win;
      // the stage's atoms (the same on every producer)
      Member mem[GA];
      int ng = 0, tot = 0, next = a + wn;
      bool big = false;
      for (int j = 0; j < wn; ++j) {
        if (!((mask >> j) & 1u)) continue;
        Member m = member(a + j);
        if (m.nfa > FV_KC) {
          if (ng == 0) {
            mem[0] = m;
            ng = 1;
            big = true;
            next = a + j + 1;
          } else {
            next = a + j;
          }
          break;
        }
        if (tot + m.nfa > FV_KC) {
          next = a + j;
          break;
        }
        m.off = tot;
        tot += m.nfa;
        mem[ng++] = m;
      }
      a = next;
      if (ng == 0) continue;
      if (big) {
        const Member& m = mem[0];
        const int nlc = m.nc0 + m.nc1 + m.nc2;
        fetch_coef(qi, min(FV_KC, m.nfa), (min(FV_KC, m.nfa) + 3) & ~3, [&](int fi) { return m.boff + fi; });
        exps(0, m);
        fv_bar_sync(FV_BAR_PROD, FV_PROD);
        for (int f0 = 0; f0 < m.nfa; f0 += FV_KC) {
          const int nfc = min(FV_KC, m.nfa - f0), kp = (nfc + 3) & ~3;
          const int b = qi & 1;
          if (f0 > 0) fetch_coef(qi, nfc, kp, [&](int fi) { return m.boff + f0 + fi; });
          begin(b);
          double* As_b = &sm.As[b][0][0];
          for (int e = pt; e < S::BP * nlc; e += FV_PROD) item(0, m, e / S::BP, e % S::BP, f0, As_b, nfc);
          pad_rows(b, nfc, kp);
          cp_wait<0>();  // this thread's coefficient copies have landed
          finish(b, kp);
        }
        continue;
      }
      const int kp = (tot + 3) & ~3;
      fetch_coef(qi, tot, kp, [&](int fi) {
        int k = 0;
        while (k + 1 < ng && fi >= mem[k + 1].off) ++k;
        return mem[k].boff + fi - mem[k].off;
      });
      for (int k = 0; k < ng; ++k) exps(k, mem[k]);
      fv_bar_sync(FV_BAR_PROD, FV_PROD);
      const int b = qi & 1;
      begin(b);
      double* As_b = &sm.As[b][0][0];
      // all members' items in one range, so that every producer has work
      int start[GA + 1];
      start[0] = 0;
      for (int k = 0; k < ng; ++k) start[k + 1] = start[k] + S::BP * (mem[k].nc0 + mem[k].nc1 + mem[k].nc2);
      for (int e = pt; e < start[ng]; e += FV_PROD) {
        int k = 0;
        while (e >= start[k + 1]) ++k;
        const int r = e - start[k];
        item(k, mem[k], r / S::BP, r % S::BP, 0, As_b, tot);
      }
      pad_rows(b, tot, kp);
      cp_wait<0>();
      finish(b, kp);
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
    const int wr = warp % S::WR, wc = warp / S::WR;
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
        for (int nt = 0; nt < 4; ++nt) bf[nt] = sm.Bs[qi % 3][kk + (lane & 3)][wc * 32 + nt * 8 + (lane >> 2)];
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

template <int NDERV, int BN>
static cudaError_t fo_values_attr() {
  return cudaFuncSetAttribute(k_fo_values<NDERV, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sizeof(FoValSmem<NDERV, BN>));
}

cudaError_t init_contract() {
  cudaError_t e = fo_values_attr<0, 64>();
  if (e == cudaSuccess) e = fo_values_attr<1, 64>();
  if (e == cudaSuccess) e = fo_values_attr<2, 64>();
  if (e == cudaSuccess) e = fo_values_attr<0, 128>();
  if (e == cudaSuccess) e = fo_values_attr<1, 128>();
  if (e == cudaSuccess) e = fo_values_attr<2, 128>();
  return e;
}

void launch_fo_values(const BasisDev& B, int nderv, int npts, const double* px, const double* py, const double* pz,
                      const double* coef, int ldc, int ncol, double* out, size_t ldo, int bn, cudaStream_t st) {
  if (npts <= 0 || ncol <= 0) return;
#define FV(D, W)                                                                                            \
  k_fo_values<D, W><<<dim3((npts + FoValShape<D, W>::BP - 1) / FoValShape<D, W>::BP, (ncol + W - 1) / W), \
                      FV_THREADS, sizeof(FoValSmem<D, W>), st>>>(B, npts, px, py, pz, coef, ldc, ncol, out, ldo)
  if (bn == 128) {
    if (nderv == 0) FV(0, 128);
    else if (nderv == 1) FV(1, 128);
    else FV(2, 128);
  } else {
    if (nderv == 0) FV(0, 64);
    else if (nderv == 1) FV(1, 64);
    else FV(2, 64);
  }
#undef FV
}

}  // namespace flosic
