// Coulomb potential of all FOs at all mesh points, FP64 tensor-core form.
//
// For one POISSON1 call (a batch of Gaussian pairs, poisson1.f:611-1098) the
// potential of FO k at mesh point p is, at points inside RCUT of the call's
// centre CG (near points),
//     sum_{pair q} sum_{t<46} COEF[q][k][t] * G[q][t][p],
//     G[q][t][p] = F_{m(t)}(delta_q |p-C_q|^2) * mono_t(p - C_q),
// and at the other points (far points, NPOT=2) the L<=6 multipole expansion
//     sum_{lm} MV[c][k][lm] * H[c][lm][p],  H = Y_lm(u) / r^(l+1),  u = (p-CG)/r
// (poisson1.f:1224-1600), MV being the normalised moments.  COEF and MV depend
// on the FO, G and H only on geometry.  Two kernels evaluate it:
//
//   k_coulomb_shared  calls whose CG, RCUT and NPOT are the same for every FO
//                     (every single-pair call with NSPN=1: CG is the pair
//                     centre).  Near/far is then a property of the point alone,
//                     so G (near points) and H (far points) are built once per
//                     (call, point) with the other points' columns zeroed, and
//                     both are segments of ONE GEMM  V[k][p] += A[k][:] B[:][p]
//                     over all such calls, on the FP64 tensor cores
//                     (mma.sync m8n8k4 .f64).  A CTA owns 128 points and up to
//                     128 FOs.
//   k_coulomb_perfo   the remaining calls, whose CG (charge weighted,
//                     poisson1.f:503-520) differs per FO: the near field of the
//                     FOs with near points in the tile as a GEMM over compacted
//                     FO slots, added per (FO, point); the far field per
//                     (FO, point).
//
// Both near-field GEMMs run warp specialised: producer warps build the G / H
// columns and copy the A rows (cp.async) into double-buffered shared memory,
// packing consecutive segments into stages of up to 52 rows, while consumer
// warps keep the accumulators and issue only the tensor-core MMAs.
//
// Both walk their calls in order, so every per-point sum is deterministic.
// Both count the evaluations they perform: near (pair, point, FO), far
// (call, point, FO) and the multipole terms the far evaluations keep, the
// units of the reference's POISSON1 work.
#include "coulomb_common.cuh"

namespace flosic {

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// G column of one (pair, point) in the COEFICIENT slot order: slot t holds
// F_{m(t)} * POLY(mono(t)), monomials in the order of poisson1.f:925-959.
// Rows >= kn (16, 32 or 48) are not written.
template <typename T>
__device__ __forceinline__ void write_g(double* g, int kn, T x, T y, T z, const T F[5]) {
#define GW(t, v) g[(size_t)(t) * G_LD] = (double)(v)
  const T F0 = F[0], F1 = F[1], F2 = F[2], F3 = F[3], F4 = F[4];
  const T zz = z * z, yz = y * z, yy = y * y, xz = x * z, xy = x * y, xx = x * x;
  GW(0, F0);
  GW(1, F1);
  GW(2, F2);
  GW(3, F1 * z);
  GW(4, F1 * y);
  GW(5, F1 * x);
  GW(6, F2 * z);
  GW(7, F2 * y);
  GW(8, F2 * x);
  GW(9, F2 * zz);
  GW(10, F2 * yz);
  GW(11, F2 * yy);
  GW(12, F2 * xz);
  GW(13, F2 * xy);
  GW(14, F2 * xx);
  GW(15, F3 * zz);
  if (kn <= 16) return;
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
  if (kn <= 32) return;
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
  GW(46, T(0));
  GW(47, T(0));
#undef GW
}

__device__ __forceinline__ void zero_rows(double* g, int k) {
  for (int t = 0; t < k; ++t) g[(size_t)t * G_LD] = 0.0;
}

// ---------------------------------------------------------------------------
// Warp-specialised pipeline
// ---------------------------------------------------------------------------
// Eight consumer warps hold the accumulators and only multiply; four producer
// warps build the B columns (one point per thread), issue the cp.async copies
// of the A rows and pack consecutive segments into stages of at most KSEG rows.
// Stages are double buffered; buffer b is handed over through named barriers
// FULL+b (producers arrive, consumers wait) and EMPTY+b (consumers arrive,
// producers wait before refilling).  Every stage, including a final marker
// stage of -1 rows that ends the consumers' loop, is waited on exactly once on
// each side, so every barrier phase collects all WS_THREADS arrivals.
constexpr int CONS_WARPS = 8;
constexpr int PROD_WARPS = 4;
constexpr int NCONS = 32 * CONS_WARPS;
constexpr int NPROD = 32 * PROD_WARPS;
constexpr int WS_THREADS = NCONS + NPROD;   // 384
constexpr int PTS_PER_PROD = TILE / NPROD;  // 1
constexpr int BAR_FULL = 1, BAR_EMPTY = 3;  // named barrier ids 1,2 and 3,4 (0 is __syncthreads)

__device__ __forceinline__ void named_sync(int id) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(WS_THREADS) : "memory");
}
__device__ __forceinline__ void named_arrive(int id) {
  asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "r"(WS_THREADS) : "memory");
}

// Producer side of the stage hand-over.
struct StagePacker {
  int qi = 0;        // stages handed over so far
  int rows = 0;      // rows of the open stage
  int b = 0;         // its buffer
  bool open = false;
  __device__ void begin() {
    b = qi & 1;
    if (qi >= 2) named_sync(BAR_EMPTY + b);
    rows = 0;
    open = true;
  }
  __device__ void finish(int* stage_rows, int r, bool leader) {
    cp_async_wait_all();
    if (leader) stage_rows[b] = r;
    named_arrive(BAR_FULL + b);
    ++qi;
    open = false;
  }
  // Offset of a segment of r rows, closing the open stage when it is full.
  __device__ int place(int* stage_rows, int r, bool leader) {
    if (open && rows + r > KSEG) finish(stage_rows, rows, leader);
    if (!open) begin();
    const int off = rows;
    rows += r;
    return off;
  }
  // Close the last stage, hand over the end marker, and wait until the
  // consumers have released the last two stages.
  __device__ void end(int* stage_rows, bool leader) {
    if (open) finish(stage_rows, rows, leader);
    begin();
    finish(stage_rows, -1, leader);
    for (int j = max(qi - 2, 0); j < qi; ++j) named_sync(BAR_EMPTY + (j & 1));
  }
};

// Copy the first `rows` doubles of nrow rows (global row i at src_row(i), shared
// row dst_row(i) with stride KSEG, column offset off) with 16-byte cp.async,
// work split over the producer threads.
template <typename SrcRow, typename DstRow>
__device__ __forceinline__ void copy_rows(double* dst, int off, int nrow, int rows, int pt, SrcRow src_row,
                                          DstRow dst_row) {
  const int cpr = rows >> 1;  // 16-byte chunks per row
  if (cpr == 0) return;
  int r = pt / cpr, ch = pt - r * cpr;
  const int dr = NPROD / cpr, dc = NPROD - dr * cpr;
  for (int e = pt; e < nrow * cpr; e += NPROD) {
    cp_async16(dst + (size_t)dst_row(r) * KSEG + off + 2 * ch, src_row(r) + 2 * ch);
    r += dr;
    ch += dc;
    if (ch >= cpr) {
      ch -= cpr;
      ++r;
    }
  }
}

// Consumer MMA over one stage: V[k][p] += A[k][0:rows] B[0:rows][p] for the
// warp's 32 x WPTS tile; m-tiles with mt_active false are skipped.
template <int NT>
__device__ __forceinline__ void stage_mma(double (&V)[4][NT][2], const double* __restrict__ As,
                                          const double* __restrict__ Bs, int rows, const bool (&mt_active)[4]) {
  for (int kk = 0; kk < rows; kk += 4) {
    double af[4];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) af[mt] = As[mt * 8 * KSEG + kk];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const double bf = Bs[(size_t)kk * G_LD + nt * 8];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
        if (mt_active[mt]) dmma884(V[mt][nt][0], V[mt][nt][1], af[mt], bf);
    }
  }
}

template <typename T>
__device__ __forceinline__ void write_h(double* g, int kf, T dx, T dy, T dz, T r2) {
  T hn;
  if constexpr (sizeof(T) == 8) hn = 1.0 / sqrt(r2);
  else hn = rsqrtf(r2);
  const int lmx = far_degree(kf);
  T rec[LM + 1];
  rec[0] = hn;
#pragma unroll
  for (int l = 1; l <= LM; ++l) rec[l] = rec[l - 1] * hn;
  harmonics_mmajor(hn * dx, hn * dy, hn * dz, lmx,
                   [&](int row, int l, T v) { g[(size_t)row * G_LD] = (double)(v * rec[l]); });
  for (int t = (lmx + 1) * (lmx + 1); t < kf; ++t) g[(size_t)t * G_LD] = 0.0;
}

// G column of one near point of pair pg (rows [0, kn)).
template <typename T>
__device__ __forceinline__ void write_g_point(double* g, int kn, const PairGeo& pg, double x, double y, double z,
                                              const double* __restrict__ boys_tab) {
  const T rx = T(x - pg.C[0]), ry = T(y - pg.C[1]), rz = T(z - pg.C[2]);
  const T xx = T(pg.delta) * (rz * rz + ry * ry + rx * rx);
  T ex;
  if constexpr (sizeof(T) == 8) ex = exp(-xx);
  else ex = expf(-xx);
  T F[5];
  boys_fmt<T>(boys_tab, xx, ex, kn >= 48 ? 5 : (kn == 32 ? 4 : 3), F);
  write_g<T>(g, kn, rx, ry, rz, F);
}

// ---------------------------------------------------------------------------
// Shared-geometry calls
// ---------------------------------------------------------------------------
template <int WM>
struct SharedSmem {
  double A[2][32 * WM * KSEG];  // FO rows of the stage's coefficients / moments
  double B[2][KSEG * G_LD];     // G or H columns
  double px[TILE], py[TILE], pz[TILE];
  int rows[2];                  // rows of the stage in each buffer, -1 = end
};

// One (tile, FO block) of the shared-geometry calls; the body of
// k_coulomb_shared (one CTA per item) and of k_coulomb_shared_batch
// (persistent CTAs over the items of many molecules).
template <int WM, bool MIXED>
__device__ __forceinline__ void shared_tile(int tile, int fob, int ncalls, const int* __restrict__ lists,
                                            const CallShare* __restrict__ share, const CallInfo* __restrict__ calls,
                                            int nfo, const double* __restrict__ coef,
                                            const int8_t* __restrict__ pair_fmt, const PairGeo* __restrict__ pairs,
                                            const double* __restrict__ momv, const MeshDev& M,
                                            const double* __restrict__ boys_tab, double* __restrict__ vh, int ldv,
                                            unsigned long long* __restrict__ cnt) {
  constexpr int FOB = 32 * WM, WN = CONS_WARPS / WM, WPTS = TILE / WN, NT = WPTS / 8;
  using PT = typename std::conditional<MIXED, float, double>::type;  // producer arithmetic
  extern __shared__ __align__(128) unsigned char smraw[];
  SharedSmem<WM>& S = *reinterpret_cast<SharedSmem<WM>*>(smraw);
  const int k0 = fob * FOB;
  const int nk = min(FOB, nfo - k0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p0 = tile * TILE;
  const int np = min(TILE, M.n - p0);
  for (int i = tid; i < TILE; i += WS_THREADS) {
    const bool a = i < np;
    S.px[i] = a ? M.x[p0 + i] : 0.0;
    S.py[i] = a ? M.y[p0 + i] : 0.0;
    S.pz[i] = a ? M.z[p0 + i] : 0.0;
  }
  __syncthreads();
  unsigned long long my_near = 0, my_far = 0, my_terms = 0;

  if (warp >= CONS_WARPS) {
    // ---- producers
    const int pt = tid - NCONS;
    const bool leader = pt == 0;
    const bool count_terms = fob == 0;  // kept terms are summed over all FOs once per (call, point)
    SegmentWalker W;
    W.list = lists;
    W.n = lists[2 * ncalls];
    W.share = share;
    W.calls = calls;
    W.pair_fmt = pair_fmt;
    for (int d = 0; d < 3; ++d) {
      W.lo[d] = M.tile_lo[3 * tile + d];
      W.hi[d] = M.tile_hi[3 * tile + d];
    }
    W.li = 0;
    W.sub = -1;
    W.c = W.p0 = W.np = W.cls = W.kf = W.ksum = 0;
    W.npot = 1;
    W.cx = W.cy = W.cz = W.rc2 = 0.0;
    StagePacker P;
    Segment s;
    while (W.next(s)) {
      if (s.rows == 0) {
        // far segment of a call whose FOs keep no multipole term: count only
        for (int j = 0; j < PTS_PER_PROD; ++j) {
          const int p = pt + j * NPROD;
          if (p < np && (s.cls == 1 || sqdist_rn2(S.px[p], S.py[p], S.pz[p], s.cx, s.cy, s.cz) > s.rc2)) ++my_far;
        }
        continue;
      }
      const int off = P.place(S.rows, s.rows, leader);
      const int b = P.b;
      const double* src = s.far ? momv + ((size_t)s.idx * nfo + k0) * MOM_LD
                                : coef + ((size_t)s.idx * nfo + k0) * COEF_LD;
      copy_rows(S.A[b], off, nk, s.rows, pt, [&](int r) { return src + (size_t)r * KSEG; },
                [](int r) { return r; });
      cp_async_commit();
      for (int j = 0; j < PTS_PER_PROD; ++j) {
        const int p = pt + j * NPROD;
        double* g = &S.B[b][(size_t)off * G_LD + p];
        const double x = S.px[p], y = S.py[p], z = S.pz[p];
        if (!s.far) {
          bool nr = p < np;
          if (nr && s.cls == 2) nr = !(sqdist_rn2(x, y, z, s.cx, s.cy, s.cz) > s.rc2);
          if (nr) {
            ++my_near;
            write_g_point<PT>(g, s.rows, pairs[s.idx], x, y, z, boys_tab);
          } else {
            zero_rows(g, s.rows);
          }
        } else {
          double r2 = 0.0;
          bool fr = p < np;
          if (fr) {
            r2 = sqdist_rn2(x, y, z, s.cx, s.cy, s.cz);
            if (s.cls == 2) fr = r2 > s.rc2;
          }
          if (fr) {
            ++my_far;
            if (count_terms) my_terms += (unsigned long long)s.ksum;
            write_h<PT>(g, s.rows, PT(x - s.cx), PT(y - s.cy), PT(z - s.cz), PT(r2));
          } else {
            zero_rows(g, s.rows);
          }
        }
      }
    }
    P.end(S.rows, leader);
  } else {
    // ---- consumers
    const int wn = warp % WN, wm = warp / WN;
    double V[4][NT][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < NT; ++b) V[a][b][0] = V[a][b][1] = 0.0;
    bool mt_active[4];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) mt_active[mt] = wm * 32 + mt * 8 < nk;
    for (int qi = 0;; ++qi) {
      const int b = qi & 1;
      named_sync(BAR_FULL + b);
      const int r = S.rows[b];
      if (r > 0)
        stage_mma(V, &S.A[b][(wm * 32 + (lane >> 2)) * KSEG + (lane & 3)],
                  &S.B[b][(lane & 3) * G_LD + wn * WPTS + (lane >> 2)], r, mt_active);
      named_arrive(BAR_EMPTY + b);
      if (r < 0) break;
    }
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
      const int k = wm * 32 + mt * 8 + (lane >> 2);
      if (k >= nk) continue;
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int p = wn * WPTS + nt * 8 + 2 * (lane & 3) + i;
          if (p < np) vh[(size_t)(k0 + k) * ldv + p0 + p] = V[mt][nt][i];
        }
    }
  }
  count_add(cnt, my_near * (unsigned long long)nk, my_far * (unsigned long long)nk, my_terms);
}

// ---------------------------------------------------------------------------
// Per-FO-geometry calls
// ---------------------------------------------------------------------------
// A CTA owns 128 points and up to 32*WM FOs and walks the per-FO calls in
// order.  For each call it classifies the tile against every FO's sphere and
// compacts the FOs with near points into slots; the producers stream the G
// columns of the call's pairs and the slots' coefficient rows, the consumers
// contract them on the active slot m-tiles only (up to 32*WC slots per pass),
// so the tensor work follows the FOs that are near rather than the whole FO
// block.  The call's near field is added, masked per (FO, point), to the CTA's
// own slice of vh (L2 resident); its far field follows, one FO per warp with
// lanes over points.
template <int WM>
struct PerFOSmem {
  static constexpr int WC = WM < 2 ? WM : 2;  // consumer warp rows: slot capacity 32*WC per pass
  double A[2][32 * WC * KSEG];  // slot rows of the stage's coefficients
  double B[2][KSEG * G_LD];     // G columns
  double MV[32 * WM * MOM_LD];  // far phase: the FOs' moments
  double px[TILE], py[TILE], pz[TILE];
  double cg[32 * WM][3];
  double rc2[32 * WM];
  int stat[32 * WM];
  int npot[32 * WM];
  int lmax[32 * WM];
  int nkeep[32 * WM];
  int fo_of[32 * WM];           // slot -> FO (block-local)
  double lo[3], hi[3];          // tile bounding box
  unsigned bal[WM];             // per warp of the status phase: FOs with near points
  unsigned balf[WM];            // per warp of the status phase: FOs with far points
  int na;
  int rows[2];
};

// Physical A row of pass-local slot s: slots fill m-tiles round robin over the
// WC warp rows, so that a few active FOs keep several warps busy.
template <int WC>
__device__ __forceinline__ int slot_row(int s) {
  const int g = s >> 3;
  return (g % WC) * 32 + (g / WC) * 8 + (s & 7);
}

// Far-field potential of one FO at one point, sum_lm MV[lm] Y_lm(u) / r^(l+1),
// summed per degree l and scaled once per degree; degree LMX at compile time.
template <typename T, int LMX>
__device__ __forceinline__ T multipole(const T* __restrict__ mv, T ux, T uy, T uz, T hn) {
  T acc[LMX + 1];
#pragma unroll
  for (int l = 0; l <= LMX; ++l) acc[l] = T(0);
  harmonics_mmajor(ux, uy, uz, LMX, [&](int row, int l, T v) { acc[l] += mv[row] * v; });
  T pot = T(0), rec = hn;
#pragma unroll
  for (int l = 0; l <= LMX; ++l) {
    pot += acc[l] * rec;
    rec *= hn;
  }
  return pot;
}

// Far field of one FO over the tile's points, lanes over points with the
// TILE/32 points of a lane evaluated together (independent chains; points
// that are near or past np are evaluated on a dummy radius and not added).
// The near/far decision is the FP64 distance test of poisson1.f; T is the
// arithmetic of the expansion.
template <typename T, int LMX>
__device__ __forceinline__ void far_points(const T* __restrict__ mv, const double* __restrict__ px,
                                           const double* __restrict__ py, const double* __restrict__ pz, int np,
                                           double cx, double cy, double cz, double rc2, double* __restrict__ vk,
                                           int lane, unsigned long long& nfar) {
#pragma unroll
  for (int j = 0; j < TILE / 32; ++j) {
    const int p = lane + 32 * j;
    const double x = px[p], y = py[p], z = pz[p];
    const double r2 = sqdist_rn2(x, y, z, cx, cy, cz);
    const bool f = p < np && r2 > rc2;
    T pot;
    if constexpr (sizeof(T) == 4) {
      const float hn = rsqrtf(f ? (float)r2 : 1.f);
      pot = multipole<float, LMX>(mv, hn * (float)(x - cx), hn * (float)(y - cy), hn * (float)(z - cz), hn);
    } else {
      const double hn = 1.0 / sqrt(f ? r2 : 1.0);
      pot = multipole<double, LMX>(mv, hn * (x - cx), hn * (y - cy), hn * (z - cz), hn);
    }
    if (f) {
      vk[p] += (double)pot;
      ++nfar;
    }
  }
}

// One (tile, FO block) of the per-FO-geometry calls; the body of
// k_coulomb_perfo and of k_coulomb_perfo_batch.
template <int WM, bool MIXED>
__device__ __forceinline__ void perfo_tile(int tile, int fob, int ncalls, const int* __restrict__ lists,
                                           int accumulate, const CallInfo* __restrict__ calls,
                                           const PairGeo* __restrict__ pairs, int nfo,
                                           const double* __restrict__ coef, const int8_t* __restrict__ pair_fmt,
                                           const CallFO* __restrict__ cfo, const double* __restrict__ momv,
                                           const MeshDev& M, const double* __restrict__ boys_tab,
                                           double* __restrict__ vh, int ldv, unsigned long long* __restrict__ cnt) {
  constexpr int FOB = 32 * WM, WC = PerFOSmem<WM>::WC, SC = 32 * WC;
  using PT = typename std::conditional<MIXED, float, double>::type;  // producer and far-field arithmetic
  constexpr int WN = CONS_WARPS / WC, WPTS = TILE / WN, NT = WPTS / 8;
  const int* list = lists + ncalls;
  const int nl = lists[2 * ncalls + 1];
  if (accumulate && nl == 0) return;
  extern __shared__ __align__(128) unsigned char smraw[];
  PerFOSmem<WM>& S = *reinterpret_cast<PerFOSmem<WM>*>(smraw);
  const int k0 = fob * FOB;
  const int nk = min(FOB, nfo - k0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p0 = tile * TILE;
  const int np = min(TILE, M.n - p0);
  for (int i = tid; i < TILE; i += WS_THREADS) {
    const bool a = i < np;
    S.px[i] = a ? M.x[p0 + i] : 0.0;
    S.py[i] = a ? M.y[p0 + i] : 0.0;
    S.pz[i] = a ? M.z[p0 + i] : 0.0;
  }
  if (!accumulate)
    for (int e = tid; e < nk * TILE; e += WS_THREADS) {
      const int k = e / TILE, p = e - k * TILE;
      if (p < np) vh[(size_t)(k0 + k) * ldv + p0 + p] = 0.0;
    }
  if (tid < 3) {
    S.lo[tid] = M.tile_lo[3 * tile + tid];
    S.hi[tid] = M.tile_hi[3 * tile + tid];
  }
  unsigned long long my_near = 0, my_far = 0, my_terms = 0;

  for (int li = 0; li < nl; ++li) {
    const int c = list[li];
    const CallInfo ci = calls[c];
    __syncthreads();  // the previous call is done with every shared buffer and with vh
    // status of every FO of the block for this tile, and the active slots
    if (tid < FOB) {
      int st = 1, npot = 2, lmx = 0, nkeep = 0;
      double cgx = 0, cgy = 0, cgz = 0, rc2 = 0;
      if (tid < nk) {
        const CallFO f = cfo[(size_t)c * nfo + k0 + tid];
        cgx = f.cg[0];
        cgy = f.cg[1];
        cgz = f.cg[2];
        rc2 = f.rcut2;
        npot = f.npot;
        st = (npot == 1) ? 0 : tile_class(S.lo, S.hi, cgx, cgy, cgz, rc2);
        if (st != 0 && npot == 2) {
          lmx = f.lmax;
          nkeep = __popcll(f.keep);
        }
      }
      S.stat[tid] = st;
      S.npot[tid] = npot;
      S.cg[tid][0] = cgx;
      S.cg[tid][1] = cgy;
      S.cg[tid][2] = cgz;
      S.rc2[tid] = rc2;
      S.lmax[tid] = lmx;
      S.nkeep[tid] = nkeep;
      const unsigned b = __ballot_sync(0xffffffffu, tid < nk && st != 1);
      const unsigned bf = __ballot_sync(0xffffffffu, tid < nk && st != 0 && npot == 2);
      if (lane == 0) {
        S.bal[warp] = b;
        S.balf[warp] = bf;
      }
    }
    __syncthreads();
    if (tid < FOB) {
      int before = 0;
      for (int w = 0; w < warp; ++w) before += __popc(S.bal[w]);
      const unsigned b = S.bal[warp];
      if ((b >> lane) & 1u) S.fo_of[before + __popc(b & ((1u << lane) - 1u))] = tid;
      if (tid == FOB - 1) S.na = before + __popc(b);
    }
    __syncthreads();
    const int na = S.na;
    bool anyfar = false;
#pragma unroll
    for (int w = 0; w < WM; ++w) anyfar = anyfar || S.balf[w] != 0u;

    for (int c0 = 0; c0 < na; c0 += SC) {
      const int nac = min(SC, na - c0);
      const int* fo = S.fo_of + c0;
      if (warp >= CONS_WARPS) {
        // ---- producers: the call's pairs, packed into stages
        const int pt = tid - NCONS;
        const bool leader = pt == 0;
        StagePacker P;
        for (int qi = 0; qi < ci.np; ++qi) {
          const int q = ci.p0 + qi;
          const int kq = near_rows(pair_fmt[q]);
          const int off = P.place(S.rows, kq, leader);
          const int b = P.b;
          const double* src = coef + ((size_t)q * nfo + k0) * COEF_LD;
          copy_rows(S.A[b], off, nac, kq, pt, [&](int s) { return src + (size_t)fo[s] * COEF_LD; },
                    [](int s) { return slot_row<WC>(s); });
          cp_async_commit();
          const PairGeo& pg = pairs[q];
          for (int j = 0; j < PTS_PER_PROD; ++j) {
            const int p = pt + j * NPROD;
            double* g = &S.B[b][(size_t)off * G_LD + p];
            if (p < np) write_g_point<PT>(g, kq, pg, S.px[p], S.py[p], S.pz[p], boys_tab);
            else zero_rows(g, kq);
          }
        }
        P.end(S.rows, leader);
      } else {
        // ---- consumers
        const int wn = warp % WN, wm = warp / WN;
        double T[4][NT][2];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < NT; ++b) T[a][b][0] = T[a][b][1] = 0.0;
        bool mt_active[4];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) mt_active[mt] = (mt * WC + wm) * 8 < nac;
        for (int qi = 0;; ++qi) {
          const int b = qi & 1;
          named_sync(BAR_FULL + b);
          const int r = S.rows[b];
          if (r > 0)
            stage_mma(T, &S.A[b][(wm * 32 + (lane >> 2)) * KSEG + (lane & 3)],
                      &S.B[b][(lane & 3) * G_LD + wn * WPTS + (lane >> 2)], r, mt_active);
          named_arrive(BAR_EMPTY + b);
          if (r < 0) break;
        }
        // masked add of the call's near field to vh
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
          const int s = (mt * WC + wm) * 8 + (lane >> 2);
          if (s >= nac) continue;
          const int k = fo[s];
          const int st = S.stat[k];
          const double cx = S.cg[k][0], cy = S.cg[k][1], cz = S.cg[k][2], rc2 = S.rc2[k];
          double* vk = vh + (size_t)(k0 + k) * ldv + p0;
#pragma unroll
          for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const int p = wn * WPTS + nt * 8 + 2 * (lane & 3) + i;
              if (p >= np) continue;
              bool nr = (st == 0);
              if (st == 2) nr = !(sqdist_rn2(S.px[p], S.py[p], S.pz[p], cx, cy, cz) > rc2);
              if (nr) {
                vk[p] += T[mt][nt][i];
                my_near += (unsigned long long)ci.np;
              }
            }
        }
      }
    }

    if (anyfar) {
      __syncthreads();  // the near phase is done with vh
      // the FOs' moments in the arithmetic of the expansion (FP32 in the mixed path)
      PT* MVp = reinterpret_cast<PT*>(S.MV);
      const double* mg = momv + ((size_t)c * nfo + k0) * MOM_LD;
      for (int e = tid; e < nk * MOM_LD; e += WS_THREADS) MVp[e] = (PT)mg[e];
      __syncthreads();
      for (int k = warp; k < nk; k += WS_THREADS / 32) {
        if (S.stat[k] == 0 || S.npot[k] == 1) continue;
        const double cx = S.cg[k][0], cy = S.cg[k][1], cz = S.cg[k][2], rc2 = S.rc2[k];
        const PT* mv = MVp + k * MOM_LD;
        double* vk = vh + (size_t)(k0 + k) * ldv + p0;
        unsigned long long nf = 0;
        switch (S.lmax[k]) {
#define FAR_CASE(L)                                                                          \
  case L:                                                                                    \
    far_points<PT, L>(mv, S.px, S.py, S.pz, np, cx, cy, cz, rc2, vk, lane, nf); \
    break;
          FAR_CASE(0)
          FAR_CASE(1)
          FAR_CASE(2)
          FAR_CASE(3)
          FAR_CASE(4)
          FAR_CASE(5)
          default: FAR_CASE(6)
#undef FAR_CASE
        }
        my_far += nf;
        my_terms += nf * (unsigned long long)S.nkeep[k];
      }
    }
  }
  count_add(cnt, my_near, my_far, my_terms);
}

template <int WM, bool MIXED>
__global__ void __launch_bounds__(WS_THREADS, 1)
k_coulomb_shared(int ncalls, const int* __restrict__ lists, const CallShare* __restrict__ share,
                 const CallInfo* __restrict__ calls, int nfo, const double* __restrict__ coef,
                 const int8_t* __restrict__ pair_fmt, const PairGeo* __restrict__ pairs,
                 const double* __restrict__ momv, MeshDev M, const double* __restrict__ boys_tab,
                 double* __restrict__ vh, int ldv, unsigned long long* __restrict__ cnt) {
  shared_tile<WM, MIXED>(blockIdx.x, blockIdx.y, ncalls, lists, share, calls, nfo, coef, pair_fmt, pairs, momv, M,
                         boys_tab, vh, ldv, cnt);
}

template <int WM, bool MIXED>
__global__ void __launch_bounds__(WS_THREADS, 1)
k_coulomb_perfo(int ncalls, const int* __restrict__ lists, int accumulate, const CallInfo* __restrict__ calls,
                const PairGeo* __restrict__ pairs, int nfo, const double* __restrict__ coef,
                const int8_t* __restrict__ pair_fmt, const CallFO* __restrict__ cfo,
                const double* __restrict__ momv, MeshDev M, const double* __restrict__ boys_tab,
                double* __restrict__ vh, int ldv, unsigned long long* __restrict__ cnt) {
  perfo_tile<WM, MIXED>(blockIdx.x, blockIdx.y, ncalls, lists, accumulate, calls, pairs, nfo, coef, pair_fmt, cfo,
                        momv, M, boys_tab, vh, ldv, cnt);
}

// ---------------------------------------------------------------------------
// Many molecules in one launch
// ---------------------------------------------------------------------------
// Persistent CTAs (one per SM) walk a list of (job, tile, FO block) items
// spanning every molecule and spin of a batch, taking the next item from a
// global counter (items of uneven cost balance themselves); a job is one
// (molecule, spin) with its own calls, coefficients, mesh and output.  Each
// item is the same work as one CTA of the per-molecule kernels and writes its
// own outputs, so every potential is the same bit for bit whichever CTA runs it.
__device__ __forceinline__ int next_item(int* counter, int* slot) {
  __syncthreads();  // every thread is done with the previous item (and its shared memory)
  if (threadIdx.x == 0) *slot = atomicAdd(counter, 1);
  __syncthreads();
  return *slot;
}

template <int WM, bool MIXED>
__global__ void __launch_bounds__(WS_THREADS, 1)
k_coulomb_shared_batch(const CoulombJob* __restrict__ jobs, const int4* __restrict__ items, int nitems,
                       int* __restrict__ counter, const double* __restrict__ boys_tab) {
  __shared__ int slot;
  for (int it = next_item(counter, &slot); it < nitems; it = next_item(counter, &slot)) {
    const int4 w = items[it];
    const CoulombJob J = jobs[w.x];
    shared_tile<WM, MIXED>(w.y, w.z, J.ncalls, J.lists, J.share, J.calls, J.nfo, J.coef, J.pair_fmt, J.pairs,
                           J.momv, J.M, boys_tab, J.vh, J.ldv, J.cnt);
  }
}

template <int WM, bool MIXED>
__global__ void __launch_bounds__(WS_THREADS, 1)
k_coulomb_perfo_batch(const CoulombJob* __restrict__ jobs, const int4* __restrict__ items, int nitems,
                      int* __restrict__ counter, const double* __restrict__ boys_tab) {
  __shared__ int slot;
  for (int it = next_item(counter, &slot); it < nitems; it = next_item(counter, &slot)) {
    const int4 w = items[it];
    const CoulombJob J = jobs[w.x];
    perfo_tile<WM, MIXED>(w.y, w.z, J.ncalls, J.lists, 1, J.calls, J.pairs, J.nfo, J.coef, J.pair_fmt, J.cfo,
                          J.momv, J.M, boys_tab, J.vh, J.ldv, J.cnt);
  }
}

// ---------------------------------------------------------------------------
// Call classification
// ---------------------------------------------------------------------------
// Largest Boys variant over the FOs of each pair (the G tile is shared by all FOs).
__global__ void k_pair_fmt(int npairs, int nfo, const int8_t* __restrict__ maxfmt, int8_t* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npairs) return;
  int m = 3;
  for (int k = 0; k < nfo; ++k) m = max(m, (int)maxfmt[(size_t)q * nfo + k]);
  out[q] = (int8_t)m;
}

// One warp per call: is (CG, RCUT^2, NPOT) bitwise the same for every FO, and
// how many moment rows do the FOs keep.
__global__ void k_call_share(int ncalls, int nfo, const CallFO* __restrict__ cfo, CallShare* __restrict__ out) {
  const int c = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= ncalls) return;
  const CallFO f0 = cfo[(size_t)c * nfo];
  bool same = true;
  int lmx = -1, ksum = 0;
  for (int k = lane; k < nfo; k += 32) {
    const CallFO f = cfo[(size_t)c * nfo + k];
    same = same && f.cg[0] == f0.cg[0] && f.cg[1] == f0.cg[1] && f.cg[2] == f0.cg[2] && f.rcut2 == f0.rcut2 &&
           f.npot == f0.npot;
    if (f.npot == 2 && f.keep != 0ull) {
      lmx = max(lmx, f.lmax);
      ksum += __popcll(f.keep);
    }
  }
  same = __all_sync(0xffffffffu, same);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lmx = max(lmx, __shfl_xor_sync(0xffffffffu, lmx, o));
    ksum += __shfl_xor_sync(0xffffffffu, ksum, o);
  }
  if (lane == 0) {
    CallShare s;
    s.cg[0] = f0.cg[0];
    s.cg[1] = f0.cg[1];
    s.cg[2] = f0.cg[2];
    s.rcut2 = f0.rcut2;
    s.npot = f0.npot;
    s.kf = (lmx < 0) ? 0 : (((lmx + 1) * (lmx + 1) + 3) / 4) * 4;
    s.shared = same ? 1 : 0;
    s.ksum = ksum;
    out[c] = s;
  }
}

// Stable partition of the calls into lists[0..ns) (shared geometry) and
// lists[ncalls..ncalls+nf) (per-FO geometry); lists[2 ncalls] = ns,
// lists[2 ncalls + 1] = nf.  One block.
constexpr int LIST_THREADS = 1024;
__global__ void __launch_bounds__(LIST_THREADS) k_call_lists(int ncalls, int per_fo_only,
                                                             const CallShare* __restrict__ share,
                                                             int* __restrict__ lists) {
  __shared__ int wsum[LIST_THREADS / 32];
  __shared__ int base;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) base = 0;
  __syncthreads();
  for (int c0 = 0; c0 < ncalls; c0 += LIST_THREADS) {
    const int c = c0 + tid;
    const bool valid = c < ncalls;
    const bool sh = valid && !per_fo_only && share[c].shared;
    const unsigned bal = __ballot_sync(0xffffffffu, sh);
    if (lane == 0) wsum[wid] = __popc(bal);
    __syncthreads();
    int before = base;
    for (int w = 0; w < wid; ++w) before += wsum[w];
    const int rank_s = before + __popc(bal & ((1u << lane) - 1u));
    if (valid) {
      if (sh) lists[rank_s] = c;
      else lists[ncalls + (c - rank_s)] = c;  // c minus the shared calls before it
    }
    __syncthreads();
    if (tid == 0) {
      int t = 0;
      for (int w = 0; w < LIST_THREADS / 32; ++w) t += wsum[w];
      base += t;
    }
    __syncthreads();
  }
  if (tid == 0) {
    lists[2 * ncalls] = base;
    lists[2 * ncalls + 1] = ncalls - base;
  }
}

template <int WM>
static void set_shared_attr() {
  cudaFuncSetAttribute(k_coulomb_shared<WM, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(SharedSmem<WM>));
  cudaFuncSetAttribute(k_coulomb_shared<WM, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(SharedSmem<WM>));
}

template <int WM>
static void set_batch_attr() {
  cudaFuncSetAttribute(k_coulomb_shared_batch<WM, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(SharedSmem<WM>));
  cudaFuncSetAttribute(k_coulomb_shared_batch<WM, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(SharedSmem<WM>));
  cudaFuncSetAttribute(k_coulomb_perfo_batch<WM, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(PerFOSmem<WM>));
  cudaFuncSetAttribute(k_coulomb_perfo_batch<WM, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(PerFOSmem<WM>));
}

template <int WM>
static void set_perfo_attr() {
  cudaFuncSetAttribute(k_coulomb_perfo<WM, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(PerFOSmem<WM>));
  cudaFuncSetAttribute(k_coulomb_perfo<WM, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(PerFOSmem<WM>));
}

// Per-device set-up: the dynamic shared-memory opt-ins.
void init_coulomb_mma() {
  set_shared_attr<1>();
  set_shared_attr<2>();
  set_shared_attr<4>();
  set_perfo_attr<1>();
  set_perfo_attr<2>();
  set_perfo_attr<4>();
  set_batch_attr<1>();
  set_batch_attr<2>();
  set_batch_attr<4>();
}

template <int WM>
static void launch_shared(int ncalls, const int* lists, const CallShare* share, const CallInfo* calls, int nfo,
                          const double* coef, const int8_t* pair_fmt, const PairGeo* pairs, const double* momv,
                          const MeshDev& M, const double* boys_tab, double* vh, int ldv, unsigned long long* cnt,
                          bool mixed, cudaStream_t st) {
  dim3 grid(M.ntiles, (nfo + 32 * WM - 1) / (32 * WM));
  if (mixed)
    k_coulomb_shared<WM, true><<<grid, WS_THREADS, sizeof(SharedSmem<WM>), st>>>(
        ncalls, lists, share, calls, nfo, coef, pair_fmt, pairs, momv, M, boys_tab, vh, ldv, cnt);
  else
    k_coulomb_shared<WM, false><<<grid, WS_THREADS, sizeof(SharedSmem<WM>), st>>>(
        ncalls, lists, share, calls, nfo, coef, pair_fmt, pairs, momv, M, boys_tab, vh, ldv, cnt);
}

template <int WM>
static void launch_perfo(int ncalls, const int* lists, int acc, const CallInfo* calls, const PairGeo* pairs, int nfo,
                         const double* coef, const int8_t* pair_fmt, const CallFO* cfo, const double* momv,
                         const MeshDev& M, const double* boys_tab, double* vh, int ldv, unsigned long long* cnt,
                         bool mixed, cudaStream_t st) {
  dim3 grid(M.ntiles, (nfo + 32 * WM - 1) / (32 * WM));
  if (mixed)
    k_coulomb_perfo<WM, true><<<grid, WS_THREADS, sizeof(PerFOSmem<WM>), st>>>(
        ncalls, lists, acc, calls, pairs, nfo, coef, pair_fmt, cfo, momv, M, boys_tab, vh, ldv, cnt);
  else
    k_coulomb_perfo<WM, false><<<grid, WS_THREADS, sizeof(PerFOSmem<WM>), st>>>(
        ncalls, lists, acc, calls, pairs, nfo, coef, pair_fmt, cfo, momv, M, boys_tab, vh, ldv, cnt);
}

void launch_coulomb_classify(int ncalls, int npairs, int nfo, const int8_t* maxfmt, const CallFO* cfo,
                             const CoulombScratch& scr, bool per_fo_only, cudaStream_t st) {
  if (npairs > 0) k_pair_fmt<<<(npairs + 127) / 128, 128, 0, st>>>(npairs, nfo, maxfmt, scr.pair_fmt);
  if (ncalls > 0) k_call_share<<<(ncalls + 7) / 8, 256, 0, st>>>(ncalls, nfo, cfo, scr.share);
  k_call_lists<<<1, LIST_THREADS, 0, st>>>(ncalls, per_fo_only ? 1 : 0, scr.share, scr.lists);
}

template <int WM>
static void launch_batch_wm(const CoulombJob* jobs, const int4* items, int nitems, int* counters, bool mixed,
                            const double* boys_tab, int nctas, cudaStream_t st) {
  if (mixed) {
    k_coulomb_shared_batch<WM, true><<<nctas, WS_THREADS, sizeof(SharedSmem<WM>), st>>>(jobs, items, nitems,
                                                                                          counters, boys_tab);
    k_coulomb_perfo_batch<WM, true><<<nctas, WS_THREADS, sizeof(PerFOSmem<WM>), st>>>(jobs, items, nitems,
                                                                                        counters + 1, boys_tab);
  } else {
    k_coulomb_shared_batch<WM, false><<<nctas, WS_THREADS, sizeof(SharedSmem<WM>), st>>>(jobs, items, nitems,
                                                                                           counters, boys_tab);
    k_coulomb_perfo_batch<WM, false><<<nctas, WS_THREADS, sizeof(PerFOSmem<WM>), st>>>(jobs, items, nitems,
                                                                                         counters + 1, boys_tab);
  }
}

void launch_coulomb_batch(const CoulombJob* jobs, const int4* items, int nitems, int* counters, int wm, bool mixed,
                          const double* boys_tab, int nctas, cudaStream_t st) {
  if (nitems <= 0) return;
  nctas = std::max(1, std::min(nctas, nitems));
  cudaMemsetAsync(counters, 0, 2 * sizeof(int), st);
  if (wm == 4) launch_batch_wm<4>(jobs, items, nitems, counters, mixed, boys_tab, nctas, st);
  else if (wm == 2) launch_batch_wm<2>(jobs, items, nitems, counters, mixed, boys_tab, nctas, st);
  else launch_batch_wm<1>(jobs, items, nitems, counters, mixed, boys_tab, nctas, st);
}

cudaError_t launch_coulomb_mma(int ncalls, const CallInfo* calls, const PairGeo* pairs, int npairs, int nfo,
                               const double* coef, const int8_t* maxfmt, const CallFO* cfo, const double* momv,
                               const MeshDev& M, const double* boys_tab, double* vh, int ldv,
                               const CoulombConfig& cfg, bool mixed, const CoulombScratch& scr,
                               unsigned long long* cnt, cudaEvent_t mid, cudaStream_t st) {
  const bool per_fo_only = cfg.per_fo_only;
  unsigned long long* cnt_perfo = cnt + 3;  // the per-FO kernel counts apart from the shared-geometry one
  launch_coulomb_classify(ncalls, npairs, nfo, maxfmt, cfo, scr, per_fo_only, st);
  if (!per_fo_only && mixed && cfg.shared_tc) {
    const size_t nc = (size_t)npairs * nfo * COEF_LD, nm = (size_t)ncalls * nfo * MOM_LD;
    launch_split_tf32((size_t)npairs, nfo, coef, scr.coef_hl, st);
    launch_split_tf32((size_t)ncalls, nfo, momv, scr.momv_hl, st);
    const cudaError_t e = launch_coulomb_shared_tc(ncalls, scr.lists, scr.share, calls, nfo, scr.coef_hl, nc,
                                                   scr.pair_fmt, pairs, scr.momv_hl, nm, M, boys_tab, vh, ldv, cnt,
                                                   scr.err, cfg.wait_limit, st);
    if (e != cudaSuccess) return e;
  } else if (!per_fo_only) {
    if (nfo > 64)
      launch_shared<4>(ncalls, scr.lists, scr.share, calls, nfo, coef, scr.pair_fmt, pairs, momv, M, boys_tab, vh,
                       ldv, cnt, mixed, st);
    else if (nfo > 32)
      launch_shared<2>(ncalls, scr.lists, scr.share, calls, nfo, coef, scr.pair_fmt, pairs, momv, M, boys_tab, vh,
                       ldv, cnt, mixed, st);
    else
      launch_shared<1>(ncalls, scr.lists, scr.share, calls, nfo, coef, scr.pair_fmt, pairs, momv, M, boys_tab, vh,
                       ldv, cnt, mixed, st);
  }
  if (mid) cudaEventRecord(mid, st);
  const int acc = per_fo_only ? 0 : 1;
  const int wm = cfg.perfo_wm > 0 ? cfg.perfo_wm : (nfo > 64 ? 4 : (nfo > 32 ? 2 : 1));
  if (wm == 4)
    launch_perfo<4>(ncalls, scr.lists, acc, calls, pairs, nfo, coef, scr.pair_fmt, cfo, momv, M, boys_tab, vh, ldv,
                    cnt_perfo, mixed, st);
  else if (wm == 2)
    launch_perfo<2>(ncalls, scr.lists, acc, calls, pairs, nfo, coef, scr.pair_fmt, cfo, momv, M, boys_tab, vh, ldv,
                    cnt_perfo, mixed, st);
  else
    launch_perfo<1>(ncalls, scr.lists, acc, calls, pairs, nfo, coef, scr.pair_fmt, cfo, momv, M, boys_tab, vh, ldv,
                    cnt_perfo, mixed, st);
  return cudaGetLastError();
}

}  // namespace flosic
