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
//                     128 FOs; segments are double buffered (A by cp.async, B by
//                     the first four warps while the others multiply).
//   k_coulomb_perfo   the remaining calls, whose CG (charge weighted,
//                     poisson1.f:503-520) differs per FO: the near field of the
//                     FOs with near points in the tile as a GEMM over compacted
//                     FO slots, added per (FO, point); the far field per
//                     (FO, point).
//
// Both walk their calls in order, so every per-point sum is deterministic.
// Both count the evaluations they perform: near (pair, point, FO), far
// (call, point, FO) and the multipole terms the far evaluations keep, the
// units of the reference's POISSON1 work.
#include <cfloat>

#include "device_math.cuh"
#include "kernels.cuh"

namespace flosic {

constexpr int MMA_THREADS = 256;            // 8 warps
constexpr int G_LD = TILE + 4;              // 132 (= 4 mod 16 doubles): conflict-free B fragment loads
constexpr int KSEG = 52;                    // rows of one B segment (46 coefficients or 49 moments, padded)
static_assert(COEF_LD == KSEG && MOM_LD == KSEG, "segment rows and global row strides must agree");

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ double sqdist_rn2(double x, double y, double z, double cx, double cy, double cz) {
  const double dx = __dadd_rn(x, -cx), dy = __dadd_rn(y, -cy), dz = __dadd_rn(z, -cz);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Tile classification against a sphere: 0 every point inside, 1 every point
// outside, 2 decided per point.  The 1e-9 margins leave boundary cases to the
// exact per-point test.
__device__ __forceinline__ int tile_class(const double lo[3], const double hi[3], double cx, double cy, double cz,
                                          double rc2) {
  const double cgv[3] = {cx, cy, cz};
  double dmin2 = 0.0, dmax2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double a = lo[d] - cgv[d], b = cgv[d] - hi[d];
    const double m = fmax(fmax(a, b), 0.0);
    dmin2 += m * m;
    const double e = fmax(fabs(cgv[d] - lo[d]), fabs(hi[d] - cgv[d]));
    dmax2 += e * e;
  }
  if (dmin2 > rc2 * (1.0 + 1e-9)) return 1;
  if (dmax2 < rc2 * (1.0 - 1e-9)) return 0;
  return 2;
}

// Unnormalised harmonics of harmonics.f in the row order of the moments
// (l*l + j; j = 0 for m = 0, 2m-1 and 2m for the two m > 0 partners), for
// l <= lmx.  The recursion of harmonics.f runs level by level; here it runs
// m-major so that only a few values are live, but every value is formed by
// the same operations on the same operands:
//   m = l (sectoral):  C_l = (2l-1)(C_{l-1} ux - S_{l-1} uy),  S_l = (2l-1)(S_{l-1} ux + C_{l-1} uy)
//   m < l:             P_l = ((2l-1)/(l-m)) P_{l-1} uz - ((l+m-1)/(l-m)) P_{l-2}
// op(row, l, value) receives each term; the caller applies 1/r^(l+1).
template <typename Op>
__device__ __forceinline__ void harmonics_mmajor(double ux, double uy, double uz, int lmx, Op op) {
  // m = 0
  {
    op(0, 0, 1.0);
    if (lmx >= 1) op(1, 1, uz);
    double p2 = 1.0, p1 = uz;
#pragma unroll
    for (int l = 2; l <= LM; ++l) {
      if (l > lmx) break;
      const double facrc = 1.0 / l;
      const double aa = facrc * (2 * l - 1), bb = facrc * (l - 1);
      const double cu = aa * p1 * uz - bb * p2;
      op(l * l, l, cu);
      p2 = p1;
      p1 = cu;
    }
  }
  double sc = ux, ss = uy;  // sectoral pair at l = m
#pragma unroll
  for (int m = 1; m <= LM; ++m) {
    if (m > lmx) break;
    if (m > 1) {
      const double ifc = (double)(2 * m - 1);
      const double nc = ifc * (sc * ux - ss * uy);
      const double ns = ifc * (ss * ux + sc * uy);
      sc = nc;
      ss = ns;
    }
    op(m * m + 2 * m - 1, m, sc);
    op(m * m + 2 * m, m, ss);
    double c2 = 0.0, s2 = 0.0, c1 = sc, s1 = ss;
#pragma unroll
    for (int l = m + 1; l <= LM; ++l) {
      if (l > lmx) break;
      const double facrc = 1.0 / (l - m);
      const double aa = facrc * (2 * l - 1);
      const double bb = (m == l - 1) ? 0.0 : facrc * (l + m - 1);
      const double cc = aa * c1 * uz - bb * c2;
      const double cs = aa * s1 * uz - bb * s2;
      op(l * l + 2 * m - 1, l, cc);
      op(l * l + 2 * m, l, cs);
      c2 = c1;
      s2 = s1;
      c1 = cc;
      s1 = cs;
    }
  }
}

// Boys values F_0..F_{fmt-1} of the FFFMTC3/4/5 variant (same arithmetic as
// boys_all); absent orders are zero.
__device__ __forceinline__ void boys_fmt(const double* __restrict__ tab, double x, double chgd, int fmt,
                                         double F[5]) {
  if (x > 16.0) {
    const double ROOTPI = 1.77245385090551602728;
    const double pol1 = -chgd;
    const double rt = __dmul_rn(sqrt(x), ROOTPI);
    const double rect1 = 0.5 / x;
    F[0] = rect1 * (rt + pol1);
    F[1] = rect1 * (F[0] + pol1);
    F[2] = rect1 * (3 * F[1] + pol1);
    F[3] = (fmt >= 4) ? rect1 * (5 * F[2] + pol1) : 0.0;
    F[4] = (fmt >= 5) ? rect1 * (7 * F[3] + pol1) : 0.0;
    return;
  }
  const int it = (int)(100 * x + 1.5);
  const double pol1 = chgd;
  const double rect1 = 2 * x;
  const double dt = (1.0e-2) * (it - 1) - x;
  const double* f = tab + (size_t)(it - 1) * BOYS_NC;
  const double o7 = 1.0 / 7.0, o5 = 1.0 / 5.0, o3 = 1.0 / 3.0;
  if (fmt == 5) {
    F[4] = f[2] + dt * (f[3] + dt * (f[6] + dt * f[9]));
    F[3] = (F[4] * rect1 + pol1) * o7;
    F[2] = (F[3] * rect1 + pol1) * o5;
  } else if (fmt == 4) {
    F[4] = 0.0;
    F[3] = f[1] + dt * (f[2] + dt * (f[5] + dt * f[8]));
    F[2] = (F[3] * rect1 + pol1) * o5;
  } else {
    F[4] = 0.0;
    F[3] = 0.0;
    F[2] = f[0] + dt * (f[1] + dt * (f[4] + dt * f[7]));
  }
  F[1] = (F[2] * rect1 + pol1) * o3;
  F[0] = (F[1] * rect1 + pol1);
}

// Rows of the near segment used by a pair whose largest Boys variant is fmt:
// slots 15.. carry F_3 and slots 31.. carry F_4 (COEFICIENT order,
// poisson1.f:402-482).
__device__ __forceinline__ int near_rows(int fmt) { return fmt >= 5 ? 48 : (fmt == 4 ? 32 : 16); }

// G column of one (pair, point) in the COEFICIENT slot order: slot t holds
// F_{m(t)} * POLY(mono(t)), monomials in the order of poisson1.f:925-959.
// Rows >= kn (16, 32 or 48) are not written.
__device__ __forceinline__ void write_g(double* g, int kn, double x, double y, double z, const double F[5]) {
#define GW(t, v) g[(size_t)(t) * G_LD] = (v)
  const double F0 = F[0], F1 = F[1], F2 = F[2], F3 = F[3], F4 = F[4];
  const double zz = z * z, yz = y * z, yy = y * y, xz = x * z, xy = x * y, xx = x * x;
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
  GW(46, 0.0);
  GW(47, 0.0);
#undef GW
}

__device__ __forceinline__ void zero_rows(double* g, int k) {
  for (int t = 0; t < k; ++t) g[(size_t)t * G_LD] = 0.0;
}

// cnt[0] near (pair, point, FO), cnt[1] far (call, point, FO), cnt[2] multipole
// terms kept by the skip rule summed over the far evaluations.
__device__ __forceinline__ void count_add(unsigned long long* cnt, unsigned long long near, unsigned long long far,
                                          unsigned long long terms) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    near += __shfl_down_sync(0xffffffffu, near, o);
    far += __shfl_down_sync(0xffffffffu, far, o);
    terms += __shfl_down_sync(0xffffffffu, terms, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (near) atomicAdd(&cnt[0], near);
    if (far) atomicAdd(&cnt[1], far);
    if (terms) atomicAdd(&cnt[2], terms);
  }
}

// ---------------------------------------------------------------------------
// Shared-geometry calls
// ---------------------------------------------------------------------------
template <int WM>
struct SharedSmem {
  double A[2][32 * WM * KSEG];  // FO rows of the segment's coefficients / moments
  double B[2][KSEG * G_LD];     // G or H columns
  double px[TILE], py[TILE], pz[TILE];
};

// One segment of the shared GEMM: the near part of one pair or the far part of
// one call, restricted to this tile.
struct Segment {
  int far;       // 0 near (pair q), 1 far (call c)
  int idx;       // q or c
  int rows;      // contraction length, a multiple of 4
  int cls;       // tile class against the call's sphere
  int ksum;      // kept multipole terms summed over all FOs (far segments)
  double cx, cy, cz, rc2;
};

// Walks the shared calls of the list in order and yields their segments for a
// tile: near segments for each pair unless the tile is entirely far, then the
// far segment unless the tile is entirely near or NPOT=1.  Every thread runs
// it identically.
struct SegmentWalker {
  const int* list;
  int n;
  const CallShare* share;
  const CallInfo* calls;
  const int8_t* pair_fmt;
  double lo[3], hi[3];
  int li, sub;
  int c, p0, np, cls, kf, npot, ksum;
  double cx, cy, cz, rc2;
  unsigned long long direct_far;  // far points of all-far tiles of calls without kept moments

  __device__ bool next(Segment& s, int npts) {
    while (li < n) {
      if (sub < 0) {
        c = list[li];
        const CallShare sh = share[c];
        const CallInfo ci = calls[c];
        cx = sh.cg[0];
        cy = sh.cg[1];
        cz = sh.cg[2];
        rc2 = sh.rcut2;
        kf = sh.kf;
        ksum = sh.ksum;
        npot = sh.npot;
        p0 = ci.p0;
        np = ci.np;
        cls = (npot == 1) ? 0 : tile_class(lo, hi, cx, cy, cz, rc2);
        sub = (cls == 1) ? np : 0;
      }
      if (sub < np) {
        const int q = p0 + sub;
        ++sub;
        s = Segment{0, q, near_rows(pair_fmt[q]), cls, 0, cx, cy, cz, rc2};
        return true;
      }
      const bool want_far = npot == 2 && cls != 0;
      sub = -1;
      ++li;
      if (want_far) {
        if (kf > 0 || cls == 2) {
          s = Segment{1, c, kf, cls, ksum, cx, cy, cz, rc2};
          return true;
        }
        direct_far += (unsigned long long)npts;
      }
    }
    return false;
  }
};

template <int WM>
__global__ void __launch_bounds__(MMA_THREADS, 1)
k_coulomb_shared(int ncalls, const int* __restrict__ lists, const CallShare* __restrict__ share,
                 const CallInfo* __restrict__ calls, int nfo, const double* __restrict__ coef,
                 const int8_t* __restrict__ pair_fmt, const PairGeo* __restrict__ pairs,
                 const double* __restrict__ momv, MeshDev M, const double* __restrict__ boys_tab,
                 double* __restrict__ vh, int ldv, unsigned long long* __restrict__ cnt) {
  constexpr int FOB = 32 * WM, WN = 8 / WM, WPTS = TILE / WN, NT = WPTS / 8;
  extern __shared__ __align__(128) unsigned char smraw[];
  SharedSmem<WM>& S = *reinterpret_cast<SharedSmem<WM>*>(smraw);
  const int tile = blockIdx.x;
  const int k0 = blockIdx.y * FOB;
  const int nk = min(FOB, nfo - k0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WM, wn = warp / WM;
  const int p0 = tile * TILE;
  const int np = min(TILE, M.n - p0);
  for (int i = tid; i < TILE; i += MMA_THREADS) {
    const bool a = i < np;
    S.px[i] = a ? M.x[p0 + i] : 0.0;
    S.py[i] = a ? M.y[p0 + i] : 0.0;
    S.pz[i] = a ? M.z[p0 + i] : 0.0;
  }
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
  W.direct_far = 0ull;
  __syncthreads();

  double V[4][NT][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < NT; ++b) V[a][b][0] = V[a][b][1] = 0.0;
  unsigned long long my_near = 0, my_far = 0, my_terms = 0;
  const bool count_terms = blockIdx.y == 0;  // kept terms are summed over all FOs once per (call, point)

  // Stage segment s into buffer b: A rows by cp.async (all threads), B columns
  // by threads 0..127 (one point each).
  auto stage = [&](const Segment& s, int b) {
    if (s.rows > 0) {
      const double* src = s.far ? momv + ((size_t)s.idx * nfo + k0) * MOM_LD
                                : coef + ((size_t)s.idx * nfo + k0) * COEF_LD;
      const int nchunk = nk * (KSEG / 2);
      double* dst = S.A[b];
      for (int i = tid; i < nchunk; i += MMA_THREADS) cp_async16(dst + 2 * i, src + 2 * i);
    }
    cp_async_commit();
    if (tid < TILE) {
      const int p = tid;
      double* g = &S.B[b][p];
      const double x = S.px[p], y = S.py[p], z = S.pz[p];
      if (!s.far) {
        bool nr = p < np;
        if (nr && s.cls == 2) nr = !(sqdist_rn2(x, y, z, s.cx, s.cy, s.cz) > s.rc2);
        if (nr) {
          ++my_near;
          const PairGeo& pg = pairs[s.idx];
          const double rx = x - pg.C[0], ry = y - pg.C[1], rz = z - pg.C[2];
          const double xx = pg.delta * (rz * rz + ry * ry + rx * rx);
          double F[5];
          boys_fmt(boys_tab, xx, exp(-xx), s.rows >= 48 ? 5 : (s.rows == 32 ? 4 : 3), F);
          write_g(g, s.rows, rx, ry, rz, F);
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
          if (s.rows > 0) {
            const double hn = 1.0 / sqrt(r2);
            const int kr = s.rows;
            double rec[LM + 1];
            rec[0] = hn;
#pragma unroll
            for (int l = 1; l <= LM; ++l) rec[l] = rec[l - 1] * hn;
            harmonics_mmajor(hn * (x - s.cx), hn * (y - s.cy), hn * (z - s.cz), LM, [&](int row, int l, double v) {
              if (row < kr) g[(size_t)row * G_LD] = v * rec[l];
            });
            for (int t = NMOM; t < kr; ++t) g[(size_t)t * G_LD] = 0.0;
          }
        } else {
          zero_rows(g, s.rows);
        }
      }
    }
  };

  Segment cur, nxt;
  bool have = W.next(cur, np);
  if (have) stage(cur, 0);
  cp_async_wait_all();
  __syncthreads();
  int buf = 0;
  while (have) {
    const bool more = W.next(nxt, np);
    if (more) stage(nxt, buf ^ 1);
    if (wm * 32 < nk && cur.rows > 0) {
      const double* As = &S.A[buf][(wm * 32 + (lane >> 2)) * KSEG + (lane & 3)];
      const double* Bs = &S.B[buf][(lane & 3) * G_LD + wn * WPTS + (lane >> 2)];
      for (int kk = 0; kk < cur.rows; kk += 4) {
        double af[4], bf[NT];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) af[mt] = As[mt * 8 * KSEG + kk];
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) bf[nt] = Bs[(size_t)kk * G_LD + nt * 8];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) dmma884(V[mt][nt][0], V[mt][nt][1], af[mt], bf[nt]);
      }
    }
    cp_async_wait_all();
    __syncthreads();
    have = more;
    cur = nxt;
    buf ^= 1;
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
  if (tid == 0) my_far += W.direct_far;
  count_add(cnt, my_near * (unsigned long long)nk, my_far * (unsigned long long)nk, my_terms);
}

// ---------------------------------------------------------------------------
// Per-FO-geometry calls
// ---------------------------------------------------------------------------
// A CTA owns 128 points and up to 32*WM FOs and walks the per-FO calls in
// order.  For each call it classifies the tile against every FO's sphere,
// compacts the FOs with near points into slots, and contracts the G columns
// of one pair per stage (double buffered) with the slots' coefficient rows
// only, so the tensor work follows the FOs that are near rather than the
// whole FO block.  The per-call result is added, masked per (FO, point), to
// the CTA's own slice of vh (L2 resident); the far field of the call follows,
// one FO per warp at a time with lanes over points.
template <int WM>
struct PerFOSmem {
  double A[2][32 * WM * KSEG];  // slot rows of the stage's coefficients; far phase: the FOs' moments (A[0])
  double B[2][KSEG * G_LD];     // G columns of the stage's pair
  double px[TILE], py[TILE], pz[TILE];
  double cg[32 * WM][3];
  double rc2[32 * WM];
  int stat[32 * WM];
  int npot[32 * WM];
  int lmax[32 * WM];
  int nkeep[32 * WM];
  int fo_of[32 * WM];           // slot -> FO (block-local)
  unsigned bal[WM];             // per warp of the status phase: FOs with near points
  unsigned balf[WM];            // per warp of the status phase: FOs with far points
  int na;
};

// Physical A row of slot s: slots fill m-tiles round robin over the WM warp
// rows, so that a few active FOs keep several warps busy.
template <int WM>
__device__ __forceinline__ int slot_row(int s) {
  const int g = s >> 3;
  return (g % WM) * 32 + (g / WM) * 8 + (s & 7);
}

// Far-field potential of one FO at one point, sum_lm MV[lm] Y_lm(u) / r^(l+1),
// summed per degree l and scaled once per degree.
__device__ __forceinline__ double multipole(const double* __restrict__ mv, int lmx, double ux, double uy, double uz,
                                            double hn) {
  double acc[LM + 1];
#pragma unroll
  for (int l = 0; l <= LM; ++l) acc[l] = 0.0;
  harmonics_mmajor(ux, uy, uz, lmx, [&](int row, int l, double v) { acc[l] += mv[row] * v; });
  double pot = 0.0, rec = hn;
#pragma unroll
  for (int l = 0; l <= LM; ++l) {
    pot += acc[l] * rec;
    rec *= hn;
  }
  return pot;
}

template <int WM>
__global__ void __launch_bounds__(MMA_THREADS, 1)
k_coulomb_perfo(int ncalls, const int* __restrict__ lists, int accumulate, const CallInfo* __restrict__ calls,
                const PairGeo* __restrict__ pairs, int nfo, const double* __restrict__ coef,
                const int8_t* __restrict__ pair_fmt, const CallFO* __restrict__ cfo,
                const double* __restrict__ momv, MeshDev M, const double* __restrict__ boys_tab,
                double* __restrict__ vh, int ldv, unsigned long long* __restrict__ cnt) {
  constexpr int FOB = 32 * WM, WN = 8 / WM, WPTS = TILE / WN, NT = WPTS / 8;
  const int* list = lists + ncalls;
  const int nl = lists[2 * ncalls + 1];
  if (accumulate && nl == 0) return;
  extern __shared__ __align__(128) unsigned char smraw[];
  PerFOSmem<WM>& S = *reinterpret_cast<PerFOSmem<WM>*>(smraw);
  const int tile = blockIdx.x;
  const int k0 = blockIdx.y * FOB;
  const int nk = min(FOB, nfo - k0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WM, wn = warp / WM;
  const int p0 = tile * TILE;
  const int np = min(TILE, M.n - p0);
  for (int i = tid; i < TILE; i += MMA_THREADS) {
    const bool a = i < np;
    S.px[i] = a ? M.x[p0 + i] : 0.0;
    S.py[i] = a ? M.y[p0 + i] : 0.0;
    S.pz[i] = a ? M.z[p0 + i] : 0.0;
  }
  if (!accumulate)
    for (int e = tid; e < nk * TILE; e += MMA_THREADS) {
      const int k = e / TILE, p = e - k * TILE;
      if (p < np) vh[(size_t)(k0 + k) * ldv + p0 + p] = 0.0;
    }
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = M.tile_lo[3 * tile + d];
    hi[d] = M.tile_hi[3 * tile + d];
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
        st = (npot == 1) ? 0 : tile_class(lo, hi, cgx, cgy, cgz, rc2);
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
      const bool act = tid < nk && st != 1;
      const unsigned b = __ballot_sync(0xffffffffu, act);
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

    if (na > 0) {
      double T[4][NT][2];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < NT; ++b) T[a][b][0] = T[a][b][1] = 0.0;
      auto stage = [&](int q, int b) {
        const double* src = coef + (size_t)q * nfo * COEF_LD;
        double* dst = S.A[b];
        for (int e = tid; e < na * (KSEG / 2); e += MMA_THREADS) {
          const int s = e / (KSEG / 2), ch = e - s * (KSEG / 2);
          cp_async16(dst + slot_row<WM>(s) * KSEG + 2 * ch, src + (size_t)(k0 + S.fo_of[s]) * COEF_LD + 2 * ch);
        }
        cp_async_commit();
        if (tid < TILE) {
          const int p = tid;
          double* g = &S.B[b][p];
          const int kn = near_rows(pair_fmt[q]);
          if (p < np) {
            const PairGeo& pg = pairs[q];
            const double rx = S.px[p] - pg.C[0], ry = S.py[p] - pg.C[1], rz = S.pz[p] - pg.C[2];
            const double xx = pg.delta * (rz * rz + ry * ry + rx * rx);
            double F[5];
            boys_fmt(boys_tab, xx, exp(-xx), kn >= 48 ? 5 : (kn == 32 ? 4 : 3), F);
            write_g(g, kn, rx, ry, rz, F);
          } else {
            zero_rows(g, kn);
          }
        }
      };
      stage(ci.p0, 0);
      cp_async_wait_all();
      __syncthreads();
      int buf = 0;
      for (int qi = 0; qi < ci.np; ++qi) {
        const int q = ci.p0 + qi;
        if (qi + 1 < ci.np) stage(q + 1, buf ^ 1);
        const int kq = near_rows(pair_fmt[q]);
        const double* As = &S.A[buf][(wm * 32 + (lane >> 2)) * KSEG + (lane & 3)];
        const double* Bs = &S.B[buf][(lane & 3) * G_LD + wn * WPTS + (lane >> 2)];
        for (int kk = 0; kk < kq; kk += 4) {
          double af[4], bf[NT];
#pragma unroll
          for (int mt = 0; mt < 4; ++mt) af[mt] = As[mt * 8 * KSEG + kk];
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) bf[nt] = Bs[(size_t)kk * G_LD + nt * 8];
#pragma unroll
          for (int mt = 0; mt < 4; ++mt) {
            if ((mt * WM + wm) * 8 >= na) continue;
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) dmma884(T[mt][nt][0], T[mt][nt][1], af[mt], bf[nt]);
          }
        }
        cp_async_wait_all();
        __syncthreads();
        buf ^= 1;
      }
      // masked add of the call's near field to vh
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int s = (mt * WM + wm) * 8 + (lane >> 2);
        if (s >= na) continue;
        const int k = S.fo_of[s];
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

    if (anyfar) {
      __syncthreads();  // near phase done with A
      const double* mg = momv + ((size_t)c * nfo + k0) * MOM_LD;
      for (int e = tid; e < nk * MOM_LD; e += MMA_THREADS) S.A[0][e] = mg[e];
      __syncthreads();
      for (int k = warp; k < nk; k += MMA_THREADS / 32) {
        if (S.stat[k] == 0 || S.npot[k] == 1) continue;
        const double cx = S.cg[k][0], cy = S.cg[k][1], cz = S.cg[k][2], rc2 = S.rc2[k];
        const int lmx = S.lmax[k];
        const unsigned long long nkeep = (unsigned long long)S.nkeep[k];
        const double* mv = &S.A[0][k * MOM_LD];
        double* vk = vh + (size_t)(k0 + k) * ldv + p0;
        for (int p = lane; p < np; p += 32) {
          const double x = S.px[p], y = S.py[p], z = S.pz[p];
          const double r2 = sqdist_rn2(x, y, z, cx, cy, cz);
          if (r2 > rc2) {
            ++my_far;
            my_terms += nkeep;
            const double hn = 1.0 / sqrt(r2);
            vk[p] += multipole(mv, lmx, hn * (x - cx), hn * (y - cy), hn * (z - cz), hn);
          }
        }
      }
    }
  }
  count_add(cnt, my_near, my_far, my_terms);
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
  cudaFuncSetAttribute(k_coulomb_shared<WM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(SharedSmem<WM>));
}

template <int WM>
static void set_perfo_attr() {
  cudaFuncSetAttribute(k_coulomb_perfo<WM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
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
}

template <int WM>
static void launch_shared(int ncalls, const int* lists, const CallShare* share, const CallInfo* calls, int nfo,
                          const double* coef, const int8_t* pair_fmt, const PairGeo* pairs, const double* momv,
                          const MeshDev& M, const double* boys_tab, double* vh, int ldv, unsigned long long* cnt,
                          cudaStream_t st) {
  dim3 grid(M.ntiles, (nfo + 32 * WM - 1) / (32 * WM));
  k_coulomb_shared<WM><<<grid, MMA_THREADS, sizeof(SharedSmem<WM>), st>>>(
      ncalls, lists, share, calls, nfo, coef, pair_fmt, pairs, momv, M, boys_tab, vh, ldv, cnt);
}

template <int WM>
static void launch_perfo(int ncalls, const int* lists, int acc, const CallInfo* calls, const PairGeo* pairs, int nfo,
                         const double* coef, const int8_t* pair_fmt, const CallFO* cfo, const double* momv,
                         const MeshDev& M, const double* boys_tab, double* vh, int ldv, unsigned long long* cnt,
                         cudaStream_t st) {
  dim3 grid(M.ntiles, (nfo + 32 * WM - 1) / (32 * WM));
  k_coulomb_perfo<WM><<<grid, MMA_THREADS, sizeof(PerFOSmem<WM>), st>>>(ncalls, lists, acc, calls, pairs, nfo, coef,
                                                                         pair_fmt, cfo, momv, M, boys_tab, vh, ldv,
                                                                         cnt);
}

void launch_coulomb_mma(int ncalls, const CallInfo* calls, const PairGeo* pairs, int npairs, int nfo,
                        const double* coef, const int8_t* maxfmt, const CallFO* cfo, const double* momv,
                        const MeshDev& M, const double* boys_tab, double* vh, int ldv, bool per_fo_only,
                        const CoulombScratch& scr, unsigned long long* cnt, cudaStream_t st) {
  if (npairs > 0) k_pair_fmt<<<(npairs + 127) / 128, 128, 0, st>>>(npairs, nfo, maxfmt, scr.pair_fmt);
  if (ncalls > 0) k_call_share<<<(ncalls + 7) / 8, 256, 0, st>>>(ncalls, nfo, cfo, scr.share);
  k_call_lists<<<1, LIST_THREADS, 0, st>>>(ncalls, per_fo_only ? 1 : 0, scr.share, scr.lists);
  if (!per_fo_only) {
    if (nfo > 64)
      launch_shared<4>(ncalls, scr.lists, scr.share, calls, nfo, coef, scr.pair_fmt, pairs, momv, M, boys_tab, vh,
                       ldv, cnt, st);
    else if (nfo > 32)
      launch_shared<2>(ncalls, scr.lists, scr.share, calls, nfo, coef, scr.pair_fmt, pairs, momv, M, boys_tab, vh,
                       ldv, cnt, st);
    else
      launch_shared<1>(ncalls, scr.lists, scr.share, calls, nfo, coef, scr.pair_fmt, pairs, momv, M, boys_tab, vh,
                       ldv, cnt, st);
  }
  const int acc = per_fo_only ? 0 : 1;
  if (nfo > 64)
    launch_perfo<4>(ncalls, scr.lists, acc, calls, pairs, nfo, coef, scr.pair_fmt, cfo, momv, M, boys_tab, vh, ldv,
                    cnt, st);
  else if (nfo > 32)
    launch_perfo<2>(ncalls, scr.lists, acc, calls, pairs, nfo, coef, scr.pair_fmt, cfo, momv, M, boys_tab, vh, ldv,
                    cnt, st);
  else
    launch_perfo<1>(ncalls, scr.lists, acc, calls, pairs, nfo, coef, scr.pair_fmt, cfo, momv, M, boys_tab, vh, ldv,
                    cnt, st);
}

}  // namespace flosic
