// Device helpers shared by the FP64 (coulomb_mma.cu) and the mixed-precision
// tensor-core (coulomb_tc.cu) Coulomb kernels: call/tile geometry, Boys values,
// harmonics, the segment walk over single-pair calls, and work counters.
#pragma once

#include <cfloat>
#include <type_traits>

#include "device_math.cuh"
#include "kernels.cuh"

namespace flosic {

constexpr int G_LD = TILE + 4;              // 132 (= 4 mod 16 doubles): conflict-free B fragment loads
constexpr int KSEG = 52;                    // rows of one B segment (46 coefficients or 49 moments, padded)
static_assert(COEF_LD == KSEG && MOM_LD == KSEG, "segment rows and global row strides must agree");

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
template <typename T, typename Op>
__device__ __forceinline__ void harmonics_mmajor(T ux, T uy, T uz, int lmx, Op op) {
  // m = 0
  {
    op(0, 0, T(1));
    if (lmx >= 1) op(1, 1, uz);
    T p2 = T(1), p1 = uz;
#pragma unroll
    for (int l = 2; l <= LM; ++l) {
      if (l > lmx) break;
      const T facrc = T(1) / T(l);
      const T aa = facrc * T(2 * l - 1), bb = facrc * T(l - 1);
      const T cu = aa * p1 * uz - bb * p2;
      op(l * l, l, cu);
      p2 = p1;
      p1 = cu;
    }
  }
  T sc = ux, ss = uy;  // sectoral pair at l = m
#pragma unroll
  for (int m = 1; m <= LM; ++m) {
    if (m > lmx) break;
    if (m > 1) {
      const T ifc = T(2 * m - 1);
      const T nc = ifc * (sc * ux - ss * uy);
      const T ns = ifc * (ss * ux + sc * uy);
      sc = nc;
      ss = ns;
    }
    op(m * m + 2 * m - 1, m, sc);
    op(m * m + 2 * m, m, ss);
    T c2 = T(0), s2 = T(0), c1 = sc, s1 = ss;
#pragma unroll
    for (int l = m + 1; l <= LM; ++l) {
      if (l > lmx) break;
      const T facrc = T(1) / T(l - m);
      const T aa = facrc * T(2 * l - 1);
      const T bb = (m == l - 1) ? T(0) : facrc * T(l + m - 1);
      const T cc = aa * c1 * uz - bb * c2;
      const T cs = aa * s1 * uz - bb * s2;
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
// boys_all); absent orders are zero.  T = float evaluates the same steps in
// single precision (the mixed-precision path).
template <typename T>
__device__ __forceinline__ void boys_fmt(const double* __restrict__ tab, T x, T chgd, int fmt, T F[5]) {
  if (x > T(16)) {
    const T ROOTPI = T(1.77245385090551602728);
    const T pol1 = -chgd;
    T rt;
    if constexpr (sizeof(T) == 8) rt = __dmul_rn(sqrt(x), ROOTPI);
    else rt = sqrtf(x) * ROOTPI;
    const T rect1 = T(0.5) / x;
    F[0] = rect1 * (rt + pol1);
    F[1] = rect1 * (F[0] + pol1);
    F[2] = rect1 * (T(3) * F[1] + pol1);
    F[3] = (fmt >= 4) ? rect1 * (T(5) * F[2] + pol1) : T(0);
    F[4] = (fmt >= 5) ? rect1 * (T(7) * F[3] + pol1) : T(0);
    return;
  }
  const int it = (int)(T(100) * x + T(1.5));
  const T pol1 = chgd;
  const T rect1 = T(2) * x;
  const T dt = T(1.0e-2) * T(it - 1) - x;
  const double* f = tab + (size_t)(it - 1) * BOYS_NC;
  const T o7 = T(1) / T(7), o5 = T(1) / T(5), o3 = T(1) / T(3);
  if (fmt == 5) {
    F[4] = T(f[2]) + dt * (T(f[3]) + dt * (T(f[6]) + dt * T(f[9])));
    F[3] = (F[4] * rect1 + pol1) * o7;
    F[2] = (F[3] * rect1 + pol1) * o5;
  } else if (fmt == 4) {
    F[4] = T(0);
    F[3] = T(f[1]) + dt * (T(f[2]) + dt * (T(f[5]) + dt * T(f[8])));
    F[2] = (F[3] * rect1 + pol1) * o5;
  } else {
    F[4] = T(0);
    F[3] = T(0);
    F[2] = T(f[0]) + dt * (T(f[1]) + dt * (T(f[4]) + dt * T(f[7])));
  }
  F[1] = (F[2] * rect1 + pol1) * o3;
  F[0] = (F[1] * rect1 + pol1);
}

// Rows of the near segment used by a pair whose largest Boys variant is fmt:
// slots 15.. carry F_3 and slots 31.. carry F_4 (COEFICIENT order,
// poisson1.f:402-482).
__device__ __forceinline__ int near_rows(int fmt) { return fmt >= 5 ? 48 : (fmt == 4 ? 32 : 16); }

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

// Degree whose harmonics fill kf moment rows ((l+1)^2 rounded up to 4).
__device__ __forceinline__ int far_degree(int kf) {
  return kf <= 4 ? 1 : (kf <= 12 ? 2 : (kf <= 16 ? 3 : (kf <= 28 ? 4 : (kf <= 36 ? 5 : 6))));
}

// H column (rows [0, kf)) of one far point: harmonics times 1/r^(l+1), zero padded.
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
// far segment unless the tile is entirely near or NPOT=1.
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

  __device__ bool next(Segment& s) {
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
        s = Segment{1, c, kf, cls, ksum, cx, cy, cz, rc2};
        return true;
      }
    }
    return false;
  }
};

}  // namespace flosic
