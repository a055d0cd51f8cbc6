// Mixed-precision Coulomb potential of the shared-geometry calls on the
// 5th-generation tensor cores (tcgen05, tensor-memory accumulators).
//
// Same contraction as k_coulomb_shared (csrc/coulomb_mma.cu): for every
// single-pair call whose CG/RCUT/NPOT are the same for all FOs,
//     V[k][p] += sum_t A[k][t] B[t][p]
// with A the FOs' potential coefficients (near segment) or normalised moments
// (far segment) and B the Boys-monomial (near points) or harmonic (far points)
// columns.  Here the B columns are formed in FP32, both operands are split into
// TF32 pairs x = hi + lo, and each product is hi*hi + hi*lo + lo*hi on
// tcgen05.mma kind::tf32 with FP32 accumulation in tensor memory.  Every two
// 32-row windows the FP32 accumulator is folded into a hi/lo FP32 pair, also in
// tensor memory, by an error-free two-sum; the pair is summed in FP64 at the end.
//
// One CTA per tile of 128 points and block of 128 FOs, 512 threads:
//   warp 0       allocates tensor memory; lane 0 issues the MMAs
//   warps 4-7    epilogue: tensor-memory lanes 0-127 (= FO rows)
//   warps 8-15   producers, two per point: stage the calls 128 at a time in
//                shared memory (one coalesced load each, tile class computed
//                once), then walk them; both producers of a point follow the
//                operand windows, the owner of each segment (alternating)
//                writes its B rows (its point); eight producer threads, one per
//                4-row position of a window, load the A rows of all 128 FOs of
//                every chunk with one TMA tiled copy each (cp.async.bulk.tensor:
//                the hi and lo parts, 2 KB each, side by side)
// Operand windows (32 K rows; hi and lo parts of A and B; 64 KB) are triple
// buffered in shared memory in a no-swizzle K-major core-matrix layout (8 rows
// x 16 bytes per core matrix) whose 4-column chunks are 2 KB blocks of all 128
// rows, so that one TMA box lands as one chunk.  Hand-over: mbarriers full (the
// producers' stores) and tma (the copies' transaction bytes) per window buffer,
// empty per window buffer, accfull/accempty per accumulator, done at the end of
// the tile; every
// wait has an iteration limit after which the CTA sets an abort flag, drains its
// copies and MMAs, frees tensor memory and returns with an error flag set.
#include <algorithm>

#include <cuda.h>

#include "coulomb_common.cuh"

namespace flosic {

constexpr int TC_THREADS = 512;
constexpr int TC_KW = 32;                // K rows per operand window
constexpr int TC_NB = 3;                 // window buffers
constexpr int TC_FLUSH = 2;              // windows per FP32 accumulation group
constexpr int TC_EPI0 = 4;               // first epilogue warp
constexpr int TC_PROD0 = 8;              // first producer warp
constexpr int TC_NPROD = 256;            // producer threads: two per point, alternate segments
constexpr int TC_NSTAGE = 128;           // calls staged per chunk
constexpr int TC_BAR_PROD = 5;           // named barrier of the producer warps
constexpr uint32_t TC_TMEM_COLS = 512;   // D0 | D1 | V_hi | V_lo, 128 columns each
constexpr long TC_SPIN_LIMIT = 1L << 25;  // default poll limit of every wait; drains always use it

// One shared-geometry call as the producers walk it.
struct TcCall {
  double cx, cy, cz, rc2;    // centre of gravity and RCUT^2
  double Cx, Cy, Cz, delta;  // pair centre and exponent sum (single-pair calls)
  int c, p0, np, kf, ksum, cls, fmt, pad;
};

struct TcSmem {
  float A[TC_NB][TC_KW / 4][2][TILE * 4];  // [buffer][4-column chunk][hi, lo] FO rows x 4 columns
  float B[TC_NB][2][TILE * TC_KW];  // [buffer][hi, lo] point rows x K
  double px[TILE], py[TILE], pz[TILE];
  TcCall calls[TC_NSTAGE];
  uint64_t full[TC_NB], tma[TC_NB], empty[TC_NB], accfull[2], accempty[2], done, drain;
  int win_rows[TC_NB], win_last[TC_NB];
  int ngroups;
  uint32_t tmem;
  int abort;
};

// Float offset of (row, k) in the no-swizzle K-major core-matrix layout: core
// matrices (8 rows x 4 columns, 128 bytes) of one 4-column chunk follow each
// other over the 128 rows (SBO 128 bytes), chunks follow each other (LBO 2 KB).
constexpr int TC_CHUNK = TILE * 4;  // floats of one 4-column chunk of all rows
__device__ __forceinline__ int cm_off(int row, int k) {
  return (k >> 2) * TC_CHUNK + (row >> 3) * 32 + (row & 7) * 4 + (k & 3);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok)
               : "r"(smem_u32(b)), "r"(parity)
               : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity; false (and the abort flag
// set) when `limit` polls are reached or another role has aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort, long limit) {
  for (long it = 0; it < limit; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 255) == 255) {
      if (*abort) return false;
      __nanosleep(128);
    }
  }
  *abort = 1;
  return false;
}
// Bounded wait that ignores the abort flag: drains the CTA's own MMAs, which
// complete without any other role.
__device__ __forceinline__ bool mbar_wait_drain(uint64_t* b, uint32_t parity) {
  for (long it = 0; it < TC_SPIN_LIMIT; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 255) == 255) __nanosleep(128);
  }
  return false;
}

// Expect `bytes` more transaction bytes on b in its current phase.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
// TMA tiled load of the box at (0, y, z, w) of a 4-D tensor map into shared
// memory; its bytes complete on b.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int y, int z, int w, uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(y), "r"(z), "r"(w), "r"(smem_u32(b))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void producer_sync() {
  asm volatile("bar.sync %0, %1;\n" ::"r"(TC_BAR_PROD), "r"(TC_NPROD) : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* b) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(b))
               : "memory");
}

// Shared-memory matrix descriptor: no swizzle, K-major; lbo = byte step between
// core matrices along K, sbo = byte step between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::tf32: D f32, A and B tf32, both K-major.
__host__ __device__ constexpr uint32_t tf32_idesc(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tc_mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

#define TC_REG32(v)                                                                                         \
  "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), \
      "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),  \
      "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), \
      "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
#define TC_IN32(v)                                                                                          \
  "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]), \
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]), "r"(v[17]),           \
      "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]),            \
      "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])

// 32 consecutive 32-bit columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : TC_REG32(v)
      : "r"(taddr));
}
__device__ __forceinline__ void tc_st32(uint32_t taddr, const uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,"
      "%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n" ::"r"(taddr),
      TC_IN32(v)
      : "memory");
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tc_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// Round to TF32 (nearest, ties away); the low 13 mantissa bits become zero.
__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// x = hi + lo with hi, lo TF32 values.
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo) {
  hi = tf32_round(x);
  lo = tf32_round(x - hi);
}

// G column values (COEFICIENT order, rows 46..51 zero) of one near point.
__device__ __forceinline__ void g_values(float (&v)[KSEG], double Cx, double Cy, double Cz, double delta, double x,
                                         double y, double z, int kn, const double* __restrict__ boys_tab) {
  const float rx = (float)(x - Cx), ry = (float)(y - Cy), rz = (float)(z - Cz);
  const float xx = (float)delta * (rz * rz + ry * ry + rx * rx);
  float F[5];
  boys_fmt<float>(boys_tab, xx, expf(-xx), kn >= 48 ? 5 : (kn == 32 ? 4 : 3), F);
  const float zz = rz * rz, yz = ry * rz, yy = ry * ry, xz = rx * rz, xy = rx * ry, xq = rx * rx;
  v[0] = F[0];
  v[1] = F[1];
  v[2] = F[2];
  v[3] = F[1] * rz;
  v[4] = F[1] * ry;
  v[5] = F[1] * rx;
  v[6] = F[2] * rz;
  v[7] = F[2] * ry;
  v[8] = F[2] * rx;
  v[9] = F[2] * zz;
  v[10] = F[2] * yz;
  v[11] = F[2] * yy;
  v[12] = F[2] * xz;
  v[13] = F[2] * xy;
  v[14] = F[2] * xq;
  v[15] = F[3] * zz;
  v[16] = F[3] * yz;
  v[17] = F[3] * yy;
  v[18] = F[3] * xz;
  v[19] = F[3] * xy;
  v[20] = F[3] * xq;
  v[21] = F[3] * (rz * zz);
  v[22] = F[3] * (ry * zz);
  v[23] = F[3] * (rz * yy);
  v[24] = F[3] * (ry * yy);
  v[25] = F[3] * (rx * zz);
  v[26] = F[3] * (rx * yz);
  v[27] = F[3] * (rx * yy);
  v[28] = F[3] * (rz * xq);
  v[29] = F[3] * (ry * xq);
  v[30] = F[3] * (rx * xq);
  v[31] = F[4] * (zz * zz);
  v[32] = F[4] * (zz * yz);
  v[33] = F[4] * (yy * zz);
  v[34] = F[4] * (yy * yz);
  v[35] = F[4] * (yy * yy);
  v[36] = F[4] * (zz * xz);
  v[37] = F[4] * (xy * zz);
  v[38] = F[4] * (xy * yz);
  v[39] = F[4] * (yy * xy);
  v[40] = F[4] * (xq * zz);
  v[41] = F[4] * (xq * yz);
  v[42] = F[4] * (xq * yy);
  v[43] = F[4] * (xz * xq);
  v[44] = F[4] * (xy * xq);
  v[45] = F[4] * (xq * xq);
#pragma unroll
  for (int t = 46; t < KSEG; ++t) v[t] = 0.f;
}

// H column values (harmonics / r^(l+1) in moment row order) of one far point
// up to degree LMX, zero up to the next multiple of 4 rows.
template <int LMX>
__device__ __forceinline__ void h_values(float (&v)[KSEG], float dx, float dy, float dz, float r2) {
  constexpr int NR = (LMX + 1) * (LMX + 1), NR4 = (NR + 3) / 4 * 4;
  const float hn = rsqrtf(r2);
  float rec[LMX + 1];
  rec[0] = hn;
#pragma unroll
  for (int l = 1; l <= LMX; ++l) rec[l] = rec[l - 1] * hn;
  harmonics_mmajor<float>(hn * dx, hn * dy, hn * dz, LMX, [&](int row, int l, float h) { v[row] = h * rec[l]; });
#pragma unroll
  for (int t = NR; t < NR4; ++t) v[t] = 0.f;
}

// Dispatch on the moment rows kf = ((lmax + 1)^2 rounded up to 4).
__device__ __forceinline__ void h_values_kf(float (&v)[KSEG], int kf, float dx, float dy, float dz, float r2) {
  switch (kf) {
    case 4: h_values<1>(v, dx, dy, dz, r2); break;
    case 12: h_values<2>(v, dx, dy, dz, r2); break;
    case 16: h_values<3>(v, dx, dy, dz, r2); break;
    case 28: h_values<4>(v, dx, dy, dz, r2); break;
    case 36: h_values<5>(v, dx, dy, dz, r2); break;
    default: h_values<6>(v, dx, dy, dz, r2); break;
  }
}

__global__ void __launch_bounds__(TC_THREADS, 1)
k_coulomb_shared_tc(int ncalls, const int* __restrict__ lists, const CallShare* __restrict__ share,
                    const CallInfo* __restrict__ calls, int nfo, const __grid_constant__ CUtensorMap tm_coef,
                    const int8_t* __restrict__ pair_fmt, const PairGeo* __restrict__ pairs,
                    const __grid_constant__ CUtensorMap tm_mom, MeshDev M,
                    const double* __restrict__ boys_tab, double* __restrict__ vh, int ldv,
                    unsigned long long* __restrict__ cnt, int* __restrict__ err, long wait_limit) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(smraw);
  const int tile = blockIdx.x;
  const int k0 = blockIdx.y * TILE;
  const int nk = min(TILE, nfo - k0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p0 = tile * TILE;
  const int np = min(TILE, M.n - p0);
  volatile int* abort = &S.abort;
  for (int i = tid; i < TILE; i += TC_THREADS) {
    const bool a = i < np;
    S.px[i] = a ? M.x[p0 + i] : 0.0;
    S.py[i] = a ? M.y[p0 + i] : 0.0;
    S.pz[i] = a ? M.z[p0 + i] : 0.0;
  }
  if (tid == 0) {
    for (int b = 0; b < TC_NB; ++b) {
      mbar_init(&S.full[b], TC_NPROD);  // per producer: its stores
      mbar_init(&S.tma[b], TC_KW / 4);  // the 8 loading threads, plus the copies' transaction bytes
      mbar_init(&S.empty[b], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&S.accfull[a], 1);
      mbar_init(&S.accempty[a], 128);
    }
    mbar_init(&S.done, 1);
    mbar_init(&S.drain, 1);
    S.abort = 0;
    S.ngroups = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&S.tmem)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem;
  unsigned long long my_near = 0, my_far = 0, my_terms = 0;

  if (warp >= TC_PROD0) {
    // ---------------- producers
    const int pt = (tid - TC_PROD0 * 32) & (TILE - 1);  // point p = pt, and A row (FO) pt
    const int half = (tid - TC_PROD0 * 32) >> 7;       // owns segments with (index & 1) == half
    const int p = pt;
    const bool count_terms = blockIdx.y == 0;  // kept terms are summed over all FOs once per (call, point)
    const int nsh = lists[2 * ncalls];
    double lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
      lo[d] = M.tile_lo[3 * tile + d];
      hi[d] = M.tile_hi[3 * tile + d];
    }
    const double x = S.px[p], y = S.py[p], z = S.pz[p];
    // eight threads (two per warp of the second producer half) load the A
    // chunks: the one of window position tma_pos loads every chunk that lands
    // there, and arrives once per window on the window's tma barrier
    const int tma_pos = (half == 1 && (pt & 15) == 0) ? (pt >> 4) : -1;
    int w = 0, fill = 0, buf = 0;
    bool open = false, ok = true, open_ok = false;  // open_ok: this thread's wait for the open window succeeded
    auto win_open = [&]() {
      buf = w % TC_NB;
      open_ok = w < TC_NB || mbar_wait(&S.empty[buf], (uint32_t)((w / TC_NB - 1) & 1), abort, wait_limit);
      if (!open_ok) ok = false;
      fill = 0;
      open = true;
    };
    auto win_close = [&](int rows, int last) {
      // the thread's own st.shared become visible to the tensor core (async
      // proxy); the A chunks' TMA copies complete on the window's tma barrier
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      if (pt == 0 && half == 0) {
        S.win_rows[buf] = rows;
        S.win_last[buf] = last;
      }
      if (tma_pos >= 0) mbar_arrive(&S.tma[buf]);
      mbar_arrive(&S.full[buf]);
      ++w;
      open = false;
    };
    // one segment: B rows of this point (v, rows; zeros when !live), and, by the
    // loading thread of each chunk's window position, the A rows of the block's
    // 128 FOs from chunk z0 of map tm
    auto emit = [&](const float (&v)[KSEG], bool mine, bool live, int rows, const CUtensorMap* tm, int z0) {
#pragma unroll
      for (int j4 = 0; j4 < KSEG / 4; ++j4) {
        if (4 * j4 >= rows || !ok) break;
        if (!open) {
          win_open();
          if (!ok) break;
        }
        if (tma_pos == (fill >> 2)) {
          // one box = the chunk's hi and lo parts, which lie next to each other
          mbar_expect_tx(&S.tma[buf], 2u * TC_CHUNK * (uint32_t)sizeof(float));
          tma_load_4d(S.A[buf][fill >> 2][0], tm, k0, z0 + j4, 0, &S.tma[buf]);
        }
        const int o = cm_off(p, fill);
        if (!mine) {
          // the other producer of this point writes this segment
        } else if (live) {
          float h4[4], l4[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) tf32_split(v[4 * j4 + e], h4[e], l4[e]);
          *reinterpret_cast<float4*>(&S.B[buf][0][o]) = make_float4(h4[0], h4[1], h4[2], h4[3]);
          *reinterpret_cast<float4*>(&S.B[buf][1][o]) = make_float4(l4[0], l4[1], l4[2], l4[3]);
        } else {
          *reinterpret_cast<float4*>(&S.B[buf][0][o]) = make_float4(0.f, 0.f, 0.f, 0.f);
          *reinterpret_cast<float4*>(&S.B[buf][1][o]) = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        fill += 4;
        if (fill == TC_KW) win_close(TC_KW, 0);
      }
    };
    // Every producer takes the same sequence of named-barrier steps (the chunk
    // loop does not depend on ok); only the work inside is skipped after an abort.
    int seg = 0;  // index of the next segment that writes rows
    for (int li0 = 0; li0 < nsh; li0 += TC_NSTAGE) {
      const int nchunk = min(TC_NSTAGE, nsh - li0);
      producer_sync();  // the previous chunk has been walked by every producer
      if (half == 0 && pt < nchunk) {
        TcCall e;
        e.c = lists[li0 + pt];
        const CallShare sh = share[e.c];
        const CallInfo ci = calls[e.c];
        e.cx = sh.cg[0];
        e.cy = sh.cg[1];
        e.cz = sh.cg[2];
        e.rc2 = sh.rcut2;
        e.kf = sh.kf;
        e.ksum = sh.ksum;
        e.p0 = ci.p0;
        e.np = ci.np;
        e.cls = (sh.npot == 1) ? 0 : tile_class(lo, hi, e.cx, e.cy, e.cz, e.rc2);
        e.fmt = pair_fmt[ci.p0];
        const PairGeo& pg = pairs[ci.p0];
        e.Cx = pg.C[0];
        e.Cy = pg.C[1];
        e.Cz = pg.C[2];
        e.delta = pg.delta;
        e.pad = 0;
        S.calls[pt] = e;
      }
      producer_sync();
      for (int i = 0; i < nchunk && ok; ++i) {
        const TcCall& e = S.calls[i];
        float v[KSEG];
        if (e.cls != 1) {  // near segments, one per pair
          for (int qi = 0; qi < e.np && ok; ++qi) {
            const int q = e.p0 + qi;
            const int kn = near_rows(qi == 0 ? e.fmt : pair_fmt[q]);
            const bool mine = (seg++ & 1) == half;
            bool nr = mine && p < np;
            if (nr && e.cls == 2) nr = !(sqdist_rn2(x, y, z, e.cx, e.cy, e.cz) > e.rc2);
            if (nr) {
              ++my_near;
              if (qi == 0) {
                g_values(v, e.Cx, e.Cy, e.Cz, e.delta, x, y, z, kn, boys_tab);
              } else {
                const PairGeo& pg = pairs[q];
                g_values(v, pg.C[0], pg.C[1], pg.C[2], pg.delta, x, y, z, kn, boys_tab);
              }
            }
            emit(v, mine, nr, kn, &tm_coef, q * (KSEG / 4));
          }
        }
        if (e.cls != 0) {  // far segment (NPOT=2)
          // near/far of a point on a boundary tile is decided in FP64, as in the
          // reference; the harmonics use the FP32 offset
          const bool mine = e.kf > 0 ? (seg++ & 1) == half : half == 0;
          bool fr = mine && p < np;
          if (fr && e.cls == 2) fr = sqdist_rn2(x, y, z, e.cx, e.cy, e.cz) > e.rc2;
          if (fr) {
            ++my_far;
            if (count_terms) my_terms += (unsigned long long)e.ksum;
          }
          if (e.kf > 0) {
            if (fr) {
              const float dx = (float)(x - e.cx), dy = (float)(y - e.cy), dz = (float)(z - e.cz);
              h_values_kf(v, e.kf, dx, dy, dz, dx * dx + dy * dy + dz * dz);
            }
            emit(v, mine, fr, e.kf, &tm_mom, e.c * (KSEG / 4));
          }
        }
      }
    }
    if (ok) {
      if (!open) {
        win_open();
        if (ok) win_close(0, 1);
      } else {
        if (fill & 7) {  // pad the last k-step of 8 rows with zeros
          if (half == 0) {
          const int o = cm_off(p, fill);
          *reinterpret_cast<float4*>(&S.B[buf][0][o]) = make_float4(0.f, 0.f, 0.f, 0.f);
          *reinterpret_cast<float4*>(&S.B[buf][1][o]) = make_float4(0.f, 0.f, 0.f, 0.f);
          *reinterpret_cast<float4*>(&S.A[buf][fill >> 2][0][4 * pt]) = make_float4(0.f, 0.f, 0.f, 0.f);
          *reinterpret_cast<float4*>(&S.A[buf][fill >> 2][1][4 * pt]) = make_float4(0.f, 0.f, 0.f, 0.f);
          }
          fill += 4;
        }
        win_close(fill, 1);
      }
    }
    if (tma_pos >= 0) {
      // every copy lands before the tile ends: a loading thread whose wait for
      // a window left open by an abort succeeded takes its part of that
      // window's phase (the buffer's previous phase has completed), then waits
      // for the last phase of each buffer (the earlier ones completed before
      // their buffer was reused); a phase that a failed wait left incomplete
      // ends this wait at its limit
      int wl = w;
      if (open && open_ok) {
        mbar_arrive(&S.tma[buf]);
        wl = w + 1;
      }
      for (int j = max(0, wl - TC_NB); j < wl; ++j)
        if (!mbar_wait_drain(&S.tma[j % TC_NB], (uint32_t)((j / TC_NB) & 1))) *abort = 1;
    }
  } else if (warp == 0) {
    // ---------------- MMA issue
    if (lane == 0) {
      constexpr uint32_t idesc = tf32_idesc(TILE, TILE);
      // B: chunks of one part follow each other (2 KB); A: a chunk's hi and lo
      // parts lie together, so its chunks are 4 KB apart
      constexpr uint32_t LBO = TC_CHUNK * sizeof(float), LBO_A = 2 * LBO, SBO = 128;
      int a = 0, nin = 0, g = 0;
      for (int w = 0;; ++w) {
        const int b = w % TC_NB;
        if (!mbar_wait(&S.full[b], (uint32_t)((w / TC_NB) & 1), abort, wait_limit)) break;
        if (!mbar_wait(&S.tma[b], (uint32_t)((w / TC_NB) & 1), abort, wait_limit)) break;
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        tc_fence_after();
        const int r = S.win_rows[b], last = S.win_last[b];
        if (r > 0) {
          if (nin == 0 && g >= 2) {
            if (!mbar_wait(&S.accempty[a], (uint32_t)((g / 2 - 1) & 1), abort, wait_limit)) break;
            tc_fence_after();
          }
          const uint32_t d = tmem + (uint32_t)(a * TILE);
          const uint32_t ah = smem_u32(S.A[b][0][0]), al = smem_u32(S.A[b][0][1]);
          const uint32_t bh = smem_u32(S.B[b][0]), bl = smem_u32(S.B[b][1]);
          for (int ks = 0; ks < r / 8; ++ks) {
            const uint32_t offa = (uint32_t)ks * 2u * LBO_A, offb = (uint32_t)ks * 2u * LBO;  // 8 K columns
            const uint64_t dah = smem_desc(ah + offa, LBO_A, SBO), dal = smem_desc(al + offa, LBO_A, SBO);
            const uint64_t dbh = smem_desc(bh + offb, LBO, SBO), dbl = smem_desc(bl + offb, LBO, SBO);
            tc_mma_tf32(d, dah, dbh, idesc, (nin > 0 || ks > 0) ? 1u : 0u);
            tc_mma_tf32(d, dah, dbl, idesc, 1u);
            tc_mma_tf32(d, dal, dbh, idesc, 1u);
          }
          ++nin;
        }
        tc_commit(&S.empty[b]);
        if (nin > 0 && (nin == TC_FLUSH || last)) {
          tc_commit(&S.accfull[a]);
          a ^= 1;
          nin = 0;
          ++g;
        }
        if (last) break;
      }
      // every MMA issued so far completes before the tile ends
      tc_commit(&S.drain);
      if (!mbar_wait_drain(&S.drain, 0u)) *abort = 1;
      S.ngroups = g;
      mbar_arrive(&S.done);
    }
    __syncwarp();
  } else if (warp >= TC_EPI0 && warp < TC_EPI0 + 4) {
    // ---------------- epilogue: lanes 32q..32q+31 of tensor memory
    const int q = warp & 3;
    const uint32_t lb = tmem + ((uint32_t)(32 * q) << 16);
    uint32_t zero[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) zero[j] = 0u;
#pragma unroll
    for (int c0 = 0; c0 < TILE; c0 += 32) {
      tc_st32(lb + 2 * TILE + c0, zero);
      tc_st32(lb + 3 * TILE + c0, zero);
    }
    tc_wait_st();
    for (int g = 0;; ++g) {
      const int a = g & 1;
      bool have = false;
      for (long it = 0; it < wait_limit; ++it) {
        if (mbar_try(&S.accfull[a], (uint32_t)((g / 2) & 1))) {
          have = true;
          break;
        }
        if ((it & 255) == 255) {
          if (*abort) break;
          if (mbar_try(&S.done, 0u) && g >= S.ngroups) break;
          __nanosleep(128);
        }
        if (it == wait_limit - 1) *abort = 1;
      }
      if (!have) break;
      tc_fence_after();
#pragma unroll 1
      for (int c0 = 0; c0 < TILE; c0 += 32) {
        uint32_t dv[32], hv[32], lv[32];
        tc_ld32(lb + (uint32_t)(a * TILE) + c0, dv);
        tc_ld32(lb + 2 * TILE + c0, hv);
        tc_ld32(lb + 3 * TILE + c0, lv);
        tc_wait_ld();
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const float d = __uint_as_float(dv[j]), h = __uint_as_float(hv[j]);
          const float s = h + d;
          const float bb = s - h;
          const float e = (h - (s - bb)) + (d - bb);
          hv[j] = __float_as_uint(s);
          lv[j] = __float_as_uint(__uint_as_float(lv[j]) + e);
        }
        tc_st32(lb + 2 * TILE + c0, hv);
        tc_st32(lb + 3 * TILE + c0, lv);
      }
      tc_wait_st();
      tc_fence_before();
      mbar_arrive(&S.accempty[a]);
    }
    if (!*abort) {
      const int k = 32 * q + lane;
#pragma unroll 1
      for (int c0 = 0; c0 < TILE; c0 += 32) {
        uint32_t hv[32], lv[32];
        tc_ld32(lb + 2 * TILE + c0, hv);
        tc_ld32(lb + 3 * TILE + c0, lv);
        tc_wait_ld();
        if (k < nk) {
          double* o = vh + (size_t)(k0 + k) * ldv + p0 + c0;
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (c0 + j < np) o[j] = (double)__uint_as_float(hv[j]) + (double)__uint_as_float(lv[j]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_TMEM_COLS)
                 : "memory");
  if (tid == 0 && S.abort) atomicExch(err, 1);
  count_add(cnt, my_near * (unsigned long long)nk, my_far * (unsigned long long)nk, my_terms);
}

// hi/lo TF32 split of rows [nrow][nfo][KSEG] doubles into the chunk-major
// layout the producers copy from, [nrow][KSEG/4][nfo][4] floats (hi at out,
// lo at out + part): the 128 FOs' values of one 4-row chunk are contiguous, so
// a warp's copies of a chunk are coalesced.
__global__ void k_split_tf32(size_t nrow, int nfo, const double* __restrict__ src, float* __restrict__ out,
                             size_t part) {
  const size_t n = nrow * nfo * KSEG;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / ((size_t)nfo * KSEG);
    const int k = (int)((i / KSEG) % nfo), t = (int)(i % KSEG);
    const double x = src[i];
    const float hi = tf32_round((float)x);
    const float lo = tf32_round((float)(x - (double)hi));
    const size_t o = ((r * (KSEG / 4) + t / 4) * nfo + k) * 4 + (t & 3);
    out[o] = hi;
    out[part + o] = lo;
  }
}

void init_coulomb_tc() {
  cudaFuncSetAttribute(k_coulomb_shared_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem));
}

void launch_split_tf32(size_t nrow, int nfo, const double* src, float* out, cudaStream_t st) {
  const size_t n = nrow * nfo * KSEG;
  if (n == 0) return;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_split_tf32<<<blocks, 256, 0, st>>>(nrow, nfo, src, out, n);
}

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, looked up once through the runtime (the
// library links no driver library).
EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<EncodeTiledFn>(nullptr);
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Tensor map of TF32 hi/lo rows in the split layout [nrow][KSEG/4][nfo][4]
// floats, lo part at + part floats: dimensions (4 columns, nfo FOs, nrow*KSEG/4
// chunks, 2 parts), box (4, 128, 1, 2) = one 2 KB chunk of a 128-FO block in
// both parts (hi, then lo); FOs past nfo read as zero.  Every stride is a multiple of 16 bytes (nfo*16;
// part is a multiple of 4 floats since KSEG is).
bool rows_map(CUtensorMap* m, const float* base, int nfo, size_t nrow, size_t part) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc || !base || nfo <= 0) return false;
  const size_t nchunk = std::max<size_t>(nrow, 1) * (KSEG / 4);
  const size_t pstride = std::max(part, nchunk * (size_t)nfo * 4) * sizeof(float);
  const cuuint64_t dims[4] = {4, (cuuint64_t)nfo, (cuuint64_t)nchunk, 2};
  const cuuint64_t strides[3] = {16, (cuuint64_t)nfo * 16, (cuuint64_t)pstride};
  const cuuint32_t box[4] = {4, TILE, 1, 2};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

cudaError_t launch_coulomb_shared_tc(int ncalls, const int* lists, const CallShare* share, const CallInfo* calls,
                                     int nfo, const float* coef_hl, size_t coef_part, const int8_t* pair_fmt,
                                     const PairGeo* pairs, const float* momv_hl, size_t mom_part, const MeshDev& M,
                                     const double* boys_tab, double* vh, int ldv, unsigned long long* cnt, int* err,
                                     long long wait_limit, cudaStream_t st) {
  static_assert(KSEG % 4 == 0, "the split layout's parts start on 16-byte boundaries");
  CUtensorMap tm_coef, tm_mom;
  const size_t npairs = coef_part / ((size_t)nfo * KSEG), nmom = mom_part / ((size_t)nfo * KSEG);
  if (!rows_map(&tm_coef, coef_hl, nfo, npairs, coef_part) || !rows_map(&tm_mom, momv_hl, nfo, nmom, mom_part))
    return cudaErrorInvalidValue;
  dim3 grid(M.ntiles, (nfo + TILE - 1) / TILE);
  const long lim = wait_limit > 0 ? (long)wait_limit : TC_SPIN_LIMIT;
  k_coulomb_shared_tc<<<grid, TC_THREADS, sizeof(TcSmem), st>>>(ncalls, lists, share, calls, nfo, tm_coef, pair_fmt,
                                                                   pairs, tm_mom, M, boys_tab, vh, ldv, cnt, err, lim);
  return cudaGetLastError();
}

}  // namespace flosic
