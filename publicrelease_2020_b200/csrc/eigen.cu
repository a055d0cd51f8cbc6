// Symmetric eigen-decomposition of the FO overlap on the GPU: the role of
// DIAGGE_FO / EWEVGE_FO (diagon_sic.f:45-232, Householder tridiagonalisation
// and implicit QL) in LOWSIC (lowden_files.f:2-172), done here by the cyclic
// Jacobi method with the round-robin (tournament) ordering, which rotates
// n/2 disjoint index pairs at once.  One CTA holds the whole problem (N_o is at
// most a few hundred): the matrix in shared memory when it fits, the
// accumulated rotations in global memory (L2 resident, rows contiguous).
//
// Each round: every pair (p, q) gets the rotation that zeroes A(p,q) (the
// symmetric Schur decomposition with t = sign(tau)/(|tau| + sqrt(1 + tau^2))),
// then all row updates A <- J^T A, then all column updates A <- A J and
// V <- V J.  An off-diagonal entry below eps/2 sqrt|A(p,p) A(q,q)| is not
// rotated; a sweep (m - 1 rounds, m = n rounded up to even) without any
// rotation ends the iteration.  Eigenvalues are returned in ascending order,
// as EWEVGE_FO returns them with IORD = -1 (diagon_sic.f:64), with their
// eigenvectors in the same order.  Everything is FP64.
#include <cfloat>

#include "kernels.cuh"

namespace flosic {

constexpr int EIG_THREADS = 1024;
constexpr int EIG_MAX_N = 1024;          // pairs held in shared memory: EIG_MAX_N / 2
constexpr int EIG_SMEM_MAX_N = 160;      // matrix in shared memory up to 160 x 161 doubles (206 KB)
constexpr int EIG_MAX_SWEEPS = 60;

// A(i, j) at A[i * (n + 1) + j]: the odd pitch spreads a column over the
// shared-memory banks.  The rotations are accumulated transposed, Vt(m, k) =
// component k of vector m, so that a column update of V is a row update of Vt
// (contiguous in memory).
__global__ void __launch_bounds__(EIG_THREADS, 1)
k_sym_eigen(int n, const double* __restrict__ ain, double* __restrict__ aglob, double* __restrict__ vt,
            double* __restrict__ wout, double* __restrict__ vout, int* __restrict__ info) {
  extern __shared__ __align__(16) double eig_sm[];
  __shared__ double rc[EIG_MAX_N / 2], rs[EIG_MAX_N / 2];
  __shared__ int rp[EIG_MAX_N / 2], rq[EIG_MAX_N / 2];
  __shared__ int nrot;
  double* A = (n <= EIG_SMEM_MAX_N) ? eig_sm : aglob;
  const int ld = n + 1;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, j = e - i * n;
    A[i * ld + j] = ain[e];
    vt[e] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int m = n + (n & 1), half = m / 2;
  bool converged = (n <= 1);
  for (int sweep = 0; sweep < EIG_MAX_SWEEPS && !converged; ++sweep) {
    if (tid == 0) nrot = 0;
    __syncthreads();
    for (int r = 0; r < m - 1; ++r) {
      for (int k = tid; k < half; k += nt) {
        const int a = (k == 0) ? 0 : ((k - 1 + r) % (m - 1)) + 1;
        const int b = ((m - 2 - k + r) % (m - 1)) + 1;
        const int p = min(a, b), q = max(a, b);
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = A[p * ld + q];
          const double app = A[p * ld + p], aqq = A[q * ld + q];
          if (apq != 0.0 && fabs(apq) > 0.5 * DBL_EPSILON * sqrt(fabs(app * aqq))) {
            const double tau = (aqq - app) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
            atomicAdd(&nrot, 1);
          }
        }
        rp[k] = p;
        rq[k] = q;
        rc[k] = c;
        rs[k] = s;
      }
      __syncthreads();
      // rows p, q of A (A <- J^T A) and of Vt (V <- V J)
      for (int e = tid; e < half * n; e += nt) {
        const int k = e / n, j = e - k * n;
        const double s = rs[k];
        if (s == 0.0) continue;
        const double c = rc[k];
        const int p = rp[k], q = rq[k];
        double x = A[p * ld + j], y = A[q * ld + j];
        A[p * ld + j] = c * x - s * y;
        A[q * ld + j] = s * x + c * y;
        x = vt[p * n + j];
        y = vt[q * n + j];
        vt[p * n + j] = c * x - s * y;
        vt[q * n + j] = s * x + c * y;
      }
      __syncthreads();
      // columns p, q of A (A <- A J); lanes run over rows i
      for (int e = tid; e < half * n; e += nt) {
        const int k = e / n, i = e - k * n;
        const double s = rs[k];
        if (s == 0.0) continue;
        const double c = rc[k];
        const int p = rp[k], q = rq[k];
        const double x = A[i * ld + p], y = A[i * ld + q];
        A[i * ld + p] = c * x - s * y;
        A[i * ld + q] = s * x + c * y;
      }
      __syncthreads();
    }
    converged = (nrot == 0);
    __syncthreads();  // every thread has read nrot before it is reset
  }
  // ascending order (ties by index): rank of each eigenvalue, then scatter
  for (int i = tid; i < n; i += nt) {
    const double d = A[i * ld + i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double dj = A[j * ld + j];
      rank += (dj < d || (dj == d && j < i)) ? 1 : 0;
    }
    wout[rank] = d;
    for (int k = 0; k < n; ++k) vout[(size_t)k * n + rank] = vt[(size_t)i * n + k];
  }
  if (tid == 0) *info = converged ? 0 : 1;
}

cudaError_t init_sym_eigen() {
  return cudaFuncSetAttribute(k_sym_eigen, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sizeof(double) * EIG_SMEM_MAX_N * (EIG_SMEM_MAX_N + 1)));
}

size_t sym_eigen_work(int n) { return (size_t)n * (n + 1) + (size_t)n * n; }

bool launch_sym_eigen(int n, const double* a, double* work, double* w, double* v, int* info, cudaStream_t st) {
  if (n < 1 || n > EIG_MAX_N) return false;
  const size_t smem = (n <= EIG_SMEM_MAX_N) ? sizeof(double) * n * (n + 1) : 0;
  k_sym_eigen<<<1, EIG_THREADS, smem, st>>>(n, a, work, work + (size_t)n * (n + 1), w, v, info);
  return true;
}

}  // namespace flosic
