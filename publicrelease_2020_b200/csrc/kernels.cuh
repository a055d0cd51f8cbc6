// Kernel declarations and device-side data descriptors.
#pragma once

#include "common.cuh"

namespace flosic {

// Basis tables in device memory (general-contraction NRLMOL layout).
struct BasisDev {
  int natoms, ntypes, nbasis, nprim;
  const double* atom_pos;    // 3*natoms
  const int* atom_type;      // natoms
  const int* atom_boff;      // natoms: first basis function of the atom
  const int* atom_poff;      // natoms: first global primitive of the atom
  const int* type_nbare;     // ntypes
  const int* type_lmax;      // ntypes
  const int* type_ncon;      // 3*ntypes
  const double* type_alpha;  // MAX_BARE*ntypes
  const double* type_amin;   // ntypes: smallest exponent
  const double* type_bfcon;  // ((t*3+l)*MAX_CON+c)*MAX_BARE+ib
  const int* prim_atom;      // nprim: atom of each global primitive
  const int* prim_ib;        // nprim: bare index inside the atom type
};

struct MeshDev {
  int n, ntiles;
  const double* x;
  const double* y;
  const double* z;
  const double* w;
  const double* tile_lo;  // 3*ntiles
  const double* tile_hi;  // 3*ntiles
};

// Basis values (nderv 0,1,2 -> 1,4,10 channels) of all functions at npts points
// (px,py,pz SoA).  out[(ch*nbasis + b)*ldo + i].
void launch_basis_values(const BasisDev& B, int nderv, int npts, const double* px, const double* py,
                         const double* pz, double* out, int ldo, cudaStream_t st);

// u[(k*nprim + gp)*10 + comp] = sum_con BFCON(ib,con,l(comp)) C(k, local(l,comp,con))
void launch_prim_u(const BasisDev& B, int nfo, const double* cfo, int ldc, double* u, cudaStream_t st);

// Per (pair, FO): 46 potential coefficients (rows of COEF_LD doubles, zero
// padded), Boys variant, centre-of-gravity partials.
// dm != nullptr (nfo = 1): the pair blocks of one general density matrix
// instead of the FOs' rank-1 blocks.
void launch_pair_coef(int npairs, const PairGeo* pairs, const CallInfo* calls, int nfo, int nprim,
                      const double* u, const double* dm, int nspn, double* coef, int8_t* maxfmt, double* cgp,
                      cudaStream_t st);

// dm[(ip*10 + mu)*10 + nu] = sum_{i<norb} u_i(pi)[mu] u_i(pj)[nu]
void launch_pair_dm(int npairs, const PairGeo* pairs, int norb, int nprim, const double* u, double* dm,
                    cudaStream_t st);

// DENSOLD spin densities (+ derivatives for ngrad = 10) and PHIG from orbital values
void launch_densold(int npts, int nw0, int nw1, int nspn, int ngrad, const double* psig, int ldp, double* rhog,
                    double* phig, int ldr, cudaStream_t st);

// Per (call, FO): CG, RCUT, NPOT, skip mask and normalised multipole moments
// momv[(c*nfo + k)*MOM_LD + lm] (skipped terms and padding zero).
void init_call_setup();
// list: the nsingle calls of one slot (one pair, NSPN=1; CG/RCUT/NPOT shared
// by all FOs, set up once per call), then the other calls (once per FO).
void launch_call_setup(int ncalls, const int* list, int nsingle, const CallInfo* calls, const PairGeo* pairs,
                       int nfo, int nspn, const double* coef, const int8_t* maxfmt, const double* cgp,
                       const MeshDev& M, const double* boys_tab, CallFO* cfo, double* momv, cudaStream_t st);

// Coulomb potential of every FO at every mesh point, vh[k*ldv + p], on the
// FP64 tensor cores (csrc/coulomb_mma.cu).  Calls whose near/far geometry is
// identical for every FO go through the shared-geometry kernel, the rest
// through the per-FO kernel, which adds its part.  per_fo_only routes every
// call through the per-FO kernel (a cross-check of the two forms).  mixed
// selects the mixed-precision path: geometric columns and the per-FO far field
// in single precision, the shared-geometry GEMM on tcgen05 (TF32 split products).
// cnt[0] += near (pair, point, FO) evaluations, cnt[1] += far (call, point, FO),
// cnt[2] += multipole terms kept by the skip rule over those far evaluations.
struct CoulombScratch {
  int8_t* pair_fmt;    // npairs
  CallShare* share;    // ncalls
  int* lists;          // 2*ncalls + 2: shared calls, per-FO calls, the two counts
  float* coef_hl;      // mixed path: TF32 hi/lo split of the coefficients (2 x npairs*nfo*COEF_LD)
  float* momv_hl;      // mixed path: TF32 hi/lo split of the moments (2 x ncalls*nfo*MOM_LD)
  int* err;            // mixed path: set when a tensor-core pipeline wait reached its limit
};
// Kernel choices (all evaluate the same sums; the results differ only by the
// rounding of the chosen arithmetic).  per_fo_only: every call through the
// per-FO kernel (a cross-check of the two forms).  shared_tc: in the mixed
// path, the shared-geometry calls on tcgen05 (TF32 split products) rather
// than on the FP64 tensor cores with FP32 columns.  perfo_wm: FO block of the
// per-FO kernel in units of 32 (1, 2 or 4; 0 chooses by the FO count).
struct CoulombConfig {
  bool per_fo_only = false;
  bool shared_tc = true;
  int perfo_wm = 0;
  long long wait_limit = 0;  // polls of each tensor-core pipeline wait before it gives up (0: the default)
  int fo_values_bn = 64;     // FOs per CTA of the fused FO-value kernel (64 or 128)
};
// One (molecule, spin) of a batched Coulomb launch: the arguments of the
// per-molecule kernels (shared-geometry and per-FO calls of one spin).
struct CoulombJob {
  int ncalls, nfo, ldv, pad;
  const int* lists;
  const CallShare* share;
  const CallInfo* calls;
  const PairGeo* pairs;
  const double* coef;
  const int8_t* pair_fmt;
  const CallFO* cfo;
  const double* momv;
  MeshDev M;
  double* vh;
  unsigned long long* cnt;
};
void init_coulomb_mma();
// Pair Boys variants, shared-geometry flags and the two call lists (the set-up
// of launch_coulomb_mma before its kernels).
void launch_coulomb_classify(int ncalls, int npairs, int nfo, const int8_t* maxfmt, const CallFO* cfo,
                             const CoulombScratch& scr, bool per_fo_only, cudaStream_t st);
// Every (job, tile, FO block) item of a batch in two persistent launches
// (shared-geometry calls, then per-FO calls added): items[i] = {job, tile,
// FO block of 32*wm FOs, 0}, taken in list order from two device counters
// (counters[0..1], zeroed here); nctas persistent CTAs.
void launch_coulomb_batch(const CoulombJob* jobs, const int4* items, int nitems, int* counters, int wm, bool mixed,
                          const double* boys_tab, int nctas, cudaStream_t st);
void init_coulomb_tc();
// TF32 hi/lo split of nrow x nfo rows of KSEG doubles into the chunk-major
// [nrow][KSEG/4][nfo][4] layout (hi, then lo at + nrow*nfo*KSEG floats).
void launch_split_tf32(size_t nrow, int nfo, const double* src, float* out, cudaStream_t st);
// Mixed-precision shared-geometry Coulomb GEMM on tcgen05 (csrc/coulomb_tc.cu);
// the A rows reach shared memory by TMA through tensor maps built here.
cudaError_t launch_coulomb_shared_tc(int ncalls, const int* lists, const CallShare* share, const CallInfo* calls,
                                     int nfo, const float* coef_hl, size_t coef_part, const int8_t* pair_fmt,
                                     const PairGeo* pairs, const float* momv_hl, size_t mom_part, const MeshDev& M,
                                     const double* boys_tab, double* vh, int ldv, unsigned long long* cnt, int* err,
                                     long long wait_limit, cudaStream_t st);
// cnt[0..2]: near/far/terms of the shared-geometry kernel, cnt[3..5]: of the per-FO kernel;
// mid (may be null) is recorded between the two kernels.
cudaError_t launch_coulomb_mma(int ncalls, const CallInfo* calls, const PairGeo* pairs, int npairs, int nfo,
                               const double* coef, const int8_t* maxfmt, const CallFO* cfo, const double* momv,
                               const MeshDev& M, const double* boys_tab, double* vh, int ldv,
                               const CoulombConfig& cfg, bool mixed, const CoulombScratch& scr,
                               unsigned long long* cnt, cudaEvent_t mid, cudaStream_t st);

// Exchange-correlation of the FO densities (fully polarised, NSPN forced to 2 as
// in apotnl_sic.F:419) from the FO values/derivatives phi[(ch*nfo+k)*ldp+p];
// writes the SIC potential V = Vxc + VH*nspn/2 and Y = w V phi, and per-block
// energy partial sums part[(k*nblk + blk)*NPART + j].
constexpr int NPART = 11;
// rhog (may be null): density channels rhog[(ch*nfo + k)*ldp + p] to use in
// place of those formed from phi (the reference's pair-route density).
void launch_xc(const MeshDev& M, int nfo, int gga, int mgga, int nspn, const int* xc, const double* phi, int ldp,
               const double* rhog, double* vh, double* vpot, double* y, double* part, int nblk, cudaStream_t st);
void launch_reduce_parts(int nfo, int nblk, const double* part, double* sums, cudaStream_t st);

// FO density channels of one FO: rhog[ch*ldr + p] (10 channels for GGA).
void launch_density(int npts, int nfo, int k, int nch, const double* phi, int ldp, double* rhog, int ldr,
                    cudaStream_t st);
void launch_fo_tau(int npts, int nfo, int k, const double* phi, int ldp, double* tau, cudaStream_t st);
void launch_xc_mgga_rhog(const MeshDev& M, const double* rhog, int ldr, const double* tau, double* vxc,
                         double* mixin, double* part, int nblk, cudaStream_t st);

// Vxc of given density channels (GETVLXC entry point): vxc[2*n], parts as above (1 FO).
// Dense products on the FP64 tensor cores (csrc/contract.cu).
// dgemm: C = alpha op(A) op(B) + beta C, column-major as BLAS DGEMM; work holds
// dgemm_work(M, N, K) doubles (split-K partial products; 0: none needed).
size_t dgemm_work(int M, int N, int K);
void dgemm(bool ta, bool tb, int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
           double beta, double* C, int ldc, double* work, cudaStream_t st);
// out[(ch*ncol + k)*ldo + p] = sum_f B_ch(p, f) coef[k*ldc + f]: basis values
// (nderv 0, 1, 2 -> 1, 4, 10 channels) at npts points times ncol coefficient columns.
cudaError_t init_contract();
// bn: FOs per CTA, 64 or 128 (the basis values of a point formed once per bn FOs).
void launch_fo_values(const BasisDev& B, int nderv, int npts, const double* px, const double* py, const double* pz,
                      const double* coef, int ldc, int ncol, double* out, size_t ldo, int bn, cudaStream_t st);
// out[k*ldo + p] = w[p] a[k*lda + p]
void launch_scale_rows(int P, int N, const double* a, int lda, const double* w, double* out, int ldo,
                       cudaStream_t st);
// Symmetric eigen-decomposition (one CTA, cyclic Jacobi; csrc/eigen.cu): a is
// n x n row-major, work holds sym_eigen_work(n) doubles; w ascending,
// v[k*n + m] = component k of eigenvector m; info 0, or 1 without convergence.
cudaError_t init_sym_eigen();
size_t sym_eigen_work(int n);
bool launch_sym_eigen(int n, const double* a, double* work, double* w, double* v, int* info, cudaStream_t st);
cudaError_t preload_xc_rhog();
void launch_xc_rhog(const MeshDev& M, int gga, const int* xc, const double* rhog, int ldr, double* vxc,
                    double* part, int nblk, cudaStream_t st);

// FO densities by the reference's route (csrc/density.cu): nch channels (1,
// 4 or 10) of each of nfo FOs, rhog[(ch*nfo + k)*ldr + p] over the mesh M,
// from the pairs of every call at the points inside the call's RCUT sphere
// (poisson1.f:849-948).  u: the FOs' primitive projections; cfo: the calls'
// per-FO geometry; dc: npairs*nfo*pair_density_ld(nch) doubles of scratch.
int pair_density_ld(int nch);
void launch_pair_density(int npairs, const PairGeo* pairs, int ncalls, const CallInfo* calls, const CallFO* cfo,
                         int nfo, int nprim, const double* u, int nch, const MeshDev& M, double* dc, double* rhog,
                         size_t ldr, cudaStream_t st);

void upload_constants(const double* leb_ang, const double* leb_w);

}  // namespace flosic
