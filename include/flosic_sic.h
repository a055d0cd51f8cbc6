/*
 * libflosic_sic_b200 -- B200 (sm_100a) implementation of the FLO-SIC
 * per-Fermi-orbital self-interaction-correction hot path.
 *
 * Drop-in boundary.  Each entry point replaces one reference Fortran routine
 * (FLOSIC/PublicRelease_2020, directory flosic/) on the SIC path; the Fortran
 * host keeps mesh generation, the SCF loop and the eigensolvers and calls
 * these functions through thin iso_c_binding shims.  The reference routines
 * read their inputs from Fortran modules; here the module arrays a routine
 * reads are passed once (flosic_sic_set_geometry / flosic_sic_set_orbitals)
 * and kept resident in GPU memory.
 *
 * Conventions
 *   - every function returns 0 on success and a nonzero FLOSIC_ERR_* code on
 *     failure; nothing here calls exit() or abort().  The Fortran shim maps a
 *     nonzero status to STOPIT, as the reference does on the same conditions.
 *   - arrays are Fortran column-major with the reference's leading dimensions;
 *     spins and orbital indices are 1-based where the reference's are.
 *   - one context binds one CUDA device; calls on a context are serialised on
 *     the context's stream and return after results are in host memory.
 */
#ifndef FLOSIC_SIC_H
#define FLOSIC_SIC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  FLOSIC_OK = 0,
  FLOSIC_ERR_ARG = 1,           /* invalid argument / size                       */
  FLOSIC_ERR_CAPACITY = 2,      /* a static capacity (MAX_BARE, MAX_CON, ...)    */
  FLOSIC_ERR_LOWDEN = 3,        /* Lowdin eigenvalue < 1e-8 (lowden_files.f:71)  */
  FLOSIC_ERR_ZERO_DENSITY = 4,  /* zero density at an FOD                        */
  FLOSIC_ERR_NFRM = 5,          /* MORB .NE. NFRM (frmiorb.f:418)                */
  FLOSIC_ERR_ZERO_COULOMB = 6,  /* "COUPOT IS ZERO" (apotnl_sic.F:277-283)       */
  FLOSIC_ERR_CUDA = 7,          /* CUDA failure, or a kernel wait that gave up    */
  FLOSIC_ERR_STATE = 8          /* call order: geometry/orbitals not set         */
};

/* Static capacities shared with the reference (PARAMA2). */
#define FLOSIC_MAX_BARE 25
#define FLOSIC_MAX_CON 15
#define FLOSIC_NSPEED 25

typedef struct flosic_ctx flosic_ctx;

/* Context management (no reference counterpart: replaces the MPI job farm
   set up in cpuhog.F / senddata.F for these routines). */
int flosic_sic_create(int device, flosic_ctx** ctx);
int flosic_sic_destroy(flosic_ctx* ctx);
const char* flosic_sic_last_error(void);

/* Module state read by the SIC routines (modules2.F90:133-244 common2,
   modules.f90:206-218 mesh1).  Atoms are given in the reference order
   (function set IFNCT outer, position I_POS inner); atom_type is the 1-based
   IFNCT of each atom.
     RAT(3,natoms) BFALP(25,ntypes) BFCON(25,15,3,ntypes) N_BARE(ntypes)
     N_CON(3,ntypes) RMSH(3,nmsh) WMSH(nmsh)
   Functional: IGGA(2), IDFTYP(2) as set by SETDFTYP (setdftyp.F:61-105);
   supported: exchange PW91/PBE/revPBE/RPBE (LDA via IGGA=0), correlation
   PW91/PBE, and SCAN for both (IGGA=3, IDFTYP=11, "MGGA-SCAN*MGGA-SCAN").
   nspn = NSPN of the run (1 or 2). */
int flosic_sic_set_geometry(flosic_ctx* ctx, int natoms, const int32_t* atom_type, const double* rat,
                            int ntypes, const int32_t* n_bare, const double* bfalp,
                            const int32_t* n_con, const double* bfcon, int nmsh, const double* rmsh,
                            const double* wmsh, int nspn, const int32_t* igga, const int32_t* idftyp);

/* KS orbitals and FODs (common5 PSI_COEF/PSI after UNRAVEL for C1 symmetry,
   modules_sic.F90 FRM BFRM).  PSI(ldpsi, nwfs(1)+nwfs(2)): spin-1 orbitals
   first, basis order per atom (l, Cartesian component, contraction) as in
   unravel2.f:160-175.  BFRM(3, ldfrm, 2). */
int flosic_sic_set_orbitals(flosic_ctx* ctx, const int32_t* nwfs, const double* psi, int ldpsi,
                            const int32_t* nfrm, const double* bfrm, int ldfrm);

/* GORBDRV(NDERV,IUPDAT,IALLCTR,NPTS,PTS,IFNCT,GRAD)  -- gorbdrv.f:18.
   PTS(25,3) relative to the atom, GRAD(25,10,6,15,3), IALLCTR(15,3). */
int flosic_sic_gorbdrv(flosic_ctx* ctx, int nderv, int32_t* iupdat, int32_t* iallctr, int npts,
                       const double* pts, int ifnct, double* grad);

/* FRMORB2(0,0) -- frmorb2.F:146-346: FMAT(ld,ld,4,2) of the FO values and
   their FOD derivatives at the FODs. */
int flosic_sic_frmorb2_fmat(flosic_ctx* ctx, double* fmat, int ld);

/* FRMIORB(1,1) -- frmiorb.f:5: TMAT(ld,ld,2) (Lowdin-orthonormalised Fermi
   transformation) and the Lowdin overlap eigenvalues EVAL(ld,2). */
int flosic_sic_frmiorb(flosic_ctx* ctx, double* tmat, double* eval, int ld);

/* COUPOT_SIC(MXXD=0,KXXS,KXXO) -- coupot_sic.F:9: Coulomb potential COULOMB(nmsh)
   of the density of FO kxxo of spin kxxs, and that density RHOG(nmsh,10). */
int flosic_sic_coupot_sic(flosic_ctx* ctx, int kxxs, int kxxo, double* coulomb, double* rhog);

/* GETVLXC(NDIM,RHOG,VXC,VLO,.false.,...) SIC branch -- getvlxc.F:8 with NSPN=2
   (apotnl_sic.F:419): VXC(2*ndim) and ERGXL,ERGXN,ERGCL,ERGCN in ergs[4]. */
int flosic_sic_getvlxc(flosic_ctx* ctx, int ndim, const double* rhog, double* vxc, double* ergs);

/* GETVLXC meta-GGA branch (SCAN) -- getvlxc.F:8 with subvlxc_libxc.F90:150-157,
   293-440 and call_mgga.f90: the caller passes TAU(ndim), the FO's kinetic
   energy density |grad phi|^2/2 that GETTAU_PAR (gettau_par.f90) forms from
   the FO coefficients, with RHOG(ndim,10) (channels 1-4 read).  Returns the
   local potential VXC(2*ndim), the Hamiltonian ingredients MIXIN(4,2*ndim)
   (the MGGA#### record: dE/d|grad rho| along grad rho, and dE/dtau / 2) and
   ERGXL,ERGXN,ERGCL,ERGCN.  flosic_sic_getvlxc returns FLOSIC_ERR_ARG for a
   meta-GGA context. */
int flosic_sic_getvlxc_mgga(flosic_ctx* ctx, int ndim, const double* rhog, const double* tau, double* vxc,
                            double* mixin, double* ergs);

/* The MGGA#### record of FO iorbx of spin lspx (getvlxc.F:203-227, written
   with KXXO = IRBSIC = iorbx + (lspx-1)*NWFS(1)): MIXIN(4, 2*nmsh), the
   spin-up Hamiltonian ingredients of the FO's own density and tau, spin-down
   half zero.  SCAN contexts only; the SIC block itself keeps them on the GPU. */
int flosic_sic_mgga_mixin(flosic_ctx* ctx, int lspx, int iorbx, double* mixin);

/* Precision of the SIC path (no counterpart in the reference).
   FLOSIC_PRECISION_FP64 (default) is the drop-in: every step in FP64.
   FLOSIC_PRECISION_MIXED forms the Coulomb potential's geometric columns
   (Boys functions times monomials, harmonics) and the per-FO far field in
   single precision and contracts the single-pair calls on the tensor cores as
   TF32 split products (hi*hi + hi*lo + lo*hi) with FP32 accumulation folded
   into compensated sums; the FO construction, Lowdin orthogonalisation, XC and
   energy sums stay FP64.  Changing the mode invalidates the cached potentials. */
enum { FLOSIC_PRECISION_FP64 = 0, FLOSIC_PRECISION_MIXED = 1 };
int flosic_sic_set_precision(flosic_ctx* ctx, int mode);

/* Route of the FO density that enters the SIC exchange-correlation.
   FLOSIC_DENSITY_PHI2 (default): rho = phi^2 with its derivatives, formed from
   the FO values on the mesh.
   FLOSIC_DENSITY_PAIRS: the reference's own route (poisson1.f:849-948, with
   the pair polynomials of gtdncf.F:5-1113), which replaces the density the
   reference's POISSON1 accumulates into RHOG for APOTNL_SIC
   (apotnl_sic.F:232-430): each Poisson call adds its Gaussian pairs' density
   polynomials at the mesh points inside its RCUT sphere only, dropping
   polynomial coefficients of magnitude <= 1e-14.  It differs from phi^2 by
   that truncation (the density tails far from every call centre) and by the
   pairs the plan screens out (coupot_sic.F:228-315); gradient-corrected and
   especially meta-GGA energies amplify the difference at low density.  Costs
   one more pass over the near (pair, point) work of the Coulomb evaluation,
   in FP64 whatever the precision mode.  Changing the route invalidates the
   cached potentials. */
enum { FLOSIC_DENSITY_PHI2 = 0, FLOSIC_DENSITY_PAIRS = 1 };
int flosic_sic_set_density_mode(flosic_ctx* ctx, int mode);

/* Poll limit of every wait between the roles of the mixed-precision
   tensor-core Coulomb kernel (no counterpart in the reference).  Each wait on
   a pipeline barrier gives up after `polls` polls (polls <= 0: the default,
   2^25, far above any legitimate wait); the kernel then stops its roles,
   drains its own copies and tensor-core operations, frees its tensor memory
   and returns, and the call reports FLOSIC_ERR_CUDA with the context still
   usable.  A small limit makes the waits run out on purpose, which is how the
   error path is tested without a GPU fault; restore the default afterwards. */
int flosic_sic_set_wait_limit(flosic_ctx* ctx, int64_t polls);

/* Tile-shape autotuner (no counterpart in the reference, whose POISSON1 batch
   shapes are compile-time constants: MXPR pairs per call, coupot_sic.F:46, and
   MPX points per block, poisson1.f:62).  Times the per-FO Coulomb kernel with
   tiles of 128 mesh points by 32, 64 and 128 FO slots on this context's own
   COUPOT_SIC evaluation (the spin with the most FOs, the current precision mode
   and mesh shard; best of reps >= 1 runs after one untimed run) and keeps the
   fastest for the following calls.  Widths that would leave half a tile or more
   empty are skipped.  All widths give the same potentials bit for bit.
   perfo_fos: the chosen width; ms[3] (may be NULL): the times of widths
   32, 64, 128 in milliseconds, -1 for a skipped width.  Needs
   flosic_sic_set_orbitals; invalidates that spin's cached potentials. */
int flosic_sic_autotune(flosic_ctx* ctx, int reps, int* perfo_fos, float* ms);

/* Allocation-free form of flosic_sic_getvlxc on the caller's device buffers (no
   counterpart in the reference).  d_rhog: RHOG(ldr,10) density channels in
   device memory (channel stride ldr >= npts), d_wmsh: the npts mesh weights,
   d_vxc: VXC(2*npts) written in device memory; ERGXL,ERGXN,ERGCL,ERGCN come
   back in the host array ergs[4].  The functional is the context's (set by
   flosic_sic_set_geometry); the call runs on the context's stream and
   synchronises it before returning.  It allocates no device or host memory:
   its block partial sums live in a file-scope device array sized for
   npts <= 4,194,304 (larger npts returns FLOSIC_ERR_CAPACITY before any work).
   The first call on a device looks up that array's address
   (cudaGetSymbolAddress).  Calls that overlap in time on one device share the
   array and race on it. */
int flosic_sic_getvlxc_device(flosic_ctx* ctx, int npts, const double* d_rhog, int ldr, const double* d_wmsh,
                              double* d_vxc, double* ergs);

/* APOTNL_SIC(TOTQNUM,LSPX,IORBX) -- apotnl_sic.F:31: RESULTS(13) and CFRM(3) of
   FO iorbx, and its SIC potential POT(nmsh) = V_xc + V_H (the ZPOT record).
   The potential also stays in GPU memory for flosic_sic_siclagm. */
int flosic_sic_apotnl_sic(flosic_ctx* ctx, double* totqnum, int lspx, int iorbx, double* results,
                          double* cfrm, double* pot);

/* SICLAGM(LSPN) -- frmorb_mpi.F:2: SIC(ld,ld) = -<phi_j|V_l|phi_l> from the
   potentials of the FOs of spin lspn (kept in GPU memory instead of the
   ZPOT#### files); for SCAN also the gradient terms of frmorb_mpi.F:440-509
   with each FO's MIXIN (kept in GPU memory instead of the MGGA#### files). */
int flosic_sic_siclagm(flosic_ctx* ctx, int lspn, double* sic, int ld);

/* FRMORB2(-LSPN,-1) -- frmorb2.F:586-717: FOD forces DEBDAX(3,ld) from SIC(ld,ld). */
int flosic_sic_frmorb2_force(flosic_ctx* ctx, int lspn, const double* sic, int ld, double* debdax);

/* One SIC block of an SCF iteration (main.F:577-759): FRMORB2(0,0), FRMIORB(1,1),
   APOTNL_SIC for every FO of every spin, SICLAGM and FRMORB2(-s,-1), all FOs of a
   spin batched in the same launches.  RESULTS(13,ld,2) SIC(ld,ld,2) DEBDAX(3,ld,2)
   CFRM(3,ld,2); esic = ZSIC = sum of RESULTS(9,:,:). */
int flosic_sic_cycle(flosic_ctx* ctx, int ld, double* results, double* sic, double* debdax,
                     double* cfrm, double* esic);

/* One SIC cycle of many molecules (no single reference counterpart: the
   reference runs one molecule per job and spreads the FOs of one molecule over
   MPI groups, global_call.F90:113-160).  ctxs[0..n) are contexts on one device
   in one precision, each with its own geometry, orbitals and FODs.  Every
   molecule's FO construction, FO values, pair coefficients and call set-up run
   on its own stream; then the Coulomb potentials of all FOs of all molecules
   and both spins are evaluated by two persistent launches over one list of
   (molecule-spin, 128-point tile, block of 32*wm FOs) items (shared-geometry
   calls, then per-FO calls added); then each molecule's XC, energies, SIC
   matrix and forces.  wm = 1, 2 or 4 sets the FO block (0: from the largest
   FO count).  Outputs per molecule m at the offsets of flosic_sic_cycle times
   m: RESULTS(13,ld,2), SIC(ld,ld,2), DEBDAX(3,ld,2), CFRM(3,ld,2) and
   esic[m].  Every potential is computed by the same operations in the same
   order as in flosic_sic_cycle on the shared-geometry tensor-core GEMM
   (FLOSIC_PRECISION_FP64: bit for bit the per-molecule results; in the mixed
   mode the shared-geometry calls use the FP32-column FP64 GEMM rather than
   the tcgen05 kernel). */
int flosic_sic_batch_cycle(flosic_ctx** ctxs, int n, int wm, int ld, double* results, double* sic,
                           double* debdax, double* cfrm, double* esic);

/* Adjoint of the SIC energy with respect to the FO coefficients (no single
   reference counterpart: the basis-space form of the SIC-matrix quadrature of
   SICLMSLV, frmorb_mpi.F:184-572).  G(ldg, nfrm) = dE_SIC/dC_FO for the FOs of
   spin lspn at the current potentials: -(4/NSPN) sum_p w chi_mu V_k phi_k (and,
   for SCAN, the gradient terms), so that C_FO^T G = (4/NSPN) SIC.  The FOD
   forces and basis-centre terms follow from G by the chain rule through the
   FO construction.  On a mesh shard the result is the shard's partial sum,
   to be summed over the shards (the dE/dC part of the exchange). */
int flosic_sic_adjoint(flosic_ctx* ctx, int lspn, double* g, int ldg);

/* dE_SIC/d(FOD positions) of spin lspn, grad(3, ld) as DEBDAX (ld >= NFRM):
   the adjoint G of flosic_sic_adjoint carried through the FO construction
   (the Lowdin-orthonormalised Fermi transformation of frmiorb.f:351-480 and
   FMAT's FOD derivatives, frmorb2.F:296-346) inside the library.  It equals
   the FOD force of FRMORB2(-LSPN,-1) (frmorb2.F:586-717) times 2/NSPN, reached
   without the SIC matrix; the reference has no single routine for it.  Whole
   mesh only. */
int flosic_sic_adjoint_fod(flosic_ctx* ctx, int lspn, double* grad, int ld);

/* SICLAG_DER / SICLM_DERSLV (siclag_der.F:2-688): the basis-centre (Pulay)
   terms of the SIC atomic forces,
     DERSIC(ix, lfn, A) = sum_p w V_l(p) phi_l(p) d_ix phi_l^(A)(p)
   with phi_l^(A) the part of FO l carried by atom A's basis functions and
   lfn = l + (s-1)*NFRM(1) over both spins; for SCAN plus the meta-GGA terms of
   siclag_der.F:576-640 through the Hessian of the basis.  Doubled for NSPN=1
   (siclag_der.F:153-161).  Fortran DERSIC(3, ldo, natoms): dersic[(A*ldo +
   lfn)*3 + ix], ldo >= NFRM(1)+NFRM(2).  The caller subtracts the sum over lfn
   from the atomic force as mfpulay.F:80-95 does.  On a mesh shard
   (flosic_sic_set_shard) the result is the shard's partial sum over its
   points; the shards' results add up to the whole mesh's. */
int flosic_sic_siclag_der(flosic_ctx* ctx, double* dersic, int ldo);

/* SICHAM / APATCH / NEWWAY (sicham.F:922-944, sicmat.F:146-318), C1 symmetry:
   the basis-space SIC Hamiltonian of spin LSPN in the projector form the
   reference selects (MM=2),
     H_mu,nu = -1/2 sum_k ( <chi_mu|V_k|phi_k><phi_k|chi_nu>
                          + <chi_mu|phi_k><phi_k|V_k|chi_nu> ),
   both brackets by mesh quadrature; for SCAN, V_k acts in the weak form of
   the SIC matrix (the gradient terms of the FO's Hamiltonian ingredients).
   ADDED to ham: packed = 0, full symmetric matrix ham[mu*ldh + nu];
   packed = 1, HSTOR(INDX,2) order (mu = 1..N outer, nu = mu..N inner,
   N(N+1)/2 entries).  Whole mesh only. */
int flosic_sic_sicham(flosic_ctx* ctx, int lspn, double* ham, int ldh, int packed);

/* The DFT side of the potential on the same mesh, basis and kernels.
   DENSOLD (densold.F:5-277): the spin densities of the occupied Kohn-Sham
   orbitals given to flosic_sic_set_orbitals, RHOG(NMSH, NGRAD, NSPN) with
   NGRAD = 1 (density) or 10 (density, gradient, second derivatives xx yy zz
   xy xz yz, as densold.F:24-43 lists them), and PHIG(NMSH, NSPN) = sum_i
   |grad psi_i|^2 (zero for NGRAD = 1; phig may be NULL).  Orbital
   coefficients at or below 1e-10 in magnitude are skipped as densold.F does.
   COUPOT1 (coupot1.F:5-762, the DFTCALL branch of COUPOT_SIC): the Coulomb
   potential COULOMB(NMSH) of the total density of those orbitals (both spins;
   the spin-up density doubled for NSPN=1), by the same pair batches, POISSON1
   near field and multipole far field as the FO potentials.  Whole mesh only. */
int flosic_sic_densold(flosic_ctx* ctx, int ngrad, double* rhog, double* phig);
int flosic_sic_coupot1(flosic_ctx* ctx, double* coulomb);

/* Mesh sharding across GPUs (one context per GPU and rank).  The reference
   spreads the same work over MPI workers and sums their mesh contributions:
   MPI_REDUCE of COULOMB/RHOG in pampoiss.F:105-120 and of the SIC matrix in
   pamlmsic.F:103.  Here each context evaluates the mesh points of its shard
   (an even split of the 128-point tiles of the sorted mesh); the set-up that
   does not depend on the points (FO construction, pair coefficients, POISSON1
   call set-up incl. its far-point counts over the whole mesh) is repeated on
   every rank, so the only exchange is one sum of a small packed buffer:
     flosic_sic_set_shard(ctx, shard, nshards)   0 <= shard < nshards; call
                                                  before or after set_geometry
     flosic_sic_partial_size(ctx, &n)            doubles in the packed buffer
     flosic_sic_cycle_partial(ctx, d_buf)        writes this shard's partial
                                                  sums to DEVICE memory d_buf[n]
     (caller: sum d_buf over the ranks in place, e.g. ncclAllReduce / MPI)
     flosic_sic_cycle_combine(ctx, d_buf, ...)   RESULTS, SIC, DEBDAX, CFRM and
                                                  E_SIC as flosic_sic_cycle
   Layout of the buffer, per spin: SIC(nfrm,nfrm), the mesh sums (XCH1, XCOU,
   XEXX, XDEL, ERGXL, ERGXN, ERGCL, ERGCN, CFRM(3)) per FO, the scaled Coulomb
   potential at the farthest mesh point per FO (zero on the other shards); then
   the near/far/term work counters.  A sharded context refuses the entry points
   whose outputs cover the whole mesh (COUPOT_SIC, APOTNL_SIC, SICLAGM,
   flosic_sic_cycle) with FLOSIC_ERR_STATE. */
int flosic_sic_set_shard(flosic_ctx* ctx, int shard, int nshards);
int flosic_sic_partial_size(flosic_ctx* ctx, int64_t* ndoubles);
int flosic_sic_cycle_partial(flosic_ctx* ctx, double* d_partial);
int flosic_sic_cycle_combine(flosic_ctx* ctx, const double* d_partial, int ld, double* results, double* sic,
                             double* debdax, double* cfrm, double* esic);

/* Timing/introspection (no reference counterpart): number of kernels launched by
   the last flosic_sic_cycle, per-stage device milliseconds of the last cycle
   (ms[0]=FO construction, [1]=orbital/density, [2]=Coulomb setup, [3]=Coulomb
   evaluation, [4]=XC+energies, [5]=SIC matrix, [6]=forces), pair/call counts, and the
   Coulomb work of the last cycle: work[0] = near (pair, point, FO) evaluations,
   work[1] = far (call, point, FO) multipole evaluations, work[2] = multipole terms
   those far evaluations keep under the skip rule of poisson1.f:1252-1270. */
int flosic_sic_stats(flosic_ctx* ctx, int64_t* launches, double* stage_ms, int64_t* npairs,
                     int64_t* ncalls, int64_t* work);

/* The Coulomb evaluation of the last cycle split by kernel (no counterpart in
   the reference): ms[0] = the shared-geometry calls (call classification,
   operand splits and the shared-geometry kernel: k_coulomb_shared_tc or
   k_coulomb_shared), ms[1] = the per-FO kernel (k_coulomb_perfo), device
   milliseconds summed over the spins; work[0..2] = near / far / kept-term
   counts of the shared-geometry kernel, work[3..5] of the per-FO kernel. */
int flosic_sic_kernel_stats(flosic_ctx* ctx, double* ms, int64_t* work);

#ifdef __cplusplus
}
#endif
#endif /* FLOSIC_SIC_H */
