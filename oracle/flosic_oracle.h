/*
 * FP64 CPU oracle for the FLO-SIC per-Fermi-orbital hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, routine by routine, the
 * reference Fortran algorithm (FLOSIC/PublicRelease_2020, directory flosic/)
 * so that the CUDA product path can be checked against it.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline legs may load it; the
 * product library (libflosic_sic_b200.so) never links or calls it.
 *
 * Layout conventions (all arrays are Fortran column-major, as in the
 * reference modules; the leading dimensions are the reference's static sizes
 * MAX_BARE=25 and MAX_CON=15):
 *   BFALP(MAX_BARE, ntypes)                 exponents of bare primitives
 *   BFCON(MAX_BARE, MAX_CON, 3, ntypes)     contraction coefficients
 *   N_CON(3, ntypes), N_BARE(ntypes)
 *   RAT(3, natoms)      atom positions, atoms ordered by type (IFNCT, I_POS)
 *   RMSH(3, nmsh), WMSH(nmsh)
 *   PSI(nbasis, nwf)    KS coefficients, spin-1 orbitals first; the basis
 *                       order inside an atom is (l, Cartesian component,
 *                       contraction), contraction fastest (unravel2.f:160-175)
 *   BFRM(3, ldfrm, 2)   FOD positions per spin
 */
#ifndef FLOSIC_ORACLE_H
#define FLOSIC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_problem orc_problem;

orc_problem* orc_create(int natoms, const int* atom_type, const double* rat,
                        int ntypes, const int* n_bare, const double* bfalp,
                        const int* n_con, const double* bfcon,
                        int nmsh, const double* rmsh, const double* wmsh,
                        int nspn, int igga_x, int idftyp_x, int igga_c, int idftyp_c);
void orc_destroy(orc_problem* p);
int  orc_nbasis(const orc_problem* p);
const char* orc_last_error(void);

int orc_set_orbitals(orc_problem* p, const int* nwfs, const double* psi, int ldpsi,
                     const int* nfrm, const double* bfrm, int ldfrm);

/* gorbdrv.f:18 */
int orc_gorbdrv(orc_problem* p, int nderv, int npts, const double* pts, int ifnct,
                double* grad, int* iupdat, int* iallctr);

/* frmorb2.F:146-346 (FRMORB2(0,0)): FMAT(ld, ld, 4, 2) */
int orc_frmorb2_fmat(orc_problem* p, double* fmat, int ld);
/* frmiorb.f:5 (FRMIORB(1,1)): TMAT(ld, ld, 2), LOWDEN eigenvalues EVAL(ld, 2) */
int orc_frmiorb(orc_problem* p, double* tmat, double* lowden_eval, int ld);
/* unravel2.f (MD=0/2): FO coefficients CFO(nbasis, nfrm(spin)) */
int orc_fo_coefficients(orc_problem* p, int spin, double* cfo);

/* coupot_sic.F:9 (serial branch) for FO iorb of spin: COULOMB(nmsh), RHOG(nmsh,10) */
int orc_coupot_sic(orc_problem* p, int spin, int iorb, int exact,
                   double* coulomb, double* rhog, long long* stats);
/* getvlxc.F:8 serial branch with subvlxc_libxc.F90 (NSPN forced to 2 as in apotnl_sic.F:419) */
int orc_getvlxc_sic(orc_problem* p, const double* rhog, double* vxc, double* ergs);
/* SCAN: tau of the FO per point, MIXIN(4, nmsh) spin-up Hamiltonian ingredients */
int orc_getvlxc_mgga(orc_problem* p, const double* rhog, const double* tau, double* vxc, double* mixin,
                     double* ergs);
int orc_fo_tau(orc_problem* p, int spin, int iorb, double* tau);
/* Test knob: XC on the untruncated (every point near) pair density while the
   Coulomb potential keeps the near/far split (0 = the reference's behaviour). */
int orc_set_xc_exact_density(orc_problem* p, int on);
/* weight of a mesh point in POISSON1's near/far cost model (timing samples of a larger mesh) */
int orc_set_count_scale(orc_problem* p, double scale);
/* SICLAG_DER: DERSIC(3, ldo, natoms) as dersic[(A*ldo + lfn)*3 + ix] */
int orc_siclag_der(orc_problem* p, double* dersic, int ldo);
/* APOTNL_SIC RESULTS(13) of one orbital given by its basis coefficients */
int orc_fo_energy(orc_problem* p, int spin, const double* cfo, double* results);
/* SICHAM's basis-space SIC Hamiltonian of one spin, added to ham[mu*ldh + nu] */
int orc_sicham(orc_problem* p, int spin, double* ham, int ldh);
/* COUPOT1: Coulomb potential of the occupied orbitals' total density */
int orc_coupot1(orc_problem* p, double* coulomb);
/* DENSOLD: rhog[(s*ngrad + ch)*nmsh + i], phig[s*nmsh + i] (phig may be NULL) */
int orc_densold(orc_problem* p, int ngrad, double* rhog, double* phig);
/* Mesh-shard decomposition of one cycle (same packing as flosic_sic_cycle_partial):
   partial sums over mesh points [b, e), and the cycle's outputs from their sum. */
int orc_partial_size(orc_problem* p, long long* n);
int orc_cycle_partial(orc_problem* p, int b, int e, double* out);
int orc_cycle_combine(orc_problem* p, const double* in, int ld, double* results, double* sic, double* debdax,
                      double* cfrm, double* esic);
/* SCAN point functions (scan.f): x: out[4] = ex, vx, vxdd, amux;
   c: out[7] = ec, vc_up, vc_dn, vcdd_up, vcdd_dn, amu, (unused) */
void orc_scan_x(double rho, double drho, double tau, double* out);
void orc_scan_c(double ru, double rd, double dru, double drd, double drt, double tauu, double taud, double* out);
/* apotnl_sic.F:31: RESULTS(13), CFRM(3), POT(nmsh) = V_xc + V_H (the ZPOT record) */
int orc_apotnl_sic(orc_problem* p, int spin, int iorb, double* results, double* cfrm,
                   double* pot, double* coulomb, double* rhog, double* mixin);
/* frmorb_mpi.F:2/184 SICLAGM: SIC(ld, ld) from POT(nmsh, nfrm) */
/* zm: [nf][nmsh][4] Hamiltonian ingredients of the FOs (meta-GGA only, else NULL) */
int orc_siclagm(orc_problem* p, int spin, const double* pots, const double* zm, double* sic, int ld);
/* frmorb2.F:586-717: DEBDAX(3, ld) from SIC(ld, ld) */
int orc_frmorb2_force(orc_problem* p, int spin, const double* sic, int ld, double* debdax);

/* One SIC cycle (main.F:577-759): RESULTS(13,ld,2) SIC(ld,ld,2) DEBDAX(3,ld,2) CFRM(3,ld,2) */
int orc_sic_cycle(orc_problem* p, int ld, double* results, double* sic, double* debdax,
                  double* cfrm, double* esic, int nthreads, int fo_limit);

/* Pair-list statistics of coupot_sic.F for one FO: stats[0]=pairs kept, [1]=batches,
   [2]=weird pairs, [3]=near (pair,point) evaluations, [4]=far (batch,point) evaluations */
int orc_pair_stats(orc_problem* p, int spin, int iorb, long long* stats);

/* The POISSON1 calls of coupot_sic.F for one FO, in call order:
   calls(6, ncalls) = CG(3), RCUT, NPOT, pairs; pairs(51, npairs) = call index,
   -C(3) (the pair centre negated, as poisson1.f keeps it), delta = alpha+beta,
   COEFICIENT(1:46) (gtdncf.F).  Fails if maxc/maxp are too small. */
int orc_pair_dump(orc_problem* p, int spin, int iorb, double* calls, long long maxc, long long* ncalls,
                  double* pairs, long long maxp, long long* npairs);

/* One mesh point of SUBVLXC (subvlxc_libxc.F90) with NSPN=2 and zero spin-down
   density: r10 = total-density channels; v2 = spin-up/down potentials; e4 =
   weighted EXL, EXN, ECL, ECN. */
int orc_xc_point(int igga_x, int idftyp_x, int igga_c, int idftyp_c, const double* r10, double w,
                 double* v2, double* e4);

/* Boys values as computed by fffmtc.F/fffmt4.F/fffmt3.F (maxfmt=5/4/3): s[5] */
void orc_boys(int maxfmt, double x, double* s);
/* harmonics.f: real spherical harmonics up to lm for a unit vector, y[(lm+1)^2] */
void orc_harmonics(int lm, const double* xyz, double* y);
/* lebedev.F degree-19 mesh (146 points): ang[3*146], w[146] */
int orc_lebedev19(double* ang, double* w);

#ifdef __cplusplus
}
#endif
#endif
