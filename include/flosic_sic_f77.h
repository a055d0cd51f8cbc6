/*
 * Fortran 77 forms of the libflosic_sic_b200 C ABI (include/flosic_sic.h).
 *
 * A Fortran host without iso_c_binding interface blocks calls a routine as
 *     CALL FLOSIC_SIC_APOTNL_SIC(CTX, TOTQNUM, LSPX, IORBX, RESULTS, CFRM, POT, IERR)
 * which gfortran and ifort link to the lowercase name with one trailing
 * underscore, every argument passed by reference.  Each function here is that
 * form of the entry point of flosic_sic.h with the same name: the same
 * arguments in the same order, then IERR.
 *   - the context handle is an INTEGER*8 holding the flosic_ctx pointer
 *     (0 after FLOSIC_SIC_DESTROY);
 *   - C `int` arguments are INTEGER*4, array arguments are the same arrays;
 *   - device addresses (the d_* arguments) are INTEGER*8 values;
 *   - IERR (INTEGER*4) receives the entry point's status: 0, or a
 *     FLOSIC_ERR_* code, after which FLOSIC_SIC_LAST_ERROR(MSG) gives the
 *     message and the host calls STOPIT as the reference does.
 * The routines of the reference's SIC path keep their argument meaning:
 * apotnl_sic.F:31, coupot_sic.F:9, getvlxc.F:8, frmorb_mpi.F:2 (SICLAGM),
 * frmorb2.F:10, frmiorb.f:5, gorbdrv.f:18 (see flosic_sic.h for each).
 */
#ifndef FLOSIC_SIC_F77_H
#define FLOSIC_SIC_F77_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* FLOSIC_SIC_CREATE(DEVICE, CTX, IERR), FLOSIC_SIC_DESTROY(CTX, IERR) */
void flosic_sic_create_(const int32_t* device, int64_t* ctx, int32_t* ierr);
void flosic_sic_destroy_(int64_t* ctx, int32_t* ierr);
/* FLOSIC_SIC_LAST_ERROR(MSG): CHARACTER*(*) MSG, filled and blank-padded;
   msg_len is the hidden length argument Fortran passes for MSG. */
void flosic_sic_last_error_(char* msg, size_t msg_len);

void flosic_sic_set_geometry_(const int64_t* ctx, const int32_t* natoms, const int32_t* atom_type,
                              const double* rat, const int32_t* ntypes, const int32_t* n_bare,
                              const double* bfalp, const int32_t* n_con, const double* bfcon,
                              const int32_t* nmsh, const double* rmsh, const double* wmsh, const int32_t* nspn,
                              const int32_t* igga, const int32_t* idftyp, int32_t* ierr);
void flosic_sic_set_orbitals_(const int64_t* ctx, const int32_t* nwfs, const double* psi, const int32_t* ldpsi,
                              const int32_t* nfrm, const double* bfrm, const int32_t* ldfrm, int32_t* ierr);
void flosic_sic_gorbdrv_(const int64_t* ctx, const int32_t* nderv, int32_t* iupdat, int32_t* iallctr,
                         const int32_t* npts, const double* pts, const int32_t* ifnct, double* grad,
                         int32_t* ierr);
void flosic_sic_frmorb2_fmat_(const int64_t* ctx, double* fmat, const int32_t* ld, int32_t* ierr);
void flosic_sic_frmiorb_(const int64_t* ctx, double* tmat, double* eval, const int32_t* ld, int32_t* ierr);
void flosic_sic_coupot_sic_(const int64_t* ctx, const int32_t* kxxs, const int32_t* kxxo, double* coulomb,
                            double* rhog, int32_t* ierr);
void flosic_sic_getvlxc_(const int64_t* ctx, const int32_t* ndim, const double* rhog, double* vxc,
                         double* ergs, int32_t* ierr);
void flosic_sic_getvlxc_mgga_(const int64_t* ctx, const int32_t* ndim, const double* rhog, const double* tau,
                              double* vxc, double* mixin, double* ergs, int32_t* ierr);
void flosic_sic_mgga_mixin_(const int64_t* ctx, const int32_t* lspx, const int32_t* iorbx, double* mixin,
                            int32_t* ierr);
void flosic_sic_set_precision_(const int64_t* ctx, const int32_t* mode, int32_t* ierr);
void flosic_sic_set_wait_limit_(const int64_t* ctx, const int64_t* polls, int32_t* ierr);
void flosic_sic_set_density_mode_(const int64_t* ctx, const int32_t* mode, int32_t* ierr);
void flosic_sic_autotune_(const int64_t* ctx, const int32_t* reps, int32_t* perfo_fos, float* ms,
                          int32_t* ierr);
void flosic_sic_getvlxc_device_(const int64_t* ctx, const int32_t* npts, const int64_t* d_rhog,
                                const int32_t* ldr, const int64_t* d_wmsh, const int64_t* d_vxc, double* ergs,
                                int32_t* ierr);
void flosic_sic_apotnl_sic_(const int64_t* ctx, double* totqnum, const int32_t* lspx, const int32_t* iorbx,
                            double* results, double* cfrm, double* pot, int32_t* ierr);
void flosic_sic_siclagm_(const int64_t* ctx, const int32_t* lspn, double* sic, const int32_t* ld,
                         int32_t* ierr);
void flosic_sic_frmorb2_force_(const int64_t* ctx, const int32_t* lspn, const double* sic, const int32_t* ld,
                               double* debdax, int32_t* ierr);
void flosic_sic_cycle_(const int64_t* ctx, const int32_t* ld, double* results, double* sic, double* debdax,
                       double* cfrm, double* esic, int32_t* ierr);
void flosic_sic_adjoint_(const int64_t* ctx, const int32_t* lspn, double* g, const int32_t* ldg,
                         int32_t* ierr);
void flosic_sic_kernel_stats_(const int64_t* ctx, double* ms, int64_t* work, int32_t* ierr);
void flosic_sic_batch_cycle_(const int64_t* ctxs, const int32_t* n, const int32_t* wm, const int32_t* ld,
                             double* results, double* sic, double* debdax, double* cfrm, double* esic,
                             int32_t* ierr);
void flosic_sic_adjoint_fod_(const int64_t* ctx, const int32_t* lspn, double* grad, const int32_t* ld,
                             int32_t* ierr);
void flosic_sic_siclag_der_(const int64_t* ctx, double* dersic, const int32_t* ldo, int32_t* ierr);
void flosic_sic_sicham_(const int64_t* ctx, const int32_t* lspn, double* ham, const int32_t* ldh,
                        const int32_t* packed, int32_t* ierr);
void flosic_sic_densold_(const int64_t* ctx, const int32_t* ngrad, double* rhog, double* phig, int32_t* ierr);
void flosic_sic_coupot1_(const int64_t* ctx, double* coulomb, int32_t* ierr);
void flosic_sic_set_shard_(const int64_t* ctx, const int32_t* shard, const int32_t* nshards, int32_t* ierr);
void flosic_sic_partial_size_(const int64_t* ctx, int64_t* ndoubles, int32_t* ierr);
void flosic_sic_cycle_partial_(const int64_t* ctx, const int64_t* d_partial, int32_t* ierr);
void flosic_sic_cycle_combine_(const int64_t* ctx, const int64_t* d_partial, const int32_t* ld,
                               double* results, double* sic, double* debdax, double* cfrm, double* esic,
                               int32_t* ierr);
void flosic_sic_stats_(const int64_t* ctx, int64_t* launches, double* stage_ms, int64_t* npairs,
                       int64_t* ncalls, int64_t* work, int32_t* ierr);

#ifdef __cplusplus
}
#endif
#endif /* FLOSIC_SIC_F77_H */
