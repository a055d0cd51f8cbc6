// Fortran 77 forms of the C ABI: by-reference arguments, a trailing IERR,
// an INTEGER*8 context handle (declared in include/flosic_sic_f77.h).  Each
// forwards to the C entry point of the same name and changes nothing else.
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstring>

#include "../../include/flosic_sic.h"
#include "../../include/flosic_sic_f77.h"

namespace {

flosic_ctx* handle(const int64_t* h) { return reinterpret_cast<flosic_ctx*>(static_cast<intptr_t>(*h)); }

// A device address passed as an INTEGER*8 value.
template <class T>
T* dev(const int64_t* a) {
  return reinterpret_cast<T*>(static_cast<intptr_t>(*a));
}

}  // namespace

extern "C" {

void flosic_sic_create_(const int32_t* device, int64_t* ctx, int32_t* ierr) {
  flosic_ctx* c = nullptr;
  *ierr = flosic_sic_create(*device, &c);
  *ctx = static_cast<int64_t>(reinterpret_cast<intptr_t>(c));
}

void flosic_sic_destroy_(int64_t* ctx, int32_t* ierr) {
  *ierr = flosic_sic_destroy(handle(ctx));
  *ctx = 0;
}

void flosic_sic_last_error_(char* msg, size_t msg_len) {
  const char* e = flosic_sic_last_error();
  const size_t n = std::min(std::strlen(e), msg_len);
  std::memcpy(msg, e, n);
  std::memset(msg + n, ' ', msg_len - n);
}

void flosic_sic_set_geometry_(const int64_t* ctx, const int32_t* natoms, const int32_t* atom_type, const double* rat,
                              const int32_t* ntypes, const int32_t* n_bare, const double* bfalp, const int32_t* n_con,
                              const double* bfcon, const int32_t* nmsh, const double* rmsh, const double* wmsh,
                              const int32_t* nspn, const int32_t* igga, const int32_t* idftyp, int32_t* ierr) {
  *ierr = flosic_sic_set_geometry(handle(ctx), *natoms, atom_type, rat, *ntypes, n_bare, bfalp, n_con, bfcon, *nmsh,
                                  rmsh, wmsh, *nspn, igga, idftyp);
}

void flosic_sic_set_orbitals_(const int64_t* ctx, const int32_t* nwfs, const double* psi, const int32_t* ldpsi,
                              const int32_t* nfrm, const double* bfrm, const int32_t* ldfrm, int32_t* ierr) {
  *ierr = flosic_sic_set_orbitals(handle(ctx), nwfs, psi, *ldpsi, nfrm, bfrm, *ldfrm);
}

void flosic_sic_gorbdrv_(const int64_t* ctx, const int32_t* nderv, int32_t* iupdat, int32_t* iallctr,
                         const int32_t* npts, const double* pts, const int32_t* ifnct, double* grad, int32_t* ierr) {
  *ierr = flosic_sic_gorbdrv(handle(ctx), *nderv, iupdat, iallctr, *npts, pts, *ifnct, grad);
}

void flosic_sic_frmorb2_fmat_(const int64_t* ctx, double* fmat, const int32_t* ld, int32_t* ierr) {
  *ierr = flosic_sic_frmorb2_fmat(handle(ctx), fmat, *ld);
}

void flosic_sic_frmiorb_(const int64_t* ctx, double* tmat, double* eval, const int32_t* ld, int32_t* ierr) {
  *ierr = flosic_sic_frmiorb(handle(ctx), tmat, eval, *ld);
}

void flosic_sic_coupot_sic_(const int64_t* ctx, const int32_t* kxxs, const int32_t* kxxo, double* coulomb,
                            double* rhog, int32_t* ierr) {
  *ierr = flosic_sic_coupot_sic(handle(ctx), *kxxs, *kxxo, coulomb, rhog);
}

void flosic_sic_getvlxc_(const int64_t* ctx, const int32_t* ndim, const double* rhog, double* vxc, double* ergs,
                         int32_t* ierr) {
  *ierr = flosic_sic_getvlxc(handle(ctx), *ndim, rhog, vxc, ergs);
}

void flosic_sic_getvlxc_mgga_(const int64_t* ctx, const int32_t* ndim, const double* rhog, const double* tau,
                              double* vxc, double* mixin, double* ergs, int32_t* ierr) {
  *ierr = flosic_sic_getvlxc_mgga(handle(ctx), *ndim, rhog, tau, vxc, mixin, ergs);
}

void flosic_sic_mgga_mixin_(const int64_t* ctx, const int32_t* lspx, const int32_t* iorbx, double* mixin,
                            int32_t* ierr) {
  *ierr = flosic_sic_mgga_mixin(handle(ctx), *lspx, *iorbx, mixin);
}

void flosic_sic_set_precision_(const int64_t* ctx, const int32_t* mode, int32_t* ierr) {
  *ierr = flosic_sic_set_precision(handle(ctx), *mode);
}

void flosic_sic_set_wait_limit_(const int64_t* ctx, const int64_t* polls, int32_t* ierr) {
  *ierr = flosic_sic_set_wait_limit(handle(ctx), *polls);
}

void flosic_sic_set_density_mode_(const int64_t* ctx, const int32_t* mode, int32_t* ierr) {
  *ierr = flosic_sic_set_density_mode(handle(ctx), *mode);
}

void flosic_sic_autotune_(const int64_t* ctx, const int32_t* reps, int32_t* perfo_fos, float* ms, int32_t* ierr) {
  *ierr = flosic_sic_autotune(handle(ctx), *reps, perfo_fos, ms);
}

void flosic_sic_getvlxc_device_(const int64_t* ctx, const int32_t* npts, const int64_t* d_rhog, const int32_t* ldr,
                                const int64_t* d_wmsh, const int64_t* d_vxc, double* ergs, int32_t* ierr) {
  *ierr = flosic_sic_getvlxc_device(handle(ctx), *npts, dev<const double>(d_rhog), *ldr, dev<const double>(d_wmsh),
                                    dev<double>(d_vxc), ergs);
}

void flosic_sic_apotnl_sic_(const int64_t* ctx, double* totqnum, const int32_t* lspx, const int32_t* iorbx,
                            double* results, double* cfrm, double* pot, int32_t* ierr) {
  *ierr = flosic_sic_apotnl_sic(handle(ctx), totqnum, *lspx, *iorbx, results, cfrm, pot);
}

void flosic_sic_siclagm_(const int64_t* ctx, const int32_t* lspn, double* sic, const int32_t* ld, int32_t* ierr) {
  *ierr = flosic_sic_siclagm(handle(ctx), *lspn, sic, *ld);
}

void flosic_sic_frmorb2_force_(const int64_t* ctx, const int32_t* lspn, const double* sic, const int32_t* ld,
                               double* debdax, int32_t* ierr) {
  *ierr = flosic_sic_frmorb2_force(handle(ctx), *lspn, sic, *ld, debdax);
}

void flosic_sic_cycle_(const int64_t* ctx, const int32_t* ld, double* results, double* sic, double* debdax,
                       double* cfrm, double* esic, int32_t* ierr) {
  *ierr = flosic_sic_cycle(handle(ctx), *ld, results, sic, debdax, cfrm, esic);
}

void flosic_sic_kernel_stats_(const int64_t* ctx, double* ms, int64_t* work, int32_t* ierr) {
  *ierr = flosic_sic_kernel_stats(handle(ctx), ms, work);
}

// The handles of a batch as an INTEGER*8 array: the same bytes as the
// C array of context pointers on a 64-bit host.
static_assert(sizeof(flosic_ctx*) == sizeof(int64_t), "context handles are INTEGER*8");

void flosic_sic_batch_cycle_(const int64_t* ctxs, const int32_t* n, const int32_t* wm, const int32_t* ld,
                             double* results, double* sic, double* debdax, double* cfrm, double* esic,
                             int32_t* ierr) {
  *ierr = flosic_sic_batch_cycle(reinterpret_cast<flosic_ctx**>(const_cast<int64_t*>(ctxs)), *n, *wm, *ld, results,
                                 sic, debdax, cfrm, esic);
}

void flosic_sic_adjoint_(const int64_t* ctx, const int32_t* lspn, double* g, const int32_t* ldg, int32_t* ierr) {
  *ierr = flosic_sic_adjoint(handle(ctx), *lspn, g, *ldg);
}

void flosic_sic_adjoint_fod_(const int64_t* ctx, const int32_t* lspn, double* grad, const int32_t* ld,
                             int32_t* ierr) {
  *ierr = flosic_sic_adjoint_fod(handle(ctx), *lspn, grad, *ld);
}

void flosic_sic_siclag_der_(const int64_t* ctx, double* dersic, const int32_t* ldo, int32_t* ierr) {
  *ierr = flosic_sic_siclag_der(handle(ctx), dersic, *ldo);
}

void flosic_sic_sicham_(const int64_t* ctx, const int32_t* lspn, double* ham, const int32_t* ldh,
                        const int32_t* packed, int32_t* ierr) {
  *ierr = flosic_sic_sicham(handle(ctx), *lspn, ham, *ldh, *packed);
}

void flosic_sic_densold_(const int64_t* ctx, const int32_t* ngrad, double* rhog, double* phig, int32_t* ierr) {
  *ierr = flosic_sic_densold(handle(ctx), *ngrad, rhog, phig);
}

void flosic_sic_coupot1_(const int64_t* ctx, double* coulomb, int32_t* ierr) {
  *ierr = flosic_sic_coupot1(handle(ctx), coulomb);
}

void flosic_sic_set_shard_(const int64_t* ctx, const int32_t* shard, const int32_t* nshards, int32_t* ierr) {
  *ierr = flosic_sic_set_shard(handle(ctx), *shard, *nshards);
}

void flosic_sic_partial_size_(const int64_t* ctx, int64_t* ndoubles, int32_t* ierr) {
  *ierr = flosic_sic_partial_size(handle(ctx), ndoubles);
}

void flosic_sic_cycle_partial_(const int64_t* ctx, const int64_t* d_partial, int32_t* ierr) {
  *ierr = flosic_sic_cycle_partial(handle(ctx), dev<double>(d_partial));
}

void flosic_sic_cycle_combine_(const int64_t* ctx, const int64_t* d_partial, const int32_t* ld, double* results,
                               double* sic, double* debdax, double* cfrm, double* esic, int32_t* ierr) {
  *ierr = flosic_sic_cycle_combine(handle(ctx), dev<const double>(d_partial), *ld, results, sic, debdax, cfrm, esic);
}

void flosic_sic_stats_(const int64_t* ctx, int64_t* launches, double* stage_ms, int64_t* npairs, int64_t* ncalls,
                       int64_t* work, int32_t* ierr) {
  *ierr = flosic_sic_stats(handle(ctx), launches, stage_ms, npairs, ncalls, work);
}

}  // extern "C"
