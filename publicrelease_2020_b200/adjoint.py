"""dE_SIC / d(FOD positions) through the basis-space adjoint, as a
torch.autograd.Function (the differentiation layer: a thin binding over the
C ABI).

Forward: one SIC cycle (flosic_sic_cycle) at the given FODs -> E_SIC.
Backward: the adjoint G = dE_SIC/dC_FO of each spin (flosic_sic_adjoint, a
chunked GEMM of the basis values with the SIC-weighted FO values on the GPU)
contracted with the derivative of the FO coefficients with respect to each
FOD.  The FO coefficients are C_FO = U C_KS with U = S^-1/2 T the
Lowdin-orthonormalised Fermi transformation (frmiorb.f:351-480), T_kj =
psi_j(a_k)/sqrt(rho(a_k)), S = T T^T; row k of T depends on FOD a_k only, and
its derivatives are FMAT(.,.,2:4) (frmorb2.F:146-346).  With M = C_KS G,
A = T M and S = V diag(q) V^T,
    W = V ((V^T A V) o F) V^T,   F_ab = -1 / (sqrt(q_a) sqrt(q_b) (sqrt(q_a) + sqrt(q_b))),
    dE/dT = (W + W^T) T + (M S^-1/2)^T,
    dE/da_m = sum_j (dE/dT)[m, j] dT[m, j]/da_m.
The result is the reference's FOD force (frmorb2.F:586-717) reached through
the adjoint instead of through the SIC matrix."""
from __future__ import annotations

import numpy as np


def fod_gradient(ctx, psi, nwfs):
    """dE_SIC/dFOD, (nspn, max nfrm, 3), at the context's current orbitals and
    FODs (the potentials of the last cycle, recomputed if stale)."""
    fm = ctx.frmorb2_fmat()                       # [s][K][jfm][jwf]
    nspn = ctx.sysm.nspn
    out = np.zeros((nspn, ctx.ld, 3))
    for s in range(nspn):
        n = ctx.nfrm[s]
        if n == 0:
            continue
        G = ctx.adjoint(s + 1)                    # (nbasis, n)
        cks = np.asarray(psi)[s * nwfs[0]: s * nwfs[0] + n]   # (n, nbasis)
        M = cks @ G                               # M[j, k]
        T = fm[s, 0, :n, :n]
        q, V = np.linalg.eigh(T @ T.T)
        rq = np.sqrt(q)
        Sm = (V / rq) @ V.T
        F = -1.0 / (rq[:, None] * rq[None, :] * (rq[:, None] + rq[None, :]))
        W = V @ ((V.T @ (T @ M) @ V) * F) @ V.T
        dEdT = (W + W.T) @ T + (M @ Sm).T
        for d in range(3):
            out[s, :n, d] = np.einsum("mj,mj->m", dEdT, fm[s, 1 + d, :n, :n])
    return out


def _autograd_function():
    import torch

    class SICEnergy(torch.autograd.Function):
        """E_SIC(FODs) with its gradient from the basis-space adjoint."""

        @staticmethod
        def forward(fc, fods, ctx, psi, nwfs):
            f = fods.detach().cpu().numpy()
            ctx.set_orbitals(psi, nwfs, [f[s] for s in range(f.shape[0])])
            r = ctx.cycle()
            g = fod_gradient(ctx, psi, nwfs)
            fc.save_for_backward(torch.from_numpy(g[:, : f.shape[1]].copy()))
            return torch.tensor(r["esic"], dtype=torch.float64)

        @staticmethod
        def backward(fc, grad):
            (g,) = fc.saved_tensors
            return grad * g, None, None, None

    return SICEnergy


def sic_energy(fods, ctx, psi, nwfs):
    """E_SIC as a differentiable function of fods, a (nspn, nfrm, 3) float64
    tensor (equal FO counts per spin; pad otherwise); ctx holds the geometry."""
    return _autograd_function().apply(fods, ctx, psi, nwfs)
