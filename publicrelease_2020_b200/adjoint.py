"""dE_SIC / d(FOD positions) through the basis-space adjoint, as a
torch.autograd.Function (the differentiation layer: a thin binding over the
C ABI).

Forward: one SIC cycle (flosic_sic_cycle) at the given FODs -> E_SIC.
Backward: flosic_sic_adjoint_fod per spin -- the adjoint G = dE_SIC/dC_FO
(basis values contracted with the SIC-weighted FO values on the FP64 tensor
cores) carried through the FO construction inside the library: C_FO = U C_KS
with U = S^-1/2 T the Lowdin-orthonormalised Fermi transformation
(frmiorb.f:351-480), T_kj = psi_j(a_k)/sqrt(rho(a_k)), S = T T^T; row k of T
depends on FOD a_k only, and its derivatives are FMAT(.,.,2:4)
(frmorb2.F:146-346).  With M = C_KS G, A = T M and S = V diag(q) V^T,
    W = V ((V^T A V) o F) V^T,   F_ab = -1 / (sqrt(q_a) sqrt(q_b) (sqrt(q_a) + sqrt(q_b))),
    dE/dT = (W + W^T) T + (M S^-1/2)^T,
    dE/da_m = sum_j (dE/dT)[m, j] dT[m, j]/da_m.
The result is the reference's FOD force (frmorb2.F:586-717) times 2/NSPN,
reached through the adjoint instead of through the SIC matrix.  The gradient
is formed only when backward runs."""
from __future__ import annotations

import numpy as np


def fod_gradient(ctx, psi=None, nwfs=None):
    """dE_SIC/dFOD, (nspn, max nfrm, 3), at the context's current orbitals and
    FODs (the potentials of the last cycle, recomputed if stale)."""
    nspn = ctx.sysm.nspn
    out = np.zeros((nspn, ctx.ld, 3))
    for s in range(nspn):
        n = ctx.nfrm[s]
        if n:
            out[s, :n] = ctx.adjoint_fod(s + 1)
    return out


def _set_fods(ctx, psi, nwfs, f):
    """Orbitals and FODs into the context unless it already holds these FODs."""
    cur = getattr(ctx, "_adjoint_fods", None)
    if cur is None or cur[0] is not psi or cur[1].shape != f.shape or not np.array_equal(cur[1], f):
        ctx.set_orbitals(psi, nwfs, [f[s] for s in range(f.shape[0])])
        ctx._adjoint_fods = (psi, f.copy())


def _autograd_function():
    import torch

    class SICEnergy(torch.autograd.Function):
        """E_SIC(FODs) with its gradient from the basis-space adjoint."""

        @staticmethod
        def forward(fc, fods, ctx, psi, nwfs):
            f = fods.detach().cpu().numpy().copy()
            _set_fods(ctx, psi, nwfs, f)
            r = ctx.cycle()
            fc.sic = (ctx, psi, nwfs, f)
            return torch.tensor(r["esic"], dtype=torch.float64)

        @staticmethod
        def backward(fc, grad):
            ctx, psi, nwfs, f = fc.sic
            _set_fods(ctx, psi, nwfs, f)   # another forward may have moved the context's FODs
            g = fod_gradient(ctx)[:, : f.shape[1]]
            return grad * torch.from_numpy(np.ascontiguousarray(g)), None, None, None

    return SICEnergy


def sic_energy(fods, ctx, psi, nwfs):
    """E_SIC as a differentiable function of fods, a (nspn, nfrm, 3) float64
    tensor (equal FO counts per spin; pad otherwise); ctx holds the geometry."""
    return _autograd_function().apply(fods, ctx, psi, nwfs)
