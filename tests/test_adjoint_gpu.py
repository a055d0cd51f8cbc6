"""Basis-space adjoint G = dE_SIC/dC_FO (flosic_sic_adjoint) and the FOD
gradient built on it inside the library (flosic_sic_adjoint_fod, used by
publicrelease_2020_b200.adjoint), through the C ABI.

Checks: (1) C_FO^T G = (4/NSPN) SIC, the FO-space projection of the adjoint
is the SIC matrix (rounding level); (2) the FOD gradient from G through the
Lowdin chain rule (in the library, and restated here in numpy) equals the
reference's FOD force formula (frmorb2.F,
computed by the library from the SIC matrix), times 2/NSPN: DEBDAX is the
force on one spin's FODs, and with NSPN=1 they stand for both spins in E_SIC;
(3) on benzene (C3) the torch.autograd.Function returns that gradient, and
central finite differences of E_SIC (h = 1e-4 bohr) agree with it.

The finite differences agree with the analytic gradient once the mesh
integrates the FO densities: E_H is formed as (1/2) sum_p w rho V_H with V_H
the analytic potential, and the force formula (as the reference's) assumes
the potentials are the energy's derivatives, which holds up to that
quadrature.  Measured on benzene (largest relative difference of five FOD
coordinates): 0.39 on 39,852 mesh points (nrad 24), 0.076 on 79,463 (nrad 48),
< 5e-5 on 158,659 (nrad 96); the test uses nrad 96."""
import numpy as np
import pytest

from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W
from publicrelease_2020_b200.adjoint import fod_gradient

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "water_lda_nspn2": lambda: W.water(seed=0, nrad=18),
    "synthetic_pbe_nspn1": lambda: W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=5000, nfo=4),
    "water_scan_nspn2": lambda: W.water(seed=0, nrad=18, functional="MGGA-SCAN*MGGA-SCAN"),
}


@pytest.fixture(scope="module", params=list(SYSTEMS))
def case(request):
    sysm = SYSTEMS[request.param]()
    ctx = S.open_system(sysm)
    r = ctx.cycle()
    yield request.param, sysm, ctx, r
    ctx.close()


def test_adjoint_projects_to_sic_matrix(case):
    name, sysm, ctx, r = case
    tm, _ = ctx.frmiorb()
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        G = ctx.adjoint(s + 1)                                   # (nbasis, n)
        cks = sysm.psi[s * sysm.nwfs[0]: s * sysm.nwfs[0] + n]   # (n, nbasis)
        cfo = tm[s][:n, :n].T @ cks                              # C_FO[k] = sum_j TMAT(k, j) psi_j
        lam = r["sic"][s][:n, :n].T                              # lam[j, l] = SIC(j, l)
        proj = cfo @ G                                           # [j, l]
        assert np.max(np.abs(proj - 4.0 / sysm.nspn * lam)) <= 1e-10 * np.abs(lam).max(), name


def _chain_rule_numpy(ctx, psi, nwfs):
    """The chain rule of flosic_sic_adjoint_fod restated in numpy from the
    adjoint G and FMAT returned through the C ABI (independent eigen-solver)."""
    fm = ctx.frmorb2_fmat()                       # [s][K][jfm][jwf]
    out = np.zeros((ctx.sysm.nspn, ctx.ld, 3))
    for s in range(ctx.sysm.nspn):
        n = ctx.nfrm[s]
        G = ctx.adjoint(s + 1)                    # (nbasis, n)
        cks = np.asarray(psi)[s * nwfs[0]: s * nwfs[0] + n]
        M = cks @ G
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


def test_adjoint_fod_gradient_equals_reference_force(case):
    name, sysm, ctx, r = case
    g = fod_gradient(ctx)
    gn = _chain_rule_numpy(ctx, sysm.psi, sysm.nwfs)
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        ref = (2.0 / sysm.nspn) * r["debdax"][s][:n]
        assert np.max(np.abs(g[s, :n] - ref)) <= 1e-8 * max(1.0, np.abs(ref).max()), (name, g[s, :n], ref)
        assert np.max(np.abs(g[s, :n] - gn[s, :n])) <= 1e-10 * max(1.0, np.abs(ref).max()), name


def test_autograd_benzene_gradient_and_finite_differences():
    import torch
    from publicrelease_2020_b200.adjoint import sic_energy
    sysm = W.benzene(seed=3, nrad=96)
    ctx = S.open_system(sysm)
    try:
        f0 = np.stack(sysm.fods)
        fods = torch.tensor(f0, dtype=torch.float64, requires_grad=True)
        e = sic_energy(fods, ctx, sysm.psi, sysm.nwfs)
        e.backward()
        grad = fods.grad.numpy()
        ref = ctx.cycle()   # same FODs: the reference force formula
        for s in range(2):
            assert np.allclose(grad[s], ref["debdax"][s][:21], rtol=1e-8, atol=1e-9)
        # central differences on a few coordinates (core, bond and pi FODs)
        h = 1e-4
        picks = [(0, 0, 0), (0, 7, 1), (0, 13, 2), (1, 19, 2), (1, 3, 0)]
        rel = []
        for s, m, d in picks:
            fp, fm = f0.copy(), f0.copy()
            fp[s, m, d] += h
            fm[s, m, d] -= h
            ep = float(sic_energy(torch.tensor(fp), ctx, sysm.psi, sysm.nwfs))
            em = float(sic_energy(torch.tensor(fm), ctx, sysm.psi, sysm.nwfs))
            fd = (ep - em) / (2 * h)
            rel.append(abs(fd - grad[s, m, d]) / max(abs(grad[s, m, d]), 1e-3))
        assert max(rel) < 1e-3, rel
    finally:
        ctx.close()
