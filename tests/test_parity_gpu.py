"""GPU parity: the CUDA path (through the C ABI) against the FP64 oracle on
the same seeded inputs.

Tolerances (FP64 path): the GPU forms the FO density as phi^2 from the
orbital values, the reference (and the oracle) from the Gaussian-pair
polynomials at near points only; both are exact up to rounding relative to
max(rho).  Summation orders differ (spatially tiled mesh, tree reductions).
RESULTS entries (energies, charges) are compared at 1e-8 Ha absolute -- the
FP64 bar of matching the reference to 1e-8 Ha; most agree to 1e-11, the
largest gap is XDEL = -int rho V_xc for GGA, where the gradient-corrected
potential amplifies the density rounding at low density.  E_SIC at 1e-9 Ha,
potentials at 1e-9 relative, SIC-matrix entries at 1e-9 relative, forces at
1e-8 Ha/bohr."""
import numpy as np
import pytest

from oracle import oracle as O
from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W

pytestmark = pytest.mark.gpu

E_TOL = 1e-8       # Ha, RESULTS entries
ESIC_TOL = 1e-9    # Ha, total E_SIC
POT_RTOL = 1e-9    # potentials, relative to max |V|
SIC_RTOL = 1e-9    # SIC matrix, relative to max |lambda| (LDA)
SIC_RTOL_GGA = 1e-8  # GGA: the gradient-corrected potential amplifies the density-route rounding
F_TOL = 1e-8       # Ha/bohr, FOD forces (LDA)
F_TOL_GGA = 1e-6   # Ha/bohr: GGA forces inherit the SIC-matrix differences above (the force
                   # routine itself agrees to 1e-9 when fed the same SIC matrix, see
                   # test_siclagm_and_force_entry_points)


def systems():
    return {
        "water_lda_nspn2": W.water(seed=0, nrad=18),
        # C1 as configured: water on the reference's default NRLMOL basis (73 functions)
        "water_default_basis_lda_nspn2": W.water(seed=0, nrad=18, basis="default"),
        "synthetic_pbe_nspn1": W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=5000, nfo=4),
        "synthetic_pw91gga_nspn2": W.small_synthetic(seed=7, natoms=3, nbasis=30, nmsh=4000, nfo=3,
                                                     functional="GGA-PW91*GGA-PW91", nspn=2),
    }


@pytest.fixture(scope="module", params=list(systems().keys()))
def pair(request):
    sysm = systems()[request.param]
    ctx = S.open_system(sysm)
    orc = O.Oracle(sysm)
    yield request.param, sysm, ctx, orc
    ctx.close()


def test_cycle_matches_oracle(pair):
    name, sysm, ctx, orc = pair
    g = ctx.cycle()
    r = orc.sic_cycle(nthreads=8)
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        gr, orr = g["results"][s][:n], r["results"][s][:n]
        assert np.allclose(gr[:, 0], orr[:, 0])
        assert np.max(np.abs(gr[:, 1:] - orr[:, 1:])) < E_TOL, name
        assert np.max(np.abs(gr[:, 8] - orr[:, 8])) < ESIC_TOL, name
        lam_g, lam_o = g["sic"][s][:n, :n], r["sic"][s][:n, :n]
        tol = SIC_RTOL_GGA if (sysm.xc[0] or sysm.xc[2]) else SIC_RTOL
        assert np.max(np.abs(lam_g - lam_o)) < tol * np.abs(lam_o).max(), name
        ftol = F_TOL_GGA if (sysm.xc[0] or sysm.xc[2]) else F_TOL
        assert np.max(np.abs(g["debdax"][s][:n] - r["debdax"][s][:n])) < ftol * max(1.0, np.abs(r["debdax"][s]).max())
        assert np.max(np.abs(g["cfrm"][s][:n] - r["cfrm"][s][:n])) < 1e-9
    assert abs(g["esic"] - r["esic"]) < ESIC_TOL


def test_coupot_and_potential_match_oracle(pair):
    """The reference (poisson1.f) accumulates the FO density only at the
    points inside RCUT of each Poisson call, so its density is truncated at a
    level set by the Coulomb error bound, not by rounding: against the same
    routine with every point treated as near (exact mode) its density channels
    move by up to ~1e-8 of their maxima and a PBE potential by up to ~1e-5 of
    max|V| at low density.  The GPU forms the untruncated density phi^2.  So
    the Coulomb potential (near/far split as in the reference) is compared with
    the reference mode, the density with the exact mode, and the total
    potential with Coulomb(reference mode) + V_xc(exact-mode density)."""
    name, sysm, ctx, orc = pair
    gga = bool(sysm.xc[0] or sysm.xc[2])
    nch = 10 if gga else 1
    for k in range(1, sysm.nfrm[0] + 1):
        cg, rg = ctx.coupot_sic(1, k)
        co, ro, _ = orc.coupot_sic(1, k)
        _, rx, _ = orc.coupot_sic(1, k, exact=True)
        assert np.max(np.abs(cg - co)) < POT_RTOL * np.abs(co).max(), (name, k)
        for ch in range(nch):   # each density channel relative to its own scale
            scale = np.abs(rx[ch]).max()
            assert np.max(np.abs(rg[ch] - rx[ch])) < 1e-10 * scale + 1e-14, (name, k, ch)
            assert np.max(np.abs(rg[ch] - ro[ch])) < 1e-8 * scale + 1e-13, (name, k, ch)
        a = ctx.apotnl_sic(1, k)
        b = orc.apotnl_sic(1, k)
        vx, _ = orc.getvlxc_sic(rx)
        want = co * (sysm.nspn / 2.0) + vx[0]   # apotnl_sic.F scales COULOMB by NSPN/2
        # V_xc ~ rho^(1/3) (and its gradient terms) amplifies rounding where
        # rho is many decades below max(rho); subvlxc_libxc.F90 drops rho < 1e-20
        # altogether.  Compare pointwise above 1e-6 max(rho), and everywhere
        # weighted by the density.
        rho = rx[0]
        m = rho > 1e-6 * rho.max()
        assert np.max(np.abs(a["pot"] - want)[m]) < POT_RTOL * np.abs(want).max(), (name, k)
        assert np.sum(np.abs(a["pot"] - want) * rho * sysm.wmsh) < 1e-11, (name, k)
        assert np.max(np.abs(a["results"][1:] - b["results"][1:])) < E_TOL


def test_fo_construction_matches_oracle(pair):
    name, sysm, ctx, orc = pair
    fg = ctx.frmorb2_fmat()
    fo = orc.fmat()
    tg, eg = ctx.frmiorb()
    to, eo = orc.frmiorb()
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        assert np.allclose(fg[s, :, :n, :n], fo[s, :, :n, :n], rtol=1e-11, atol=1e-11)
        assert np.allclose(tg[s, :n, :n], to[s, :n, :n], rtol=1e-10, atol=1e-10)
        assert np.allclose(np.sort(eg[s, :n]), np.sort(eo[s, :n]), rtol=1e-11)


def test_getvlxc_matches_oracle(pair):
    name, sysm, ctx, orc = pair
    _, rho, _ = orc.coupot_sic(1, 1)
    vg, eg = ctx.getvlxc(rho)
    vo, eo = orc.getvlxc_sic(rho)
    assert np.max(np.abs(vg[0] - vo[0])) < 1e-10 * np.abs(vo[0]).max()
    assert np.max(np.abs(eg - eo)) < 1e-11 * max(1.0, np.abs(eo).max())


def test_gorbdrv_matches_oracle(pair):
    name, sysm, ctx, orc = pair
    rng = np.random.default_rng(3)
    pts = rng.normal(0, 0.8, (25, 3))
    for nderv in (0, 1, 2):
        for ifnct in range(1, min(sysm.ntypes, 3) + 1):
            gg, ug, ag = ctx.gorbdrv(nderv, pts, ifnct)
            go, uo, ao = orc.gorbdrv(nderv, pts, ifnct)
            nch = (1, 4, 10)[nderv]
            assert ug == uo
            assert np.array_equal(ag, ao)
            a, b = gg[:, :, :, :nch, :], go[:, :, :, :nch, :]
            assert np.max(np.abs(a - b)) < 1e-12 * max(1.0, np.abs(b).max())


def test_siclagm_and_force_entry_points(pair):
    name, sysm, ctx, orc = pair
    for s in range(1, sysm.nspn + 1):
        lam = ctx.siclagm(s)
        n = sysm.nfrm[s - 1]
        pots = np.stack([orc.apotnl_sic(s, k)["pot"] for k in range(1, n + 1)])
        lo = orc.siclagm(s, pots)
        tol = SIC_RTOL_GGA if (sysm.xc[0] or sysm.xc[2]) else SIC_RTOL
        assert np.max(np.abs(lam[:n, :n] - lo[:n, :n])) < tol * np.abs(lo[:n, :n]).max()
        fg = ctx.frmorb2_force(s, lo)
        fo = orc.frmorb2_force(s, lo)
        assert np.max(np.abs(fg[:n] - fo[:n])) < 1e-9 * max(1.0, np.abs(fo[:n]).max())


def test_error_codes():
    sysm = W.water(seed=0, nrad=12)
    ctx = S.open_system(sysm)
    f = [x.copy() for x in sysm.fods]
    f[0][1] = f[0][0]
    ctx.set_orbitals(sysm.psi, sysm.nwfs, f)
    with pytest.raises(S.FlosicError) as e:
        ctx.frmiorb()
    assert e.value.code == 3  # FLOSIC_ERR_LOWDEN
    with pytest.raises(S.FlosicError) as e:
        ctx.set_orbitals(sysm.psi, (5, 4), sysm.fods)
    assert e.value.code == 5  # FLOSIC_ERR_NFRM
    with pytest.raises(S.FlosicError) as e:
        ctx.apotnl_sic(1, 99)
    assert e.value.code in (1, 8)
    ctx.close()


def test_shared_and_per_fo_coulomb_kernels_agree(pair, monkeypatch):
    """The shared-geometry tensor-core kernel (calls whose CG/RCUT/NPOT are the
    same for every FO) against the per-FO kernel run on every call
    (FLOSIC_COULOMB=perfo): same sums in another order, so agreement is at
    rounding level."""
    name, sysm, ctx, orc = pair
    monkeypatch.setenv("FLOSIC_COULOMB", "perfo")
    alt = S.open_system(sysm)
    try:
        for s in range(sysm.nspn):
            for k in range(1, sysm.nfrm[s] + 1):
                a, _ = ctx.coupot_sic(s + 1, k)
                b, _ = alt.coupot_sic(s + 1, k)
                assert np.max(np.abs(a - b)) < 1e-12 * np.abs(b).max(), (name, s, k)
    finally:
        alt.close()


def test_work_counts_match_oracle(pair):
    """Near (pair, point, FO) and far (call, point, FO) evaluations counted by
    the Coulomb kernels equal the reference's POISSON1 counts (points inside /
    outside RCUT of each call and FO, NPOT=1 calls all near): the near/far split
    is the reference's.  CG and RCUT may differ from the oracle's in the last
    bit, which can move a point lying on a sphere; hence the 1e-6 slack."""
    name, sysm, ctx, orc = pair
    fresh = S.open_system(sysm)
    try:
        fresh.cycle()
        st = fresh.stats()
    finally:
        fresh.close()
    near = far = 0
    for s in range(sysm.nspn):
        for k in range(1, sysm.nfrm[s] + 1):
            d = orc.pair_stats(s + 1, k)
            near += d["near"]
            far += d["far"]
    assert near > 0
    assert abs(st["near_evals"] - near) <= 1e-6 * near, (name, st["near_evals"], near)
    assert abs(st["far_evals"] - far) <= 1e-6 * max(far, 1), (name, st["far_evals"], far)
