"""GPU parity of the reference-route FO density (FLOSIC_DENSITY_PAIRS).

POISSON1 forms each FO's density for the SIC exchange-correlation from the
Gaussian-pair polynomials of its Poisson calls, at the mesh points inside each
call's RCUT sphere only, with polynomial coefficients of magnitude <= 1e-14
dropped (poisson1.f:849-948, gtdncf.F).  In this mode the GPU forms that same
truncated density, so the quantities that the default phi^2 route can only
match to the truncation level (the gradient-corrected XDEL, GGA forces, and
for SCAN the whole low-density tail of the functional) are compared with the
oracle at the FP64 drop-in bar: RESULTS entries to 1e-8 Ha, E_SIC to 1e-9 Ha,
SIC matrices to 1e-9 of their largest entry and FOD forces to 1e-8 Ha/bohr.
The density channels themselves agree to 1e-12 of each channel's maximum
(measured: 2e-15 .. 4e-14): both sides add the same pair terms in the same
call and pair order, and differ only by the rounding of exp and of fused
multiply-adds.

One entry is held to its conditioning instead: SCAN's XDEL = -int rho V_xc
(RESULTS(7)).  Its local potential is a difference of large terms wherever
tau_unif ~ rho^(5/3) is tiny, and moving rho and tau by one unit in the last
place of their maxima -- the rounding of any evaluation of them as sums over
basis functions -- moves XDEL by 1e-6 .. 2e-2 Ha per FO (water).  The test
measures that spread with the oracle for each FO (four random draws) and
requires the GPU's XDEL within it; measured, the GPU sits at 0.00 .. 0.72 of
the spread.  Every other SCAN entry meets the 1e-8 Ha bar."""
import numpy as np
import pytest

from oracle import oracle as O
from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W
from publicrelease_2020_b200.batch import Batch

pytestmark = pytest.mark.gpu

SCAN = "MGGA-SCAN*MGGA-SCAN"
E_TOL = 1e-8        # Ha, RESULTS entries (XDEL included)
ESIC_TOL = 1e-9     # Ha, total E_SIC
SIC_RTOL = 1e-9     # SIC matrix, relative to its largest entry
F_TOL = 1e-8        # Ha/bohr, FOD forces
RHO_RTOL = 1e-12    # density channels, relative to each channel's maximum


def systems():
    return {
        "water_lda_nspn2": W.water(seed=0, nrad=18),
        "synthetic_pbe_nspn1": W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=5000, nfo=4),
        "synthetic_pw91gga_nspn2": W.small_synthetic(seed=7, natoms=3, nbasis=30, nmsh=4000, nfo=3,
                                                     functional="GGA-PW91*GGA-PW91", nspn=2),
        "water_scan_nspn2": W.water(seed=0, nrad=18, functional=SCAN),
        "synthetic_scan_nspn1": W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=5000, nfo=4, functional=SCAN),
    }


@pytest.fixture(scope="module", params=list(systems().keys()))
def pair(request):
    sysm = systems()[request.param]
    ctx = S.open_system(sysm)
    ctx.set_density_mode("pairs")
    orc = O.Oracle(sysm)
    yield request.param, sysm, ctx, orc
    ctx.close()


def test_pair_density_matches_oracle(pair):
    name, sysm, ctx, orc = pair
    nch = 4 if "scan" in name else (10 if (sysm.xc[0] or sysm.xc[2]) else 1)
    for s in range(1, sysm.nspn + 1):
        for k in range(1, sysm.nfrm[s - 1] + 1):
            _, rg = ctx.coupot_sic(s, k)
            _, ro, _ = orc.coupot_sic(s, k)
            for ch in range(nch):
                scale = np.abs(ro[ch]).max()
                assert np.max(np.abs(rg[ch] - ro[ch])) <= RHO_RTOL * scale, (name, s, k, ch)
            # outside every call's sphere both densities are exactly zero
            assert np.array_equal(rg[0] == 0.0, ro[0] == 0.0), (name, s, k)


def _scan_xdel_spread(orc, sysm, s, k, draws=4):
    """How far the oracle's XDEL (its exchange-correlation part, -sum w rho
    V_xc) moves when every density channel and tau move by up to one unit in
    the last place of their maxima."""
    w = sysm.wmsh
    _, rho, _ = orc.coupot_sic(s, k)
    tau = orc.fo_tau(s, k)
    v0, _, _ = orc.getvlxc_mgga(rho, tau)
    x0 = -np.sum(w * rho[0] * v0[0])
    rng = np.random.default_rng(k + 10 * s)
    spread = 0.0
    for _ in range(draws):
        r2 = rho.copy()
        for ch in range(4):
            r2[ch] = rho[ch] + 2.0**-52 * np.abs(rho[ch]).max() * rng.uniform(-1, 1, rho[ch].shape)
        t2 = tau + 2.0**-52 * tau.max() * rng.uniform(-1, 1, tau.shape)
        vp, _, _ = orc.getvlxc_mgga(r2, t2)
        spread = max(spread, abs(-np.sum(w * r2[0] * vp[0]) - x0))
    return spread


def test_cycle_pairs_matches_oracle(pair):
    name, sysm, ctx, orc = pair
    g = ctx.cycle()
    r = orc.sic_cycle(nthreads=8)
    scan = "scan" in name
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        gr, orr = g["results"][s][:n], r["results"][s][:n]
        assert np.allclose(gr[:, 0], orr[:, 0])
        d = np.abs(gr[:, 1:] - orr[:, 1:])
        if scan:
            for k in range(n):
                sp = _scan_xdel_spread(orc, sysm, s + 1, k + 1)
                assert d[k, 5] <= sp, (name, s, k, d[k, 5], sp)
            d[:, 5] = 0.0
        assert np.max(d) < E_TOL, (name, d.max(axis=0))
        lam_g, lam_o = g["sic"][s][:n, :n], r["sic"][s][:n, :n]
        assert np.max(np.abs(lam_g - lam_o)) < SIC_RTOL * np.abs(lam_o).max(), name
        ftol = F_TOL * max(1.0, np.abs(r["debdax"][s][:n]).max())
        assert np.max(np.abs(g["debdax"][s][:n] - r["debdax"][s][:n])) < ftol, name
    assert abs(g["esic"] - r["esic"]) < ESIC_TOL, (name, g["esic"], r["esic"])


def test_scan_mixin_pairs_matches_oracle(pair):
    """MGGA#### records (flosic_sic_mgga_mixin) from the pair-route density.
    As in the file-writer test, the reference is the oracle's SUBVLXC on the
    GPU's own FO density channels and the oracle's tau, so that the density's
    last-digit rounding stays out of the comparison.  With the pair route, rho
    and tau no longer come from the same orbital values and SCAN's ingredients
    are ill-conditioned where they disagree, so the bound is the oracle's own
    spread when rho and tau move by one unit in the last place of their maxima
    (four draws), pointwise where rho is above 1e-3 of its maximum (at least
    1e-8 of the channel's scale) and density-weighted over all points."""
    name, sysm, ctx, orc = pair
    if "scan" not in name:
        pytest.skip("MIXIN belongs to meta-GGA functionals")
    n, w = sysm.nmsh, sysm.wmsh
    for s in range(1, sysm.nspn + 1):
        for k in range(1, sysm.nfrm[s - 1] + 1):
            m = ctx.mgga_mixin(s, k)
            _, rho = ctx.coupot_sic(s, k)
            tau = orc.fo_tau(s, k)
            _, mo, _ = orc.getvlxc_mgga(rho, tau)
            r0 = rho[0]
            keep = r0 > 1e-3 * r0.max()
            assert np.all(m[n:] == 0.0)
            rng = np.random.default_rng(k + 10 * s)
            sp = np.zeros_like(mo)
            for _ in range(4):
                r2 = rho.copy()
                for ch in range(4):
                    r2[ch] = rho[ch] + 2.0**-52 * np.abs(rho[ch]).max() * rng.uniform(-1, 1, rho[ch].shape)
                t2 = tau + 2.0**-52 * tau.max() * rng.uniform(-1, 1, tau.shape)
                _, mp, _ = orc.getvlxc_mgga(r2, t2)
                sp = np.maximum(sp, np.abs(mp - mo))
            for d in range(4):
                scale = np.abs(mo[keep, d]).max()
                diff = np.abs(m[:n, d] - mo[:, d])
                assert np.all(diff[keep] <= np.maximum(1e-8 * scale, sp[keep, d])), (name, s, k, d)
                dw, sw = np.sum(diff * r0 * w), np.sum(sp[:, d] * r0 * w)
                assert dw <= max(sw, 1e-8 * scale), (name, s, k, d, dw, sw)


def test_mode_switch_restores_phi2(pair):
    """Switching back to phi^2 invalidates the cached potentials: the cycle
    then equals a fresh context's default cycle bit for bit."""
    name, sysm, ctx, orc = pair
    ctx.set_density_mode("phi2")
    try:
        a = ctx.cycle()
    finally:
        ctx.set_density_mode("pairs")
    fresh = S.open_system(sysm)
    try:
        b = fresh.cycle()
    finally:
        fresh.close()
    assert a["esic"] == b["esic"], name
    for key in ("results", "sic", "debdax"):
        assert np.array_equal(a[key], b[key]), (name, key)


def test_batched_cycle_pairs_equals_serial():
    """The batched launch forms the pair-route densities in each molecule's
    own preparation step: its results equal each molecule's serial cycle."""
    systems_ = W.alkane_batch(n=3, seed=100, max_carbons=3, nrad=(6, 8))
    b = Batch(systems_)
    try:
        for c in b.ctxs:
            c.set_density_mode("pairs")
        got = b.cycle()
        want = b.cycle_serial()
    finally:
        b.close()
    for sysm, p, q in zip(systems_, got, want):
        assert p["esic"] == q["esic"], sysm.name
        for key in ("results", "sic", "debdax", "cfrm"):
            n = q[key].shape[1]
            assert np.array_equal(p[key][:, :n, ...][..., : q[key].shape[-1]], q[key]), (sysm.name, key)
