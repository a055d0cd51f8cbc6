"""SCAN meta-GGA on the GPU (IGGA=3, IDFTYP=11 for exchange and correlation)
against the FP64 oracle's restatement of scan.f / call_mgga.f90 /
gettau_par.f90 / the meta-GGA branch of SICLMSLV, through the C ABI.

The GPU forms the FO density from phi^2 and tau = |grad phi|^2/2 from the
same FO values, so alpha = (tau - tau_W)/tau_unif is zero up to rounding; the
reference (and the oracle) take the density from the Gaussian-pair route,
truncated at far points, and tau from the FO gradients.  In the density tails
tau_unif ~ rho^(5/3) is tiny and any mismatch between rho and tau moves alpha
far from zero.  The same happens near the FOs' nodes, where a density formed
from Gaussian pairs carries relative rounding error that phi^2 does not.  The
energy density rho*e_xc stays bounded there, the local potential
d(rho e_xc)/d rho does not, so XDEL = -int rho V_xc (RESULTS(7)) is
ill-conditioned for SCAN: measured, the GPU and the oracle differ in XDEL by
up to 0.06 Ha on water through points at 1e-9 .. 1e-12 of the peak density,
whether the oracle's density is truncated or not, while E_SIC agrees to
2e-13 Ha (untruncated) / 3e-9 Ha (truncated), the SIC matrix to 1e-10
relative and the forces to 2e-7 Ha/bohr.  Hence every RESULTS entry but XDEL,
the SIC matrix and the forces at the tolerances below, XDEL to 10%.

Pointwise, SCAN's potential is ill-conditioned where the density is many
decades below its maximum (alpha and its derivatives are differences of
nearly equal large terms there), so the XC entry point is compared pointwise
above 1e-6 max(rho) and everywhere weighted by the density."""
import numpy as np
import pytest

from oracle import oracle as O
from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W

pytestmark = pytest.mark.gpu

SCAN = "MGGA-SCAN*MGGA-SCAN"
E_TOL = 1e-8       # Ha, RESULTS entries
ESIC_TOL = 1e-8    # Ha, total E_SIC
SIC_RTOL = 1e-8    # SIC matrix, relative to its largest entry
F_TOL = 1e-6       # Ha/bohr, FOD forces (they inherit the SIC-matrix differences)
XDEL_RTOL = 0.1    # RESULTS(7), relative to max(1, |XDEL|) (ill-conditioned for SCAN, see above)


def systems():
    return {
        "water_scan_nspn2": W.water(seed=0, nrad=18, functional=SCAN),
        "synthetic_scan_nspn1": W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=5000, nfo=4, functional=SCAN),
    }


@pytest.fixture(scope="module", params=list(systems().keys()))
def pair(request):
    sysm = systems()[request.param]
    ctx = S.open_system(sysm)
    orc = O.Oracle(sysm)
    yield request.param, sysm, ctx, orc
    ctx.close()


def test_scan_getvlxc_matches_oracle(pair):
    """Same density channels and tau in, same functional out: potential,
    Hamiltonian ingredients (MIXIN) and energies at rounding level."""
    name, sysm, ctx, orc = pair
    for k in range(1, sysm.nfrm[0] + 1):
        _, rho, _ = orc.coupot_sic(1, k, exact=True)
        tau = orc.fo_tau(1, k)
        vg, mg, eg = ctx.getvlxc_mgga(rho, tau)
        vo, mo, eo = orc.getvlxc_mgga(rho, tau)
        n = sysm.nmsh
        r0, w = rho[0], sysm.wmsh
        m = r0 > 1e-6 * r0.max()
        # measured: <= 1e-9 of max|V| pointwise (differences of nearly equal terms in d alpha / d rho)
        assert np.max(np.abs(vg[0] - vo[0])[m]) <= 1e-8 * np.abs(vo[0][m]).max(), (name, k)
        # Density-weighted over all points, the bound is the potential's own
        # conditioning: how far the oracle's V moves when its inputs move by one
        # unit in the last place.  The device code, compiled for the host
        # without multiply-add contraction, equals the oracle to 1e-15 here;
        # the GPU contracts multiply-adds, which moves the sum by 2.1e-10 on
        # water FO 2 (one point, rho = 2e-5 max(rho), V = 1.5e5, where
        # tau - tau_W cancels), 10-100x below this spread for every FO.
        rng = np.random.default_rng(k)
        spread = np.zeros(n)
        for _ in range(4):
            vp, _, _ = orc.getvlxc_mgga(rho * (1 + 2.0**-52 * rng.uniform(-1, 1, rho.shape)),
                                        tau * (1 + 2.0**-52 * rng.uniform(-1, 1, tau.shape)))
            spread = np.maximum(spread, np.abs(vp[0] - vo[0]))
        assert np.sum(np.abs(vg[0] - vo[0]) * r0 * w) <= np.sum(spread * r0 * w), (name, k)
        for d in range(4):
            scale = np.abs(mo[:, d][m]).max()
            assert np.max(np.abs(mg[:n, d] - mo[:, d])[m]) <= 1e-8 * scale, (name, k, d)
        assert np.all(mg[n:] == 0.0)
        assert np.max(np.abs(eg - eo)) <= 1e-11 * max(1.0, np.abs(eo).max()), (name, k, eg, eo)


@pytest.mark.parametrize("exact_density", [False, True])
def test_scan_cycle_matches_oracle(pair, exact_density):
    name, sysm, ctx, orc = pair
    g = ctx.cycle()
    orc.set_xc_exact_density(exact_density)
    try:
        r = orc.sic_cycle(nthreads=8)
    finally:
        orc.set_xc_exact_density(False)
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        gr, orr = g["results"][s][:n], r["results"][s][:n]
        d = np.abs(gr[:, 1:] - orr[:, 1:])
        assert np.all(d[:, 5] <= XDEL_RTOL * np.maximum(1.0, np.abs(orr[:, 6]))), (name, d[:, 5])
        d[:, 5] = 0.0
        assert np.max(d) < E_TOL, (name, exact_density, d.max(axis=0))
        lam_g, lam_o = g["sic"][s][:n, :n], r["sic"][s][:n, :n]
        assert np.max(np.abs(lam_g - lam_o)) < SIC_RTOL * np.abs(lam_o).max(), name
        ftol = F_TOL * max(1.0, np.abs(r["debdax"][s][:n]).max())
        assert np.max(np.abs(g["debdax"][s][:n] - r["debdax"][s][:n])) < ftol, name
    assert abs(g["esic"] - r["esic"]) < ESIC_TOL, (name, g["esic"], r["esic"])


def test_scan_sic_matrix_from_oracle_potentials(pair):
    """SICLAGM's meta-GGA terms: the GPU SIC matrix against the oracle's
    SICLAGM fed with the oracle's own potentials and MIXIN arrays."""
    name, sysm, ctx, orc = pair
    for s in range(1, sysm.nspn + 1):
        n = sysm.nfrm[s - 1]
        outs = [orc.apotnl_sic(s, k) for k in range(1, n + 1)]
        lo = orc.siclagm(s, np.stack([o["pot"] for o in outs]), np.stack([o["mixin"] for o in outs]))
        lam = ctx.siclagm(s)
        assert np.max(np.abs(lam[:n, :n] - lo[:n, :n])) < SIC_RTOL * np.abs(lo[:n, :n]).max(), name


def test_scan_mixed_precision_gate(pair):
    """The mixed path changes only the Coulomb potential: the SCAN energy and
    forces stay within the mixed form's targets."""
    name, sysm, ctx, orc = pair
    ref = ctx.cycle()
    ctx.set_precision("mixed")
    try:
        mix = ctx.cycle()
    finally:
        ctx.set_precision("fp64")
    assert abs(mix["esic"] - ref["esic"]) <= 1e-5, name
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        assert np.max(np.abs(mix["debdax"][s][:n] - ref["debdax"][s][:n])) <= 1e-4, name


def test_scan_rejects_plain_getvlxc():
    sysm = systems()["synthetic_scan_nspn1"]
    ctx = S.open_system(sysm)
    try:
        with pytest.raises(S.FlosicError) as e:
            ctx.getvlxc(np.zeros((10, sysm.nmsh)))
        assert e.value.code == 1
        assert "meta-GGA" in str(e.value)
    finally:
        ctx.close()
