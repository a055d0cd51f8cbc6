"""CPU tests pinning the FP64 oracle (oracle/) against closed forms and
identities.  The reference ships no kernel-level golden vectors and its
Fortran cannot be built here, so these analytic pins stand in: Boys values,
closed-form Coulomb potentials, the multipole far field against the exact
mode, the charge and r V(r) asymptote, LDA/PW92/PBE/SCAN reference points,
Lowdin orthonormality and the force chain rule."""
import math
import os

import numpy as np
import pytest
from scipy.special import erf

from oracle import oracle as O
from publicrelease_2020_b200 import workloads as W

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "analytic_pins.npz"))


def one_gaussian_system(alpha=0.8, centre=(0.3, -0.2, 0.1), nrad=60, l=0):
    s = W.System("one", np.array([centre]), np.zeros(1, dtype=np.int32), np.array([1], dtype=np.int32),
                 np.zeros((1, 25)), np.zeros((1, 3), dtype=np.int32), np.zeros((1, 3, 15, 25)), None, None, 2,
                 "LDA-PW91*LDA-PW91")
    s.bfalp[0, 0] = alpha
    s.n_con[0, l] = 1
    s.bfcon[0, l, 0, 0] = (2 * alpha / math.pi) ** 0.75 * (4 * alpha) ** (l / 2)
    s.rmsh, s.wmsh = W.atom_centred_mesh(s.rat, nrad=nrad, rscale=[1.0])
    nloc = s.nloc(0)
    s.psi = np.zeros((2, nloc))
    s.psi[:, 0] = 1.0
    s.nwfs = (1, 1)
    s.fods = [np.array([[centre[0] + 0.05, centre[1], centre[2]]]), np.array([[centre[0], centre[1] + 0.05, centre[2]]])]
    return s


@pytest.mark.parametrize("maxfmt", [3, 4, 5])
def test_boys_against_incomplete_gamma(maxfmt):
    xs, F = GOLD["boys_x"], GOLD["boys_F"]
    for x, ref in zip(xs, F):
        s = O.boys(maxfmt, x)
        for m in range(maxfmt):
            # table branch: Taylor error ~1e-12; x > 16: fffmtc.F keeps only the leading
            # term of the erfc tail of F_0, a ~3e-10 relative approximation
            tol = 1e-11 if x <= 16.0 else 1e-9
            assert abs(s[m] - ref[m]) <= tol * ref[m] + 1e-14, (maxfmt, x, m, s[m], ref[m])


@pytest.mark.parametrize("exact", [False, True])
def test_coulomb_of_s_gaussian_is_erf_over_r(exact):
    a = 0.8
    s = one_gaussian_system(a)
    o = O.Oracle(s)
    coul, rhog, st = o.coupot_sic(1, 1, exact=exact)
    r = np.linalg.norm(s.rmsh - s.rat[0], axis=1)
    ref = erf(np.sqrt(2 * a) * r) / r
    assert np.max(np.abs(coul - ref) / ref) < 1e-10
    rho_ref = (2 * a / math.pi) ** 1.5 * np.exp(-2 * a * r ** 2)
    assert np.max(np.abs(rhog[0] - rho_ref)) < 1e-12
    assert abs((rhog[0] * s.wmsh).sum() - 1.0) < 1e-8
    if not exact:
        assert st[4] > 0  # some points went through the multipole far field


def _multipole_potential(s, a, l, pts):
    """Potential of rho = (c x e^{-a r^2})^2 (l = 1) or (c x^2 e^{-a r^2})^2 (l = 2)
    by brute-force quadrature: the angular factor split into its degree-l'
    parts with the addition theorem on the 146-point Lebedev grid (exact to
    degree 19), the radial Green's-function integrals by adaptive quadrature."""
    from scipy import integrate
    from scipy.special import eval_legendre
    c = s.bfcon[0, l, 0, 0]
    d = pts - s.rat[0]
    r = np.linalg.norm(d, axis=1)
    u = d / r[:, None]
    ang, w = O.lebedev19()
    w = w * (4 * math.pi / w.sum())
    g_leb = (ang[:, 0] if l == 1 else ang[:, 0] ** 2) ** 2
    rk = np.round(r, 12)
    V = np.zeros(len(r))
    for lp in range(0, 2 * l + 1, 2):
        gl = (2 * lp + 1) / (4 * math.pi) * (eval_legendre(lp, u @ ang.T) * (w * g_leb)[None, :]).sum(1)
        R = {}
        for x in np.unique(rk):
            f_in = lambda t: c * c * t ** (2 * l + lp + 2) * np.exp(-2 * a * t * t)
            f_out = lambda t: c * c * t ** (2 * l + 1 - lp) * np.exp(-2 * a * t * t)
            i1 = integrate.quad(f_in, 0, x, epsabs=0, epsrel=1e-13, limit=200)[0]
            i2 = integrate.quad(f_out, x, np.inf, epsabs=0, epsrel=1e-13, limit=200)[0]
            R[x] = 4 * math.pi / (2 * lp + 1) * (x ** (-lp - 1) * i1 + x ** lp * i2)
        V += gl * np.array([R[x] for x in rk])
    return V


@pytest.mark.parametrize("l", [1, 2])
def test_coulomb_of_p_and_d_densities_vs_radial_quadrature(l):
    """COUPOT_SIC of one p_x (l=1) or d_xx (l=2) orbital: the pair-polynomial
    potential against an independent multipole/radial-quadrature evaluation."""
    a = 0.8
    s = one_gaussian_system(a, nrad=30, l=l)
    c0 = s.rat[0]
    s.fods = [np.array([c0 + [0.1, 0.05, 0.02]]), np.array([c0 + [0.07, -0.04, 0.03]])]
    o = O.Oracle(s)
    ref = _multipole_potential(s, a, l, s.rmsh)
    for exact in (False, True):
        coul, rhog, _ = o.coupot_sic(1, 1, exact=exact)
        assert np.max(np.abs(coul - ref) / np.abs(ref)) < 1e-9


def test_coupot1_and_densold_of_s_gaussian():
    """DENSOLD and COUPOT1 of one s orbital per spin: rho_s = psi^2 with its
    gradient, Hessian and PHIG = |grad psi|^2 in closed form; the Coulomb
    potential of both spins is 2 erf(sqrt(2a) r)/r."""
    a = 0.8
    s = one_gaussian_system(a)
    o = O.Oracle(s)
    d = s.rmsh - s.rat[0]
    r = np.linalg.norm(d, axis=1)
    v = o.coupot1()
    ref = 2 * erf(np.sqrt(2 * a) * r) / r
    assert np.max(np.abs(v - ref) / ref) < 1e-10
    rg, ph = o.densold(10)
    g = (2 * a / math.pi) ** 0.75 * np.exp(-a * r ** 2)
    rho = g * g
    for sp in (0, 1):
        assert np.abs(rg[sp, 0] - rho).max() < 1e-14
        assert np.abs(rg[sp, 1:4] - (-4 * a * d * rho[:, None]).T).max() < 1e-14
        assert np.abs(ph[sp] - (4 * a * a * (d ** 2).sum(1) * rho)).max() < 1e-14
        for ch, (i, j) in {4: (0, 0), 5: (1, 1), 6: (2, 2), 7: (0, 1), 8: (0, 2), 9: (1, 2)}.items():
            h = (16 * a * a * d[:, i] * d[:, j] - (4 * a if i == j else 0.0)) * rho
            assert np.abs(rg[sp, ch] - h).max() < 1e-13
    r1, _ = o.densold(1)
    assert np.array_equal(r1[:, 0], rg[:, 0])


@pytest.mark.parametrize("case", ["water", "synthetic_nspn1"])
def test_coupot1_is_sum_of_fo_potentials(case):
    """The FOs are an orthogonal rotation of the occupied orbitals, so the
    total density's potential (COUPOT1) is the sum of the FO potentials
    (COUPOT_SIC) up to the multipole truncation (EPSMULTI 1e-6), whose call
    set-up depends on the density; DENSOLD integrates to the electron count."""
    s = W.water(seed=0, nrad=14) if case == "water" else W.small_synthetic(seed=5, nspn=1)
    o = O.Oracle(s)
    v = o.coupot1()
    tot = sum(o.coupot_sic(sp, k + 1)[0] for sp in range(1, s.nspn + 1) for k in range(s.nfrm[sp - 1]))
    assert np.abs(v - tot).max() < 1e-6 * np.abs(v).max()
    rg, _ = o.densold(1)
    for sp in range(s.nspn):
        assert abs((rg[sp, 0] * s.wmsh).sum() - s.nwfs[sp]) < 1e-8


def test_lebedev_and_harmonics_orthonormal():
    ang, w = O.lebedev19()
    assert ang.shape == (146, 3)
    assert abs(w.sum() - 4 * math.pi) < 1e-12
    Y = np.array([O.harmonics(6, a) for a in ang])
    G = (Y * w[:, None]).T @ Y
    assert np.max(np.abs(G - np.eye(49))) < 1e-12


def test_multipole_far_field_close_to_exact():
    s = W.water(seed=0, nrad=24)
    o = O.Oracle(s)
    c0, r0, st0 = o.coupot_sic(1, 2, exact=False)
    c1, r1, st1 = o.coupot_sic(1, 2, exact=True)
    assert st0[4] > 0 and st1[4] == 0
    rel = np.abs(c0 - c1) / np.abs(c1)
    assert rel.max() < 5e-6            # EPSMULTI = 1e-6 design accuracy of poisson1.f
    assert abs(((c0 - c1) * r1[0] * s.wmsh).sum()) < 1e-9
    # asymptote r V -> analytic charge (coupot_sic.F:785-797): monopole-dominated
    # and identical in both modes (the mesh charge differs from the analytic one
    # because the synthetic orbitals are orthonormal in the mesh metric)
    r = np.linalg.norm(s.rmsh, axis=1)
    far = r > 0.8 * r.max()
    rv = c0[far] * r[far]
    assert np.allclose(rv, c1[far] * r[far], rtol=1e-9)
    assert rv.std() < 1e-2 * abs(rv.mean())


def test_pw92_polarised_correlation_matches_published_formula():
    # uniform fully polarised gas: ZET=1, LDA-PW91 correlation (PW92 fit, pw91lc.f)
    for rs, ecp in zip(GOLD["rs"], GOLD["ec_pol"]):
        rho = 3.0 / (4 * math.pi * rs ** 3)
        v, e = O.xc_point((0, 6, 0, 6), [rho] + [0.0] * 9, w=1.0)
        ec = e[2] / rho
        assert abs(ec - ecp) < 2e-4 * abs(ecp), (rs, ec, ecp)


def test_lda_exchange_polarised_closed_form():
    for rho in [1e-3, 0.05, 1.0, 30.0]:
        v, e = O.xc_point((0, 6, 0, 6), [rho] + [0.0] * 9, w=1.0)
        ex = -0.75 * (6.0 / math.pi) ** (1 / 3) * rho ** (4 / 3)
        assert abs(e[0] - ex) < 1e-8 * abs(ex)
        # exchange potential of the polarised gas: -(6 rho/pi)^(1/3)
        v_x, _ = O.xc_point((0, 6, 0, 0), [rho] + [0.0] * 9, w=1.0)
        assert abs(v_x[0] + (6 * rho / math.pi) ** (1 / 3)) < 1e-8 * (6 * rho / math.pi) ** (1 / 3)


def test_pbe_enhancement_factor():
    kf_rho = lambda rho: (3 * math.pi ** 2 * 2 * rho) ** (1 / 3)
    for s_val, fx in zip(GOLD["pbe_s"], GOLD["pbe_fx"]):
        rho = 0.3
        D = 2 * rho
        grad = s_val * 2 * kf_rho(rho) * D / 2.0   # |grad rho| so that s(2 rho) = s_val
        r10 = [rho, grad, 0, 0, 0, 0, 0, 0, 0, 0]
        v, e = O.xc_point((1, 7, 1, 7), r10, w=1.0)
        assert abs((e[0] + e[1]) / e[0] - fx) < 1e-10


@pytest.mark.parametrize("xc", [(0, 6, 0, 6), (1, 7, 1, 7), (1, 6, 1, 6)])
def test_lda_potential_is_energy_derivative(xc):
    # for a density without gradients the potential is d(rho e_xc)/d rho pointwise
    for rho in [0.01, 0.4, 5.0]:
        v, _ = O.xc_point(xc, [rho] + [0.0] * 9)
        h = 1e-6 * rho
        ep = sum(O.xc_point(xc, [rho + h] + [0.0] * 9)[1])
        em = sum(O.xc_point(xc, [rho - h] + [0.0] * 9)[1])
        assert abs(v[0] - (ep - em) / (2 * h)) < 1e-7 * max(1.0, abs(v[0]))


@pytest.mark.parametrize("functional", ["LDA-PW91*LDA-PW91", "MGGA-SCAN*MGGA-SCAN"])
def test_force_equals_chain_rule_of_lowdin_rotation(functional):
    """The FOD force of frmorb2.F equals the derivative of E_SIC through the
    Lowdin-orthonormalised rotation U = S^-1/2 T at fixed potentials (with the
    meta-GGA terms of the SIC matrix for SCAN)."""
    s = W.water(seed=0, nrad=20, functional=functional)
    o = O.Oracle(s)
    r = o.sic_cycle(nthreads=4)
    FM = o.fmat()
    for spin in (0, 1):
        n = s.nfrm[spin]
        T = FM[spin, 0, :n, :n]
        SIC = r["sic"][spin][:n, :n].T
        S = T @ T.T
        q, V = np.linalg.eigh(S)
        Sm = V @ np.diag(q ** -0.5) @ V.T
        U = Sm @ T
        f = -1.0 / (np.sqrt(q)[:, None] * np.sqrt(q)[None, :] * (np.sqrt(q)[:, None] + np.sqrt(q)[None, :]))
        grad = np.zeros((n, 3))
        for m in range(n):
            for d in range(3):
                dT = np.zeros_like(T)
                dT[m] = FM[spin, 1 + d, m, :n]
                dS = dT @ T.T + T @ dT.T
                dU = (V @ ((V.T @ dS @ V) * f) @ V.T) @ T + Sm @ dT
                grad[m, d] = 2 * np.sum((dU @ U.T) * SIC.T)
        assert np.allclose(r["debdax"][spin][:n], grad, atol=1e-9, rtol=1e-9)


@pytest.mark.parametrize("functional,atom,ix", [("LDA-PW91*LDA-PW91", 1, 2), ("MGGA-SCAN*MGGA-SCAN", 2, 0)])
def test_siclag_der_is_basis_centre_derivative(functional, atom, ix):
    """SICLAG_DER (siclag_der.F): 2 sum_k DERSIC(ix, k, A) is the derivative of
    E_SIC with respect to atom A's basis centre at fixed FO coefficients and a
    fixed mesh (for SCAN through the basis Hessian terms).  Central differences
    agree to the quadrature error of the analytic Coulomb potential on the mesh,
    about 1e-3 for the hydrogens of the 40-shell water mesh; the oxygen core
    functions need a far finer mesh, so they are not used here."""
    import copy
    s = W.water(seed=0, nrad=40, functional=functional)
    o = O.Oracle(s)
    D = o.siclag_der()
    assert D.shape == (s.natoms, sum(s.nfrm), 3)
    h = 1e-4
    cf = [o.fo_coefficients(sp) for sp in range(1, s.nspn + 1)]
    e = []
    for sg in (1.0, -1.0):
        s2 = copy.deepcopy(s)
        r = np.array(s2.rat, dtype=float).reshape(-1, 3)
        r[atom, ix] += sg * h
        s2.rat = r
        o2 = O.Oracle(s2)
        e.append(sum(o2.fo_energy(sp + 1, c)[8] for sp in range(s.nspn) for c in cf[sp]))
    fd = (e[0] - e[1]) / (2 * h)
    an = 2 * D[atom, :, ix].sum()
    assert abs(fd - an) < 3e-3 * abs(an), (fd, an)


@pytest.mark.parametrize("functional", ["LDA-PW91*LDA-PW91", "MGGA-SCAN*MGGA-SCAN"])
def test_sicham_projects_to_symmetrised_sic_matrix(functional):
    """SICHAM's projector form (sicham.F:922-944, APATCH in sicmat.F): the FOs
    are orthonormal on the mesh, so C_FO H C_FO^T is the symmetrised SICLAGM
    matrix (SIC + SIC^T)/2 of the same spin, to rounding."""
    s = W.water(seed=0, nrad=14, functional=functional)
    o = O.Oracle(s)
    r = o.sic_cycle(nthreads=4)
    for sp in (1, 2):
        H = o.sicham(sp)
        assert np.abs(H - H.T).max() == 0.0
        C = o.fo_coefficients(sp)
        n = s.nfrm[sp - 1]
        sic_m = r["sic"][sp - 1][:n, :n]
        assert np.abs(C @ H @ C.T - 0.5 * (sic_m + sic_m.T)).max() < 1e-12 * np.abs(sic_m).max()


def test_fo_orthonormal_and_lowden():
    s = W.water(seed=3, nrad=20)
    o = O.Oracle(s)
    tm, ev = o.frmiorb()
    for spin in (0, 1):
        n = s.nfrm[spin]
        T = tm[spin][:n, :n].T   # TMAT(k, jwf)
        assert np.allclose(T @ T.T, np.eye(n), atol=1e-12)
        assert np.all(ev[spin][:n] > 1e-8)


def test_bad_fods_raise_lowden_error():
    s = W.water(seed=0, nrad=16)
    f = [x.copy() for x in s.fods]
    f[0][1] = f[0][0]           # two coincident FODs: singular FO overlap
    o = O.Oracle(s)
    o.set_orbitals(s.psi, s.nwfs, f)
    with pytest.raises(O.OracleError, match="LOWDEN"):
        o.frmiorb()


def test_pair_plan_counts_small_synthetic():
    s = W.small_synthetic()
    o = O.Oracle(s)
    st = o.pair_stats(1, 1)
    assert st["pairs"] > 0 and st["batches"] > 0 and st["weird"] <= st["pairs"]


# ---------------------------------------------------------------------------
# SCAN meta-GGA (scan.f restated in the oracle).  Pins: the uniform-gas limit
# (exchange = LDA exchange, correlation = PW92 LSD), the one-electron limit
# (correlation vanishes for a fully polarised single-orbital density), the
# hydrogen-atom exchange energy SCAN is built to reproduce (-5/16 Ha), and
# every derivative the functional returns against central differences of its
# own energy density.
AX = -0.7385587663820224058842300326808360


def _pw92_lsd(rs, zeta):
    """PW92 correlation energy per particle (Perdew & Wang 1992, eq. 8-10)."""
    def g(a, a1, b1, b2, b3, b4):
        q1 = 2 * a * (b1 * rs ** 0.5 + b2 * rs + b3 * rs ** 1.5 + b4 * rs ** 2)
        return -2 * a * (1 + a1 * rs) * np.log(1 + 1 / q1)
    eu = g(0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294)
    ep = g(0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517)
    am = -g(0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671)
    f = ((1 + zeta) ** (4 / 3) + (1 - zeta) ** (4 / 3) - 2) / (2 ** (4 / 3) - 2)
    fzz = 8 / (9 * (2 ** (4 / 3) - 2))
    return eu + am * f / fzz * (1 - zeta ** 4) + (ep - eu) * f * zeta ** 4


@pytest.mark.parametrize("rho", [1e-3, 0.1, 10.0])
def test_scan_exchange_uniform_gas_is_lda(rho):
    pi = 3.1415927  # the literal of scan.f's exchange
    tau_unif = 0.3 * (3 * pi * pi) ** (2 / 3) * rho ** (5 / 3)
    ex = O.scan_x(rho, 1e-12, tau_unif)[0]
    assert abs(ex - AX * rho ** (1 / 3)) <= 1e-12 * abs(ex)


@pytest.mark.parametrize("rho,zeta", [(0.05, 0.0), (1.0, 0.0), (0.2, 0.6)])
def test_scan_correlation_uniform_gas_is_pw92(rho, zeta):
    ru, rd = rho * (1 + zeta) / 2, rho * (1 - zeta) / 2
    ds = ((1 + zeta) ** (5 / 3) + (1 - zeta) ** (5 / 3)) / 2
    tau0 = 0.3 * (3 * math.pi ** 2) ** (2 / 3) * rho ** (5 / 3) * ds
    g = 1e-9  # |grad rho| ~ 0: t -> 0, tau = tau_W + tau0 gives alpha = 1
    ec = O.scan_c(ru, rd, g / 2, g / 2, g, tau0 / 2 + g * g / (16 * rho), tau0 / 2 + g * g / (16 * rho))[0]
    rs = (3 / (4 * math.pi * rho)) ** (1 / 3)
    assert abs(ec - _pw92_lsd(rs, zeta)) <= 1e-9 * abs(ec)


def test_scan_correlation_vanishes_for_one_orbital():
    for ru, dru in ((0.3, 0.2), (2.0, 5.0), (1e-3, 1e-3)):
        tauw = dru * dru / (8 * ru)  # alpha = 0: tau = tau_W
        ec = O.scan_c(ru, 0.0, dru, 0.0, dru, tauw, 0.0)[0]
        assert abs(ec) < 1e-10 * abs(_pw92_lsd((3 / (4 * math.pi * ru)) ** (1 / 3), 1.0))


def test_scan_exchange_of_hydrogen_atom():
    r = np.linspace(1e-6, 40.0, 20001)
    rho = np.exp(-2 * r) / np.pi
    # spin scaling E_x[rho, 0] = E_x^unp[2 rho] / 2; tau = tau_W = rho / 2 per spin
    ex = np.array([O.scan_x(2 * q, 4 * q, q)[0] for q in rho])
    w = np.full_like(r, r[1] - r[0])
    w[0] *= 0.5
    w[-1] *= 0.5
    e = np.sum(rho * ex * 4 * np.pi * r * r * w)
    assert abs(e - (-5 / 16)) < 5e-6


@pytest.mark.parametrize("alpha", [0.0, 0.4, 1.7])
def test_scan_exchange_derivatives(alpha):
    rho, drho = 0.37, 0.29
    pi = 3.1415927
    tau = alpha * 0.3 * (3 * pi * pi) ** (2 / 3) * rho ** (5 / 3) + drho * drho / (8 * rho)
    _, vx, vxdd, amu = O.scan_x(rho, drho, tau)
    e = lambda a, b, c: a * O.scan_x(a, b, c)[0]
    h = 1e-6
    assert abs(vx - (e(rho + h, drho, tau) - e(rho - h, drho, tau)) / (2 * h)) < 1e-7
    assert abs(vxdd - (e(rho, drho + h, tau) - e(rho, drho - h, tau)) / (2 * h)) < 1e-7
    assert abs(amu - (e(rho, drho, tau + h) - e(rho, drho, tau - h)) / (2 * h)) < 1e-7


@pytest.mark.parametrize("alpha", [0.3, 1.6])
def test_scan_correlation_derivatives(alpha):
    """vc = d(rho ec)/d rho_s at fixed gradients and tau; vcdd = d/d|grad rho_s|
    along grad rho_s, with |grad rho| following; amu = d/d tau."""
    gu, gd = np.array([0.21, -0.05, 0.13]), np.array([0.02, 0.11, -0.04])

    def e(ru, rd, gu, gd, tauu, taud):
        dru, drd, drt = np.linalg.norm(gu), np.linalg.norm(gd), np.linalg.norm(gu + gd)
        return (ru + rd) * O.scan_c(ru, rd, dru, drd, drt, tauu, taud)[0]

    ru, rd = 0.31, 0.12
    rt, zeta = ru + rd, (ru - rd) / (ru + rd)
    ds = ((1 + zeta) ** (5 / 3) + (1 - zeta) ** (5 / 3)) / 2
    tau0 = 0.3 * (3 * math.pi ** 2) ** (2 / 3) * rt ** (5 / 3) * ds
    tt = alpha * tau0 + np.dot(gu + gd, gu + gd) / (8 * rt)
    tauu, taud = 0.6 * tt, 0.4 * tt
    out = O.scan_c(ru, rd, np.linalg.norm(gu), np.linalg.norm(gd), np.linalg.norm(gu + gd), tauu, taud)
    _, vcu, vcd, vddu, vddd, amu = out
    h = 1e-6
    assert abs(vcu - (e(ru + h, rd, gu, gd, tauu, taud) - e(ru - h, rd, gu, gd, tauu, taud)) / (2 * h)) < 1e-7
    assert abs(vcd - (e(ru, rd + h, gu, gd, tauu, taud) - e(ru, rd - h, gu, gd, tauu, taud)) / (2 * h)) < 1e-7
    nu, nd = gu / np.linalg.norm(gu), gd / np.linalg.norm(gd)
    assert abs(vddu - (e(ru, rd, gu + h * nu, gd, tauu, taud) - e(ru, rd, gu - h * nu, gd, tauu, taud)) / (2 * h)) < 1e-7
    assert abs(vddd - (e(ru, rd, gu, gd + h * nd, tauu, taud) - e(ru, rd, gu, gd - h * nd, tauu, taud)) / (2 * h)) < 1e-7
    assert abs(amu - (e(ru, rd, gu, gd, tauu + h, taud) - e(ru, rd, gu, gd, tauu - h, taud)) / (2 * h)) < 1e-7
