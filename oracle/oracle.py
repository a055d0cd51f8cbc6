"""ctypes binding of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/liboracle_flosic.so, a restatement of the reference Fortran
routines (see flosic_oracle.cpp).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline legs may import this module; the product package
never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_flosic.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, _ip, _dp, C.c_int, _ip, _dp, _ip, _dp, C.c_int, _dp, _dp,
                                 C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_nbasis.argtypes = [C.c_void_p]
        L.orc_last_error.restype = C.c_char_p
        L.orc_set_orbitals.argtypes = [C.c_void_p, _ip, _dp, C.c_int, _ip, _dp, C.c_int]
        L.orc_gorbdrv.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _dp, _ip, _ip]
        L.orc_frmorb2_fmat.argtypes = [C.c_void_p, _dp, C.c_int]
        L.orc_frmiorb.argtypes = [C.c_void_p, _dp, _dp, C.c_int]
        L.orc_fo_coefficients.argtypes = [C.c_void_p, C.c_int, _dp]
        L.orc_coupot_sic.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp, _dp, _lp]
        L.orc_getvlxc_sic.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_apotnl_sic.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_siclagm.argtypes = [C.c_void_p, C.c_int, _dp, C.c_void_p, _dp, C.c_int]
        L.orc_getvlxc_mgga.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.orc_fo_tau.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        L.orc_set_xc_exact_density.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_count_scale.argtypes = [C.c_void_p, C.c_double]
        L.orc_siclag_der.argtypes = [C.c_void_p, _dp, C.c_int]
        L.orc_fo_energy.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.orc_sicham.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int]
        L.orc_coupot1.argtypes = [C.c_void_p, _dp]
        L.orc_densold.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.orc_partial_size.argtypes = [C.c_void_p, _lp]
        L.orc_cycle_partial.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.orc_cycle_combine.argtypes = [C.c_void_p, C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.orc_scan_x.argtypes = [C.c_double, C.c_double, C.c_double, _dp]
        L.orc_scan_x.restype = None
        L.orc_scan_c.argtypes = [C.c_double] * 7 + [_dp]
        L.orc_scan_c.restype = None
        L.orc_frmorb2_force.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int, _dp]
        L.orc_sic_cycle.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int]
        L.orc_pair_stats.argtypes = [C.c_void_p, C.c_int, C.c_int, _lp]
        L.orc_pair_dump.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_longlong, _lp, _dp, C.c_longlong,
                                    _lp]
        L.orc_xc_point.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _dp, C.c_double, _dp, _dp]
        L.orc_boys.argtypes = [C.c_int, C.c_double, _dp]
        L.orc_harmonics.argtypes = [C.c_int, _dp, _dp]
        L.orc_lebedev19.argtypes = [_dp, _dp]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _check(rc):
    if rc != 0:
        raise OracleError(f"oracle error {rc}: {lib().orc_last_error().decode()}")


class Oracle:
    """FP64 restatement of the reference SIC path for one System."""

    def __init__(self, sysm):
        L = lib()
        self.sysm = sysm
        ix, idx, ic, idc = sysm.xc
        self.h = L.orc_create(
            sysm.natoms, np.ascontiguousarray(sysm.atom_type, dtype=np.int32),
            np.ascontiguousarray(sysm.rat, dtype=np.float64), sysm.ntypes,
            np.ascontiguousarray(sysm.n_bare, dtype=np.int32), np.ascontiguousarray(sysm.bfalp),
            np.ascontiguousarray(sysm.n_con, dtype=np.int32), np.ascontiguousarray(sysm.bfcon),
            sysm.nmsh, np.ascontiguousarray(sysm.rmsh), np.ascontiguousarray(sysm.wmsh),
            sysm.nspn, ix, idx, ic, idc)
        if not self.h:
            raise OracleError(L.orc_last_error().decode())
        self.nbasis = L.orc_nbasis(self.h)
        self.ld = max(max(sysm.nfrm), 1)
        if sysm.psi is not None:
            self.set_orbitals(sysm.psi, sysm.nwfs, sysm.fods)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def set_orbitals(self, psi, nwfs, fods):
        nf = np.array([len(f) for f in fods] + [0] * (2 - len(fods)), dtype=np.int32)
        self.ld = max(int(nf.max()), 1)
        bfrm = np.zeros((2, self.ld, 3))
        for s, f in enumerate(fods):
            bfrm[s, : len(f)] = f
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        _check(lib().orc_set_orbitals(self.h, np.array(nwfs, dtype=np.int32), psi, psi.shape[1], nf,
                                      bfrm, self.ld))

    def gorbdrv(self, nderv, pts, ifnct):
        """pts (npts<=25, 3) relative to the atom; returns GRAD(25,10,6,15,3) as C array [3][15][6][10][25]."""
        P = np.zeros((3, 25))
        P[:, : len(pts)] = np.asarray(pts).T
        grad = np.zeros(25 * 10 * 6 * 15 * 3)
        iup = np.zeros(1, dtype=np.int32)
        iall = np.zeros(45, dtype=np.int32)
        _check(lib().orc_gorbdrv(self.h, nderv, len(pts), np.ascontiguousarray(P), ifnct, grad, iup, iall))
        return grad.reshape(3, 15, 6, 10, 25), bool(iup[0]), iall.reshape(3, 15)

    def fmat(self):
        out = np.zeros(2 * 4 * self.ld * self.ld)
        _check(lib().orc_frmorb2_fmat(self.h, out, self.ld))
        return out.reshape(2, 4, self.ld, self.ld)   # [s][K][jfm][jwf]

    def frmiorb(self):
        tm = np.zeros(2 * self.ld * self.ld)
        ev = np.zeros(2 * self.ld)
        _check(lib().orc_frmiorb(self.h, tm, ev, self.ld))
        return tm.reshape(2, self.ld, self.ld), ev.reshape(2, self.ld)  # tm[s][jwf][k] = TMAT(k,jwf,s)

    def fo_coefficients(self, spin):
        nf = self.sysm.nfrm[spin - 1]
        out = np.zeros(nf * self.nbasis)
        _check(lib().orc_fo_coefficients(self.h, spin, out))
        return out.reshape(nf, self.nbasis)

    def coupot_sic(self, spin, iorb, exact=False):
        n = self.sysm.nmsh
        coul = np.zeros(n)
        rhog = np.zeros(10 * n)
        st = np.zeros(9, dtype=np.int64)
        _check(lib().orc_coupot_sic(self.h, spin, iorb, int(exact), coul, rhog, st))
        return coul, rhog.reshape(10, n), st

    def getvlxc_sic(self, rhog):
        n = self.sysm.nmsh
        vxc = np.zeros(2 * n)
        ergs = np.zeros(4)
        _check(lib().orc_getvlxc_sic(self.h, np.ascontiguousarray(rhog, dtype=np.float64).reshape(-1), vxc, ergs))
        return vxc.reshape(2, n), ergs

    def apotnl_sic(self, spin, iorb):
        """One FO; for a meta-GGA also 'mixin' (nmsh, 4): MIXIN(1:4) of the spin-up half."""
        n = self.sysm.nmsh
        res = np.zeros(13)
        cf = np.zeros(3)
        pot = np.zeros(n)
        coul = np.zeros(n)
        rhog = np.zeros(10 * n)
        mix = np.zeros(4 * n)
        _check(lib().orc_apotnl_sic(self.h, spin, iorb, res, cf, pot, coul, rhog, mix))
        return dict(results=res, cfrm=cf, pot=pot, coulomb=coul, rhog=rhog.reshape(10, n),
                    mixin=mix.reshape(n, 4))

    def siclagm(self, spin, pots, mixins=None):
        """pots (nf, nmsh); mixins (nf, nmsh, 4) for a meta-GGA."""
        sic = np.zeros(self.ld * self.ld)
        zm = None if mixins is None else np.ascontiguousarray(mixins, dtype=np.float64)
        _check(lib().orc_siclagm(self.h, spin, np.ascontiguousarray(pots, dtype=np.float64),
                                 zm.ctypes.data_as(C.c_void_p) if zm is not None else None, sic, self.ld))
        return sic.reshape(self.ld, self.ld)   # [l][j] = SIC(j,l)

    def getvlxc_mgga(self, rhog, tau):
        """Meta-GGA GETVLXC: density channels (10, n), tau (n) -> vxc (2, n), mixin (n, 4), ergs (4)."""
        n = self.sysm.nmsh
        vxc = np.zeros(2 * n)
        mix = np.zeros(4 * n)
        ergs = np.zeros(4)
        _check(lib().orc_getvlxc_mgga(self.h, np.ascontiguousarray(rhog, dtype=np.float64).reshape(-1),
                                      np.ascontiguousarray(tau, dtype=np.float64), vxc, mix, ergs))
        return vxc.reshape(2, n), mix.reshape(n, 4), ergs

    def siclag_der(self):
        """DERSIC (natoms, nfrm(1)+nfrm(2), 3): SICLAG_DER's site derivatives."""
        ldo = max(1, self.sysm.nfrm[0] + (self.sysm.nfrm[1] if self.sysm.nspn == 2 else 0))
        out = np.zeros(self.sysm.natoms * ldo * 3)
        _check(lib().orc_siclag_der(self.h, out, ldo))
        return out.reshape(self.sysm.natoms, ldo, 3)

    def coupot1(self):
        """COUPOT1: Coulomb potential (nmsh) of the KS orbitals' total density."""
        v = np.zeros(self.sysm.nmsh)
        _check(lib().orc_coupot1(self.h, v))
        return v

    def densold(self, ngrad=10):
        """DENSOLD: (rhog (nspn, ngrad, nmsh), phig (nspn, nmsh))."""
        n, ns = self.sysm.nmsh, self.sysm.nspn
        r = np.zeros(ns * ngrad * n)
        ph = np.zeros(ns * n)
        _check(lib().orc_densold(self.h, ngrad, r, ph))
        return r.reshape(ns, ngrad, n), ph.reshape(ns, n)

    def sicham(self, spin):
        """SICHAM's basis-space SIC Hamiltonian (nbasis, nbasis) of one spin."""
        h = np.zeros((self.nbasis, self.nbasis))
        _check(lib().orc_sicham(self.h, spin, h.reshape(-1), self.nbasis))
        return h

    def fo_energy(self, spin, cfo):
        """APOTNL_SIC RESULTS(13) of the orbital with basis coefficients cfo."""
        res = np.zeros(13)
        _check(lib().orc_fo_energy(self.h, spin, np.ascontiguousarray(cfo, dtype=np.float64), res))
        return res

    def set_xc_exact_density(self, on):
        """XC on the untruncated pair density (the GPU's phi^2), Coulomb unchanged."""
        _check(lib().orc_set_xc_exact_density(self.h, int(bool(on))))

    def set_count_scale(self, scale):
        """Weight of each mesh point in POISSON1's near/far cost model: m when this
        mesh is every m-th point of a larger one (timing samples)."""
        _check(lib().orc_set_count_scale(self.h, float(scale)))

    def fo_tau(self, spin, iorb):
        """tau = |grad phi_k|^2 / 2 of one FO at the mesh points (GETTAU_PAR)."""
        tau = np.zeros(self.sysm.nmsh)
        _check(lib().orc_fo_tau(self.h, spin, iorb, tau))
        return tau

    def frmorb2_force(self, spin, sic):
        deb = np.zeros(3 * self.ld)
        _check(lib().orc_frmorb2_force(self.h, spin, np.ascontiguousarray(sic, dtype=np.float64).reshape(-1),
                                       self.ld, deb))
        return deb.reshape(self.ld, 3)

    def sic_cycle(self, nthreads=1, fo_limit=0):
        ld = self.ld
        res = np.zeros(2 * ld * 13)
        sic = np.zeros(2 * ld * ld)
        deb = np.zeros(2 * ld * 3)
        cfrm = np.zeros(2 * ld * 3)
        esic = np.zeros(1)
        _check(lib().orc_sic_cycle(self.h, ld, res, sic, deb, cfrm, esic, nthreads, fo_limit))
        return dict(results=res.reshape(2, ld, 13), sic=sic.reshape(2, ld, ld), debdax=deb.reshape(2, ld, 3),
                    cfrm=cfrm.reshape(2, ld, 3), esic=float(esic[0]))

    def pair_stats(self, spin=1, iorb=1):
        st = np.zeros(9, dtype=np.int64)
        _check(lib().orc_pair_stats(self.h, spin, iorb, st))
        return dict(pairs=int(st[0]), batches=int(st[1]), weird=int(st[2]), near=int(st[3]), far=int(st[4]),
                    near_multi=int(st[5]), far_multi=int(st[6]), npot1_multi=int(st[7]), calls_multi=int(st[8]))

    def pair_dump(self, spin=1, iorb=1, maxc=200000, maxp=400000):
        """POISSON1 calls of one FO: calls (n, 6) = CG(3), RCUT, NPOT, pairs;
        pairs (m, 51) = call index, -C(3), delta, COEFICIENT(1:46)."""
        calls = np.zeros(6 * maxc)
        pairs = np.zeros(51 * maxp)
        nc = np.zeros(1, dtype=np.int64)
        npr = np.zeros(1, dtype=np.int64)
        _check(lib().orc_pair_dump(self.h, spin, iorb, calls, maxc, nc, pairs, maxp, npr))
        return calls[:6 * nc[0]].reshape(-1, 6), pairs[:51 * npr[0]].reshape(-1, 51)


def xc_point(xc, r10, w=1.0):
    """(IGGA_x, IDFTYP_x, IGGA_c, IDFTYP_c), density channels -> (v_up, v_dn), (EXL, EXN, ECL, ECN)."""
    v = np.zeros(2)
    e = np.zeros(4)
    lib().orc_xc_point(xc[0], xc[1], xc[2], xc[3], np.ascontiguousarray(r10, dtype=np.float64), float(w), v, e)
    return v, e


def boys(maxfmt, x):
    s = np.zeros(5)
    lib().orc_boys(maxfmt, float(x), s)
    return s


def harmonics(lm, xyz):
    y = np.zeros((lm + 1) ** 2)
    lib().orc_harmonics(lm, np.ascontiguousarray(xyz, dtype=np.float64), y)
    return y


def lebedev19():
    a = np.zeros(146 * 3)
    w = np.zeros(146)
    lib().orc_lebedev19(a, w)
    return a.reshape(146, 3), w


def scan_x(rho, drho, tau):
    """SCAN exchange (VSCANxUNP): ex per particle, d(rho ex)/d rho, d/d|grad rho|, d/d tau."""
    out = np.zeros(4)
    lib().orc_scan_x(rho, drho, tau, out)
    return out


def scan_c(ru, rd, dru, drd, drt, tauu, taud):
    """SCAN correlation (VSCANc): ec, vc_up, vc_dn, vcdd_up, vcdd_dn, amu (d/d tau)."""
    out = np.zeros(7)
    lib().orc_scan_c(ru, rd, dru, drd, drt, tauu, taud, out)
    return out[:6]


class OracleShard:
    """The oracle as one shard of a mesh-sharded cycle: mesh points [b, e) of
    the system, the same partial/combine protocol (and packing) as the CUDA
    library's flosic_sic_cycle_partial / _combine, on host buffers."""

    def __init__(self, orc, b, e):
        self.orc, self.b, self.e = orc, int(b), int(e)

    def partial_size(self):
        n = np.zeros(1, dtype=np.int64)
        _check(lib().orc_partial_size(self.orc.h, n))
        return int(n[0])

    def cycle_partial(self, address):
        _check(lib().orc_cycle_partial(self.orc.h, self.b, self.e, C.c_void_p(int(address))))

    def cycle_combine(self, address):
        ld = self.orc.ld
        res = np.zeros(2 * ld * 13)
        sic = np.zeros(2 * ld * ld)
        deb = np.zeros(2 * ld * 3)
        cfrm = np.zeros(2 * ld * 3)
        esic = np.zeros(1)
        _check(lib().orc_cycle_combine(self.orc.h, C.c_void_p(int(address)), ld, res, sic, deb, cfrm, esic))
        return dict(results=res.reshape(2, ld, 13), sic=sic.reshape(2, ld, ld), debdax=deb.reshape(2, ld, 3),
                    cfrm=cfrm.reshape(2, ld, 3), esic=float(esic[0]))
