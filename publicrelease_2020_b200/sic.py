"""Python binding of libflosic_sic_b200 (ctypes over the C ABI in
include/flosic_sic.h).

The methods keep the names and argument meaning of the reference routines
they replace (APOTNL_SIC, COUPOT_SIC, GETVLXC, SICLAGM, FRMORB2, FRMIORB,
GORBDRV in FLOSIC/PublicRelease_2020 flosic/), with numpy arrays in place of
the Fortran module state.  Errors from the library are raised as
``FlosicError`` carrying the library's status code, mirroring the reference's
STOPIT on the same conditions.  There is no CPU implementation behind this
class: without the CUDA library or a GPU it raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libflosic_sic_b200.so")

ERRORS = {
    1: "FLOSIC_ERR_ARG", 2: "FLOSIC_ERR_CAPACITY", 3: "FLOSIC_ERR_LOWDEN", 4: "FLOSIC_ERR_ZERO_DENSITY",
    5: "FLOSIC_ERR_NFRM", 6: "FLOSIC_ERR_ZERO_COULOMB", 7: "FLOSIC_ERR_CUDA", 8: "FLOSIC_ERR_STATE",
}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_vp = C.c_void_p

EXPORTS = [
    "flosic_sic_create", "flosic_sic_destroy", "flosic_sic_last_error", "flosic_sic_set_geometry",
    "flosic_sic_set_orbitals", "flosic_sic_gorbdrv", "flosic_sic_frmorb2_fmat", "flosic_sic_frmiorb",
    "flosic_sic_coupot_sic", "flosic_sic_getvlxc", "flosic_sic_apotnl_sic", "flosic_sic_siclagm",
    "flosic_sic_frmorb2_force", "flosic_sic_cycle", "flosic_sic_stats", "flosic_sic_getvlxc_device",
    "flosic_sic_set_precision", "flosic_sic_getvlxc_mgga", "flosic_sic_set_shard", "flosic_sic_partial_size",
    "flosic_sic_cycle_partial", "flosic_sic_cycle_combine", "flosic_sic_adjoint", "flosic_sic_mgga_mixin",
    "flosic_sic_siclag_der", "flosic_sic_sicham", "flosic_sic_densold", "flosic_sic_coupot1",
    "flosic_sic_autotune", "flosic_sic_adjoint_fod", "flosic_sic_set_wait_limit", "flosic_sic_batch_cycle",
    "flosic_sic_kernel_stats", "flosic_sic_set_density_mode",
]
PRECISION = {"fp64": 0, "mixed": 1}
DENSITY = {"phi2": 0, "pairs": 1}

_lib = None


class FlosicError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def load_library(path=LIB_PATH):
    """Load the CUDA library and declare the C ABI (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: run __graft_entry__.build() (no CPU fallback exists)")
    L = C.CDLL(path)
    L.flosic_sic_create.argtypes = [C.c_int, C.POINTER(_vp)]
    L.flosic_sic_destroy.argtypes = [_vp]
    L.flosic_sic_last_error.restype = C.c_char_p
    L.flosic_sic_set_geometry.argtypes = [_vp, C.c_int, _ip, _dp, C.c_int, _ip, _dp, _ip, _dp, C.c_int, _dp, _dp,
                                          C.c_int, _ip, _ip]
    L.flosic_sic_set_orbitals.argtypes = [_vp, _ip, _dp, C.c_int, _ip, _dp, C.c_int]
    L.flosic_sic_gorbdrv.argtypes = [_vp, C.c_int, _ip, _ip, C.c_int, _dp, C.c_int, _dp]
    L.flosic_sic_frmorb2_fmat.argtypes = [_vp, _dp, C.c_int]
    L.flosic_sic_frmiorb.argtypes = [_vp, _dp, _dp, C.c_int]
    L.flosic_sic_coupot_sic.argtypes = [_vp, C.c_int, C.c_int, _dp, _dp]
    L.flosic_sic_getvlxc.argtypes = [_vp, C.c_int, _dp, _dp, _dp]
    L.flosic_sic_getvlxc_mgga.argtypes = [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp]
    L.flosic_sic_set_precision.argtypes = [_vp, C.c_int]
    L.flosic_sic_set_wait_limit.argtypes = [_vp, C.c_int64]
    L.flosic_sic_set_density_mode.argtypes = [_vp, C.c_int]
    L.flosic_sic_kernel_stats.argtypes = [_vp, _dp, _i64]
    L.flosic_sic_batch_cycle.argtypes = [C.POINTER(_vp), C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp]
    L.flosic_sic_autotune.argtypes = [_vp, C.c_int, _ip, np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")]
    L.flosic_sic_getvlxc_device.argtypes = [_vp, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, _dp]
    L.flosic_sic_apotnl_sic.argtypes = [_vp, _dp, C.c_int, C.c_int, _dp, _dp, _dp]
    L.flosic_sic_siclagm.argtypes = [_vp, C.c_int, _dp, C.c_int]
    L.flosic_sic_frmorb2_force.argtypes = [_vp, C.c_int, _dp, C.c_int, _dp]
    L.flosic_sic_cycle.argtypes = [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp]
    L.flosic_sic_stats.argtypes = [_vp, _i64, _dp, _i64, _i64, _i64]
    L.flosic_sic_set_shard.argtypes = [_vp, C.c_int, C.c_int]
    L.flosic_sic_adjoint.argtypes = [_vp, C.c_int, _dp, C.c_int]
    L.flosic_sic_adjoint_fod.argtypes = [_vp, C.c_int, _dp, C.c_int]
    L.flosic_sic_mgga_mixin.argtypes = [_vp, C.c_int, C.c_int, _dp]
    L.flosic_sic_siclag_der.argtypes = [_vp, _dp, C.c_int]
    L.flosic_sic_sicham.argtypes = [_vp, C.c_int, _dp, C.c_int, C.c_int]
    L.flosic_sic_densold.argtypes = [_vp, C.c_int, _dp, C.c_void_p]
    L.flosic_sic_coupot1.argtypes = [_vp, _dp]
    L.flosic_sic_partial_size.argtypes = [_vp, _i64]
    L.flosic_sic_cycle_partial.argtypes = [_vp, C.c_void_p]
    L.flosic_sic_cycle_combine.argtypes = [_vp, C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp]
    _lib = L
    return L


class FlosicSIC:
    """One GPU context holding the SIC-path module state."""

    def __init__(self, device=0):
        self.L = load_library()
        h = _vp()
        self._check(self.L.flosic_sic_create(int(device), C.byref(h)))
        self.h = h
        self.sysm = None
        self.ld = 1

    def close(self):
        if getattr(self, "h", None):
            self.L.flosic_sic_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise FlosicError(rc, self.L.flosic_sic_last_error().decode())

    # -- module state ------------------------------------------------------
    def set_geometry(self, sysm):
        ix, idx, ic, idc = sysm.xc
        self.sysm = sysm
        self._check(self.L.flosic_sic_set_geometry(
            self.h, sysm.natoms, np.ascontiguousarray(sysm.atom_type + 1, dtype=np.int32),
            np.ascontiguousarray(sysm.rat, dtype=np.float64), sysm.ntypes,
            np.ascontiguousarray(sysm.n_bare, dtype=np.int32), np.ascontiguousarray(sysm.bfalp),
            np.ascontiguousarray(sysm.n_con, dtype=np.int32), np.ascontiguousarray(sysm.bfcon), sysm.nmsh,
            np.ascontiguousarray(sysm.rmsh), np.ascontiguousarray(sysm.wmsh), sysm.nspn,
            np.array([ix, ic], dtype=np.int32), np.array([idx, idc], dtype=np.int32)))

    def set_orbitals(self, psi, nwfs, fods):
        nf = np.array([len(f) for f in fods] + [0] * (2 - len(fods)), dtype=np.int32)
        self.ld = max(int(nf.max()), 1)
        bfrm = np.zeros((2, self.ld, 3))
        for s, f in enumerate(fods):
            bfrm[s, : len(f)] = f
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        self._check(self.L.flosic_sic_set_orbitals(self.h, np.array(list(nwfs) + [0] * (2 - len(nwfs)), dtype=np.int32),
                                                   psi, psi.shape[1], nf, bfrm, self.ld))
        self.nfrm = tuple(int(x) for x in nf)
        self._adjoint_fods = None  # FODs set through publicrelease_2020_b200.adjoint, if any

    # -- reference routines ------------------------------------------------
    def gorbdrv(self, nderv, pts, ifnct):
        """GORBDRV: pts (npts<=25, 3) relative to the atom of function set ifnct (1-based);
        returns GRAD(25,10,6,15,3) as a C array [3][15][6][10][25], IUPDAT, IALLCTR(15,3)."""
        P = np.zeros((3, 25))
        P[:, : len(pts)] = np.asarray(pts).T
        grad = np.zeros(25 * 10 * 6 * 15 * 3)
        iup = np.zeros(1, dtype=np.int32)
        iall = np.zeros(45, dtype=np.int32)
        self._check(self.L.flosic_sic_gorbdrv(self.h, nderv, iup, iall, len(pts), np.ascontiguousarray(P), ifnct, grad))
        return grad.reshape(3, 15, 6, 10, 25), bool(iup[0]), iall.reshape(3, 15)

    def frmorb2_fmat(self):
        out = np.zeros(2 * 4 * self.ld * self.ld)
        self._check(self.L.flosic_sic_frmorb2_fmat(self.h, out, self.ld))
        return out.reshape(2, 4, self.ld, self.ld)

    def frmiorb(self):
        tm = np.zeros(2 * self.ld * self.ld)
        ev = np.zeros(2 * self.ld)
        self._check(self.L.flosic_sic_frmiorb(self.h, tm, ev, self.ld))
        return tm.reshape(2, self.ld, self.ld), ev.reshape(2, self.ld)

    def coupot_sic(self, kxxs, kxxo):
        n = self.sysm.nmsh
        coul = np.zeros(n)
        rhog = np.zeros(10 * n)
        self._check(self.L.flosic_sic_coupot_sic(self.h, kxxs, kxxo, coul, rhog))
        return coul, rhog.reshape(10, n)

    def getvlxc(self, rhog):
        n = self.sysm.nmsh
        vxc = np.zeros(2 * n)
        ergs = np.zeros(4)
        self._check(self.L.flosic_sic_getvlxc(self.h, n, np.ascontiguousarray(rhog, dtype=np.float64).reshape(-1),
                                              vxc, ergs))
        return vxc.reshape(2, n), ergs

    def getvlxc_mgga(self, rhog, tau):
        """Meta-GGA GETVLXC: RHOG (10, n), TAU (n) -> VXC (2, n), MIXIN (2n, 4), ergs (4)."""
        n = self.sysm.nmsh
        vxc = np.zeros(2 * n)
        mix = np.zeros(8 * n)
        ergs = np.zeros(4)
        self._check(self.L.flosic_sic_getvlxc_mgga(self.h, n, np.ascontiguousarray(rhog, dtype=np.float64).reshape(-1),
                                                   np.ascontiguousarray(tau, dtype=np.float64), vxc, mix, ergs))
        return vxc.reshape(2, n), mix.reshape(2 * n, 4), ergs

    def set_precision(self, mode):
        """"fp64" (the drop-in, default) or "mixed"."""
        self._check(self.L.flosic_sic_set_precision(self.h, PRECISION[mode]))

    def set_density_mode(self, mode):
        """FO density route of the SIC exchange-correlation: "phi2" (default,
        rho = phi^2 from the FO values) or "pairs" (the reference's POISSON1
        route: Gaussian-pair polynomials at the points inside each call's RCUT
        sphere, coefficients below 1e-14 dropped)."""
        self._check(self.L.flosic_sic_set_density_mode(self.h, DENSITY[mode]))

    def set_wait_limit(self, polls):
        """Poll limit of the mixed-precision tensor-core kernel's pipeline waits
        (<= 0: the default)."""
        self._check(self.L.flosic_sic_set_wait_limit(self.h, int(polls)))

    def autotune(self, reps=2):
        """Time the per-FO Coulomb kernel's FO-slot widths (32, 64, 128) on this
        system and keep the fastest; returns (width, {width: ms}) with skipped
        widths left out."""
        fos = np.zeros(1, dtype=np.int32)
        ms = np.zeros(3, dtype=np.float32)
        self._check(self.L.flosic_sic_autotune(self.h, int(reps), fos, ms))
        return int(fos[0]), {32 << i: float(t) for i, t in enumerate(ms) if t >= 0}

    def getvlxc_device(self, npts, d_rhog, ldr, d_wmsh, d_vxc):
        """Allocation-free GETVLXC on device buffers given as raw device addresses
        (e.g. torch CUDA tensors' data_ptr()); returns ERGXL, ERGXN, ERGCL, ERGCN."""
        ergs = np.zeros(4)
        self._check(self.L.flosic_sic_getvlxc_device(self.h, int(npts), C.c_void_p(int(d_rhog)), int(ldr),
                                                     C.c_void_p(int(d_wmsh)), C.c_void_p(int(d_vxc)), ergs))
        return ergs

    def apotnl_sic(self, lspx, iorbx):
        n = self.sysm.nmsh
        totq = np.zeros(1)
        res = np.zeros(13)
        cf = np.zeros(3)
        pot = np.zeros(n)
        self._check(self.L.flosic_sic_apotnl_sic(self.h, totq, lspx, iorbx, res, cf, pot))
        return dict(totqnum=float(totq[0]), results=res, cfrm=cf, pot=pot)

    def siclagm(self, lspn):
        sic = np.zeros(self.ld * self.ld)
        self._check(self.L.flosic_sic_siclagm(self.h, lspn, sic, self.ld))
        return sic.reshape(self.ld, self.ld)

    def frmorb2_force(self, lspn, sic):
        deb = np.zeros(3 * self.ld)
        self._check(self.L.flosic_sic_frmorb2_force(self.h, lspn, np.ascontiguousarray(sic, dtype=np.float64).reshape(-1),
                                                    self.ld, deb))
        return deb.reshape(self.ld, 3)

    def cycle(self, out=None):
        ld = self.ld
        if out is None:
            out = dict(results=np.zeros(2 * ld * 13), sic=np.zeros(2 * ld * ld), debdax=np.zeros(2 * ld * 3),
                       cfrm=np.zeros(2 * ld * 3), esic=np.zeros(1))
        self._check(self.L.flosic_sic_cycle(self.h, ld, out["results"], out["sic"], out["debdax"], out["cfrm"],
                                            out["esic"]))
        return dict(results=out["results"].reshape(2, ld, 13), sic=out["sic"].reshape(2, ld, ld),
                    debdax=out["debdax"].reshape(2, ld, 3), cfrm=out["cfrm"].reshape(2, ld, 3),
                    esic=float(out["esic"][0]))

    def mgga_mixin(self, lspx, iorbx):
        """MIXIN(4, 2*nmsh) of one FO (the MGGA#### record) as an array (2*nmsh, 4)."""
        n = self.sysm.nmsh
        m = np.zeros(8 * n)
        self._check(self.L.flosic_sic_mgga_mixin(self.h, lspx, iorbx, m))
        return m.reshape(2 * n, 4)

    def adjoint(self, lspn):
        """G = dE_SIC/dC_FO (nbasis, nfrm) of spin lspn (flosic_sic_adjoint)."""
        nb = self.sysm.nbasis
        g = np.zeros(nb * self.nfrm[lspn - 1])
        self._check(self.L.flosic_sic_adjoint(self.h, lspn, g, nb))
        return g.reshape(self.nfrm[lspn - 1], nb).T

    def adjoint_fod(self, lspn):
        """dE_SIC/dFOD (nfrm, 3) of spin lspn from the adjoint, chain rule in the
        library (flosic_sic_adjoint_fod)."""
        n = self.nfrm[lspn - 1]
        g = np.zeros(3 * max(n, 1))
        self._check(self.L.flosic_sic_adjoint_fod(self.h, lspn, g, max(n, 1)))
        return g.reshape(-1, 3)[:n]

    def siclag_der(self):
        """DERSIC (natoms, nfrm(1)+nfrm(2), 3): the basis-centre SIC force terms
        (flosic_sic_siclag_der, SICLAG_DER in siclag_der.F)."""
        ldo = max(1, self.nfrm[0] + (self.nfrm[1] if self.sysm.nspn == 2 else 0))
        out = np.zeros(self.sysm.natoms * ldo * 3)
        self._check(self.L.flosic_sic_siclag_der(self.h, out, ldo))
        return out.reshape(self.sysm.natoms, ldo, 3)

    def sicham(self, lspn, ham=None, packed=False):
        """Add the basis-space SIC Hamiltonian of spin lspn to ham (flosic_sic_sicham,
        SICHAM's projector form); a new zero matrix (nbasis, nbasis), or the
        N(N+1)/2 HSTOR-ordered vector when packed, if ham is None."""
        nb = self.sysm.nbasis
        if ham is None:
            ham = np.zeros(nb * (nb + 1) // 2 if packed else (nb, nb))
        if ham.dtype != np.float64 or not ham.flags.c_contiguous:
            raise ValueError("ham must be a C-contiguous float64 array")
        self._check(self.L.flosic_sic_sicham(self.h, int(lspn), ham.reshape(-1), nb, int(bool(packed))))
        return ham

    def densold(self, ngrad=10):
        """DENSOLD: (rhog (nspn, ngrad, nmsh), phig (nspn, nmsh)) of the KS orbitals."""
        n, ns = self.sysm.nmsh, self.sysm.nspn
        rhog = np.zeros(ns * ngrad * n)
        phig = np.zeros(ns * n)
        self._check(self.L.flosic_sic_densold(self.h, int(ngrad), rhog, phig.ctypes.data_as(C.c_void_p)))
        return rhog.reshape(ns, ngrad, n), phig.reshape(ns, n)

    def coupot1(self):
        """COUPOT1: Coulomb potential (nmsh) of the KS orbitals' total density."""
        v = np.zeros(self.sysm.nmsh)
        self._check(self.L.flosic_sic_coupot1(self.h, v))
        return v

    def set_shard(self, shard, nshards):
        """Evaluate only mesh shard `shard` of `nshards` (flosic_sic_set_shard)."""
        self._check(self.L.flosic_sic_set_shard(self.h, int(shard), int(nshards)))

    def partial_size(self):
        n = np.zeros(1, dtype=np.int64)
        self._check(self.L.flosic_sic_partial_size(self.h, n))
        return int(n[0])

    def cycle_partial(self, d_partial):
        """This shard's packed partial sums into device memory at address d_partial."""
        self._check(self.L.flosic_sic_cycle_partial(self.h, C.c_void_p(int(d_partial))))

    def cycle_combine(self, d_partial):
        """The cycle's outputs from the summed partials at device address d_partial."""
        ld = self.ld
        out = dict(results=np.zeros(2 * ld * 13), sic=np.zeros(2 * ld * ld), debdax=np.zeros(2 * ld * 3),
                   cfrm=np.zeros(2 * ld * 3), esic=np.zeros(1))
        self._check(self.L.flosic_sic_cycle_combine(self.h, C.c_void_p(int(d_partial)), ld, out["results"],
                                                    out["sic"], out["debdax"], out["cfrm"], out["esic"]))
        return dict(results=out["results"].reshape(2, ld, 13), sic=out["sic"].reshape(2, ld, ld),
                    debdax=out["debdax"].reshape(2, ld, 3), cfrm=out["cfrm"].reshape(2, ld, 3),
                    esic=float(out["esic"][0]))

    def stats(self):
        la = np.zeros(1, dtype=np.int64)
        ms = np.zeros(7)
        npairs = np.zeros(1, dtype=np.int64)
        ncalls = np.zeros(1, dtype=np.int64)
        work = np.zeros(3, dtype=np.int64)
        self._check(self.L.flosic_sic_stats(self.h, la, ms, npairs, ncalls, work))
        return dict(launches=int(la[0]), stage_ms=ms, npairs=int(npairs[0]), ncalls=int(ncalls[0]),
                    near_evals=int(work[0]), far_evals=int(work[1]), far_terms=int(work[2]))

    def kernel_stats(self):
        """The last cycle's Coulomb evaluation by kernel: {'shared': (ms, near,
        far, terms), 'perfo': (ms, near, far, terms)} (flosic_sic_kernel_stats)."""
        ms = np.zeros(2)
        w = np.zeros(6, dtype=np.int64)
        self._check(self.L.flosic_sic_kernel_stats(self.h, ms, w))
        return {"shared": (float(ms[0]), int(w[0]), int(w[1]), int(w[2])),
                "perfo": (float(ms[1]), int(w[3]), int(w[4]), int(w[5]))}


def batch_cycle(ctxs, wm=0):
    """One SIC cycle of every context in ctxs (flosic_sic_batch_cycle: the
    Coulomb potentials of all molecules in two persistent launches); a list of
    outputs shaped as FlosicSIC.cycle's."""
    n = len(ctxs)
    L = load_library()
    ld = max(c.ld for c in ctxs)
    res, sic = np.zeros(n * 2 * ld * 13), np.zeros(n * 2 * ld * ld)
    deb, cfr, es = np.zeros(n * 2 * ld * 3), np.zeros(n * 2 * ld * 3), np.zeros(n)
    arr = (_vp * n)(*[c.h for c in ctxs])
    rc = L.flosic_sic_batch_cycle(arr, n, int(wm), ld, res, sic, deb, cfr, es)
    if rc != 0:
        raise FlosicError(rc, L.flosic_sic_last_error().decode())
    out = []
    for m in range(n):
        out.append(dict(results=res.reshape(n, 2, ld, 13)[m], sic=sic.reshape(n, 2, ld, ld)[m],
                        debdax=deb.reshape(n, 2, ld, 3)[m], cfrm=cfr.reshape(n, 2, ld, 3)[m], esic=float(es[m])))
    return out


def open_system(sysm, device=0, shard=None):
    """Context with geometry and orbitals of a workloads.System loaded;
    shard = (index, count) makes it evaluate one mesh shard."""
    ctx = FlosicSIC(device)
    if shard is not None:
        ctx.set_shard(*shard)
    ctx.set_geometry(sysm)
    ctx.set_orbitals(sysm.psi, sysm.nwfs, sysm.fods)
    return ctx
