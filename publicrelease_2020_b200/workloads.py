"""Seeded synthetic inputs with the shapes of the FLO-SIC benchmark systems.

The reference ships no kernel-level inputs (no mesh, no converged KS
orbitals), so every system here is generated from a seed:

* ``water``      -- O at the origin, H at (+-0.757, 0, 0.587) A, an
  even-tempered basis with the NRLMOL default shapes (O: 13 bare primitives,
  5s4p3d; H: 6 bare primitives, 4s3p1d; 73 functions) or, with
  basis="default", the reference's default NRLMOL basis itself
  (nrlmol_default_type), an atom-centred radial x Lebedev mesh standing in
  for the variational mesh (vmesh.F), 5+5 FODs at a 1s + tetrahedral guess
  perturbed by N(0, 0.05 bohr).
* ``synthetic``  -- N atoms uniform in a cube (min separation 1.8 bohr),
  contracted Cartesian s/p/d functions with 3 primitives each (exponents
  log-uniform in [0.05, 1e4]), jittered uniform mesh with weights summing to
  the box volume, N_o FODs near the atoms.

KS orbitals are random coefficient vectors orthonormalised in the mesh
overlap metric S = B^T W B.  All arrays use the reference's Fortran layouts
(BFALP(MAX_BARE,ntypes), BFCON(MAX_BARE,MAX_CON,3,ntypes), RMSH(3,nmsh),
PSI(nbasis,nwf), BFRM(3,ld,2)); see modules2.F90:133-331 and modules.f90:206.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

MAX_BARE = 25
MAX_CON = 15
BOHR_PER_ANG = 1.0 / 0.529177210903

# Cartesian components in the order of gorbdrv.f (s; x y z; xx yy zz xy xz yz)
_POWS = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (0, 2, 0), (0, 0, 2),
         (1, 1, 0), (1, 0, 1), (0, 1, 1)]
_NCOMP = (1, 3, 6)
_SHIFT = (0, 1, 4)

# functional codes: (IGGA_x, IDFTYP_x, IGGA_c, IDFTYP_c) as set by setdftyp.F
FUNCTIONALS = {
    "LDA-PW91*LDA-PW91": (0, 6, 0, 6),
    "GGA-PBE*GGA-PBE": (1, 7, 1, 7),
    "GGA-PW91*GGA-PW91": (1, 6, 1, 6),
    "MGGA-SCAN*MGGA-SCAN": (3, 11, 3, 11),
}


@dataclasses.dataclass
class System:
    name: str
    rat: np.ndarray          # (natoms, 3)   bohr, atoms grouped by type
    atom_type: np.ndarray    # (natoms,)     0-based type index
    n_bare: np.ndarray       # (ntypes,)
    bfalp: np.ndarray        # (ntypes, MAX_BARE)              == BFALP(MAX_BARE, ntypes)
    n_con: np.ndarray        # (ntypes, 3)                     == N_CON(3, ntypes)
    bfcon: np.ndarray        # (ntypes, 3, MAX_CON, MAX_BARE)  == BFCON(MAX_BARE, MAX_CON, 3, ntypes)
    rmsh: np.ndarray         # (nmsh, 3)
    wmsh: np.ndarray         # (nmsh,)
    nspn: int
    functional: str
    psi: np.ndarray | None = None     # (nwf, nbasis) == PSI(nbasis, nwf)
    nwfs: tuple = (0, 0)
    fods: list = dataclasses.field(default_factory=list)  # per spin (nfrm, 3)

    @property
    def natoms(self):
        return int(self.rat.shape[0])

    @property
    def ntypes(self):
        return int(self.n_bare.shape[0])

    @property
    def nmsh(self):
        return int(self.rmsh.shape[0])

    def nloc(self, t):
        return int(sum(_NCOMP[l] * self.n_con[t, l] for l in range(3)))

    @property
    def nbasis(self):
        return int(sum(self.nloc(t) for t in self.atom_type))

    @property
    def xc(self):
        return FUNCTIONALS[self.functional]

    @property
    def nfrm(self):
        return tuple(len(f) for f in self.fods) + (0,) * (2 - len(self.fods))

    def bfrm(self, ld=None):
        """FOD positions as BFRM(3, ld, 2) (C order: [2][ld][3])."""
        ld = ld or max(self.nfrm)
        out = np.zeros((2, ld, 3))
        for s, f in enumerate(self.fods):
            out[s, : len(f)] = f
        return out


# ---------------------------------------------------------------------------
# basis evaluation in numpy (input preparation only: overlap metric)
# ---------------------------------------------------------------------------
def basis_values(sysm: System, pts: np.ndarray) -> np.ndarray:
    """Values of all contracted functions at pts, (npts, nbasis), local order
    (l, component, contraction) per atom as in unravel2.f."""
    cols = []
    for a in range(sysm.natoms):
        t = int(sysm.atom_type[a])
        d = pts - sysm.rat[a]
        r2 = np.einsum("ij,ij->i", d, d)
        nb = int(sysm.n_bare[t])
        alp = sysm.bfalp[t, :nb]
        g = np.exp(-np.minimum(np.outer(r2, alp), 700.0))
        g[np.outer(r2, alp) >= 40.0] = 0.0
        for l in range(3):
            nc = int(sysm.n_con[t, l])
            if nc == 0:
                continue
            rad = g @ sysm.bfcon[t, l, :nc, :nb].T      # (npts, nc)
            for mu in range(_NCOMP[l]):
                px, py, pz = _POWS[_SHIFT[l] + mu]
                ang = d[:, 0] ** px * d[:, 1] ** py * d[:, 2] ** pz
                cols.append(rad * ang[:, None])
    return np.concatenate(cols, axis=1)


def mesh_overlap(sysm: System, chunk=100000) -> np.ndarray:
    nb = sysm.nbasis
    S = np.zeros((nb, nb))
    for i0 in range(0, sysm.nmsh, chunk):
        B = basis_values(sysm, sysm.rmsh[i0:i0 + chunk])
        S += (B * sysm.wmsh[i0:i0 + chunk, None]).T @ B
    return S


def orthonormal_orbitals(sysm: System, nwf: int, rng) -> np.ndarray:
    """nwf random orbitals orthonormal in S = B^T W B; returns (nwf, nbasis)."""
    S = mesh_overlap(sysm)
    nb = S.shape[0]
    C = rng.standard_normal((nb, nwf))
    M = C.T @ S @ C
    w, U = np.linalg.eigh(M)
    C = C @ (U / np.sqrt(w)) @ U.T
    return np.ascontiguousarray(C.T)


# ---------------------------------------------------------------------------
# basis sets
# ---------------------------------------------------------------------------
def _even_tempered(nprim, amin, amax):
    return np.geomspace(amax, amin, nprim)


def _primitive_norm(alpha, l):
    # normalisation of x^l exp(-a r^2) (axis component)
    return (2 * alpha / math.pi) ** 0.75 * (4 * alpha) ** (l / 2) / math.sqrt(
        float(np.prod([2 * k - 1 for k in range(1, l + 1)]) if l > 0 else 1.0)
    )


def _nrlmol_like_type(nprim, ncon, amin, amax, rng):
    """General-contraction type: ncon[l] contractions over a shared set of
    nprim bare primitives (the NRLMOL layout, PDF pp.14-16)."""
    alp = _even_tempered(nprim, amin, amax)
    con = np.zeros((3, MAX_CON, MAX_BARE))
    for l in range(3):
        for c in range(ncon[l]):
            if c < ncon[l] - 1:
                # contracted: coefficients over the tighter primitives
                w = np.exp(-0.5 * ((np.arange(nprim) - (c * nprim) / max(ncon[l], 1)) / 2.0) ** 2)
                w[nprim - ncon[l] + c + 1:] = 0.0
            else:
                # most diffuse function: a single primitive with coefficient 1 (times norm)
                w = np.zeros(nprim)
                w[nprim - 1 - (l > 0)] = 1.0
            for i in range(nprim):
                con[l, c, i] = w[i] * _primitive_norm(alp[i], l)
    return alp, con


_NRLMOL_TABLES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "nrlmol_default_basis.npz")


def nrlmol_default_type(z):
    """The reference's default all-electron basis for element z (H, C or O).

    The tables are the NRLMOL bare exponents and full contractions that
    flosic/bdallbas.f stores, kept in data/nrlmol_default_basis.npz.  To them
    SALLBAS adds, per l, single-primitive functions with coefficient 1
    (sallbas.f:86-104, 133-153): three on the most diffuse primitives for s
    and p, and three on the next-to-most-diffuse ones for d.  An atom without
    p contractions (H) moves its p singles one primitive tighter and gets one
    d single on the third most diffuse primitive.  The supplementary set
    NBASF(2, l) is left out, as READINP does unless EXTRABASIS asks for it
    (readinp.F:137-186).  The exponents are already in the descending order
    READINP sorts them into.  Returns (alpha, con[l, c, i], n_con)."""
    tab = np.load(_NRLMOL_TABLES)
    nspd, alph, coef = tab[f"nspd_{z}"], tab[f"alph_{z}"], tab[f"coef_{z}"]
    nalp = len(alph)
    if not np.all(np.diff(alph) < 0):
        raise ValueError("NRLMOL exponents must be in descending order")
    nadd, ibofs = [3, 3, 3], [0, 0, 1]
    if nspd[1] == 0:
        ibofs[1], nadd[2], ibofs[2] = 1, 1, 2
    con = np.zeros((3, MAX_CON, MAX_BARE))
    for l in range(3):
        con[l, : nspd[l], :nalp] = coef[l, : nspd[l]]
        for i in range(1, nadd[l] + 1):
            con[l, nspd[l] + i - 1, nalp - ibofs[l] - nadd[l] + i - 1] = 1.0
    return np.array(alph), con, tuple(int(nspd[l] + nadd[l]) for l in range(3))


def _pack_types(types):
    nt = len(types)
    n_bare = np.array([len(t[0]) for t in types], dtype=np.int32)
    bfalp = np.zeros((nt, MAX_BARE))
    bfcon = np.zeros((nt, 3, MAX_CON, MAX_BARE))
    n_con = np.zeros((nt, 3), dtype=np.int32)
    for i, (alp, con, ncon) in enumerate(types):
        bfalp[i, : len(alp)] = alp
        bfcon[i] = con
        n_con[i] = ncon
    return n_bare, bfalp, n_con, bfcon


# ---------------------------------------------------------------------------
# meshes
# ---------------------------------------------------------------------------
def lebedev146():
    """Degree-19 Lebedev mesh (146 points, weights summing to 4 pi): published
    Lebedev parameters as tabulated in lebedev.F:165-190."""
    A1, A2, A3 = 0.00753519001311713812, 0.09265184700375432421, 0.09061000833610514010
    B = (0.09518264418191036893, 0.08487112439121475736, 0.08942676055004592969)
    AL = (0.15746766720390817632, 0.41749612279654533594, 0.67644104001142636987)
    AM = (0.97488864367717323548, 0.80708981835958250163, 0.29129888220952674629)
    D1, AR, AU, AW = 0.08785259467896816188, 0.14035538117131832857, 0.44933283232695573488, 0.88227001126032263192
    pts, w = [], []
    for i in range(3):
        for s in (1, -1):
            p = [0.0, 0.0, 0.0]
            p[i] = s
            pts.append(p)
            w.append(A1)
    r2 = 1 / math.sqrt(2)
    for i in range(3):
        for s1 in (1, -1):
            for s2 in (1, -1):
                p = [0.0, 0.0, 0.0]
                p[(i + 1) % 3] = s1 * r2
                p[(i + 2) % 3] = s2 * r2
                pts.append(p)
                w.append(A2)
    r3 = 1 / math.sqrt(3)
    for s1 in (1, -1):
        for s2 in (1, -1):
            for s3 in (1, -1):
                pts.append([s1 * r3, s2 * r3, s3 * r3])
                w.append(A3)
    for g in range(3):
        for i in range(3):
            for s0 in (1, -1):
                for s1 in (1, -1):
                    for s2 in (1, -1):
                        p = [0.0, 0.0, 0.0]
                        p[i] = s0 * AM[g]
                        p[(i + 1) % 3] = s1 * AL[g]
                        p[(i + 2) % 3] = s2 * AL[g]
                        pts.append(p)
                        w.append(B[g])
    import itertools
    for perm in itertools.permutations((AR, AU, AW)):
        for s in itertools.product((1, -1), repeat=3):
            pts.append([s[0] * perm[0], s[1] * perm[1], s[2] * perm[2]])
            w.append(D1)
    return np.array(pts), np.array(w)


def atom_centred_mesh(rat, nrad=40, rscale=None, seed=0):
    """Becke-partitioned radial x Lebedev-146 mesh around each atom (stand-in
    for the variational mesh of vmesh.F, which needs the Fortran build)."""
    ang, wang = lebedev146()
    rng = np.random.default_rng(seed)
    pts, wts = [], []
    nat = len(rat)
    rscale = rscale or [1.0] * nat
    for a in range(nat):
        # Gauss-Chebyshev (second kind) radial grid mapped to (0, inf)
        i = np.arange(1, nrad + 1)
        x = np.cos(i * math.pi / (nrad + 1))
        w_x = math.pi / (nrad + 1) * np.sin(i * math.pi / (nrad + 1)) ** 2 / np.sqrt(1 - x ** 2)
        r = rscale[a] * (1 + x) / (1 - x)
        dr = rscale[a] * 2 / (1 - x) ** 2
        wr = w_x * dr * r ** 2
        # random rotation of the angular grid per atom
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        angr = ang @ q
        p = (r[:, None, None] * angr[None, :, :]).reshape(-1, 3) + rat[a]
        w = (wr[:, None] * wang[None, :]).reshape(-1)
        # Becke fuzzy-cell weights
        if nat > 1:
            dist = np.linalg.norm(p[:, None, :] - rat[None, :, :], axis=2)
            Rab = np.linalg.norm(rat[:, None] - rat[None, :], axis=2)
            cell = np.ones((len(p), nat))
            # cell[:, A] = prod over B != A (ascending) of s(mu_AB), all A at once
            with np.errstate(divide="ignore", invalid="ignore"):
                for B in range(nat):
                    mu = (dist - dist[:, B:B + 1]) / Rab[:, B]
                    f = mu
                    for _ in range(3):
                        f = 1.5 * f - 0.5 * (f * f * f)
                    sB = 0.5 * (1 - f)
                    sB[:, B] = 1.0
                    cell *= sB
            w = w * cell[:, a] / cell.sum(axis=1)
        keep = w > 1e-14
        pts.append(p[keep])
        wts.append(w[keep])
    return np.concatenate(pts), np.concatenate(wts)


# ---------------------------------------------------------------------------
# systems
# ---------------------------------------------------------------------------
def water(seed=0, nrad=40, functional="LDA-PW91*LDA-PW91", basis="nrlmol-like"):
    """C1: water, 5+5 FODs, NSPN=2; LDA-PW91*LDA-PW91 unless another functional
    is named.  basis="default" is the reference's default NRLMOL basis
    (nrlmol_default_type: O 5s4p3d, H 4s3p1d, 73 functions); "nrlmol-like"
    has the same shape with even-tempered exponents."""
    rng = np.random.default_rng(seed)
    b = BOHR_PER_ANG
    rat = np.array([[0.0, 0.0, 0.0], [0.757 * b, 0.0, 0.587 * b], [-0.757 * b, 0.0, 0.587 * b]])
    if basis == "default":
        types = [nrlmol_default_type(8), nrlmol_default_type(1)]
    else:
        types = []
        alp, con = _nrlmol_like_type(13, (5, 4, 3), 0.12, 6.0e4, rng)
        types.append((alp, con, (5, 4, 3)))
        alp, con = _nrlmol_like_type(6, (4, 3, 1), 0.08, 80.0, rng)
        types.append((alp, con, (4, 3, 1)))
    n_bare, bfalp, n_con, bfcon = _pack_types(types)
    rmsh, wmsh = atom_centred_mesh(rat, nrad=nrad, rscale=[0.7, 0.5, 0.5], seed=seed + 1)
    sysm = System("water", rat, np.array([0, 1, 1], dtype=np.int32), n_bare, bfalp, n_con, bfcon,
                  rmsh, wmsh, 2, functional)
    nocc = 5
    C = orthonormal_orbitals(sysm, 2 * nocc, rng)
    sysm.psi = np.ascontiguousarray(np.concatenate([C[:nocc], C[nocc:]], axis=0))
    sysm.nwfs = (nocc, nocc)
    # FOD guess: 1s at O, two O-H bond points, two lone pairs (tetrahedral)
    oh1 = 0.6 * rat[1]
    oh2 = 0.6 * rat[2]
    lp1 = np.array([0.0, 0.55, -0.45])
    lp2 = np.array([0.0, -0.55, -0.45])
    base = np.array([[0.0, 0.0, 0.0], oh1, oh2, lp1, lp2])
    sysm.fods = [base + rng.normal(0, 0.05, base.shape), base + rng.normal(0, 0.05, base.shape)]
    return sysm


def synthetic(natoms=40, nbasis=512, nmsh=1_000_000, nfo=128, box_ang=12.0, seed=1,
              functional="GGA-PBE*GGA-PBE", nspn=1, min_sep=1.8):
    """C2-shaped synthetic system (one spin channel of nfo FOs by default)."""
    rng = np.random.default_rng(seed)
    L = box_ang * BOHR_PER_ANG
    rat = []
    while len(rat) < natoms:
        p = rng.uniform(0.1 * L, 0.9 * L, 3)
        if all(np.linalg.norm(p - q) >= min_sep for q in rat):
            rat.append(p)
    rat = np.array(rat)
    # distribute nbasis functions over atoms: each atom gets s/p/d contractions
    # (s:1 fn, p:3 fns, d:6 fns), 3 primitives per contraction (general contraction:
    # contraction c of every l uses primitives 3c..3c+2 of the atom)
    ncon = np.zeros((natoms, 3), dtype=np.int32)
    ncon[:, 0] = 1
    total = natoms
    order = rng.permutation(natoms)
    k = 0
    while total < nbasis:
        a = order[k % natoms]
        rem = nbasis - total
        choice = rng.choice([0, 1, 2], p=[0.3, 0.45, 0.25])
        size = (1, 3, 6)[choice]
        if size > rem:
            choice, size = 0, 1
        if ncon[a, choice] < 4:
            ncon[a, choice] += 1
            total += size
        k += 1
    types = []
    for a in range(natoms):
        nc = ncon[a]
        nprim = 3 * int(nc.max())
        alp = np.sort(np.exp(rng.uniform(math.log(0.05), math.log(1.0e4), nprim)))[::-1]
        con = np.zeros((3, MAX_CON, MAX_BARE))
        for l in range(3):
            for c in range(nc[l]):
                for j in range(3):
                    i = 3 * c + j
                    con[l, c, i] = rng.uniform(0.3, 1.0) * _primitive_norm(alp[i], l)
        types.append((alp, con, tuple(int(x) for x in nc)))
    n_bare, bfalp, n_con, bfcon = _pack_types(types)
    # jittered uniform mesh, weights summing to the box volume
    n1 = int(round(nmsh ** (1 / 3)))
    while n1 ** 3 < nmsh:
        n1 += 1
    h = L / n1
    idx = np.stack(np.meshgrid(*[np.arange(n1)] * 3, indexing="ij"), -1).reshape(-1, 3)[:nmsh]
    rmsh = (idx + 0.5 + rng.uniform(-0.35, 0.35, idx.shape)) * h
    wmsh = rng.uniform(0.5, 1.5, nmsh)
    wmsh *= L ** 3 / wmsh.sum()
    sysm = System("synthetic", rat, np.arange(natoms, dtype=np.int32), n_bare, bfalp, n_con, bfcon,
                  rmsh, wmsh, nspn, functional)
    nb = sysm.nbasis
    assert nb == nbasis, (nb, nbasis)
    C = orthonormal_orbitals(sysm, nfo * nspn, rng)
    sysm.psi = C
    sysm.nwfs = (nfo, nfo if nspn == 2 else 0)
    sysm.fods = [place_fods(sysm, C[s * nfo:(s + 1) * nfo], rng) for s in range(nspn)]
    return sysm


def place_fods(sysm, C, rng, min_eig=1e-3, tries=200):
    """FODs near the atoms, redrawn one at a time until the Fermi-orbital
    overlap T T^T (frmiorb.f:426-438) is safely non-singular."""
    nfo = C.shape[0]
    at = rng.integers(0, sysm.natoms, nfo)
    fods = sysm.rat[at] + rng.normal(0, 0.6, (nfo, 3))

    def lowden_min(f):
        psi = basis_values(sysm, f) @ C.T            # (nfod, nwf)
        rho = np.einsum("ij,ij->i", psi, psi)
        T = psi / np.sqrt(rho)[:, None]
        return np.linalg.eigvalsh(T @ T.T)

    for _ in range(tries):
        ev = lowden_min(fods)
        if ev.min() > min_eig:
            break
        # move the FOD with the largest weight in the softest eigenvector
        psi = basis_values(sysm, fods) @ C.T
        rho = np.einsum("ij,ij->i", psi, psi)
        T = psi / np.sqrt(rho)[:, None]
        w, V = np.linalg.eigh(T @ T.T)
        k = int(np.argmax(np.abs(V[:, 0])))
        fods[k] = sysm.rat[rng.integers(0, sysm.natoms)] + rng.normal(0, 0.6, 3)
    return fods


def small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=6000, nfo=4, functional="GGA-PBE*GGA-PBE", nspn=1):
    """Seconds-sized synthetic system for parity tests."""
    return synthetic(natoms=natoms, nbasis=nbasis, nmsh=nmsh, nfo=nfo, box_ang=4.0, seed=seed,
                     functional=functional, nspn=nspn, min_sep=1.8)


def _fods_conditioned(sysm, fods, rng, sigma=0.05, min_eig=1e-4, tries=50):
    """Perturb structured FOD guesses by N(0, sigma) until the Fermi-orbital
    overlap T T^T (frmiorb.f:426-438) of every spin is safely non-singular."""
    out = []
    for s, base in enumerate(fods):
        C = sysm.psi[s * sysm.nwfs[0]: s * sysm.nwfs[0] + sysm.nwfs[s]]
        f = base + rng.normal(0, sigma, base.shape)
        for _ in range(tries):
            psi = basis_values(sysm, f) @ C.T
            rho = np.einsum("ij,ij->i", psi, psi)
            T = psi / np.sqrt(rho)[:, None]
            if np.linalg.eigvalsh(T @ T.T).min() > min_eig:
                break
            f = base + rng.normal(0, sigma, base.shape)
        out.append(f)
    return out


def benzene(seed=3, nrad=40, functional="LDA-PW91*LDA-PW91", basis="nrlmol-like"):
    """C3: benzene, planar D6h (C-C 1.39 A, C-H 1.09 A), C 5s4p3d = 35
    functions, H 4s3p1d = 19 (324 in all), 21+21 FODs at core, C-H and C-C
    bond and pi positions, perturbed by N(0, 0.05 bohr); NSPN=2.
    basis="default" is the reference's default NRLMOL basis
    (nrlmol_default_type); "nrlmol-like" has the same shape with
    even-tempered exponents."""
    rng = np.random.default_rng(seed)
    b = BOHR_PER_ANG
    ang = np.arange(6) * np.pi / 3
    ring = np.stack([np.cos(ang), np.sin(ang), np.zeros(6)], axis=1)
    rc, rh = 1.39 * b, (1.39 + 1.09) * b
    rat = np.concatenate([rc * ring, rh * ring])
    if basis == "default":
        types = [nrlmol_default_type(6), nrlmol_default_type(1)]
    else:
        types = []
        alp, con = _nrlmol_like_type(14, (5, 4, 3), 0.08, 2.2e4, rng)
        types.append((alp, con, (5, 4, 3)))
        alp, con = _nrlmol_like_type(6, (4, 3, 1), 0.08, 80.0, rng)
        types.append((alp, con, (4, 3, 1)))
    n_bare, bfalp, n_con, bfcon = _pack_types(types)
    rmsh, wmsh = atom_centred_mesh(rat, nrad=nrad, rscale=[0.7] * 6 + [0.5] * 6, seed=seed + 1)
    sysm = System("benzene", rat, np.array([0] * 6 + [1] * 6, dtype=np.int32), n_bare, bfalp, n_con, bfcon,
                  rmsh, wmsh, 2, functional)
    nocc = 21
    C = orthonormal_orbitals(sysm, 2 * nocc, rng)
    sysm.psi = np.ascontiguousarray(np.concatenate([C[:nocc], C[nocc:]], axis=0))
    sysm.nwfs = (nocc, nocc)
    cc = 0.5 * (rat[:6] + np.roll(rat[:6], -1, axis=0))        # C-C bond midpoints
    ch = rat[:6] + 0.5 * (rat[6:] - rat[:6])                    # C-H bond points
    z = np.array([0.0, 0.0, 0.9])
    up = np.concatenate([rat[:6], ch, cc, cc[0::2] + z])        # pi FODs above the plane
    dn = np.concatenate([rat[:6], ch, cc, cc[1::2] - z])        # and below, on the other bonds
    sysm.fods = _fods_conditioned(sysm, [up, dn], rng)
    return sysm


def _truncated_icosahedron():
    """The 60 vertices (edge length 2) of the truncated icosahedron: even
    permutations of (0, +-1, +-3p), (+-1, +-(2+p), +-2p), (+-p, +-2, +-(2p+1)),
    p the golden ratio."""
    p = (1 + 5 ** 0.5) / 2
    base = [(0.0, 1.0, 3 * p), (1.0, 2 + p, 2 * p), (p, 2.0, 2 * p + 1)]
    pts = set()
    for x, y, z in base:
        for sx in (1, -1):
            for sy in (1, -1):
                for sz in (1, -1):
                    v = (sx * x, sy * y, sz * z)
                    for k in range(3):  # cyclic (even) permutations
                        pts.add(tuple(round(c, 12) for c in (v[k], v[(k + 1) % 3], v[(k + 2) % 3])))
    return np.array(sorted(pts))


def c60(seed=4, nrad=40, functional="MGGA-SCAN*MGGA-SCAN", rscale=0.7):
    """C5: C60 (truncated icosahedron, radius 3.55 A), carbon 3s2p1d basis (15
    functions, 900 in all), 180+180 FODs: 60 cores, one per single (5-6) bond,
    two per double (6-6) bond, perturbed by N(0, 0.05 bohr); SCAN; NSPN=2.
    nrad sets the radial shells of the atom-centred mesh (60 x nrad x 146
    points before the cut-off)."""
    rng = np.random.default_rng(seed)
    v = _truncated_icosahedron()
    rat = v / np.linalg.norm(v[0]) * 3.55 * BOHR_PER_ANG
    d = np.linalg.norm(rat[:, None] - rat[None], axis=2)
    bond = d[0][d[0] > 1e-6].min()
    edges = [(i, j) for i in range(60) for j in range(i + 1, 60) if abs(d[i, j] - bond) < 0.05 * bond]
    # 6-6 (double) bonds: edges whose two atoms share no pentagon, found as the
    # edges not on any 5-cycle
    nb = {i: [j for j in range(60) if j != i and abs(d[i, j] - bond) < 0.05 * bond] for i in range(60)}
    pent = set()
    for i in range(60):
        for j in nb[i]:
            for k in nb[j]:
                if k == i:
                    continue
                for l in nb[k]:
                    if l in (i, j):
                        continue
                    for m in nb[l]:
                        if m in (i, j, k) or i not in nb[m]:
                            continue
                        for e in ((i, j), (j, k), (k, l), (l, m), (m, i)):
                            pent.add(tuple(sorted(e)))
    single = [e for e in edges if e in pent]
    double = [e for e in edges if e not in pent]
    assert len(edges) == 90 and len(single) == 60 and len(double) == 30
    types = []
    alp, con = _nrlmol_like_type(9, (3, 2, 1), 0.1, 5.0e3, rng)
    types.append((alp, con, (3, 2, 1)))
    n_bare, bfalp, n_con, bfcon = _pack_types(types)
    rmsh, wmsh = atom_centred_mesh(rat, nrad=nrad, rscale=[rscale] * 60, seed=seed + 1)
    sysm = System("c60", rat, np.zeros(60, dtype=np.int32), n_bare, bfalp, n_con, bfcon, rmsh, wmsh, 2,
                  functional)
    nocc = 180
    C = orthonormal_orbitals(sysm, 2 * nocc, rng)
    sysm.psi = np.ascontiguousarray(np.concatenate([C[:nocc], C[nocc:]], axis=0))
    sysm.nwfs = (nocc, nocc)
    mid_s = np.array([0.5 * (rat[i] + rat[j]) for i, j in single])
    out = []
    for sgn in (1.0, -1.0):
        dbl = []
        for i, j in double:
            m = 0.5 * (rat[i] + rat[j])
            rad = m / np.linalg.norm(m)
            tan = np.cross(rat[j] - rat[i], rad)
            tan /= np.linalg.norm(tan)
            dbl += [m + 0.6 * rad * sgn, m + 0.6 * tan * sgn]
        out.append(np.concatenate([rat, mid_s, np.array(dbl)]))
    sysm.fods = _fods_conditioned(sysm, out, rng)
    return sysm


def alkane(ncarbon, ring=False, seed=0, nrad=12, functional="LDA-PW91*LDA-PW91"):
    """An alkane chain C_nH_(2n+2) or cycloalkane ring C_nH_2n (n >= 3) of
    tetrahedral carbons (C-C 1.54 A, C-H 1.09 A), carbon 3s2p1d (15 functions)
    and hydrogen 2s1p (5 functions) bases, an atom-centred mesh of nrad
    radial shells per atom, random orthonormal occupied orbitals and FODs near
    the atoms; NSPN=2, one FO per occupied orbital of each spin."""
    rng = np.random.default_rng(seed)
    b = BOHR_PER_ANG
    cc, chd = 1.54 * b, 1.09 * b
    tet = np.deg2rad(109.47)
    if ring:
        if ncarbon < 3:
            raise ValueError("a ring needs at least three carbons")
        rad = cc / (2 * np.sin(np.pi / ncarbon))
        ang = 2 * np.pi * np.arange(ncarbon) / ncarbon
        carb = np.stack([rad * np.cos(ang), rad * np.sin(ang), 0.3 * b * (-1) ** np.arange(ncarbon)], axis=1)
    else:
        carb = np.zeros((ncarbon, 3))
        for i in range(1, ncarbon):  # planar zigzag
            carb[i] = carb[i - 1] + cc * np.array([np.sin(tet / 2), (-1) ** i * np.cos(tet / 2), 0.0])
    hyd = []
    for i in range(ncarbon):
        nbr = [j for j in range(ncarbon) if j != i and np.linalg.norm(carb[j] - carb[i]) < 1.1 * cc]
        nh = 4 - len(nbr)
        axis = -sum((carb[j] - carb[i]) for j in nbr) if nbr else np.array([0.0, 0.0, 1.0])
        axis = axis / np.linalg.norm(axis) if np.linalg.norm(axis) > 1e-9 else np.array([0.0, 0.0, 1.0])
        perp = np.cross(axis, [0.0, 0.0, 1.0] if abs(axis[2]) < 0.9 else [1.0, 0.0, 0.0])
        perp /= np.linalg.norm(perp)
        for h in range(nh):
            phi = 2 * np.pi * h / max(nh, 1) + rng.uniform(0, 0.2)
            rot = np.cos(phi) * perp + np.sin(phi) * np.cross(axis, perp)
            d = axis * np.cos(np.pi - tet) + rot * np.sin(np.pi - tet) if nh > 1 else axis
            hyd.append(carb[i] + chd * d / np.linalg.norm(d))
    rat = np.concatenate([carb, np.array(hyd)]) if hyd else carb
    types = []
    alp, con = _nrlmol_like_type(9, (3, 2, 1), 0.1, 5.0e3, rng)
    types.append((alp, con, (3, 2, 1)))
    alp, con = _nrlmol_like_type(5, (2, 1, 0), 0.08, 50.0, rng)
    types.append((alp, con, (2, 1, 0)))
    n_bare, bfalp, n_con, bfcon = _pack_types(types)
    atype = np.array([0] * ncarbon + [1] * len(hyd), dtype=np.int32)
    rmsh, wmsh = atom_centred_mesh(rat, nrad=nrad, rscale=[0.7] * ncarbon + [0.5] * len(hyd), seed=seed + 1)
    name = f"c{ncarbon}h{len(hyd)}" + ("-ring" if ring else "")
    sysm = System(name, rat, atype, n_bare, bfalp, n_con, bfcon, rmsh, wmsh, 2, functional)
    nocc = (6 * ncarbon + len(hyd)) // 2
    C = orthonormal_orbitals(sysm, 2 * nocc, rng)
    sysm.psi = np.ascontiguousarray(np.concatenate([C[:nocc], C[nocc:]], axis=0))
    sysm.nwfs = (nocc, nocc)
    sysm.fods = [place_fods(sysm, C[:nocc], rng), place_fods(sysm, C[nocc:], rng)]
    return sysm


def alkane_batch(n=64, seed=100, max_carbons=9, nrad=(8, 40)):
    """C4: n molecules of uneven size from consecutive seeds -- chains and
    rings of 1..max_carbons carbons (2..29 atoms), meshes of nrad[0]..nrad[1]
    radial shells per atom."""
    out = []
    for i in range(n):
        rng = np.random.default_rng(seed + i)
        ring = bool(rng.integers(0, 2)) and max_carbons >= 3
        nc = int(rng.integers(3 if ring else 1, max_carbons + 1))
        out.append(alkane(nc, ring=ring, seed=seed + i, nrad=int(rng.integers(nrad[0], nrad[1] + 1))))
    return out
