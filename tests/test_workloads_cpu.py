"""CPU checks of the seeded stand-in inputs (publicrelease_2020_b200/workloads):
the atom-centred Becke mesh integrates what a molecular mesh must, and
every generator is reproducible from its seed.  The GPU and the oracle always consume the same arrays, so
these checks are about the inputs being physically sensible, not parity."""
import numpy as np
import pytest

from publicrelease_2020_b200 import workloads as W


def _gaussians(r, centres, alpha):
    """Sum of normalised s-Gaussians exp(-alpha |r - c|^2) (alpha / pi)^1.5."""
    d2 = ((r[:, None, :] - centres[None, :, :]) ** 2).sum(-1)
    return (np.exp(-alpha * d2) * (alpha / np.pi) ** 1.5).sum(1)


@pytest.mark.parametrize("alpha", [0.5, 2.0, 20.0])
def test_becke_mesh_integrates_atom_centred_gaussians(alpha):
    s = W.water(seed=0, nrad=40)
    r, w = np.asarray(s.rmsh).reshape(-1, 3), np.asarray(s.wmsh)
    rat = np.asarray(s.rat).reshape(-1, 3)
    assert np.all(w > 0)
    got = np.sum(w * _gaussians(r, rat, alpha))
    assert got == pytest.approx(len(rat), rel=2e-5)


def test_becke_mesh_integrates_off_centre_gaussian():
    s = W.benzene(nrad=24)
    r, w = np.asarray(s.rmsh).reshape(-1, 3), np.asarray(s.wmsh)
    rat = np.asarray(s.rat).reshape(-1, 3)
    mid = 0.5 * (rat[0] + rat[1])[None, :]   # a bond midpoint
    assert np.sum(w * _gaussians(r, mid, 1.0)) == pytest.approx(1.0, rel=1e-3)


def test_cell_weights_partition_unity():
    """A mesh of two atoms integrates a wide density centred between them,
    which both atoms' cells share: the cell weights of every point add to one."""
    rat = np.array([[0.0, 0.0, 0.0], [1.4, 0.0, 0.0]])
    r, w = W.atom_centred_mesh(rat, nrad=60)
    assert np.sum(w * _gaussians(r, rat.mean(0)[None, :], 0.1)) == pytest.approx(1.0, rel=1e-4)


@pytest.mark.parametrize("make", [lambda: W.water(seed=0, nrad=12),
                                  lambda: W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=3000, nfo=4),
                                  lambda: W.benzene(nrad=8)])
def test_generators_are_reproducible(make):
    a, b = make(), make()
    for key in ("rmsh", "wmsh", "psi"):
        assert np.array_equal(np.asarray(getattr(a, key)), np.asarray(getattr(b, key))), key
    for s in range(a.nspn):
        assert np.array_equal(np.asarray(a.fods[s]), np.asarray(b.fods[s]))


def test_nrlmol_default_basis_shapes():
    """SALLBAS's default basis: O and C 5s4p3d, H 4s3p1d, singles with
    coefficient 1 on the primitives sallbas.f picks."""
    for z, nbare, ncon in ((8, 13, (5, 4, 3)), (6, 12, (5, 4, 3)), (1, 6, (4, 3, 1))):
        alp, con, n = W.nrlmol_default_type(z)
        assert len(alp) == nbare and n == ncon and np.all(np.diff(alp) < 0)
        nspd = (1, 0, 0) if z == 1 else (2, 1, 0)
        singles = {8: ([10, 11, 12], [10, 11, 12], [9, 10, 11]), 6: ([9, 10, 11], [9, 10, 11], [8, 9, 10]),
                   1: ([3, 4, 5], [2, 3, 4], [3])}[z]
        for l in range(3):
            for i, prim in enumerate(singles[l]):
                row = con[l, nspd[l] + i]
                assert row[prim] == 1.0 and np.count_nonzero(row) == 1, (z, l, i)
            assert np.count_nonzero(con[l, n[l]:]) == 0
    w = W.water(seed=0, nrad=8, basis="default")
    b = W.benzene(nrad=6, basis="default")
    assert w.nbasis == 73 and b.nbasis == 324


def test_default_basis_water_sic_cycle_is_physical():
    """With the reference's default basis the oracle's FO charges integrate
    to one on the stand-in mesh and the per-FO SIC energies are a few mHa to
    tens of mHa, as for a real molecule."""
    from oracle import oracle as O
    s = W.water(seed=0, nrad=16, basis="default")
    r = O.Oracle(s).sic_cycle(nthreads=4)
    for sp in range(2):
        res = r["results"][sp][:5]
        assert np.allclose(res[:, 1], 1.0, atol=0.03)          # XCH1
        assert np.all((res[:, 8] > 0.0) & (res[:, 8] < 0.1))   # per-FO SIC energy
    assert 0.05 < r["esic"] < 0.5
