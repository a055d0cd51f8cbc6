"""Edge cases of the SIC block through the C ABI, against the FP64 oracle
where there is a result: unequal FO counts per spin, a spin without FOs, a
mesh smaller than one 128-point tile, and the refusals of sizes beyond the
reference's static capacities (PARAMA2: MAX_BARE=25, MAX_CON=15) and of bad
shapes, which the library reports as status codes."""
import numpy as np
import pytest

from oracle import oracle as O
from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _drop_orbitals(sysm, keep):
    """The same system with only keep[s] orbitals and FODs in spin s."""
    n0 = sysm.nwfs[0]
    rows = list(range(keep[0])) + [n0 + i for i in range(keep[1])]
    sysm.psi = np.ascontiguousarray(sysm.psi[rows])
    sysm.nwfs = tuple(keep)
    sysm.fods = [sysm.fods[0][: keep[0]], sysm.fods[1][: keep[1]]]
    return sysm


def _compare(sysm, g, r, e_tol=1e-8):
    assert abs(g["esic"] - r["esic"]) < 1e-9
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        if n == 0:
            continue
        assert np.max(np.abs(g["results"][s][:n, 1:] - r["results"][s][:n, 1:])) < e_tol
        lam = r["sic"][s][:n, :n]
        assert np.max(np.abs(g["sic"][s][:n, :n] - lam)) < 1e-9 * np.abs(lam).max()
        assert np.max(np.abs(g["debdax"][s][:n] - r["debdax"][s][:n])) < 1e-8 * max(1.0, np.abs(r["debdax"][s][:n]).max())


@pytest.mark.parametrize("keep", [(5, 4), (3, 1)])
def test_unequal_fo_counts_per_spin(keep):
    sysm = _drop_orbitals(W.water(seed=0, nrad=14), keep)
    ctx = S.open_system(sysm)
    try:
        _compare(sysm, ctx.cycle(), O.Oracle(sysm).sic_cycle(nthreads=8))
    finally:
        ctx.close()


def test_spin_without_fos():
    sysm = _drop_orbitals(W.water(seed=0, nrad=14), (2, 0))
    ctx = S.open_system(sysm)
    try:
        g = ctx.cycle()
        r = O.Oracle(sysm).sic_cycle(nthreads=8)
        _compare(sysm, g, r)
        assert np.all(g["results"][1] == 0.0) and np.all(g["debdax"][1] == 0.0)
    finally:
        ctx.close()


def test_mesh_smaller_than_one_tile():
    sysm = W.water(seed=0, nrad=14)
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(sysm.nmsh, 77, replace=False))
    sysm.rmsh = np.ascontiguousarray(sysm.rmsh[idx])
    sysm.wmsh = np.ascontiguousarray(sysm.wmsh[idx] * 50.0)
    ctx = S.open_system(sysm)
    try:
        _compare(sysm, ctx.cycle(), O.Oracle(sysm).sic_cycle(nthreads=8))
    finally:
        ctx.close()


def test_capacity_and_shape_refusals():
    sysm = W.water(seed=0, nrad=10)
    ctx = S.FlosicSIC(0)
    try:
        bad = W.water(seed=0, nrad=10)
        bad.n_bare = bad.n_bare.copy()
        bad.n_bare[0] = 26                        # > MAX_BARE
        with pytest.raises(S.FlosicError) as e:
            ctx.set_geometry(bad)
        assert e.value.code == 2
        bad = W.water(seed=0, nrad=10)
        bad.n_con = bad.n_con.copy()
        bad.n_con[0, 0] = 16                      # > MAX_CON
        with pytest.raises(S.FlosicError) as e:
            ctx.set_geometry(bad)
        assert e.value.code == 2
        bad = W.water(seed=0, nrad=10)
        bad.nspn = 3
        with pytest.raises(S.FlosicError) as e:
            ctx.set_geometry(bad)
        assert e.value.code == 1
        with pytest.raises(S.FlosicError) as e:       # no geometry yet
            ctx.cycle()
        assert e.value.code == 8
        ctx.set_geometry(sysm)
        with pytest.raises(S.FlosicError) as e:       # no orbitals yet
            ctx.cycle()
        assert e.value.code == 8
    finally:
        ctx.close()
