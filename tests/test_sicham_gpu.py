"""SICHAM's basis-space SIC Hamiltonian on the GPU (flosic_sic_sicham) against
the oracle's restatement of sicham.F / APATCH: full and HSTOR-packed layouts,
accumulation into the caller's matrix, LDA/GGA/SCAN, NSPN 1 and 2."""
import numpy as np
import pytest

from oracle import oracle as O
from publicrelease_2020_b200 import sic, workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("functional", ["LDA-PW91*LDA-PW91", "GGA-PBE*GGA-PBE", "MGGA-SCAN*MGGA-SCAN"])
def test_sicham_water(functional):
    s = W.water(seed=0, nrad=14, functional=functional)
    o = O.Oracle(s)
    ctx = sic.open_system(s)
    try:
        for sp in (1, 2):
            ref = o.sicham(sp)
            h = ctx.sicham(sp)
            assert np.abs(h - ref).max() < 1e-9 * np.abs(ref).max()
            # packed HSTOR order, added on top of what the caller holds
            nb = s.nbasis
            base = np.arange(nb * (nb + 1) // 2, dtype=np.float64)
            hp = ctx.sicham(sp, ham=base.copy(), packed=True)
            iu = np.triu_indices(nb)
            assert np.abs(hp - base - ref[iu]).max() < 1e-9 * np.abs(ref).max()
    finally:
        ctx.close()


def test_sicham_closed_shell():
    s = W.small_synthetic(seed=5, nspn=1)
    ref = O.Oracle(s).sicham(1)
    ctx = sic.open_system(s)
    try:
        h = ctx.sicham(1)
        with pytest.raises(sic.FlosicError):
            ctx.sicham(2)
    finally:
        ctx.close()
    assert np.abs(h - ref).max() < 1e-9 * np.abs(ref).max()
