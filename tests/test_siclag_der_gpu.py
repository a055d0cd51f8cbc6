"""SICLAG_DER on the GPU (flosic_sic_siclag_der) against the oracle's
restatement of siclag_der.F: the basis-centre SIC force terms DERSIC(3, lfn,
atom) over both spins, LDA/GGA and SCAN, NSPN 1 and 2."""
import numpy as np
import pytest

from oracle import oracle as O
from publicrelease_2020_b200 import sic, workloads as W

pytestmark = pytest.mark.gpu


def _dersic_pair(sysm, precision="fp64"):
    ctx = sic.open_system(sysm)
    try:
        ctx.set_precision(precision)
        d = ctx.siclag_der()
    finally:
        ctx.close()
    return d, O.Oracle(sysm).siclag_der()


@pytest.mark.parametrize("functional", ["LDA-PW91*LDA-PW91", "GGA-PBE*GGA-PBE", "MGGA-SCAN*MGGA-SCAN"])
def test_siclag_der_water(functional):
    s = W.water(seed=0, nrad=14, functional=functional)
    d, ref = _dersic_pair(s)
    assert d.shape == ref.shape == (s.natoms, sum(s.nfrm), 3)
    scale = np.abs(ref).max()
    assert np.abs(d - ref).max() < 1e-8 * scale, np.abs(d - ref).max() / scale


def test_siclag_der_closed_shell_doubles():
    """NSPN=1: one spin of FOs and DERSIC doubled (siclag_der.F:153-161)."""
    s = W.small_synthetic(seed=5, nspn=1)
    d, ref = _dersic_pair(s)
    assert d.shape == ref.shape == (s.natoms, s.nfrm[0], 3)
    assert np.abs(d - ref).max() < 1e-8 * np.abs(ref).max()


def test_siclag_der_mixed_precision():
    """The mixed Coulomb path feeds the same potentials into DERSIC within the
    precision mode's potential error."""
    s = W.water(seed=0, nrad=14)
    d, ref = _dersic_pair(s, "mixed")
    assert np.abs(d - ref).max() < 1e-5 * np.abs(ref).max()


def test_siclag_der_refuses_short_ldo():
    s = W.water(seed=0, nrad=14)
    ctx = sic.open_system(s)
    try:
        out = np.zeros(s.natoms * 3 * 3)
        with pytest.raises(sic.FlosicError):
            ctx._check(ctx.L.flosic_sic_siclag_der(ctx.h, out, 3))
    finally:
        ctx.close()
