"""The DFT side on the GPU: DENSOLD (flosic_sic_densold) and COUPOT1
(flosic_sic_coupot1) against the oracle's restatements of densold.F and
coupot1.F, and against closed forms for one s orbital per spin."""
import math

import numpy as np
import pytest
from scipy.special import erf

from oracle import oracle as O
from publicrelease_2020_b200 import sic, workloads as W

from test_oracle_pins import one_gaussian_system

pytestmark = pytest.mark.gpu

CASES = {
    "water_lda": lambda: W.water(seed=0, nrad=14),
    "water_pbe": lambda: W.water(seed=0, nrad=14, functional="GGA-PBE*GGA-PBE"),
    "synthetic_pbe_nspn1": lambda: W.small_synthetic(seed=5, nspn=1),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_densold_and_coupot1(case):
    s = CASES[case]()
    o = O.Oracle(s)
    ctx = sic.open_system(s)
    try:
        for ngrad in (1, 10):
            rg, ph = ctx.densold(ngrad)
            rref, pref = o.densold(ngrad)
            assert np.abs(rg - rref).max() < 1e-12 * np.abs(rref).max()
            assert np.abs(ph - pref).max() <= 1e-12 * max(np.abs(pref).max(), 1.0)
        v = ctx.coupot1()
        vref = o.coupot1()
        assert np.abs(v - vref).max() < 1e-9 * np.abs(vref).max()
        ctx.set_precision("mixed")
        vm = ctx.coupot1()
        assert np.abs(vm - vref).max() < 1e-5 * np.abs(vref).max()
    finally:
        ctx.close()


def test_dft_side_closed_forms():
    a = 0.8
    s = one_gaussian_system(a)
    ctx = sic.open_system(s)
    try:
        v = ctx.coupot1()
        rg, ph = ctx.densold(10)
    finally:
        ctx.close()
    r = np.linalg.norm(s.rmsh - s.rat[0], axis=1)
    ref = 2 * erf(np.sqrt(2 * a) * r) / r
    assert np.max(np.abs(v - ref) / ref) < 1e-10
    rho = (2 * a / math.pi) ** 1.5 * np.exp(-2 * a * r ** 2)
    assert np.abs(rg[:, 0] - rho).max() < 1e-14
