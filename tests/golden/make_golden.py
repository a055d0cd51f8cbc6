"""Generates tests/golden/analytic_pins.npz: independent closed-form values
used to pin the oracle (the reference ships no kernel-level golden vectors
and cannot be built here).  Only scipy/numpy special functions and the
published formulas are used -- no code of this repository.

    python tests/golden/make_golden.py
"""
import os

import numpy as np
from scipy.special import gamma, gammainc

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "analytic_pins.npz")


def boys(m, x):
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    small = x < 1e-8
    out[small] = 1.0 / (2 * m + 1)
    xs = x[~small]
    out[~small] = gamma(m + 0.5) * gammainc(m + 0.5, xs) / (2 * xs ** (m + 0.5))
    return out


def pw92_g(rs, A, a1, b1, b2, b3, b4):
    """PW92 interpolation G(rs) with p=1 (Perdew & Wang, PRB 45, 13244, eq. 10)."""
    q0 = -2 * A * (1 + a1 * rs)
    q1 = 2 * A * (b1 * np.sqrt(rs) + b2 * rs + b3 * rs ** 1.5 + b4 * rs ** 2)
    return q0 * np.log(1 + 1 / q1)


def main():
    xs = np.array([0.0, 1e-3, 0.37, 2.5, 7.99, 12.345, 15.9, 16.0, 16.5, 30.0, 100.0])
    F = np.stack([boys(m, xs) for m in range(5)], axis=1)
    rs = np.array([0.1, 0.5, 1.0, 2.0, 5.0, 10.0])
    # fully polarised correlation energy per electron (PW92 table I, polarised column)
    ecp = pw92_g(rs, 0.015545, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517)
    ecu = pw92_g(rs, 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294)
    s = np.array([0.0, 0.1, 0.5, 1.0, 2.0, 3.0])
    kappa, mu = 0.804, 0.2195149727645171
    fx_pbe = 1 + kappa - kappa / (1 + mu * s ** 2 / kappa)
    np.savez(OUT, boys_x=xs, boys_F=F, rs=rs, ec_pol=ecp, ec_unpol=ecu, pbe_s=s, pbe_fx=fx_pbe)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
