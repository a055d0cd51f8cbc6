"""Exact-integer form of the near-field contraction, emulated on the CPU with
the oracle's own POISSON1 data (orc_pair_dump).

A multi-pair call's near potential at a point is V = sum_k a_k g_k over the
call's K = 46 x pairs rows: a_k = COEFICIENT(1:46) of each pair (gtdncf.F),
g_k = F_m(delta r^2) times a monomial of r - C up to degree 4 (the ERP sums of
poisson1.f:1000-1117).  Cut each operand into int8 slices, multiply them with
exact int32 sums (as an integer tensor-core MMA would) and scale back.  With
one scale per FO row and one per point column this loses most of its digits,
because the rows of a pair span many decades.  A power-of-two balance per row,
d_k = 2^round(log2(max|g_k| / max|a_k|) / 2) with a_k d_k and g_k / d_k, is
exact and keeps 4 slices (10 triangular products) within 1e-7 of max|V|.
These tests pin that property of the data; the GPU kernels contract the same
rows in FP64."""
import numpy as np
import pytest
from scipy.special import gamma, gammainc

from oracle import oracle as O
from publicrelease_2020_b200 import workloads as W

# (Boys order m, monomial j) of COEFICIENT(k+1), k = 0..45, in the order the
# ERP sums of poisson1.f use them
KM = ([(0, 0), (1, 0), (2, 0)] + [(1, j) for j in range(1, 4)] + [(2, j) for j in range(1, 10)]
      + [(3, j) for j in range(4, 20)] + [(4, j) for j in range(20, 35)])
MK = np.array([m for m, _ in KM])
JK = np.array([j for _, j in KM])
# monomials of poisson1.f's POLY(35): index -> (earlier index, factor index)
PROD = {5: (2, 1), 7: (3, 1), 8: (3, 2), 10: (1, 4), 11: (2, 4), 12: (1, 6), 13: (2, 6), 14: (3, 4),
        15: (3, 5), 16: (3, 6), 17: (1, 9), 18: (2, 9), 19: (3, 9), 20: (4, 4), 21: (4, 5), 22: (6, 4),
        23: (6, 5), 24: (6, 6), 25: (4, 7), 26: (8, 4), 27: (8, 5), 28: (6, 8), 29: (9, 4), 30: (9, 5),
        31: (9, 6), 32: (7, 9), 33: (8, 9), 34: (9, 9)}


def g_rows(r, cn, delta):
    """g_k at points r (n, 3) for a pair with -C = cn and exponent sum delta."""
    d = r + cn
    p = np.zeros((len(r), 35))
    p[:, 0] = 1.0
    p[:, 1], p[:, 2], p[:, 3] = d[:, 2], d[:, 1], d[:, 0]
    p[:, 4], p[:, 6], p[:, 9] = d[:, 2] ** 2, d[:, 1] ** 2, d[:, 0] ** 2
    for i in sorted(PROD):
        a, b = PROD[i]
        p[:, i] = p[:, a] * p[:, b]
    x = np.maximum(delta * (d * d).sum(1), 1e-300)
    F = np.stack([np.where(x < 1e-8, 1.0 / (2 * m + 1),
                           gamma(m + 0.5) * gammainc(m + 0.5, x) / (2 * x ** (m + 0.5))) for m in range(5)], 1)
    return F[:, MK] * p[:, JK]


def int8_slices(v, scale, n):
    r, out = v / scale, []
    for t in range(n):
        q = np.clip(np.rint(r * 2.0 ** (7 * (t + 1))), -127, 127)
        out.append(q.astype(np.int64))
        r = r - q * 2.0 ** (-7 * (t + 1))
    return out


def sliced_dot(G, a, n):
    """G (points, K) . a (K) from n int8 slices of each, triangular products,
    exact integer sums; one scale for a, one per point for G."""
    sa = np.abs(a).max()
    sg = np.abs(G).max(1)
    sg[sg == 0] = 1.0
    qa, qg = int8_slices(a, sa, n), int8_slices(G, sg[:, None], n)
    v = np.zeros(len(G))
    for t in range(n):
        for u in range(n - t):
            v += (qg[u] @ qa[t]).astype(np.float64) * 2.0 ** (-7 * (t + u + 2))
    return v * sa * sg


@pytest.fixture(scope="module")
def near_calls():
    s = W.synthetic(natoms=10, nbasis=128, nmsh=20000, nfo=4, box_ang=7.56, seed=1)
    orc = O.Oracle(s)
    calls, pairs = orc.pair_dump(1, 1)
    r = np.asarray(s.rmsh).reshape(-1, 3)[::5]
    out = []
    for ci, (c0, c1, c2, rc, npot, n) in enumerate(calls):
        if n <= 1:
            continue
        near = np.ones(len(r), bool) if npot == 1 else ((r - [c0, c1, c2]) ** 2).sum(1) <= rc * rc
        if not near.any():
            continue
        cp = pairs[pairs[:, 0] == ci]
        G = np.concatenate([g_rows(r[near], q[1:4], q[4]) for q in cp], axis=1)
        out.append((G, cp[:, 5:51].reshape(-1)))
    assert len(out) > 10
    return out, orc, s


def test_g_rows_reproduce_exact_mode_potential(near_calls):
    _, orc, s = near_calls
    calls, pairs = orc.pair_dump(1, 1)
    r = np.asarray(s.rmsh).reshape(-1, 3)[::97]
    v = sum(g_rows(r, q[1:4], q[4]) @ q[5:51] for q in pairs)
    ex = orc.coupot_sic(1, 1, exact=True)
    ex = (ex[0] if isinstance(ex, tuple) else ex)[::97]
    assert np.abs(v - ex).max() < 1e-9 * np.abs(ex).max()


def _max_rel_error(near_calls, balance, n):
    calls, _, _ = near_calls
    err, vmax = 0.0, 0.0
    for G, a in calls:
        exact = G @ a
        if balance:
            ga, aa = np.abs(G).max(0), np.abs(a)
            d = np.ones(len(a))
            ok = (ga > 0) & (aa > 0)
            d[ok] = 2.0 ** np.rint(0.5 * np.log2(ga[ok] / aa[ok]))
            G, a = G / d, a * d
        err = max(err, np.abs(sliced_dot(G, a, n) - exact).max())
        vmax = max(vmax, np.abs(exact).max())
    return err / vmax


def test_balanced_int8_slices_reach_fp32_class_accuracy(near_calls):
    assert _max_rel_error(near_calls, True, 4) < 1e-7
    assert _max_rel_error(near_calls, True, 3) < 1e-5


def test_unbalanced_int8_slices_lose_the_potential(near_calls):
    assert _max_rel_error(near_calls, False, 4) > 1e-4


def test_balance_shared_by_an_fo_block(near_calls):
    """One balance per (pair, row) for a block of FOs (the largest |a_k| over
    the block), one scale per FO row: every FO keeps the accuracy."""
    _, orc, s = near_calls
    dumps = [orc.pair_dump(1, k) for k in range(1, 5)]
    calls = dumps[0][0]
    assert all(np.array_equal(d[1][:, :5], dumps[0][1][:, :5]) for d in dumps)  # one pair plan
    r = np.asarray(s.rmsh).reshape(-1, 3)[::5]
    err, vmax = np.zeros(4), np.zeros(4)
    for ci, (c0, c1, c2, rc, npot, n) in enumerate(calls):
        if n <= 1:
            continue
        near = np.ones(len(r), bool) if npot == 1 else ((r - [c0, c1, c2]) ** 2).sum(1) <= rc * rc
        if not near.any():
            continue
        sel = dumps[0][1][:, 0] == ci
        G = np.concatenate([g_rows(r[near], q[1:4], q[4]) for q in dumps[0][1][sel]], axis=1)
        A = np.stack([d[1][sel][:, 5:51].reshape(-1) for d in dumps])
        ga, aa = np.abs(G).max(0), np.abs(A).max(0)
        d = np.ones(A.shape[1])
        ok = (ga > 0) & (aa > 0)
        d[ok] = 2.0 ** np.rint(0.5 * np.log2(ga[ok] / aa[ok]))
        for f in range(4):
            exact = G @ A[f]
            err[f] = max(err[f], np.abs(sliced_dot(G / d, A[f] * d, 4) - exact).max())
            vmax[f] = max(vmax[f], np.abs(exact).max())
    assert np.all(err / vmax < 1e-7), err / vmax


def test_one_g_scale_per_call(near_calls):
    """The G side needs no per-point scale: one scale per call (the largest
    balanced |g|) keeps 4 slices within 1e-7."""
    calls, _, _ = near_calls
    err, vmax = 0.0, 0.0
    for G, a in calls:
        exact = G @ a
        ga, aa = np.abs(G).max(0), np.abs(a)
        d = np.ones(len(a))
        ok = (ga > 0) & (aa > 0)
        d[ok] = 2.0 ** np.rint(0.5 * np.log2(ga[ok] / aa[ok]))
        Gb, ab = G / d, a * d
        sa, sg = np.abs(ab).max(), np.abs(Gb).max()
        qa, qg = int8_slices(ab, sa, 4), int8_slices(Gb, sg, 4)
        v = sum((qg[u] @ qa[t]).astype(np.float64) * 2.0 ** (-7 * (t + u + 2))
                for t in range(4) for u in range(4 - t))
        err = max(err, np.abs(v * sa * sg - exact).max())
        vmax = max(vmax, np.abs(exact).max())
    assert err / vmax < 1e-7
