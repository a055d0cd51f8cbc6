"""Writes nrlmol_default_basis.npz: the NRLMOL all-electron basis tables
(D. Porezag and M. R. Pederson) for H, C and O as the reference stores them
in flosic/bdallbas.f -- per element NG bare exponents ALPH, the NSPD(1:3)
fully contracted s/p/d functions and their coefficients COEF.  The seeded
workloads (publicrelease_2020_b200/workloads.py) build the reference's
default basis from these tables with the supplement rule of flosic/sallbas.f.

Run once with the path of a reference checkout (the directory that holds
flosic/bdallbas.f), which it reads as data:

    python publicrelease_2020_b200/data/make_nrlmol_default_basis.py <reference checkout>
"""
import os
import re
import sys

import numpy as np

ELEMENTS = (1, 6, 8)


def _numbers(text):
    return [float(x.replace("D", "E").replace("d", "e")) for x in re.findall(r"[-+]?\d+\.\d+[DdEe][-+]?\d+", text)]


def _block(src, header):
    """Numbers of the DATA statement whose header matches, up to its closing '/'."""
    m = re.search(re.escape(header).replace(r"\ ", r"\s*") + r"\s*/(.*?)/", src, re.S)
    if not m:
        raise ValueError(f"missing DATA block {header}")
    return _numbers(m.group(1))


def parse(path):
    src = open(path).read()
    out = {}
    for z in ELEMENTS:
        m = re.search(r"DATA \(NSPD\(I,\s*%d\), I=1,3\), NG\(\s*%d\)/\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+)/" % (z, z), src)
        nspd = [int(m.group(i)) for i in (1, 2, 3)]
        ng = int(m.group(4))
        alph = _block(src, "DATA (ALPH(I, %3d), I=1, %2d)" % (z, ng))
        assert len(alph) == ng, (z, len(alph), ng)
        coef = np.zeros((3, max(max(nspd), 1), ng))
        for l in range(3):
            for c in range(nspd[l]):
                v = _block(src, "DATA (COEF(I, %d, %d, %2d), I=1, %2d)" % (c + 1, l + 1, z, ng))
                assert len(v) == ng, (z, l, c, len(v))
                coef[l, c] = v
        out[z] = (np.array(nspd, dtype=np.int32), np.array(alph), coef)
    return out


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_nrlmol_default_basis.py <reference checkout holding flosic/bdallbas.f>")
    ref = sys.argv[1]
    tables = parse(os.path.join(ref, "flosic", "bdallbas.f"))
    arrays = {}
    for z, (nspd, alph, coef) in tables.items():
        arrays[f"nspd_{z}"], arrays[f"alph_{z}"], arrays[f"coef_{z}"] = nspd, alph, coef
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "nrlmol_default_basis.npz")
    np.savez(out, **arrays)
    for z, (nspd, alph, _) in tables.items():
        print(z, "NSPD", nspd.tolist(), "NG", len(alph), "alpha", alph[0], "...", alph[-1])
