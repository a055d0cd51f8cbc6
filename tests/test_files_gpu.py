"""The SIC files written from real cycles (publicrelease_2020_b200/files.py):
ZPOT#### hold the APOTNL_SIC potentials bit for bit, MGGA#### the FOs'
Hamiltonian ingredients (against the oracle's SUBVLXC on the same FO
density), SICD.DAT / SIC_ENERGY / fforce.dat the cycle's
SIC matrix, RESULTS and DEBDAX to their printed precision."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from publicrelease_2020_b200 import files as F
from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("functional", ["LDA-PW91*LDA-PW91", "MGGA-SCAN*MGGA-SCAN"])
def test_cycle_files(tmp_path, functional):
    sysm = W.water(seed=0, nrad=18, functional=functional)
    ctx = S.open_system(sysm)
    try:
        out = ctx.cycle()
        F.write_cycle_files(str(tmp_path), ctx, out)
        names = sorted(os.listdir(tmp_path))
        zp = [f"ZPOT{i:04d}" for i in range(1, 11)]
        assert all(z in names for z in zp)
        assert ("MGGA0001" in names) == (functional.startswith("MGGA"))
        for s in range(2):
            for k in range(1, 6):
                recs = F.read_unformatted(str(tmp_path / f"ZPOT{k + 5 * s:04d}"))
                assert np.array_equal(np.concatenate(recs), ctx.apotnl_sic(s + 1, k)["pot"])
        if functional.startswith("MGGA"):
            # the FO's Hamiltonian ingredients: the oracle's SUBVLXC on the GPU's
            # FO density and the oracle's tau (the same functions up to rounding;
            # SCAN amplifies rounding where rho << max rho, hence the masks)
            orc = O.Oracle(sysm)
            _, rho = ctx.coupot_sic(1, 1)
            _, mo, _ = orc.getvlxc_mgga(rho, orc.fo_tau(1, 1))
            m = np.stack(F.read_unformatted(str(tmp_path / "MGGA0001")))
            n = sysm.nmsh
            assert m.shape == (2 * n, 4) and np.all(m[n:] == 0.0)
            r0 = rho[0]
            keep = r0 > 1e-3 * r0.max()
            for d in range(4):
                scale = np.abs(mo[keep, d]).max()
                assert np.max(np.abs(m[:n][keep, d] - mo[keep, d])) <= 1e-8 * scale, d
                assert np.sum(np.abs(m[:n, d] - mo[:, d]) * r0 * sysm.wmsh) <= 1e-8 * scale, d
        sicd = np.array([float(v) for ln in open(tmp_path / "SICD.DAT") for v in ln.split()]).reshape(10, 5)
        ref = np.concatenate([out["sic"][s][:5, :5] for s in range(2)])
        assert np.max(np.abs(sicd - ref)) <= 5e-6
        ff = np.array([float(v) for ln in open(tmp_path / "fforce.dat") for v in ln.split()]).reshape(10, 3)
        assert np.max(np.abs(ff - np.concatenate([out["debdax"][s][:5] for s in range(2)]))) <= 5e-12 * max(
            1.0, np.abs(ff).max())
    finally:
        ctx.close()
