"""The whole-mesh SIC cycle in passes on one GPU (shard.chunked_cycle): one
context re-sharded between passes (flosic_sic_set_shard after the geometry and
orbitals are set), its packed partial sums added on the device and combined.
It must equal the one-pass cycle to rounding (1e-10 relative, the bar of the
multi-context shard tests), again when repeated, and the context must run
the whole mesh again after set_shard(0, 1); in both FO density routes (the
reference's pair route forms each point's density from the calls whose sphere
holds it, whichever pass the point falls in).  The file sorts after the other
GPU tests, before the allocation-free entry point's."""
import numpy as np
import pytest

from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W
from publicrelease_2020_b200.shard import chunked_cycle

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "water_lda_nspn2": lambda: W.water(seed=0, nrad=18),
    "water_scan_nspn2": lambda: W.water(seed=0, nrad=18, functional="MGGA-SCAN*MGGA-SCAN"),
    "synthetic_pbe_nspn1": lambda: W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=5000, nfo=4),
}


def _close(a, b, sysm):
    assert abs(a["esic"] - b["esic"]) < 1e-10 * max(1.0, abs(b["esic"]))
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        assert np.allclose(a["results"][s][:n], b["results"][s][:n], rtol=1e-10, atol=1e-11)
        assert np.allclose(a["sic"][s][:n, :n], b["sic"][s][:n, :n], rtol=1e-10, atol=1e-12)
        assert np.allclose(a["debdax"][s][:n], b["debdax"][s][:n], rtol=1e-9, atol=1e-10)
        assert np.allclose(a["cfrm"][s][:n], b["cfrm"][s][:n], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("density", ["phi2", "pairs"])
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_chunked_cycle_equals_one_pass(name, density):
    sysm = SYSTEMS[name]()
    ctx = S.open_system(sysm)
    try:
        ctx.set_density_mode(density)
        ref = ctx.cycle()
        st = ctx.stats()
        got = chunked_cycle(ctx, 3, device="cuda:0")
        _close(got, ref, sysm)
        w = ctx.stats()
        assert (w["near_evals"], w["far_evals"], w["far_terms"]) == \
            (st["near_evals"], st["far_evals"], st["far_terms"])
        _close(chunked_cycle(ctx, 3, device="cuda:0"), ref, sysm)
        ctx.set_shard(0, 1)
        _close(ctx.cycle(), ref, sysm)
    finally:
        ctx.close()
