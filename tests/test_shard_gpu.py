"""Mesh sharding through the C ABI (flosic_sic_set_shard / _cycle_partial /
_cycle_combine) on one GPU: the partial sums of the shards, added, give the
unsharded cycle.  Shards run as separate contexts in one process (sum on the
device) and as two spawned ranks of a gloo process group on the same GPU (the
sum goes through host memory; no kernel waits on another rank).  The packed
sums are added in another order than the single-context reductions, so the
comparison is at rounding level (1e-10 relative)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "water_lda_nspn2": lambda: W.water(seed=0, nrad=18),
    "synthetic_pbe_nspn1": lambda: W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=5000, nfo=4),
    "water_scan_nspn2": lambda: W.water(seed=0, nrad=18, functional="MGGA-SCAN*MGGA-SCAN"),
}


def _close(a, b, sysm):
    assert abs(a["esic"] - b["esic"]) < 1e-10 * max(1.0, abs(b["esic"]))
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        assert np.allclose(a["results"][s][:n], b["results"][s][:n], rtol=1e-10, atol=1e-11)
        assert np.allclose(a["sic"][s][:n, :n], b["sic"][s][:n, :n], rtol=1e-10, atol=1e-12)
        assert np.allclose(a["debdax"][s][:n], b["debdax"][s][:n], rtol=1e-9, atol=1e-10)
        assert np.allclose(a["cfrm"][s][:n], b["cfrm"][s][:n], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("nshards", [2, 3])
def test_shard_partials_sum_to_unsharded_cycle(name, nshards):
    import torch
    sysm = SYSTEMS[name]()
    whole = S.open_system(sysm)
    ref = whole.cycle()
    st = whole.stats()
    whole.close()
    ctxs = [S.open_system(sysm, shard=(r, nshards)) for r in range(nshards)]
    try:
        n = ctxs[0].partial_size()
        bufs = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in ctxs]
        for c, b in zip(ctxs, bufs):
            c.cycle_partial(b.data_ptr())
        total = torch.stack(bufs).sum(0)
        torch.cuda.synchronize()
        for c in ctxs:   # every rank combines the same sum into the same outputs
            got = c.cycle_combine(total.data_ptr())
            _close(got, ref, sysm)
            w = c.stats()
            assert (w["near_evals"], w["far_evals"], w["far_terms"]) == (st["near_evals"], st["far_evals"], st["far_terms"])
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("name", ["water_lda_nspn2", "water_scan_nspn2", "synthetic_pbe_nspn1"])
def test_shard_adjoint_and_dersic_sum_to_whole_mesh(name):
    """dE/dC_FO and DERSIC on mesh shards are partial sums over the shards' points."""
    sysm = SYSTEMS[name]()
    whole = S.open_system(sysm)
    g_ref = [whole.adjoint(sp) for sp in range(1, sysm.nspn + 1)]
    d_ref = whole.siclag_der()
    whole.close()
    ctxs = [S.open_system(sysm, shard=(r, 2)) for r in range(2)]
    try:
        for sp in range(1, sysm.nspn + 1):
            g = sum(c.adjoint(sp) for c in ctxs)
            assert np.abs(g - g_ref[sp - 1]).max() < 1e-10 * np.abs(g_ref[sp - 1]).max()
        d = sum(c.siclag_der() for c in ctxs)
        assert np.abs(d - d_ref).max() < 1e-10 * np.abs(d_ref).max()
    finally:
        for c in ctxs:
            c.close()


def test_sharded_context_refuses_whole_mesh_entry_points():
    sysm = SYSTEMS["water_lda_nspn2"]()
    ctx = S.open_system(sysm, shard=(1, 2))
    try:
        for call in (lambda: ctx.cycle(), lambda: ctx.apotnl_sic(1, 1), lambda: ctx.siclagm(1),
                     lambda: ctx.coupot_sic(1, 1)):
            with pytest.raises(S.FlosicError) as e:
                call()
            assert e.value.code == 8  # FLOSIC_ERR_STATE
        with pytest.raises(S.FlosicError) as e:
            ctx.set_shard(2, 2)
        assert e.value.code == 1
    finally:
        ctx.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from publicrelease_2020_b200 import sic as S2
    from publicrelease_2020_b200.shard import sharded_adjoint, sharded_cycle, sharded_siclag_der
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sysm = SYSTEMS["synthetic_pbe_nspn1"]()
        ctx = S2.open_system(sysm, shard=(rank, world))
        r = sharded_cycle(ctx, device="cuda:0")
        res = {k: (np.array(v) if not isinstance(v, float) else v) for k, v in r.items()}
        res["g1"] = sharded_adjoint(ctx, 1, device="cuda:0")
        res["dersic"] = sharded_siclag_der(ctx, device="cuda:0")
        out[rank] = res
        ctx.close()
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo_on_one_gpu():
    sysm = SYSTEMS["synthetic_pbe_nspn1"]()
    whole = S.open_system(sysm)
    ref = whole.cycle()
    g_ref = whole.adjoint(1)
    d_ref = whole.siclag_der()
    whole.close()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=600)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        got = [dict(out[r]) for r in range(2)]
    for g in got:
        _close(g, ref, sysm)
        assert np.abs(g["g1"] - g_ref).max() < 1e-10 * np.abs(g_ref).max()
        assert np.abs(g["dersic"] - d_ref).max() < 1e-10 * np.abs(d_ref).max()
