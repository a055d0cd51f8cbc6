"""The mesh-sharded cycle on CPU: world_size-2 gloo process groups (127.0.0.1)
driving publicrelease_2020_b200.shard.sharded_cycle with the oracle as each
rank's shard (mesh points split in two), against the unsharded oracle cycle.
This covers the N>1 orchestration (partial sums, the one all-reduce, the
combine) and the decomposition itself: which sums the ranks must exchange
(SIC matrix, APOTNL_SIC's mesh sums, the farthest point's potential) and that
everything else is replicated.  The GPU form of the same protocol is in
tests/test_shard_gpu.py."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from publicrelease_2020_b200 import workloads as W

SYSTEMS = {
    "water_lda_nspn2": lambda: W.water(seed=0, nrad=12),
    "synthetic_pbe_nspn1": lambda: W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=3000, nfo=4),
    "water_scan_nspn2": lambda: W.water(seed=0, nrad=12, functional="MGGA-SCAN*MGGA-SCAN"),
}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, name, out):
    import torch.distributed as dist
    from oracle import oracle as O
    from publicrelease_2020_b200.shard import sharded_cycle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sysm = SYSTEMS[name]()
        orc = O.Oracle(sysm)
        n = sysm.nmsh
        b, e = n * rank // world, n * (rank + 1) // world
        r = sharded_cycle(O.OracleShard(orc, b, e))
        out[rank] = {k: (np.array(v) if not isinstance(v, float) else v) for k, v in r.items()}
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_two_rank_gloo_cycle_equals_unsharded(name):
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, name, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=600)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        got = [dict(out[r]) for r in range(2)]
    sysm = SYSTEMS[name]()
    ref = O.Oracle(sysm).sic_cycle(nthreads=4)
    for g in got:   # every rank holds the full result
        assert abs(g["esic"] - ref["esic"]) < 1e-10 * max(1.0, abs(ref["esic"]))
        for s in range(sysm.nspn):
            n = sysm.nfrm[s]
            assert np.allclose(g["results"][s][:n], ref["results"][s][:n], rtol=1e-10, atol=1e-11)
            assert np.allclose(g["sic"][s][:n, :n], ref["sic"][s][:n, :n], rtol=1e-10, atol=1e-12)
            assert np.allclose(g["debdax"][s][:n], ref["debdax"][s][:n], rtol=1e-9, atol=1e-10)
            assert np.allclose(g["cfrm"][s][:n], ref["cfrm"][s][:n], rtol=1e-10, atol=1e-12)
    assert all(np.array_equal(got[0][k], got[1][k]) for k in ("results", "sic", "debdax"))


class _PartialCtx:
    """A shard context stand-in whose partial sums are known: rank r holds
    (r + 1) * base, so the sum over two ranks is 3 * base."""

    def __init__(self, rank):
        self.rank = rank

    def adjoint(self, lspn):
        return (self.rank + 1) * np.arange(12.0).reshape(4, 3) * lspn

    def siclag_der(self):
        return (self.rank + 1) * np.linspace(-1.0, 1.0, 18).reshape(3, 2, 3)


def _rank_sums(rank, world, port, out):
    import torch.distributed as dist
    from publicrelease_2020_b200.shard import sharded_adjoint, sharded_siclag_der
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = _PartialCtx(rank)
        out[rank] = (sharded_adjoint(c, 2), sharded_siclag_der(c))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_basis_space_sums():
    """sharded_adjoint / sharded_siclag_der add the ranks' partial arrays."""
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_sums, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        got = [out[r] for r in range(2)]
    for g, d in got:
        assert np.array_equal(g, 3 * np.arange(12.0).reshape(4, 3) * 2)
        assert np.allclose(d, 3 * np.linspace(-1.0, 1.0, 18).reshape(3, 2, 3), rtol=0, atol=1e-15)


class _OracleChunks:
    """The oracle behind the set_shard protocol of the CUDA context: shard i
    of n is the mesh-point range [n_pts * i // n, n_pts * (i + 1) // n)."""

    def __init__(self, orc, npts):
        self.orc, self.npts, self.cur, self.log = orc, npts, None, []

    def set_shard(self, i, n):
        from oracle import oracle as O
        self.cur = O.OracleShard(self.orc, self.npts * i // n, self.npts * (i + 1) // n)
        self.log.append((i, n))

    def partial_size(self):
        from oracle import oracle as O
        return O.OracleShard(self.orc, 0, self.npts).partial_size()

    def cycle_partial(self, address):
        self.cur.cycle_partial(address)

    def cycle_combine(self, address):
        return self.cur.cycle_combine(address)


@pytest.mark.parametrize("nchunks", [1, 3])
def test_chunked_cycle_equals_one_pass(nchunks):
    """chunked_cycle (one device, the mesh in passes) adds every chunk's
    partial sums once and combines them into the one-pass cycle."""
    from oracle import oracle as O
    from publicrelease_2020_b200.shard import chunked_cycle
    sysm = SYSTEMS["water_scan_nspn2"]()
    orc = O.Oracle(sysm)
    ref = orc.sic_cycle(nthreads=4)
    ch = _OracleChunks(orc, sysm.nmsh)
    got = chunked_cycle(ch, nchunks)
    assert ch.log == [(i, nchunks) for i in range(nchunks)]
    assert abs(got["esic"] - ref["esic"]) < 1e-10 * max(1.0, abs(ref["esic"]))
    for s in range(sysm.nspn):
        n = sysm.nfrm[s]
        assert np.allclose(got["results"][s][:n], ref["results"][s][:n], rtol=1e-10, atol=1e-11)
        assert np.allclose(got["sic"][s][:n, :n], ref["sic"][s][:n, :n], rtol=1e-10, atol=1e-12)
        assert np.allclose(got["debdax"][s][:n], ref["debdax"][s][:n], rtol=1e-9, atol=1e-10)
