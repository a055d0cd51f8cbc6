"""Mesh-sharded SIC cycle: one process (rank) per GPU, each context evaluating
one shard of the mesh points, and one in-place sum of the packed partial sums
over the ranks -- the exchange step the reference performs with MPI_REDUCE of
the mesh contributions (pampoiss.F:105-120) and of the SIC matrix
(pamlmsic.F:103).

The sum runs on the GPU buffer with an NCCL process group (over NVLink /
NVSwitch on one node); with a gloo group the buffer goes through host memory.
Any object with partial_size(), cycle_partial(address) and
cycle_combine(address) can be driven: the CUDA library (sic.FlosicSIC) and,
in the CPU tests, the FP64 CPU restatement of the same decomposition.

The basis-space results (dE/dC_FO and the atomic SIC force terms DERSIC) are
sums over mesh points too: each rank computes its shard's part and one more
sum completes them (sharded_adjoint, sharded_siclag_der)."""
from __future__ import annotations

import numpy as np


def allreduce_array(a, group=None, device=None):
    """Sum a host array over the ranks of `group` (through `device` for NCCL)."""
    import torch
    import torch.distributed as dist

    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
    if dist.get_backend(group) == "nccl":
        t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.cpu().numpy()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.numpy()


def sharded_adjoint(ctx, lspn, group=None, device=None):
    """G = dE_SIC/dC_FO of spin lspn over the whole mesh from the ranks' shards."""
    return allreduce_array(ctx.adjoint(lspn), group, device)


def sharded_siclag_der(ctx, group=None, device=None):
    """DERSIC over the whole mesh from the ranks' shards."""
    return allreduce_array(ctx.siclag_der(), group, device)


def chunked_cycle(ctx, nchunks, device=None):
    """One SIC cycle of the whole mesh on one device in nchunks passes, for a
    system whose per-FO mesh arrays (FO values and their derivatives, Coulomb
    and SIC potentials, the SIC-weighted Y channels: several doubles per
    point and FO of each spin) would not fit in device memory at once.  Pass
    i evaluates mesh shard i of nchunks (flosic_sic_set_shard), so those
    arrays are sized for one chunk; the packed partial sums of the passes are
    added and flosic_sic_cycle_combine completes the cycle, exactly as the
    ranks of sharded_cycle do, so the outputs equal the one-pass cycle to
    rounding.  The FO set-up and the POISSON1 call set-up are recomputed in
    every pass.  The context is left on its last chunk."""
    import torch

    n = ctx.partial_size()
    on_gpu = device is not None and torch.device(device).type == "cuda"
    total = torch.zeros(n, dtype=torch.float64, device=device if on_gpu else "cpu")
    part = torch.zeros_like(total)
    for i in range(nchunks):
        ctx.set_shard(i, nchunks)
        ctx.cycle_partial(part.data_ptr())
        total += part
        if on_gpu:   # the next pass rewrites `part` on the library's stream
            torch.cuda.synchronize(total.device)
    return ctx.cycle_combine(total.data_ptr())


def sharded_cycle(ctx, group=None, device=None):
    """One SIC cycle over the ranks of `group` (torch.distributed default group
    if None).  Every rank calls it with its own shard's context; every rank
    returns the full cycle's outputs (RESULTS, SIC, DEBDAX, CFRM, E_SIC)."""
    import torch
    import torch.distributed as dist

    n = ctx.partial_size()
    backend = dist.get_backend(group)
    on_gpu = device is not None and torch.device(device).type == "cuda"
    buf = torch.zeros(n, dtype=torch.float64, device=device if on_gpu else "cpu")
    ctx.cycle_partial(buf.data_ptr())
    if on_gpu and backend == "nccl":
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        torch.cuda.synchronize(buf.device)   # the library reads the sum on its own stream
    elif on_gpu:
        host = buf.cpu()
        dist.all_reduce(host, op=dist.ReduceOp.SUM, group=group)
        buf.copy_(host)
        torch.cuda.synchronize(buf.device)
    else:
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    return ctx.cycle_combine(buf.data_ptr())
