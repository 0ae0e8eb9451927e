"""Multi-GPU plumbing for the (omega, py) data parallelism.

The reference spreads frequencies over MPI process groups
(``mkMPIgroups.f:61-97``, ``IFREQ = (IFREQL-1)*NPGROUPS + IPGROUP + 1`` at
``funcgradh.f90:155``) and sums the per-group gradients with
``MPI_REDUCE(GRADL, ..., MPI_SUM, MYHD_COMM)`` (``funcgradh.f90:428``).
Here one process drives one GPU; systems are independent, so

* assembly needs no collective (each rank assembles its own systems), and
* the gradient is the sum over ranks of each rank's partial gradient: one
  FP64 all-reduce of 3 x NNPG values.

Pairs are assigned longest-processing-time first by an estimated cost.  A
rank that fails reports it through the process group's store before the
collective, so the others raise instead of waiting in the all-reduce.
"""
from __future__ import annotations

import heapq
from datetime import timedelta
from typing import Callable, Sequence


def shard_lpt(costs: Sequence[float], world: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment of items to ``world`` ranks.
    Returns, per rank, the item indices in ascending order."""
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: -costs[k]):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(v) for v in out]


def pair_costs(freqs: Sequence[float], nsrc: int = 1) -> list[float]:
    """Cost model of one (omega, py) pair: a unit per source plus the share of
    its frequency's PML delta (built once per frequency by the batched
    assembly), which makes pairs of sparsely sampled frequencies dearer."""
    per_f: dict[float, int] = {}
    for f in freqs:
        per_f[f] = per_f.get(f, 0) + 1
    return [nsrc + 0.5 / per_f[f] for f in freqs]


class RankFailure(RuntimeError):
    pass


def _store():
    import torch.distributed as dist
    from torch.distributed import distributed_c10d as c10d
    return c10d._get_default_store() if dist.is_initialized() else None


def report_and_check(tag: str, ok: bool, msg: str = "", timeout_s: float = 60.0):
    """Every rank publishes its status under ``tag`` and reads the others'
    before the next collective; any failure raises RankFailure on all ranks."""
    import torch.distributed as dist
    rank, world = dist.get_rank(), dist.get_world_size()
    st = _store()
    st.set(f"fem25/{tag}/{rank}", ("ok" if ok else "fail:" + msg))
    keys = [f"fem25/{tag}/{r}" for r in range(world)]
    try:
        st.wait(keys, timedelta(seconds=timeout_s))
    except Exception:  # a rank that died or hangs never reports
        missing = [r for r, k in enumerate(keys) if not st.check([k])]
        raise RankFailure(f"rank(s) {missing} did not report within {timeout_s:g} s")
    bad = []
    for r, k in enumerate(keys):
        v = st.get(k).decode()
        if v != "ok":
            bad.append(f"rank {r}: {v[5:]}")
    if bad:
        raise RankFailure("; ".join(bad))


def distributed_gradient(pairs: Sequence[tuple[float, float]], partial: Callable, nnpg: int,
                         step: int = 0, device=None, timeout_s: float = 60.0):
    """Sum over ranks of ``partial(my_pair_indices) -> tensor[3, nnpg]``.

    ``partial`` computes this rank's gradient over its pairs (on the GPU in
    production).  The all-reduce replaces MPI_REDUCE(GRADL) of the reference;
    the status exchange before it turns a failing rank into an exception on
    every rank instead of a hang."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_initialized() else 1
    rank = dist.get_rank() if dist.is_initialized() else 0
    mine = shard_lpt(pair_costs([p[0] for p in pairs]), world)[rank]
    g, err = None, ""
    try:
        g = partial(mine)
    except Exception as e:  # reported to the other ranks below
        err = f"{type(e).__name__}: {e}"
    if world > 1:
        report_and_check(f"grad{step}", g is not None, err, timeout_s)
    elif g is None:
        raise RankFailure(err)
    if world > 1:
        g = g.to(torch.float64)
        if g.is_cuda and dist.get_backend() != "nccl":
            # a host collective (gloo): reduce a host copy
            h = g.cpu()
            dist.all_reduce(h, op=dist.ReduceOp.SUM)
            g.copy_(h)
        else:
            dist.all_reduce(g, op=dist.ReduceOp.SUM)
    return g


def sharded_gradient(ctx, pairs: Sequence[tuple[float, float]], nsrc: int, fields: Callable,
                     step: int = 0, stream=None, timeout_s: float = 60.0):
    """The exact gradient of all ``pairs`` over the ranks of the process group,
    each rank on its own GPU context ``ctx``: the rank accumulates the field
    covariances of its longest-processing-time share of the pairs
    (``fields(k) -> (u, lam)``, device tensors [1, nsrc, NDOF] of pair k) in
    split precision, contracts them once, and the per-rank FP64 gradients
    are summed by one all-reduce (NCCL on GPUs) -- the MPI_REDUCE(GRADL) of
    funcgradh.f90:428.  Returns the summed gradient [3, NNPG] on every rank."""
    import torch
    dev = torch.device("cuda", ctx.device)

    def partial(mine):
        g = torch.zeros((3, ctx.mesh.nnpg), dtype=torch.float64, device=dev)
        for k in mine:
            u, lam = fields(k)
            ctx.gradient_accumulate([pairs[k][0]], [pairs[k][1]], nsrc, u, lam, stream=stream)
        ctx.gradient_finalize(g, stream=stream)
        ctx.sync_status(stream)
        return g

    return distributed_gradient(pairs, partial, ctx.mesh.nnpg, step=step, timeout_s=timeout_s)
