"""Multi-process host logic on CPU (gloo, world size 2): LPT pair sharding,
the gradient all-reduce, and failure detection through the store (a rank
that raises makes every rank raise; nobody waits in the collective)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fem25_b200.parallel import pair_costs, shard_lpt


def test_lpt_balances_and_covers():
    freqs = [0.1 * (i + 1) for i in range(24) for _ in range(int(np.ceil(16 * (i + 1))))]
    costs = pair_costs(freqs, nsrc=64)
    for world in (1, 2, 4, 8):
        parts = shard_lpt(costs, world)
        allk = sorted(k for p in parts for k in p)
        assert allk == list(range(len(freqs)))
        loads = [sum(costs[k] for k in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=30))
    import oracle
    from fem25_b200 import synth
    from fem25_b200.parallel import RankFailure, distributed_gradient
    mesh, pairs, _ = synth.make_config(0, nx=6, nz=4)
    g = oracle.graph_build(mesh)
    sel = pairs[:6]
    rng = np.random.default_rng(7)
    u = rng.standard_normal((len(sel), 1, g.ndof)) + 1j * rng.standard_normal((len(sel), 1, g.ndof))
    lam = rng.standard_normal((len(sel), 1, g.ndof)) + 1j * rng.standard_normal((len(sel), 1, g.ndof))

    if mode == "exit" and rank == 1:
        return  # this rank dies before the gradient: it never reports
    def partial(idx):
        if mode == "fail" and rank == 1:
            raise ValueError("injected host failure")
        out_g = np.zeros((3, mesh.nnpg))
        for k in idx:
            oracle.grad_exact(mesh, g, sel[k][0], sel[k][1], u[k], lam[k], out=out_g)
        return torch.from_numpy(out_g)

    try:
        res = distributed_gradient(sel, partial, mesh.nnpg, step=0,
                                   timeout_s=5.0 if mode == "exit" else 60.0)
        if rank == 0:
            ref = np.zeros((3, mesh.nnpg))
            for k in range(len(sel)):
                oracle.grad_exact(mesh, g, sel[k][0], sel[k][1], u[k], lam[k], out=ref)
            out.put(("ok", float(np.abs(res.numpy() - ref).max() / np.abs(ref).max())))
    except RankFailure as e:
        out.put(("failure", rank, str(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["ok", "fail", "exit"])
def test_two_rank_gradient(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    msgs = [q.get(timeout=5) for _ in range({"ok": 1, "fail": 2, "exit": 1}[mode])]
    if mode == "ok":
        assert msgs[0][0] == "ok" and msgs[0][1] < 1e-12
    elif mode == "exit":
        # the surviving rank learns of the dead one from the store, not a hang
        assert msgs[0][:2] == ("failure", 0) and "rank(s) [1] did not report" in msgs[0][2]
    else:
        assert sorted(m[1] for m in msgs) == [0, 1]
        assert all("injected host failure" in m[2] for m in msgs)


def _gpu_worker(rank, world, port, out):
    """Rank 0 computes its share on the GPU (sharded_gradient's accumulate /
    finalize on a Context), rank 1 with the oracle on the CPU; gloo sums."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import oracle
    from fem25_b200 import synth
    from fem25_b200.parallel import distributed_gradient, sharded_gradient
    mesh, pairs, _ = synth.make_config(2, nx=14, nz=8)
    g = oracle.graph_build(mesh)
    sel = [pairs[k] for k in (3, 70, 140, 200, 333, 480)]
    nsrc = 8
    u = synth.smooth_fields(mesh, g, sel, nsrc, seed=5).numpy()
    lam = synth.smooth_fields(mesh, g, sel, nsrc, seed=6).numpy()
    try:
        if rank == 0:
            from fem25_b200 import Context
            ctx = Context(mesh, g)
            dev = torch.device("cuda:0")
            res = sharded_gradient(ctx, sel, nsrc, lambda k: (torch.from_numpy(u[k:k + 1]).to(dev),
                                                              torch.from_numpy(lam[k:k + 1]).to(dev)))
            res = res.cpu().numpy()
            ref = np.zeros((3, mesh.nnpg))
            for k in range(len(sel)):
                oracle.grad_exact(mesh, g, sel[k][0], sel[k][1], u[k], lam[k], out=ref)
            err = max(float(np.linalg.norm(res[m] - ref[m]) / np.linalg.norm(ref[m])) for m in range(3))
            out.put(("ok", err))
            ctx.close()
        else:
            def partial(idx):
                o = np.zeros((3, mesh.nnpg))
                for k in idx:
                    oracle.grad_exact(mesh, g, sel[k][0], sel[k][1], u[k], lam[k], out=o)
                return torch.from_numpy(o)
            distributed_gradient(sel, partial, mesh.nnpg)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_rank_gradient_gpu_and_oracle_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    tag, err = q.get(timeout=5)
    assert tag == "ok" and err <= 1e-6, err
