"""CUDA-graph capture of the batched assembly + gradient pipeline.

After one uncaptured call (which builds the affine basis, picks the
streaming variant and uploads the tensor-core tables), fem25_assemble_batch_dev
and fem25_gradient_dev record into a CUDA graph with no host synchronisation:
the per-launch system and pair tables travel as kernel parameters.  A replay
must reproduce the eager results (assembly bit-exact; the gradient's
cross-element atomic sums to 1e-12 relative), including after the input
fields are overwritten in place.  Calls that would need set-up during a
capture fail with an error instead of breaking it.
"""
import numpy as np
import pytest

import oracle
from fem25_b200 import (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE,
                        Context, Fem25Error, synth)
from tests import helpers

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dev():
    return torch.device("cuda:0")


def _rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.mark.parametrize("prec", [FEM25_PREC_FP64, FEM25_PREC_TF32X3,
                                  FEM25_PREC_TF32X3_POINTWISE])
def test_graph_replay_matches_eager(prec):
    mesh, pairs, _ = synth.make_config(0, nx=12, nz=8)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    sel = [pairs[1], pairs[4], pairs[9], pairs[12], pairs[15]]
    n, nslots, nsrc = len(sel), 3, 5
    cft = ["B", "S", "B", "B", "S"]
    freqs, pys = [p[0] for p in sel], [p[1] for p in sel]
    stride = 2 * g.nzero + 4
    rng = np.random.default_rng(21)
    shape = (n, nsrc, g.ndof)
    u = torch.from_numpy(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).to(_dev())
    lam = torch.from_numpy(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).to(_dev())

    ring_e = torch.zeros(nslots * stride, dtype=torch.float64, device=_dev())
    grad_e = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
    ctx.assemble_batch(cft, freqs, pys, ring_e, stride, nslots)
    ctx.gradient(freqs, pys, nsrc, u, lam, grad_e, prec)
    torch.cuda.synchronize()

    ring_g = torch.zeros_like(ring_e)
    grad_g = torch.zeros_like(grad_e)
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            st = torch.cuda.current_stream()
            grad_g.zero_()
            ctx.assemble_batch(cft, freqs, pys, ring_g, stride, nslots, stream=st)
            ctx.gradient(freqs, pys, nsrc, u, lam, grad_g, prec, stream=st)
    torch.cuda.current_stream().wait_stream(side)
    for rep in range(2):
        ring_g.zero_()
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(ring_g, ring_e), rep
        assert _rel(grad_g, grad_e) <= 1e-12, rep

    # the graph reads the fields through their device pointers: new values
    # written in place are picked up by the next replay
    u.mul_(0.5 + 0.25j)
    graph.replay()
    grad_e2 = torch.zeros_like(grad_e)
    ctx.gradient(freqs, pys, nsrc, u, lam, grad_e2, prec)
    torch.cuda.synchronize()
    assert _rel(grad_g, grad_e2) <= 1e-12
    assert _rel(grad_g, grad_e) > 1e-3

    # the replayed assembly still matches the oracle
    r = ring_g.view(nslots, stride)
    for k in range(n - nslots, n):
        ref128, _ = oracle.asmble(mesh, g, cft[k], freqs[k], pys[k], want64=False)
        got = r[k % nslots, :2 * g.nzero].cpu().numpy()
        assert helpers.row_norm_err(got[0::2] + 1j * got[1::2], ref128, g.irptr) <= 1e-12
    del graph
    ctx.close()


def test_gradient_more_pairs_than_one_launch():
    """More (omega, py) pairs than one launch's parameter table holds: the
    entry point splits them over several launches that add into grad."""
    mesh, pairs, _ = synth.make_config(0, nx=6, nz=4)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    npairs, nsrc = 70, 1
    use = [pairs[k % len(pairs)] for k in range(npairs)]
    use = [(f * (1.0 + 0.01 * k), py) for k, (f, py) in enumerate(use)]
    rng = np.random.default_rng(5)
    shape = (npairs, nsrc, g.ndof)
    u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    lam = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ref = np.zeros((3, mesh.nnpg))
    for p, (f, py) in enumerate(use):
        oracle.grad_exact(mesh, g, f, py, u[p], lam[p], out=ref)
    d_u = torch.from_numpy(u).to(_dev())
    d_l = torch.from_numpy(lam).to(_dev())
    for prec, tol in ((FEM25_PREC_FP64, 1e-10), (FEM25_PREC_TF32X3, 2e-5),
                      (FEM25_PREC_TF32X3_POINTWISE, 2e-5)):
        d_g = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
        ctx.gradient([p[0] for p in use], [p[1] for p in use], nsrc, d_u, d_l, d_g, prec)
        got = d_g.cpu().numpy()
        for m in range(3):
            rel = np.linalg.norm(got[m] - ref[m]) / np.linalg.norm(ref[m])
            assert rel <= tol, (prec, m, rel)
    ctx.close()


def test_capture_before_setup_is_rejected():
    mesh, pairs, _ = synth.make_config(0, nx=6, nz=4)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    stride = 2 * g.nzero
    ring = torch.zeros(stride, dtype=torch.float64, device=_dev())
    u = torch.zeros((1, 1, g.ndof), dtype=torch.complex128, device=_dev())
    grad = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            st = torch.cuda.current_stream()
            with pytest.raises(Fem25Error):
                ctx.assemble_batch("B", [pairs[0][0]], [pairs[0][1]], ring, stride, 1, stream=st)
            for prec in (FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE):
                with pytest.raises(Fem25Error):
                    ctx.gradient([pairs[0][0]], [pairs[0][1]], 1, u, u, grad, prec, stream=st)
            with pytest.raises(Fem25Error):
                ctx.assemble("B", pairs[0][0], pairs[0][1], ring, stream=st)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    del graph
    # the same calls work once made outside a capture
    ctx.assemble_batch("B", [pairs[0][0]], [pairs[0][1]], ring, stride, 1)
    for prec in (FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE):
        ctx.gradient([pairs[0][0]], [pairs[0][1]], 1, u, u, grad, prec)
    torch.cuda.synchronize()
    ctx.close()
