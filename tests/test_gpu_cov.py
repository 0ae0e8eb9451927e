"""Covariance form of the split-precision gradient (FEM25_PREC_TF32X3,
fem25_gradient_accumulate_dev / fem25_gradient_finalize_dev).

Per element the weighted covariances sum conj(lam) u^T of the nodal fields
are accumulated over (pair, source) on tcgen05 tensor cores in 3xTF32 and
contracted once in FP64.  Checks: the oracle's exact gradient (grad_exact,
a loop-for-loop restatement of the KM25ISOQ derivative sums) on the
half-space, jittered, topographic and layered layouts with source counts
that fill 8-source stages partly (1, 5, 17, 33 sources); the FP64 kernel; the
split calls against the one-shot call; the accumulator's empty / pending
states; split calls recorded into a CUDA graph.

Tolerances: 2e-5 relative (2-norm per parameter) against the oracle, as
for the pointwise split-precision kernel; split vs one-shot 1e-12 (the same
FP32 tensor-memory sums, FP64 additions in another order).
"""
import numpy as np
import pytest

import oracle
from fem25_b200 import FEM25_PREC_FP64, FEM25_PREC_TF32X3, Context, synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dev():
    return torch.device("cuda:0")


def _fields(rng, npairs, nsrc, ndof):
    shape = (npairs, nsrc, ndof)
    u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    lam = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return u, lam


def _rel(got, ref):
    return max(float(np.linalg.norm(got[m] - ref[m]) / np.linalg.norm(ref[m])) for m in range(3))


@pytest.mark.parametrize("idx,nx,nz,nsrc", [(0, 10, 6, 1), (3, 14, 8, 5), (4, 18, 10, 17),
                                            (1, 12, 8, 33)],
                         ids=["halfspace-1src", "jittered-5src", "topographic-17src",
                              "layered-33src"])
def test_cov_gradient_matches_oracle(idx, nx, nz, nsrc):
    mesh, pairs, _ = synth.make_config(idx, nx=nx, nz=nz)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    use = [pairs[1], pairs[len(pairs) // 2], pairs[-1]]
    rng = np.random.default_rng(61 + idx)
    u, lam = _fields(rng, len(use), nsrc, g.ndof)
    ref = np.zeros((3, mesh.nnpg))
    for p, (f, py) in enumerate(use):
        oracle.grad_exact(mesh, g, f, py, u[p], lam[p], out=ref)
    d_u, d_l = torch.from_numpy(u).to(_dev()), torch.from_numpy(lam).to(_dev())
    d_g = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
    ctx.gradient([p[0] for p in use], [p[1] for p in use], nsrc, d_u, d_l, d_g, FEM25_PREC_TF32X3)
    got = d_g.cpu().numpy()
    assert _rel(got, ref) <= 2e-5
    # the FP64 kernel on the same fields
    d_g64 = torch.zeros_like(d_g)
    ctx.gradient([p[0] for p in use], [p[1] for p in use], nsrc, d_u, d_l, d_g64, FEM25_PREC_FP64)
    assert _rel(got, d_g64.cpu().numpy()) <= 2e-5
    ctx.close()


def test_split_calls_equal_one_shot():
    mesh, pairs, _ = synth.make_config(3, nx=12, nz=8)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    use = [pairs[k] for k in (0, 3, 7, 11, 15)]
    nsrc = 6
    rng = np.random.default_rng(71)
    u, lam = _fields(rng, len(use), nsrc, g.ndof)
    d_u, d_l = torch.from_numpy(u).to(_dev()), torch.from_numpy(lam).to(_dev())
    freqs, pys = [p[0] for p in use], [p[1] for p in use]
    one = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
    ctx.gradient(freqs, pys, nsrc, d_u, d_l, one, FEM25_PREC_TF32X3)
    split = torch.zeros_like(one)
    ctx.gradient_finalize(split)  # nothing pending: unchanged
    torch.cuda.synchronize()
    assert float(split.abs().max()) == 0.0
    for k in range(len(use)):  # one pair per call, as an inversion loop solves them
        ctx.gradient_accumulate([freqs[k]], [pys[k]], nsrc, d_u[k:k + 1], d_l[k:k + 1])
    ctx.gradient_finalize(split)
    before = split.clone()
    ctx.gradient_finalize(split)  # emptied by the first finalize
    torch.cuda.synchronize()
    assert torch.equal(split, before)
    rel = float(torch.linalg.norm(split - one) / torch.linalg.norm(one))
    assert rel <= 1e-12
    # a one-shot call flushes a pending accumulation into its own grad
    ctx.gradient_accumulate(freqs[:2], pys[:2], nsrc, d_u[:2], d_l[:2])
    both = torch.zeros_like(one)
    ctx.gradient(freqs[2:], pys[2:], nsrc, d_u[2:], d_l[2:], both, FEM25_PREC_TF32X3)
    rel = float(torch.linalg.norm(both - one) / torch.linalg.norm(one))
    assert rel <= 1e-12
    ctx.sync_status()  # no Jacobian failure or timed-out wait recorded
    ctx.close()


def test_split_calls_record_into_a_graph():
    """Accumulate calls recorded together with the finalize that consumes
    them replay to the eager result on every replay, including after the
    fields are overwritten in place."""
    mesh, pairs, _ = synth.make_config(0, nx=10, nz=6)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    use = [pairs[2], pairs[7], pairs[12]]
    nsrc = 5
    rng = np.random.default_rng(83)
    u, lam = _fields(rng, len(use), nsrc, g.ndof)
    d_u, d_l = torch.from_numpy(u).to(_dev()), torch.from_numpy(lam).to(_dev())
    freqs, pys = [p[0] for p in use], [p[1] for p in use]
    eager = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
    for k in range(len(use)):  # the uncaptured first call allocates the accumulators
        ctx.gradient_accumulate([freqs[k]], [pys[k]], nsrc, d_u[k:k + 1], d_l[k:k + 1])
    ctx.gradient_finalize(eager)
    torch.cuda.synchronize()
    got = torch.zeros_like(eager)
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            st = torch.cuda.current_stream()
            got.zero_()
            for k in range(len(use)):
                ctx.gradient_accumulate([freqs[k]], [pys[k]], nsrc, d_u[k:k + 1], d_l[k:k + 1],
                                        stream=st)
            ctx.gradient_finalize(got, stream=st)
    torch.cuda.current_stream().wait_stream(side)
    for rep in range(2):
        graph.replay()
        torch.cuda.synchronize()
        rel = float(torch.linalg.norm(got - eager) / torch.linalg.norm(eager))
        assert rel <= 1e-12, (rep, rel)
    d_u.mul_(0.5 - 0.5j)
    graph.replay()
    again = torch.zeros_like(eager)
    ctx.gradient(freqs, pys, nsrc, d_u, d_l, again, FEM25_PREC_TF32X3)
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(got - again) / torch.linalg.norm(again)) <= 1e-12
    assert float(torch.linalg.norm(got - eager) / torch.linalg.norm(eager)) > 1e-3
    del graph
    ctx.close()
