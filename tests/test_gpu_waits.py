"""The bounded pipeline waits of the tensor-core gradient kernels.

Every hand-off of k_grad_cov (covariance form) and k_grad_tc (pointwise
form) is an mbarrier wait with a limit; a wait that runs out records an
error code, the CTA drains its schedule without waiting (its MMAs are
awaited and its tensor memory freed before it exits) and the host reads the
code with fem25_sync_status.  Here the test hook fem25_test_waits makes one
producer warp withhold its first arrival under a short limit (about 1 ms of
SM clock), so a wait runs out on purpose: no fault, no trap, and every wait
still ends.  Checked: the status is FEM25_ERR_CUDA with the time-out message,
the context stays usable, and the next normal call is correct (split
precision within 2e-5 of the FP64 kernel, as in the parity tests)."""
import numpy as np
import pytest

from fem25_b200 import (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE,
                        Context, Fem25Error, synth)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

LIMIT = 2_000_000  # SM clocks, about 1 ms


@pytest.fixture(scope="module")
def case():
    mesh, pairs, _ = synth.make_config(2, nx=24, nz=12)
    ctx = Context(mesh)
    dev = torch.device("cuda:0")
    gen = torch.Generator(device=dev)
    gen.manual_seed(71)
    nsrc = 8
    shape = (2, nsrc, ctx.ndof)
    u = torch.randn(shape, dtype=torch.complex128, device=dev, generator=gen)
    lam = torch.randn(shape, dtype=torch.complex128, device=dev, generator=gen)
    pp = [pairs[5], pairs[300]]
    fr, py = [p[0] for p in pp], [p[1] for p in pp]
    g64 = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=dev)
    ctx.gradient(fr, py, nsrc, u, lam, g64, FEM25_PREC_FP64)
    torch.cuda.synchronize()
    yield mesh, ctx, fr, py, nsrc, u, lam, g64
    ctx.close()


def _rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.mark.parametrize("prec", [FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE])
def test_timed_out_wait_reports_and_recovers(case, prec):
    mesh, ctx, fr, py, nsrc, u, lam, g64 = case
    out = torch.zeros_like(g64)
    ctx.gradient(fr, py, nsrc, u, lam, out, prec)  # set-up call (tables, accumulators)
    ctx.sync_status()
    ctx.test_waits(LIMIT, inject=True)
    try:
        out.zero_()
        ctx.gradient(fr, py, nsrc, u, lam, out, prec)
        with pytest.raises(Fem25Error) as ei:
            ctx.sync_status()
        assert ei.value.code == 4 and "timed out" in str(ei.value), str(ei.value)
    finally:
        ctx.test_waits(0, inject=False)
    ctx.sync_status()  # the error word was cleared by the report
    out.zero_()
    ctx.gradient(fr, py, nsrc, u, lam, out, prec)
    ctx.sync_status()
    rel = _rel(out, g64)
    assert rel <= 2e-5, rel


def test_timed_out_accumulation_is_discarded(case):
    """A drained accumulation invalidates the covariances accumulated since the
    last finalize: the report discards them, the next finalize adds nothing and
    a fresh accumulate + finalize is correct."""
    mesh, ctx, fr, py, nsrc, u, lam, g64 = case
    out = torch.zeros_like(g64)
    ctx.gradient_accumulate(fr[:1], py[:1], nsrc, u[:1], lam[:1])
    ctx.test_waits(LIMIT, inject=True)
    try:
        ctx.gradient_accumulate(fr[1:], py[1:], nsrc, u[1:], lam[1:])
        with pytest.raises(Fem25Error) as ei:
            ctx.sync_status()
        assert ei.value.code == 4
    finally:
        ctx.test_waits(0, inject=False)
    ctx.gradient_finalize(out)
    torch.cuda.synchronize()
    assert float(out.abs().max()) == 0.0
    ctx.gradient_accumulate(fr, py, nsrc, u, lam)
    ctx.gradient_finalize(out)
    ctx.sync_status()
    rel = _rel(out, g64)
    assert rel <= 2e-5, rel
