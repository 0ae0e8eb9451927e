"""Split-precision (3xTF32) gradients at the target accuracy, per parameter.

The adjoint-gradient workload's fields: seeded complex128 nodal fields of
unit RMS per (pair, source) with a lognormal(0, 0.1) amplitude and a smooth
phase exp(i (k0 x + phi)), phi correlated over 5 km (synth.smooth_fields), on
the layered 400x120 layout at 24x12 elements, two (omega, py) pairs with 32
and 64 sources each.  Both split-precision forms (covariance,
FEM25_PREC_TF32X3, and pointwise, FEM25_PREC_TF32X3_POINTWISE) must agree
with the oracle's exact FP64 gradient (grad_exact) to 1e-6 relative
(2-norm) separately for lambda, mu and rho -- the target accuracy -- and the
FP64 kernel to 1e-10.  (White-noise fields, a harder case for cancellation,
are covered at 2e-5 by the parity tests.)"""
import numpy as np
import pytest

import oracle
from fem25_b200 import (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE,
                        Context, synth)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def layered():
    mesh, pairs, _ = synth.make_config(2, nx=24, nz=12)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    yield mesh, pairs, g, ctx
    ctx.close()


@pytest.mark.parametrize("nsrc", [32, 64])
def test_split_precision_per_parameter_1e6(layered, nsrc):
    mesh, pairs, g, ctx = layered
    use = [pairs[70], pairs[400]]
    u = synth.smooth_fields(mesh, g, use, nsrc, seed=100 + nsrc)
    lam = synth.smooth_fields(mesh, g, use, nsrc, seed=200 + nsrc)
    ref = np.zeros((3, mesh.nnpg))
    un, ln = u.numpy(), lam.numpy()
    for p, (f, py) in enumerate(use):
        oracle.grad_exact(mesh, g, f, py, un[p], ln[p], out=ref)
    dev = torch.device("cuda:0")
    d_u, d_l = u.to(dev), lam.to(dev)
    errs = {}
    for prec, tol in ((FEM25_PREC_FP64, 1e-10), (FEM25_PREC_TF32X3, 1e-6),
                      (FEM25_PREC_TF32X3_POINTWISE, 1e-6)):
        d_g = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=dev)
        ctx.gradient([p[0] for p in use], [p[1] for p in use], nsrc, d_u, d_l, d_g, prec)
        ctx.sync_status()
        got = d_g.cpu().numpy()
        errs[prec] = [float(np.linalg.norm(got[m] - ref[m]) / np.linalg.norm(ref[m]))
                      for m in range(3)]
        assert max(errs[prec]) <= tol, (prec, errs[prec])
    print(f"nsrc {nsrc}: per-parameter errors (lambda, mu, rho): {errs}")
