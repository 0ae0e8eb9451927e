"""GPU parity on the layouts of the larger benchmark configurations, at small
element counts: the three-layer model of the 400x120 layout, the jittered
300x150 layout (anchors moved by up to 20 %) and the jittered, topographic
600x200 layout with its 4-element strip.  Distorted elements exercise the
Jacobian, the PML depths and the anchor interpolation away from the
rectangular half-space the other parity tests use.

Tolerances as in test_gpu_parity.py: plain FP64 CSR and the reference's
COMPLEX*8 CDIST bit-exact (dispersive media included); batched CSR <= 1e-12
per row; exact gradient FP64 <= 1e-10 and 3xTF32 <= 2e-5 relative (2-norm);
both split-precision forms (covariance and pointwise) as well;
reference-compatible gradient and the Hessian-path kernels (MET225_MOD,
CADJ_NU_ALPHA, PCHADJ) bit-exact.
"""
import numpy as np
import pytest

import oracle
from fem25_b200 import (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE,
                        Context, synth)
from tests import helpers

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dev():
    return torch.device("cuda:0")


@pytest.fixture(scope="module", params=[(1, 16, 8), (3, 14, 8), (4, 18, 10)],
                ids=["layered", "jittered", "topographic"])
def layout(request):
    idx, nx, nz = request.param
    mesh, pairs, _ = synth.make_config(idx, nx=nx, nz=nz)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    yield mesh, pairs, g, ctx
    ctx.close()


def test_plain_and_batched_assembly(layout):
    mesh, pairs, g, ctx = layout
    sel = [pairs[0], pairs[len(pairs) // 2], pairs[-1]]
    cft = ["B", "S", "B"]
    for (f, py), c in zip(sel, cft):
        ref128, ref64 = oracle.asmble(mesh, g, c, f, py)
        o128 = torch.zeros(g.nzero, dtype=torch.complex128, device=_dev())
        o64 = torch.zeros(g.nzero, dtype=torch.complex64, device=_dev())
        ctx.assemble(c, f, py, o128, o64)
        torch.cuda.synchronize()
        assert np.array_equal(o128.cpu().numpy(), ref128)
        assert np.array_equal(o64.cpu().numpy().view(np.uint32), ref64.view(np.uint32))
    stride = (2 * g.nzero + 15) // 16 * 16
    ring = torch.zeros(len(sel) * stride, dtype=torch.float64, device=_dev())
    ctx.assemble_batch(cft, [p[0] for p in sel], [p[1] for p in sel], ring, stride, len(sel))
    torch.cuda.synchronize()
    r = ring.view(len(sel), stride).cpu().numpy()
    for k, ((f, py), c) in enumerate(zip(sel, cft)):
        ref128, _ = oracle.asmble(mesh, g, c, f, py, want64=False)
        got = r[k, :2 * g.nzero:2] + 1j * r[k, 1:2 * g.nzero:2]
        assert helpers.row_norm_err(got, ref128, g.irptr) <= 1e-12, k


def test_exact_gradient_both_precisions(layout):
    mesh, pairs, g, ctx = layout
    use = [pairs[1], pairs[-2]]
    nsrc = 6
    rng = np.random.default_rng(37)
    shape = (len(use), nsrc, g.ndof)
    u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    lam = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ref = np.zeros((3, mesh.nnpg))
    for p, (f, py) in enumerate(use):
        oracle.grad_exact(mesh, g, f, py, u[p], lam[p], out=ref)
    d_u, d_l = torch.from_numpy(u).to(_dev()), torch.from_numpy(lam).to(_dev())
    for prec, tol in ((FEM25_PREC_FP64, 1e-10), (FEM25_PREC_TF32X3, 2e-5),
                      (FEM25_PREC_TF32X3_POINTWISE, 2e-5)):
        d_g = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
        ctx.gradient([p[0] for p in use], [p[1] for p in use], nsrc, d_u, d_l, d_g, prec)
        got = d_g.cpu().numpy()
        for m in range(3):
            rel = np.linalg.norm(got[m] - ref[m]) / np.linalg.norm(ref[m])
            assert rel <= tol, (prec, m, rel)


def test_reference_gradient(layout):
    mesh, pairs, g, ctx = layout
    rg = oracle.RefGrad(mesh, g)
    rng = np.random.default_rng(41)
    wave = (rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
    lam = (rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
    f, py = pairs[len(pairs) // 3]
    for cinv in ("PP", "SS"):
        fm = rg.cfmat(f, py, wave, lisp=(cinv == "PP"))
        ref = rg.adjflam(fm, lam)
        d_g = torch.zeros(rg.nnpinv, dtype=torch.float32, device=_dev())
        ctx.cfmat_adjgrad(cinv, 1.7320508075688772, f, py, torch.from_numpy(wave).to(_dev()),
                          torch.from_numpy(lam).to(_dev()), d_g)
        assert np.array_equal(d_g.cpu().numpy().view(np.uint32), ref.view(np.uint32)), cinv


def test_dispersive_plain_assembly(layout):
    """KMDAMP / CMDAMP with VCMPLX complex velocities on the distorted layout:
    FP64 CSR and COMPLEX*8 CDIST bit-exact to the oracle."""
    mesh, pairs, _, _ = layout
    dmesh = synth.make_dispersive(mesh, 13)
    g = oracle.graph_build(dmesh)
    ctx = Context(dmesh, g)
    for f, py in (pairs[2], pairs[-3]):
        ref128, ref64 = oracle.asmble(dmesh, g, "B", f, py)
        o128 = torch.zeros(g.nzero, dtype=torch.complex128, device=_dev())
        o64 = torch.zeros(g.nzero, dtype=torch.complex64, device=_dev())
        ctx.assemble("B", f, py, o128, o64)
        torch.cuda.synchronize()
        assert np.array_equal(o128.cpu().numpy(), ref128)
        assert np.array_equal(o64.cpu().numpy().view(np.uint32), ref64.view(np.uint32))
    ctx.close()


def test_hessian_path_kernels(layout):
    """MET225_MOD, CADJ_NU_ALPHA and PCHADJ ('PS') on the distorted layout,
    bit-identical to the oracle."""
    mesh, pairs, g, ctx = layout
    rg = oracle.RefGrad(mesh, g)
    rng = np.random.default_rng(47)
    vec = [(rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
           for _ in range(4)]
    d = [torch.from_numpy(v).to(_dev()) for v in vec]
    f, py = pairs[len(pairs) // 2]
    r1, r2 = rg.met225(f, py, *vec, cinvtype="PS")
    p1 = torch.zeros(r1.shape, dtype=torch.float32, device=_dev())
    p2 = torch.zeros(r2.shape, dtype=torch.float32, device=_dev())
    ctx.met225("PS", f, py, *d, p1, p2)
    assert np.array_equal(p1.cpu().numpy().view(np.uint32), r1.view(np.uint32))
    assert np.array_equal(p2.cpu().numpy().view(np.uint32), r2.view(np.uint32))
    v = rng.standard_normal(2 * rg.nnpinv).astype(np.float32)
    rb, ra, p3 = rg.cadj_nu_alpha(f, py, v, vec[0], vec[3], cinvtype="PS")
    d_b = torch.zeros(g.ndof, dtype=torch.complex64, device=_dev())
    d_a = torch.zeros(g.ndof, dtype=torch.complex64, device=_dev())
    d_p = torch.zeros(p3.shape, dtype=torch.float32, device=_dev())
    ctx.cadj_nu_alpha("PS", f, py, torch.from_numpy(v).to(_dev()), d[0], d[3], d_b, d_a, d_p)
    assert np.array_equal(d_b.cpu().numpy().view(np.uint32), rb.view(np.uint32))
    assert np.array_equal(d_a.cpu().numpy().view(np.uint32), ra.view(np.uint32))
    assert np.array_equal(d_p.cpu().numpy().view(np.uint32), p3.view(np.uint32))
    nrhs = 5
    grns = (rng.standard_normal((nrhs, g.ndof)) + 1j * rng.standard_normal((nrhs, g.ndof))
            ).astype(np.complex64)
    fmat = (rng.standard_normal((2, rg.nz)) + 1j * rng.standard_normal((2, rg.nz))
            ).astype(np.complex64)
    hess = np.zeros(rg.nnpinv * 4, np.float32)
    d_h = torch.zeros(rg.nnpinv * 4, dtype=torch.float32, device=_dev())
    jacl = rg.pchadj(grns, fmat, hess)
    d_j = torch.zeros((rg.nnpinv * 2, nrhs), dtype=torch.complex64, device=_dev())
    ctx.pchadj(2, nrhs, torch.from_numpy(grns).to(_dev()), torch.from_numpy(fmat).to(_dev()),
               d_h, d_j)
    assert np.array_equal(d_j.cpu().numpy().view(np.uint32), jacl.view(np.uint32))
    assert np.array_equal(d_h.cpu().numpy().view(np.uint32), hess.view(np.uint32))
