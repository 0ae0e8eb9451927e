"""The adjoint-gradient check of the 400x120 configuration at full size: the
exact lambda/mu/rho gradient against central finite differences of the L2
misfit through the whole loop on the GPU -- assembly of the 2.3 M-DOF
system, sparse LU (fem25_sparse_factor_dev), forward solve, misfit, adjoint
solve with A^H -- on 10 seeded random directions of the anchor model (away
from the PML, where the gradient is not defined: the damping depends on Vp).

Two (omega, py) pairs, two surface point-force sources each, 20 surface
receivers.  Tolerances: FP64 gradient vs central differences (h = 2e-5
relative, Richardson-extrapolated) <= 1e-6 relative per direction -- the
measured agreement is 1e-10 to 1e-8; at h = 1e-4 the extrapolated
differences still carry their O(h^4) truncation, up to 4e-6 on this 200 km
mesh at 1 Hz, where a relative model change moves the phase of ~100
wavelengths (measured: 4.2e-6, 7.1e-9 and 3.5e-9 at h = 1e-4, 2e-5, 5e-6); split
precision vs the FP64 gradient, per parameter (2-norm): the pointwise form
<= 1e-6 for lambda, mu and rho; the covariance form <= 1e-6 for mu and rho
and <= 1e-5 for lambda.  Its lambda error (2.3e-6 here, 3.8e-6 with 32
sources per pair) is the split operands' precision (about 22 bits of each
deviation) amplified twice by the lambda gradient's divergence, a small
difference of large derivatives for shear-dominated solved fields; the
pointwise form forms each divergence in FP64 and amplifies it once."""
import numpy as np
import pytest

from fem25_b200 import (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE, Context,
                        graph_build, synth)
from tests import helpers

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_fullsize_gradient_against_finite_differences():
    dev = torch.device("cuda:0")
    mesh, pairs, _ = synth.make_config(2)
    g = graph_build(mesh)
    ctx = Context(mesh, g)
    mrdof = helpers.surface_receivers(mesh, g, 20)
    rdofs = torch.from_numpy(mrdof.reshape(-1).astype(np.int64) - 1).to(dev)
    use = [pairs[10], pairs[4 * 64 + 37]]  # 0.2 Hz, and 1.0 Hz at a larger ky
    nsrc = 2
    src = torch.zeros((nsrc, g.ndof), dtype=torch.complex128, device=dev)
    for s, r in enumerate((5, 14)):
        src[s] = torch.from_numpy(helpers.point_force_rhs(g, mrdof[r])).to(dev)
    rng = np.random.default_rng(2027)
    obs = [torch.from_numpy((rng.standard_normal((nsrc, rdofs.numel())) +
                             1j * rng.standard_normal((nsrc, rdofs.numel()))) * 1e-10).to(dev)
           for _ in use]
    a = torch.zeros(g.nzero, dtype=torch.complex128, device=dev)

    def chi_grad(want):
        chi = 0.0
        us, lams = [], []
        for (f, py), ob in zip(use, obs):
            ctx.assemble("B", f, py, a)
            ctx.sparse_factor(a)
            u = src.clone()
            ctx.sparse_solve(u, 0)
            est = u[:, rdofs]
            chi += 0.5 * float(torch.sum(torch.abs(ob - est) ** 2))
            if want:
                lam = torch.zeros_like(u)
                lam[:, rdofs] = ob - est
                ctx.sparse_solve(lam, 2)  # lam = A^{-H} R^T r
                us.append(u)
                lams.append(lam)
        return chi, us, lams

    _, us, lams = chi_grad(True)
    fr, py = [p[0] for p in use], [p[1] for p in use]
    u = torch.stack(us)
    lam = torch.stack(lams)
    g64 = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=dev)
    ctx.gradient(fr, py, nsrc, u, lam, g64, FEM25_PREC_FP64)
    for prec, tols in ((FEM25_PREC_TF32X3_POINTWISE, (1e-6, 1e-6, 1e-6)),
                       (FEM25_PREC_TF32X3, (1e-5, 1e-6, 1e-6))):
        g32 = torch.zeros_like(g64)
        ctx.gradient(fr, py, nsrc, u, lam, g32, prec)
        torch.cuda.synchronize()
        for m in range(3):
            rel = float(torch.linalg.norm(g32[m] - g64[m]) / torch.linalg.norm(g64[m]))
            assert rel <= tols[m], (prec, m, rel)
    grad = g64.cpu().numpy()
    del u, lam, us, lams, g32

    touch = np.zeros(mesh.nnpg, bool)
    for e in range(mesh.nelem):
        if chr(mesh.cdomain[e]) == "A":
            touch[mesh.ieng[e] - 1] = True
    base = np.stack([mesh.ecoeff[0], mesh.ecoeff[1], mesh.dens])

    def chi_at(m3):
        ctx.update_model(m3[:2], m3[2])
        return chi_grad(False)[0]

    h = 2e-5
    for trial in range(10):
        dm = rng.standard_normal((3, mesh.nnpg)) * ~touch * base
        an = float(np.sum(grad * dm))
        fd1 = (chi_at(base + h * dm) - chi_at(base - h * dm)) / (2 * h)
        fd2 = (chi_at(base + h / 2 * dm) - chi_at(base - h / 2 * dm)) / h
        fd = (4 * fd2 - fd1) / 3
        assert abs(fd - an) <= 1e-6 * abs(an), (trial, fd, an)
    ctx.update_model(base[:2], base[2])
    ctx.close()
