"""Direct solve on the GPU for small meshes (fem25_dense_factor_dev /
fem25_dense_solve_dev): agreement with a host sparse LU, and the whole
assemble -> solve -> misfit -> adjoint solve -> gradient loop on the device
checked against central finite differences.

Tolerances: solution vs host sparse LU <= 1e-9 relative (2-norm, both are
backward-stable LUs of the same matrix); residual ||op(A) x - b|| / ||b||
<= 1e-12; gradient vs central differences (h = 1e-4 relative,
Richardson-extrapolated) <= 1e-6 relative.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import oracle
from fem25_b200 import FEM25_PREC_FP64, Context, Fem25Error, synth
from tests import helpers

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dev():
    return torch.device("cuda:0")


def test_dense_solve_matches_host_lu():
    mesh, pairs, _ = synth.make_config(0, nx=12, nz=6)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    f, py = pairs[7]
    a = torch.zeros(g.nzero, dtype=torch.complex128, device=_dev())
    ctx.assemble("B", f, py, a)
    ctx.dense_factor(a)
    A = helpers.csr_matrix(g, a.cpu().numpy()).tocsc()
    lu = spla.splu(A)
    rng = np.random.default_rng(17)
    b = rng.standard_normal((3, g.ndof)) + 1j * rng.standard_normal((3, g.ndof))
    for trans, op, mat in ((0, "N", A), (1, "T", A.T), (2, "H", A.conj().T)):
        x = torch.from_numpy(b).to(_dev())
        ctx.dense_solve(x, trans)
        got = x.cpu().numpy()
        for k in range(3):
            ref = lu.solve(b[k], trans=op)
            assert np.linalg.norm(got[k] - ref) <= 1e-9 * np.linalg.norm(ref), (trans, k)
            res = mat @ got[k] - b[k]
            assert np.linalg.norm(res) <= 1e-12 * np.linalg.norm(b[k]), (trans, k)
    ctx.close()


def test_dense_solve_requires_factor_and_valid_op():
    mesh, pairs, _ = synth.make_config(0, nx=6, nz=4)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    x = torch.zeros((1, g.ndof), dtype=torch.complex128, device=_dev())
    with pytest.raises(Fem25Error):
        ctx.dense_solve(x, 0)
    with pytest.raises(Fem25Error):
        ctx.dense_solve(x, 3)
    ctx.close()


def test_finite_difference_loop_on_device():
    """GPU assembly, GPU LU, L2 misfit (torch, FP64), GPU adjoint solve with
    A^H, GPU exact gradient vs central differences of the misfit."""
    mesh, pairs, _ = synth.make_config(0, nx=12, nz=6)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    mrdof = helpers.surface_receivers(mesh, g, 8)
    rdofs = torch.from_numpy(mrdof.reshape(-1).astype(np.int64) - 1).to(_dev())
    use = [pairs[3], pairs[10]]
    rng = np.random.default_rng(8)
    f_src = torch.from_numpy(helpers.point_force_rhs(g, mrdof[len(mrdof) // 2])).to(_dev())
    obs = [torch.from_numpy((rng.standard_normal(rdofs.numel()) +
                             1j * rng.standard_normal(rdofs.numel())) * 1e-9).to(_dev())
           for _ in use]
    a = torch.zeros(g.nzero, dtype=torch.complex128, device=_dev())

    def chi_grad(want):
        chi = 0.0
        grad = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
        for (f, py), ob in zip(use, obs):
            ctx.assemble("B", f, py, a)
            ctx.dense_factor(a)
            u = f_src.clone().view(1, -1)
            ctx.dense_solve(u, 0)
            est = u[0, rdofs]
            chi += 0.5 * float(torch.sum(torch.abs(ob - est) ** 2))
            if want:
                lam = torch.zeros_like(u)
                lam[0, rdofs] = ob - est
                ctx.dense_solve(lam, 2)  # lam = A^{-H} R^T r
                ctx.gradient([f], [py], 1, u.view(1, 1, -1), lam.view(1, 1, -1), grad,
                             FEM25_PREC_FP64)
        return chi, grad.cpu().numpy()

    _, grad = chi_grad(True)
    touch = np.zeros(mesh.nnpg, bool)
    for e in range(mesh.nelem):
        if chr(mesh.cdomain[e]) == "A":
            touch[mesh.ieng[e] - 1] = True
    base = np.stack([mesh.ecoeff[0], mesh.ecoeff[1], mesh.dens])

    def chi_at(m3):
        ctx.update_model(m3[:2], m3[2])
        return chi_grad(False)[0]

    h = 1e-4
    for trial in range(2):
        dm = rng.standard_normal((3, mesh.nnpg)) * ~touch * base
        an = float(np.sum(grad * dm))
        fd1 = (chi_at(base + h * dm) - chi_at(base - h * dm)) / (2 * h)
        fd2 = (chi_at(base + h / 2 * dm) - chi_at(base - h / 2 * dm)) / h
        fd = (4 * fd2 - fd1) / 3
        assert abs(fd - an) <= 1e-6 * abs(an), (trial, fd, an)
    ctx.update_model(base[:2], base[2])
    ctx.close()
