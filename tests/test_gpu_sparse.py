"""Sparse direct solve on the GPU (fem25_sparse_factor_dev /
fem25_sparse_solve_dev): the multifrontal LU against the dense GPU LU and a
host sparse LU on small meshes, residuals on the full small configuration and
a medium mesh, all three operators (A, A^T, A^H), and the finite-difference
loop of the gradient with the sparse solve in place of the dense one.

Tolerances: solution vs host / dense LU <= 1e-9 relative (2-norm; backward-
stable LUs of the same matrix); residual ||op(A) x - b|| / ||b|| <= 1e-11
(1e-10 on the medium mesh, whose matrix spans a wider range of scales);
gradient vs central differences (h = 1e-4 relative, Richardson-extrapolated)
<= 1e-6 relative.
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


def _rhs(ndof, n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, ndof)) + 1j * rng.standard_normal((n, ndof))


@pytest.mark.parametrize("cftype", ["B", "S"])
def test_sparse_solve_matches_host_and_dense_lu(cftype):
    mesh, pairs, _ = synth.make_config(0, nx=12, nz=6)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    f, py = pairs[7]
    a = torch.zeros(g.nzero, dtype=torch.complex128, device=_dev())
    ctx.assemble(cftype, f, py, a)
    ctx.sparse_factor(a)
    ctx.dense_factor(a)
    A = helpers.csr_matrix(g, a.cpu().numpy()).tocsc()
    lu = spla.splu(A)
    b = _rhs(g.ndof, 3, 17)
    for trans, op, mat in ((0, "N", A), (1, "T", A.T), (2, "H", A.conj().T)):
        x = torch.from_numpy(b).to(_dev())
        ctx.sparse_solve(x, trans)
        xd = torch.from_numpy(b).to(_dev())
        ctx.dense_solve(xd, trans)
        got, dense = x.cpu().numpy(), xd.cpu().numpy()
        for k in range(3):
            ref = lu.solve(b[k], trans=op)
            assert np.linalg.norm(got[k] - ref) <= 1e-9 * np.linalg.norm(ref), (trans, k)
            assert np.linalg.norm(got[k] - dense[k]) <= 1e-9 * np.linalg.norm(ref), (trans, k)
            res = mat @ got[k] - b[k]
            assert np.linalg.norm(res) <= 1e-11 * np.linalg.norm(b[k]), (trans, k)
    fronts, levels, fac_bytes, work_bytes, kmax, nmax, flops = ctx.sparse_info()
    assert fronts > 1 and levels > 1 and fac_bytes > 0 and kmax <= nmax and flops > 0
    ctx.close()


@pytest.mark.parametrize("cfg, nx, nz, tol", [(0, None, None, 1e-11), (1, 100, 40, 1e-10)])
def test_sparse_solve_residuals(cfg, nx, nz, tol):
    """The full small configuration (40x20, 39 k DOF) and the layered mesh at
    100x40 (192 k DOF, beyond the dense solve): residuals of 9 right-hand
    sides (more than one solve CTA group) for each operator; refactoring a
    second system reuses the analysis."""
    mesh, pairs, _ = synth.make_config(cfg, nx=nx, nz=nz)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    a = torch.zeros(g.nzero, dtype=torch.complex128, device=_dev())
    for f, py in (pairs[3], pairs[-2]):
        ctx.assemble("B", f, py, a)
        ctx.sparse_factor(a)
        A = helpers.csr_matrix(g, a.cpu().numpy())
        b = _rhs(g.ndof, 9, 5)
        for trans, mat in ((0, A), (1, A.T.tocsr()), (2, A.conj().T.tocsr())):
            x = torch.from_numpy(b).to(_dev())
            ctx.sparse_solve(x, trans)
            got = x.cpu().numpy()
            for k in range(9):
                res = mat @ got[k] - b[k]
                assert np.linalg.norm(res) <= tol * np.linalg.norm(b[k]), (f, trans, k)
    ctx.close()


def test_sparse_solve_requires_factor_and_valid_op():
    mesh, pairs, _ = synth.make_config(0, nx=6, nz=4)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    x = torch.zeros((1, g.ndof), dtype=torch.complex128, device=_dev())
    with pytest.raises(Fem25Error):
        ctx.sparse_solve(x, 0)
    with pytest.raises(Fem25Error):
        ctx.sparse_solve(x, 3)
    ctx.close()


def test_sparse_solve_rejects_a_singular_matrix():
    """A zero matrix has a zero pivot in its first front: refused with
    FEM25_ERR_ARG, and the context factors a regular system afterwards."""
    mesh, pairs, _ = synth.make_config(0, nx=6, nz=4)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    a = torch.zeros(g.nzero, dtype=torch.complex128, device=_dev())
    with pytest.raises(Fem25Error) as ei:
        ctx.sparse_factor(a)
    assert ei.value.code == 1
    f, py = pairs[2]
    ctx.assemble("B", f, py, a)
    ctx.sparse_factor(a)
    x = torch.ones((1, g.ndof), dtype=torch.complex128, device=_dev())
    ctx.sparse_solve(x, 0)
    A = helpers.csr_matrix(g, a.cpu().numpy())
    assert np.linalg.norm(A @ x.cpu().numpy()[0] - 1.0) <= 1e-11 * np.sqrt(g.ndof)
    ctx.close()


def test_finite_difference_loop_with_sparse_solve():
    """GPU assembly, GPU sparse LU, L2 misfit, adjoint solve with A^H, GPU
    exact gradient vs central differences of the misfit."""
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
            ctx.sparse_factor(a)
            u = f_src.clone().view(1, -1)
            ctx.sparse_solve(u, 0)
            est = u[0, rdofs]
            chi += 0.5 * float(torch.sum(torch.abs(ob - est) ** 2))
            if want:
                lam = torch.zeros_like(u)
                lam[0, rdofs] = ob - est
                ctx.sparse_solve(lam, 2)  # lam = A^{-H} R^T r
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
