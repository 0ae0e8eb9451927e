"""The Bielak identity of VERIFY_STEVE (asmble.f90:381-433) on solved systems.

With the effective force of ASMB_PEFF (asmble.f90:318-377) as right-hand
side, the solve, and ADDBLK (bielak_utils.f:1116-1125) adding the background
field u0 back on the exterior DOFs, every exterior ('E') row satisfies
    sum_{j in E, B} S_ij u0_j = sum_{j in E, B} S_ij sol_j + sum_{j in A} S_ij sol_j
VERIFY_STEVE sums only the 'E' and 'B' columns (BUFF1, BUFF2), so its
"max difference" is zero (to the solve's precision) on the 'E' rows that
have no PML ('A') column, and equals the PML coupling term on the rows next
to the PML (CNMESH, bielak_utils.f:934-1027, classes the DOFs shared by 'E'
and 'A' elements as 'A').  Both forms are checked, with the oracle's
restatement of VERIFY_STEVE, on
  * an all-oracle chain (assembly, P_eff, ADDBLK; SciPy's sparse LU stands in
    for MUMPS), with a planted sign error in the oracle's P_eff that the
    identity must catch;
  * the library's chain on the GPU: COMPLEX*8 assembly, fem25_peff_dev, the
    GPU direct solve and fem25_addblk_dev.
Tolerance: 1e-4 of max |BUFF1| (COMPLEX*8 matrix and sums; the planted error
gives O(1))."""
import numpy as np
import pytest

import oracle
from fem25_b200 import Context, synth
from tests import helpers


def _case():
    # the 4-element strip of the uneven-batch layout (2 PML + 2 Bielak
    # elements), so that some 'E' rows have no PML column
    mesh, pairs, _ = synth.make_config(4, nx=20, nz=10)
    g = oracle.graph_build(mesh)
    f, py = pairs[40]
    rng = np.random.default_rng(44)
    # a smooth background field (a plane wave with a seeded phase per component)
    nl = mesh.nord + 1
    x = np.zeros(g.ndof)
    for e in range(mesh.nelem):
        xa = mesh.xlocs[mesh.ieng[e] - 1]
        for a in range(nl * nl):
            xi = -1 + 2 * (a % nl) / (nl - 1)
            for d in g.lm[e, a]:
                if d > 0:
                    x[d - 1] = 0.5 * ((1 - xi) * xa[0] + (1 + xi) * xa[1])
    k = 2 * np.pi * f / 3000.0
    u0 = (np.exp(1j * (k * x + rng.uniform(0, 2 * np.pi, 3)[np.arange(g.ndof) % 3]))
          ).astype(np.complex64)
    return mesh, g, f, py, u0


def _identity_errors(g, c64, sol, b1, b2):
    """(error of VERIFY_STEVE on the 'E' rows without PML columns, error of
    the PML-corrected identity on every 'E' row), relative to max |BUFF1|."""
    cnp = np.asarray(g.cnp)
    A = helpers.csr_matrix(g, np.asarray(c64, np.complex128))
    cols_a = (cnp == ord("A")).astype(np.float64)
    touches_a = helpers.csr_matrix(g, np.ones(g.nzero)) @ cols_a > 0
    e_rows = cnp == ord("E")
    pure = e_rows & ~touches_a
    assert pure.sum() > 0 and (e_rows & touches_a).sum() > 0
    solA = np.where(cnp == ord("A"), np.asarray(sol, np.complex128), 0)
    pml = A @ solA
    scale = float(np.abs(b1[e_rows]).max())
    d = np.asarray(b1, np.complex128) - np.asarray(b2, np.complex128)
    return (float(np.abs(d[pure]).max()) / scale,
            float(np.abs(d[e_rows] - pml[e_rows]).max()) / scale)


def test_bielak_identity_oracle_chain():
    mesh, g, f, py, u0 = _case()
    _, c64 = oracle.asmble(mesh, g, "B", f, py)
    A = helpers.csr_matrix(g, c64.astype(np.complex128)).tocsc()
    import scipy.sparse.linalg as spla
    lu = spla.splu(A)

    def chain(peff):
        sol = lu.solve(peff.astype(np.complex128)).astype(np.complex64)
        sol = oracle.addblk(g, u0, sol)
        return sol, oracle.verify_steve(g, c64, u0, sol)

    peff = oracle.peff(g, c64, u0)
    sol, (d, b1, b2) = chain(peff)
    pure, full = _identity_errors(g, c64, sol, b1, b2)
    assert pure <= 1e-4 and full <= 1e-4, (pure, full)
    # planted mistake (in the oracle's force, on the CPU): the 'EB' term with
    # the wrong sign must break the identity
    bad = peff.copy()
    e_rows = np.asarray(g.cnp) == ord("E")
    bad[e_rows] = -bad[e_rows]
    sol_b, (d_b, b1_b, b2_b) = chain(bad)
    pure_b, full_b = _identity_errors(g, c64, sol_b, b1_b, b2_b)
    assert pure_b > 1e-1 and full_b > 1e-1, (pure_b, full_b)


@pytest.mark.gpu
def test_bielak_identity_gpu_chain():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    mesh, g, f, py, u0 = _case()
    ctx = Context(mesh, g)
    try:
        c128 = torch.zeros(g.nzero, dtype=torch.complex128, device=dev)
        c64 = torch.zeros(g.nzero, dtype=torch.complex64, device=dev)
        ctx.assemble("B", f, py, c128, c64)
        d_u0 = torch.from_numpy(u0).to(dev)
        peff = torch.zeros(g.ndof, dtype=torch.complex64, device=dev)
        ctx.asmb_peff(1, c64, d_u0, peff)
        ctx.dense_factor(c128)
        x = peff.to(torch.complex128).contiguous()
        ctx.dense_solve(x)
        sol = x.to(torch.complex64).contiguous()
        ctx.addblk(1, d_u0, sol)
        torch.cuda.synchronize()
        h64, hsol = c64.cpu().numpy(), sol.cpu().numpy()
        d, b1, b2 = oracle.verify_steve(g, h64, u0, hsol)
        pure, full = _identity_errors(g, h64, hsol, b1, b2)
        assert pure <= 1e-4 and full <= 1e-4, (pure, full)
        # the library's force on its own CSR equals the oracle's bit for bit
        assert np.array_equal(peff.cpu().numpy().view(np.uint32),
                              oracle.peff(g, c64.cpu().numpy(), u0).view(np.uint32))
    finally:
        ctx.close()
