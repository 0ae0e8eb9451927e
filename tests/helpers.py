"""Shared test utilities: CSR conversion, error metrics, a direct-solve FWI
loop (scipy SuperLU stands in for MUMPS) used by the finite-difference
gradient checks."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def csr_matrix(g, vals):
    """scipy CSR from the 1-based IRPTR/JCPTR pattern and values."""
    return sp.csr_matrix((vals, g.jcptr - 1, g.irptr - 1), shape=(g.ndof, g.ndof))


def row_norm_err(a, ref, irptr):
    """max over rows of max_j |a - ref| / ||ref_row||_inf (CSR value error)."""
    d = np.abs(np.asarray(a) - np.asarray(ref))
    r = np.abs(np.asarray(ref))
    starts = irptr[:-1] - 1
    dm = np.maximum.reduceat(d, starts)
    rm = np.maximum.reduceat(r, starts)
    rm = np.where(rm > 0, rm, 1.0)
    return float((dm / rm).max())


def surface_receivers(mesh, g, nrec):
    """Receivers at free-surface GLL nodes spread over the interior: MRDOF(3,NREC)."""
    nl = mesh.nord + 1
    top = []
    for e in range(mesh.nelem):
        if chr(mesh.cdomain[e]) != "I":
            continue
        # top edge of element: eta = +1 -> element nodes (nl-1)*nl .. nl*nl-1
        z = mesh.zlocs[mesh.ieng[e, 2] - 1]
        if abs(z - mesh.zlocs.max()) > 1e-6:
            continue
        for ilxi in range(nl - 1):
            a = (nl - 1) * nl + ilxi
            dofs = g.lm[e, a]
            if (dofs > 0).all():
                top.append(tuple(int(d) for d in dofs))
    top = sorted(set(top))
    idx = np.linspace(0, len(top) - 1, nrec).round().astype(int)
    return np.array([top[i] for i in idx], np.int32)


def point_force_rhs(g, mrdof_src, comp=2, amp=1.0):
    """Vertical (z) unit point force at a surface node, built like RESID_DRHS."""
    f = np.zeros(g.ndof, np.complex128)
    f[mrdof_src[comp] - 1] = amp
    return f


class DirectFWI:
    """Assemble (via a callable), factor, solve forward and adjoint problems."""

    def __init__(self, g, mrdof, wghts=None):
        self.g = g
        self.mrdof = mrdof
        self.rdofs = mrdof.reshape(-1) - 1
        self.w = np.ones(len(self.rdofs)) if wghts is None else wghts

    def misfit_and_fields(self, vals, f, obs):
        A = csr_matrix(self.g, vals).tocsc()
        lu = spla.splu(A)
        u = lu.solve(f)
        est = u[self.rdofs]
        res = self.w ** 2 * (obs - est)
        chi = 0.5 * float(np.sum(self.w ** 2 * np.abs(obs - est) ** 2))
        r = np.zeros(self.g.ndof, np.complex128)
        r[self.rdofs] = res
        lam = lu.solve(r, trans="H")  # lam = A^{-H} R^T r
        return chi, u, lam


def sample_rows(mesh, g, per_class=12, seed=0):
    """A seeded set of 1-based CSR rows covering every DOF class of CNMESH
    (PML 'A', Bielak strip 'E', interior 'I', strip boundary 'B'), rows of
    free-surface nodes (topography included) and the first and last rows."""
    rng = np.random.default_rng(seed)
    rows = {1, g.ndof}
    cnp = np.asarray(g.cnp)
    for c in b"AEIB":
        cand = np.nonzero(cnp == c)[0] + 1
        if len(cand):
            rows.update(int(r) for r in rng.choice(cand, min(per_class, len(cand)), replace=False))
    nl = mesh.nord + 1
    fs = np.array([bytes(mesh.cnnpg[p]) == b"FS" for p in range(mesh.nnpg)])
    top = np.nonzero(fs[mesh.ieng[:, 2] - 1] | fs[mesh.ieng[:, 3] - 1])[0]
    surf = set()
    for e in top:
        for ilxi in range(nl):
            surf.update(int(d) for d in g.lm[e, (nl - 1) * nl + ilxi] if d > 0)
    surf = np.array(sorted(surf))
    rows.update(int(r) for r in rng.choice(surf, min(per_class, len(surf)), replace=False))
    return np.array(sorted(rows), np.int64)


def rows_err(a, ref, idx, g, rows):
    """CSR value error of the sampled rows: max over rows of
    max_j |a - ref| / max_j |ref| (the per-row definition of row_norm_err)."""
    lens = (g.irptr[rows] - g.irptr[rows - 1]).astype(np.int64)
    starts = np.concatenate([[0], np.cumsum(lens)[:-1]])
    d = np.abs(np.asarray(a) - np.asarray(ref))
    r = np.abs(np.asarray(ref))
    dm = np.maximum.reduceat(d, starts)
    rm = np.maximum.reduceat(r, starts)
    return float((dm / np.where(rm > 0, rm, 1.0)).max())
