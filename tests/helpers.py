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
