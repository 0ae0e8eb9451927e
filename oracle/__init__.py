"""ctypes bindings for the CPU oracle (``oracle/fem25_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline / reference legs of ``bench.py``, to compare against.  The
product library (``fem25_b200``) never imports, links or executes it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
                os.path.join(_HERE, "fem25_oracle.c")):
            build()
        _lib = C.CDLL(_LIB)
        _setup(_lib)
    return _lib


class OrcMesh(C.Structure):
    _fields_ = [("nelem", C.c_int), ("nnpg", C.c_int), ("nord", C.c_int),
                ("ieng", C.c_void_p), ("cdomain", C.c_void_p), ("cnnpg", C.c_void_p),
                ("xlocs", C.c_void_p), ("zlocs", C.c_void_p), ("xd", C.c_void_p),
                ("zd", C.c_void_p), ("ecoeff", C.c_void_p), ("dens", C.c_void_p),
                ("xwidth", C.c_double), ("zwidth", C.c_double),
                ("rcoeff", C.c_double * 2), ("dmax", C.c_double * 2),
                ("kappa", C.c_double * 2), ("fcent", C.c_double * 2),
                ("ldisp", C.c_int), ("qp", C.c_void_p), ("qs", C.c_void_p),
                ("freq0", C.c_double)]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _setup(L):
    vp = C.c_void_p
    L.orc_lobatto.argtypes = [C.c_int, vp, vp]
    L.orc_genpts.argtypes = [C.c_int, vp]
    L.orc_tables.argtypes = [C.c_int, vp, vp]
    L.orc_element_matrix.argtypes = [vp, C.c_int, C.c_char, C.c_double, C.c_double, vp, vp]
    L.orc_asmble.argtypes = [vp, vp, vp, vp, C.c_int, C.c_char, C.c_double, C.c_double,
                             C.c_int, C.c_int, vp, vp]
    L.orc_asmble_rows.argtypes = [vp, vp, vp, vp, C.c_int, vp, C.c_char, C.c_double,
                                  C.c_double, vp, vp]
    L.orc_graph_build.argtypes = [vp, C.POINTER(C.c_int)]
    L.orc_graph_build.restype = vp
    L.orc_graph_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_longlong), C.POINTER(C.c_int)]
    L.orc_graph_copy.argtypes = [vp, vp, vp, vp, vp, vp]
    L.orc_graph_free.argtypes = [vp]
    L.orc_peff.argtypes = [C.c_int, vp, vp, vp, vp, vp, vp]
    L.orc_addblk.argtypes = [C.c_int, vp, vp, vp]
    L.orc_grad_exact.argtypes = [vp, vp, C.c_int, C.c_double, C.c_double, C.c_int, vp, vp, vp]
    L.orc_gengmask.argtypes = [vp, vp, C.c_int, vp, vp, C.POINTER(C.c_int)]
    L.orc_ncon_anchor.argtypes = [vp]
    L.orc_elem_wts.argtypes = [vp, vp, vp, C.c_int, vp]
    L.orc_gradptrs.argtypes = [vp, vp, C.c_int, vp, vp, C.c_int, vp, vp]
    L.orc_gradptrs.restype = C.c_longlong
    L.orc_cfmat_dist.argtypes = [vp, vp, C.c_int, vp, vp, C.c_int, vp, vp, vp, C.c_int,
                                 C.c_double, C.c_double, C.c_double, vp, vp, C.c_int]
    L.orc_adjflam.argtypes = [C.c_int, vp, vp, vp, vp, vp]
    L.orc_dabm_element.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_double, vp, vp, vp, vp]
    L.orc_vforce2.argtypes = [vp, vp, vp, vp, C.c_int, vp, vp, C.c_longlong, C.c_int, C.c_int,
                              C.c_double, C.c_double, vp, vp]
    L.orc_cadj_nu_alpha.argtypes = [vp, vp, C.c_int, vp, vp, C.c_int, vp, vp, vp, C.c_int,
                                    C.c_int, C.c_double, C.c_double, vp, vp, vp, C.c_int, vp,
                                    vp, vp]
    L.orc_pchadj.argtypes = [C.c_int, C.c_int, C.c_longlong, C.c_int, C.c_int, vp, vp, vp, vp,
                             vp, vp]
    L.orc_met225.argtypes = [vp, vp, vp, vp, C.c_int, vp, vp, vp, C.c_int, C.c_int, C.c_double,
                             C.c_double, vp, vp, vp, vp, C.c_int, vp, vp]
    L.orc_misfit.argtypes = [C.c_int, C.c_int, vp, vp, C.c_double, C.c_double, C.c_double,
                             vp, vp, vp, vp, vp, vp]
    L.orc_misfit.restype = C.c_float


class OracleMesh:
    """Holds the numpy arrays alive and the C struct that points at them."""

    def __init__(self, mesh):
        self.keep = dict(
            ieng=np.ascontiguousarray(mesh.ieng, np.int32),
            cdomain=np.ascontiguousarray(mesh.cdomain, np.uint8),
            cnnpg=np.ascontiguousarray(mesh.cnnpg, np.uint8),
            xlocs=np.ascontiguousarray(mesh.xlocs, np.float64),
            zlocs=np.ascontiguousarray(mesh.zlocs, np.float64),
            xd=np.ascontiguousarray(mesh.xd, np.float64),
            zd=np.ascontiguousarray(mesh.zd, np.float64),
            ecoeff=np.ascontiguousarray(mesh.ecoeff, np.float64),
            dens=np.ascontiguousarray(mesh.dens, np.float64))
        q9 = np.full(mesh.nnpg, 9999.0)
        self.keep["qp"] = np.ascontiguousarray(q9 if mesh.qp is None else mesh.qp, np.float64)
        self.keep["qs"] = np.ascontiguousarray(q9 if mesh.qs is None else mesh.qs, np.float64)
        k = self.keep
        s = OrcMesh()
        s.nelem, s.nnpg, s.nord = mesh.nelem, mesh.nnpg, mesh.nord
        for f in ("ieng", "cdomain", "cnnpg", "xlocs", "zlocs", "xd", "zd", "ecoeff", "dens"):
            setattr(s, f, _p(k[f]))
        s.xwidth, s.zwidth = mesh.xwidth, mesh.zwidth
        for f in ("rcoeff", "dmax", "kappa", "fcent"):
            getattr(s, f)[0], getattr(s, f)[1] = getattr(mesh, f)
        s.ldisp = 1 if mesh.ldisp else 0
        s.qp, s.qs = _p(k["qp"]), _p(k["qs"])
        s.freq0 = mesh.freq0
        self.s = s
        self.mesh = mesh
        self.ptr = C.cast(C.pointer(s), C.c_void_p)


class Graph:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def graph_build(mesh):
    L = lib()
    om = OracleMesh(mesh)
    ierr = C.c_int(0)
    h = L.orc_graph_build(om.ptr, C.byref(ierr))
    if ierr.value != 0:
        L.orc_graph_free(h)
        raise RuntimeError(f"oracle graph build failed: ierr={ierr.value}")
    nnp, ndof, ncon = C.c_int(), C.c_int(), C.c_int()
    nz = C.c_longlong()
    L.orc_graph_info(h, C.byref(nnp), C.byref(ndof), C.byref(nz), C.byref(ncon))
    nen = (mesh.nord + 1) ** 2
    ien = np.empty((mesh.nelem, nen), np.int32)
    lm = np.empty((mesh.nelem, nen, 3), np.int32)
    irptr = np.empty(ndof.value + 1, np.int32)
    jcptr = np.empty(nz.value, np.int32)
    cnp = np.empty(ndof.value, np.uint8)
    L.orc_graph_copy(h, _p(ien), _p(lm), _p(irptr), _p(jcptr), _p(cnp))
    L.orc_graph_free(h)
    return Graph(nnp=nnp.value, ndof=ndof.value, nzero=nz.value, ncon=ncon.value, ien=ien,
                 lm=lm, irptr=irptr, jcptr=jcptr, cnp=cnp)


def tables(nord=4):
    nint = 2 * nord + 5
    nen = (nord + 1) ** 2
    xigll = np.empty(2 * nint)
    shl = np.empty(3 * nen * nint * nint)
    lib().orc_tables(nord, _p(xigll), _p(shl))
    return xigll.reshape(2, nint), shl.reshape(nint, nint, nen, 3)


def lobatto(n):
    x = np.empty(n)
    w = np.empty(n)
    lib().orc_lobatto(n, _p(x), _p(w))
    return x, w


def element_matrix(mesh, ielem, cftype, freq, py):
    om = OracleMesh(mesh)
    nee = 3 * (mesh.nord + 1) ** 2
    me = np.empty((nee, nee), order="F")
    ce = np.empty((nee, nee), np.complex128, order="F")
    ierr = lib().orc_element_matrix(om.ptr, ielem, cftype.encode(), freq, py, _p(me), _p(ce))
    if ierr:
        raise RuntimeError(f"element {ielem}: Jacobian check failed")
    return me, ce


def dabm_element(mesh, ielem, inpg, freq, py):
    """DABMKISOB25 (dM/dalpha, dK/dalpha, dM/dbeta, dK/dbeta) of one element
    for anchor ``inpg`` (1-based), column-major 75x75."""
    om = OracleMesh(mesh)
    nee = 3 * (mesh.nord + 1) ** 2
    out = [np.empty((nee, nee), order="F"), np.empty((nee, nee), np.complex128, order="F"),
           np.empty((nee, nee), order="F"), np.empty((nee, nee), np.complex128, order="F")]
    ierr = lib().orc_dabm_element(om.ptr, ielem, inpg, freq, py, *[_p(a) for a in out])
    if ierr:
        raise RuntimeError(f"element {ielem}: Jacobian check failed")
    return out


def asmble(mesh, g, cftype, freq, py, elo=0, ehi=None, want64=True, want128=True, out=None):
    """ASMBLE_DRIVER over elements [elo, ehi): (csr128, csr64).  ``out`` =
    (csr128, csr64) arrays to add into instead of fresh zeroed ones (either
    may be None, which skips that output)."""
    om = OracleMesh(mesh)
    ehi = mesh.nelem if ehi is None else ehi
    if out is not None:
        c128, c64 = out
    else:
        c128 = np.zeros(g.nzero, np.complex128) if want128 else None
        c64 = np.zeros(g.nzero, np.complex64) if want64 else None
    ierr = lib().orc_asmble(om.ptr, _p(g.lm), _p(g.irptr), _p(g.jcptr), g.ndof,
                            cftype.encode(), freq, py, elo, ehi,
                            _p(c128) if c128 is not None else None,
                            _p(c64) if c64 is not None else None)
    if ierr:
        raise RuntimeError(f"oracle asmble ierr={ierr}")
    return c128, c64


def asmble_rows(mesh, g, rows, cftype, freq, py):
    """CSR values of the given 1-based DOF rows only: (idx, csr128, csr64) with
    idx the 0-based CSR positions of the rows' entries (rows in the given
    order, each in JCPTR order) and the values at those positions, equal bit
    for bit to the full ``asmble`` there."""
    om = OracleMesh(mesh)
    rows = np.asarray(rows, np.int64)
    if len(np.unique(rows)) != len(rows) or rows.min() < 1 or rows.max() > g.ndof:
        raise ValueError("rows must be distinct 1-based DOFs")
    starts = g.irptr[rows - 1].astype(np.int64) - 1
    lens = (g.irptr[rows] - g.irptr[rows - 1]).astype(np.int64)
    rowoff = np.full(g.ndof, -1, np.int64)
    rowoff[rows - 1] = np.concatenate([[0], np.cumsum(lens)[:-1]])
    n = int(lens.sum())
    idx = np.concatenate([np.arange(s0, s0 + l) for s0, l in zip(starts, lens)])
    c128 = np.zeros(n, np.complex128)
    c64 = np.zeros(n, np.complex64)
    ierr = lib().orc_asmble_rows(om.ptr, _p(np.ascontiguousarray(g.lm, np.int32)),
                                 _p(np.ascontiguousarray(g.irptr, np.int32)),
                                 _p(np.ascontiguousarray(g.jcptr, np.int32)), g.ndof, _p(rowoff),
                                 cftype.encode(), freq, py, _p(c128), _p(c64))
    if ierr:
        raise RuntimeError(f"oracle asmble_rows ierr={ierr}")
    return idx, c128, c64


def peff(g, cdist64, ue64):
    out = np.zeros(g.ndof, np.complex64)
    lib().orc_peff(g.ndof, _p(g.irptr), _p(g.jcptr), _p(g.cnp),
                   _p(np.ascontiguousarray(cdist64, np.complex64)),
                   _p(np.ascontiguousarray(ue64, np.complex64)), _p(out))
    return out


def addblk(g, ue64, sol64):
    """ADDBLK: sol + ue on the 'E' DOFs (COMPLEX*8), returned as a new array."""
    out = np.array(sol64, np.complex64, copy=True)
    lib().orc_addblk(g.ndof, _p(g.cnp), _p(np.ascontiguousarray(ue64, np.complex64)), _p(out))
    return out


def verify_steve(g, cdist64, u0, sol):
    """VERIFY_STEVE: (DIF1, BUFF1, BUFF2) of the Bielak identity on the 'E'
    rows for the COMPLEX*8 CSR, background field u0 and total solution sol."""
    L = lib()
    L.orc_verify_steve.restype = C.c_float
    L.orc_verify_steve.argtypes = [C.c_int] + [C.c_void_p] * 8
    b1 = np.zeros(g.ndof, np.complex64)
    b2 = np.zeros(g.ndof, np.complex64)
    d = L.orc_verify_steve(g.ndof, _p(g.irptr), _p(g.jcptr), _p(g.cnp),
                           _p(np.ascontiguousarray(cdist64, np.complex64)),
                           _p(np.ascontiguousarray(u0, np.complex64)),
                           _p(np.ascontiguousarray(sol, np.complex64)), _p(b1), _p(b2))
    return float(d), b1, b2


def grad_exact(mesh, g, freq, py, u, lam, out=None):
    """g[3, nnpg] += sum_s Re(lam_s^H dA/dm u_s); u, lam complex128 [nsrc, ndof]."""
    om = OracleMesh(mesh)
    u = np.ascontiguousarray(u, np.complex128)
    lam = np.ascontiguousarray(lam, np.complex128)
    if out is None:
        out = np.zeros((3, mesh.nnpg))
    ierr = lib().orc_grad_exact(om.ptr, _p(g.lm), g.ndof, freq, py, u.shape[0], _p(u), _p(lam),
                                _p(out))
    if ierr:
        raise RuntimeError("oracle grad ierr")
    return out


class RefGrad:
    """GENGMASK / ELEM_WTS / GRADPTRS products for the reference-compatible gradient."""

    def __init__(self, mesh, g):
        L = lib()
        om = OracleMesh(mesh)
        self.om = om
        ncon = L.orc_ncon_anchor(om.ptr)
        self.maskg = np.zeros(mesh.nnpg, np.int32)
        self.mconn = np.zeros((ncon, mesh.nnpg), np.int32)  # MCONN(NNPG,NCON) col-major
        nc = C.c_int()
        self.nnpinv = L.orc_gengmask(om.ptr, _p(g.lm), mesh.nord, _p(self.maskg), _p(self.mconn),
                                     C.byref(nc))
        self.ncon = nc.value
        self.elem_wts = np.zeros(mesh.nelem)
        L.orc_elem_wts(om.ptr, _p(self.maskg), _p(self.mconn), self.ncon, _p(self.elem_wts))
        nz = L.orc_gradptrs(om.ptr, _p(g.lm), mesh.nord, _p(self.maskg), _p(self.mconn),
                            self.ncon, None, None)
        self.jcsc = np.zeros(self.nnpinv + 1, np.int32)
        self.icsc = np.zeros(nz, np.int32)
        L.orc_gradptrs(om.ptr, _p(g.lm), mesh.nord, _p(self.maskg), _p(self.mconn), self.ncon,
                       _p(self.jcsc), _p(self.icsc))
        self.nz = nz
        self.g = g
        self.mesh = mesh

    def cfmat(self, freq, py, wave64, lisp=True, vpvs=1.7320508075688772,
              accumulate=False):
        out = np.zeros(self.nz, np.complex64)
        ierr = lib().orc_cfmat_dist(self.om.ptr, _p(self.g.lm), self.g.ndof, _p(self.maskg),
                                    _p(self.mconn), self.ncon, _p(self.elem_wts), _p(self.jcsc),
                                    _p(self.icsc), 1 if lisp else 0, vpvs, freq, py,
                                    _p(np.ascontiguousarray(wave64, np.complex64)), _p(out),
                                    1 if accumulate else 0)
        if ierr:
            raise RuntimeError(f"oracle cfmat ierr={ierr}")
        return out

    def vforce2(self, freq, py, wave64, cinvtype="PP"):
        """VFORCE25_2 forces with DABMKISOB25 matrices: COMPLEX*8 [nvinv, nz]."""
        lisp = cinvtype.upper() in ("PP", "PS")
        liss = cinvtype.upper() in ("SS", "PS")
        out = np.zeros((int(lisp) + int(liss), self.nz), np.complex64)
        ierr = lib().orc_vforce2(self.om.ptr, _p(self.g.lm), _p(self.maskg), _p(self.mconn),
                                 self.ncon, _p(self.jcsc), _p(self.icsc), self.nz, int(lisp),
                                 int(liss), freq, py,
                                 _p(np.ascontiguousarray(wave64, np.complex64)), _p(out))
        if ierr:
            raise RuntimeError(f"oracle vforce2 ierr={ierr}")
        return out

    def met225(self, freq, py, adjlam64, nu64, alpha64, wave64, cinvtype="PP",
               accumulate=False):
        """MET225_MOD: (P1BUF, P2BUF) REAL*4 [nnpinv * nvinv] (alpha before beta)."""
        lisp = cinvtype.upper() in ("PP", "PS")
        liss = cinvtype.upper() in ("SS", "PS")
        nv = int(lisp) + int(liss)
        p1 = np.zeros(self.nnpinv * nv, np.float32)
        p2 = np.zeros(self.nnpinv * nv, np.float32)
        c64 = lambda x: _p(np.ascontiguousarray(x, np.complex64))
        ierr = lib().orc_met225(self.om.ptr, _p(self.g.lm), _p(self.maskg), _p(self.mconn),
                                self.ncon, _p(self.elem_wts), _p(self.jcsc), _p(self.icsc),
                                int(lisp), int(liss), freq, py, c64(adjlam64), c64(nu64),
                                c64(alpha64), c64(wave64), 1 if accumulate else 0, _p(p1), _p(p2))
        if ierr:
            raise RuntimeError(f"oracle met225 ierr={ierr}")
        return p1, p2

    def cadj_nu_alpha(self, freq, py, v, adjlam64, wave64, cinvtype="PP", accumulate=False):
        """CADJ_NU_ALPHA without its solves: (RHSBNU, RHSALP) COMPLEX*8 [ndof] and
        P3 REAL*4 [nnpinv * nvinv]; v: REAL*4 [nnpinv * nvinv]."""
        lisp = cinvtype.upper() in ("PP", "PS")
        liss = cinvtype.upper() in ("SS", "PS")
        nv = int(lisp) + int(liss)
        rb = np.zeros(self.g.ndof, np.complex64)
        ra = np.zeros(self.g.ndof, np.complex64)
        p3 = np.zeros(self.nnpinv * nv, np.float32)
        c64 = lambda x: _p(np.ascontiguousarray(x, np.complex64))
        ierr = lib().orc_cadj_nu_alpha(self.om.ptr, _p(self.g.lm), self.g.ndof, _p(self.maskg),
                                       _p(self.mconn), self.ncon, _p(self.elem_wts),
                                       _p(self.jcsc), _p(self.icsc), int(lisp), int(liss), freq,
                                       py, _p(np.ascontiguousarray(v, np.float32)), c64(adjlam64),
                                       c64(wave64), 1 if accumulate else 0, _p(rb), _p(ra), _p(p3))
        if ierr:
            raise RuntimeError(f"oracle cadj_nu_alpha ierr={ierr}")
        return rb, ra, p3

    def pchadj(self, grns64, fmat64, hessb, want_jacl=True):
        """PCHADJ after the Green's-function solve: HESSB updated in place
        (REAL*4 [nnpinv * nvinv^2]), returns JACL COMPLEX*8 [nnpinv*nvinv, nrhs]."""
        fm = np.ascontiguousarray(fmat64, np.complex64).reshape(-1, self.nz)
        nv = fm.shape[0]
        gr = np.ascontiguousarray(grns64, np.complex64).reshape(-1, self.g.ndof)
        jacl = np.zeros((self.nnpinv * nv, gr.shape[0]), np.complex64) if want_jacl else None
        lib().orc_pchadj(self.nnpinv, nv, self.nz, self.g.ndof, gr.shape[0], _p(self.jcsc),
                         _p(self.icsc), _p(gr), _p(fm), _p(hessb),
                         _p(jacl) if jacl is not None else None)
        return jacl

    def avgrad(self, nvinv, ncasc, grad):
        """AVGRAD (float32 grad) or AVGRAD8 (float64 grad): a smoothed copy."""
        L = lib()
        g = np.array(grad, copy=True)
        ieng = np.ascontiguousarray(self.mesh.ieng, np.int32)
        fn = L.orc_avgrad8 if g.dtype == np.float64 else L.orc_avgrad
        fn.argtypes = [C.c_int] * 4 + [C.c_void_p] * 3 + [C.c_int, C.c_void_p]
        fn(self.mesh.nnpg, self.ncon, nvinv, ncasc, _p(self.maskg), _p(self.mconn), _p(ieng),
           g.size, _p(g))
        return g

    def adjflam(self, fmat, adjlam64, gradl=None):
        if gradl is None:
            gradl = np.zeros(self.nnpinv, np.float32)
        lib().orc_adjflam(self.nnpinv, _p(self.jcsc), _p(self.icsc),
                          _p(np.ascontiguousarray(fmat, np.complex64)),
                          _p(np.ascontiguousarray(adjlam64, np.complex64)), _p(gradl))
        return gradl


def wtgrad(wgrad, grad):
    """WTGRAD: grad * wgrad in REAL*4 (a new array)."""
    g = np.array(grad, np.float32, copy=True)
    lib().orc_wtgrad.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
    lib().orc_wtgrad(g.size, _p(np.ascontiguousarray(wgrad, np.float32)), _p(g))
    return g


def misfit(ndof, mrdof, yrec, freq, py, azmod, recv, sol64, obs, wghts, norm=2, irestp=3,
           ibphase=0, eps=0.0, thresh=0.0, dtmax=0.0, dtmax_obj=0.0):
    """(est[nrec,3] c64, rhs[ndof] c64, the source's sum of COBJ4 terms)."""
    L = lib()
    L.orc_misfit_opt.restype = C.c_float
    L.orc_misfit_opt.argtypes = ([C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                  C.c_double, C.c_double] + [C.c_void_p] * 4 +
                                 [C.c_int] * 3 + [C.c_float] * 4 + [C.c_void_p] * 2)
    nrec = mrdof.shape[0]
    est = np.zeros((nrec, 3), np.complex64)
    rhs = np.zeros(ndof, np.complex64)
    val = L.orc_misfit_opt(ndof, nrec, _p(np.ascontiguousarray(mrdof, np.int32)),
                           _p(np.ascontiguousarray(yrec, np.float64)), freq, py, azmod,
                           _p(np.ascontiguousarray(recv, np.complex64)),
                           _p(np.ascontiguousarray(sol64, np.complex64)),
                           _p(np.ascontiguousarray(obs, np.complex64)),
                           _p(np.ascontiguousarray(wghts, np.float32)), norm, irestp, ibphase,
                           eps, thresh, dtmax, dtmax_obj, _p(est), _p(rhs))
    return est, rhs, float(val)


def hdiffer(ibphase, freq):
    """HDIFFER(IBPHASE, FREQ) as COMPLEX*8."""
    L = lib()
    L.orc_hdiffer.argtypes = [C.c_int, C.c_double, C.c_void_p]
    h = np.zeros(2, np.float32)
    L.orc_hdiffer(ibphase, freq, _p(h))
    return complex(h[0], h[1])
