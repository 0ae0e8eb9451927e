"""ctypes binding of libfem25gpu.so and the host-side context object."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfem25gpu.so")

FEM25_OK = 0
FEM25_PREC_FP64 = 0
FEM25_PREC_TF32X3 = 1
FEM25_PREC_TF32X3_POINTWISE = 2
_CODES = {1: "ERR_ARG", 2: "ERR_JACOBIAN", 3: "ERR_PATTERN", 4: "ERR_CUDA", 5: "ERR_ALLOC",
          6: "ERR_GRAPH", 7: "ERR_UNSUPPORTED", 8: "ERR_NOMESH"}


class Fem25Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fem25 {_CODES.get(code, code)} ({code}): {msg}")
        self.code = code


class Mesh(C.Structure):
    _fields_ = [("nelem", C.c_int), ("nnpg", C.c_int), ("nord", C.c_int), ("ldisp", C.c_int),
                ("ieng", C.c_void_p), ("cdomain", C.c_void_p), ("cnnpg", C.c_void_p),
                ("xlocs", C.c_void_p), ("zlocs", C.c_void_p), ("xd", C.c_void_p),
                ("zd", C.c_void_p), ("ecoeff", C.c_void_p), ("dens", C.c_void_p),
                ("xwidth", C.c_double), ("zwidth", C.c_double),
                ("rcoeff_srf", C.c_double), ("dmax_srf", C.c_double), ("kappa_srf", C.c_double),
                ("fcent_srf", C.c_double), ("rcoeff_bdy", C.c_double), ("dmax_bdy", C.c_double),
                ("kappa_bdy", C.c_double), ("fcent_bdy", C.c_double),
                ("qp", C.c_void_p), ("qs", C.c_void_p), ("freq0", C.c_double)]


_lib = None


def lib():
    """Load libfem25gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m fem25_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, i, d, ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
        L.fem25_graph_build.argtypes = [vp, C.POINTER(vp)]
        L.fem25_graph_info.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(ll)]
        L.fem25_graph_copy.argtypes = [vp, vp, vp, vp, vp, vp]
        L.fem25_graph_free.argtypes = [vp]
        L.fem25_graph_free.restype = None
        L.fem25_graph_save.argtypes = [vp, vp, C.c_char_p]
        L.fem25_graph_load.argtypes = [vp, C.c_char_p, C.POINTER(vp)]
        L.fem25_read_mesh.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.fem25_mesh_file_get.argtypes = [vp, vp, vp, vp]
        L.fem25_mesh_file_free.argtypes = [vp]
        L.fem25_mesh_file_free.restype = None
        L.fem25_fazmod.argtypes = [d, d, d, d, C.POINTER(d)]
        L.fem25_create.argtypes = [vp, i, ll, vp, vp, vp, vp, i, C.POINTER(vp)]
        L.fem25_destroy.argtypes = [vp]
        L.fem25_destroy.restype = None
        L.fem25_last_error.argtypes = [vp, C.c_char_p, i]
        L.fem25_sizes.argtypes = [vp, C.POINTER(i), C.POINTER(ll), C.POINTER(ll)]
        L.fem25_update_model.argtypes = [vp, vp, vp]
        L.fem25_asmble_driver.argtypes = [vp, i, C.c_char, d, d, vp]
        L.fem25_assemble_dev.argtypes = [vp, C.c_char, d, d, vp, vp, vp]
        L.fem25_assemble_batch_dev.argtypes = [vp, i, vp, vp, vp, vp, ll, i, vp]
        L.fem25_peff_dev.argtypes = [vp, i, vp, vp, vp, vp]
        L.fem25_addblk_dev.argtypes = [vp, i, vp, vp, vp]
        L.fem25_dense_factor_dev.argtypes = [vp, vp, vp]
        L.fem25_dense_solve_dev.argtypes = [vp, i, i, vp, vp]
        L.fem25_sparse_factor_dev.argtypes = [vp, vp, vp]
        L.fem25_sparse_solve_dev.argtypes = [vp, i, i, vp, vp]
        L.fem25_sparse_info.argtypes = [vp, vp]
        L.fem25_sparse_plan.argtypes = [vp, vp, vp]
        L.fem25_gradient_dev.argtypes = [vp, i, vp, vp, i, vp, vp, i, vp, vp]
        L.fem25_gradient_accumulate_dev.argtypes = [vp, i, vp, vp, i, vp, vp, vp]
        L.fem25_gradient_finalize_dev.argtypes = [vp, vp, vp]
        L.fem25_sync_status.argtypes = [vp, vp]
        L.fem25_test_waits.argtypes = [vp, ll, i]
        L.fem25_plain_fma.argtypes = [vp, i]
        L.fem25_ref_gradient_dev.argtypes = [vp, C.c_char_p, d, d, d, vp, vp, i, vp, vp]
        L.fem25_ref_gradient_info.argtypes = [vp, C.POINTER(i), C.POINTER(ll), vp]
        L.fem25_ref_vforce2_dev.argtypes = [vp, C.c_char_p, d, d, vp, vp, vp]
        L.fem25_ref_met225_dev.argtypes = [vp, C.c_char_p, C.c_double, C.c_double, vp, vp, vp, vp,
                                           i, vp, vp, vp]
        L.fem25_ref_cadj_nu_alpha_dev.argtypes = [vp, C.c_char_p, C.c_double, C.c_double, vp,
                                                  vp, vp, i, vp, vp, vp, vp]
        L.fem25_ref_pchadj_dev.argtypes = [vp, i, i, vp, vp, vp, vp, vp]
        L.fem25_wtgrad_dev.argtypes = [vp, i, vp, vp, vp]
        L.fem25_avgrad_dev.argtypes = [vp, i, i, vp, vp]
        L.fem25_avgrad8_dev.argtypes = [vp, i, i, vp, vp]
        L.fem25_postsolve_dev.argtypes = [vp, i, i, vp, vp, d, d, d, vp, vp, vp, vp, vp, vp, vp,
                                          vp, vp]
        L.fem25_asmb_peff.argtypes = [vp, i, vp, vp, vp]
        L.fem25_cfmat_adjgrad.argtypes = [vp, C.c_char_p, d, d, d, vp, vp, i, vp]
        L.fem25_misfit_options.argtypes = [vp, i, i, i, C.c_float, C.c_float, C.c_float,
                                           C.c_float]
        L.fem25_misfit_dev.argtypes = [vp, i, i, vp, vp, d, d, d, vp, vp, vp, vp, vp, vp, vp, vp]
        L.fem25_misfit_noalloc_dev.argtypes = [vp, i, i, vp, vp, d, d, d, vp, vp, vp, vp, vp, vp, vp,
                                               vp]
        L.fem25_tuning.argtypes = [vp, C.POINTER(i), C.POINTER(i)]
        L.fem25_profile_enable.argtypes = [vp, i]
        L.fem25_profile_ms.argtypes = [vp, i, C.POINTER(d)]
        _lib = L
    return _lib


def _np(a):
    return a.ctypes.data_as(C.c_void_p)


def _ptr(t):
    """Device pointer of a torch tensor (or an int address)."""
    if t is None:
        return None
    if isinstance(t, int):
        return C.c_void_p(t)
    return C.c_void_p(t.data_ptr())


def _stream(s):
    if s is None:
        return None
    if isinstance(s, int):
        return C.c_void_p(s)
    return C.c_void_p(s.cuda_stream)


class _MeshKeep:
    """Contiguous numpy copies of the mesh arrays + the C struct pointing at them."""

    def __init__(self, mesh):
        self.a = dict(ieng=np.ascontiguousarray(mesh.ieng, np.int32),
                      cdomain=np.ascontiguousarray(mesh.cdomain, np.uint8),
                      cnnpg=np.ascontiguousarray(mesh.cnnpg, np.uint8),
                      xlocs=np.ascontiguousarray(mesh.xlocs, np.float64),
                      zlocs=np.ascontiguousarray(mesh.zlocs, np.float64),
                      xd=np.ascontiguousarray(mesh.xd, np.float64),
                      zd=np.ascontiguousarray(mesh.zd, np.float64),
                      ecoeff=np.ascontiguousarray(mesh.ecoeff, np.float64),
                      dens=np.ascontiguousarray(mesh.dens, np.float64))
        ldisp = bool(getattr(mesh, "ldisp", False))
        if ldisp:
            self.a["qp"] = np.ascontiguousarray(mesh.qp, np.float64)
            self.a["qs"] = np.ascontiguousarray(mesh.qs, np.float64)
        s = Mesh()
        s.nelem, s.nnpg, s.nord, s.ldisp = mesh.nelem, mesh.nnpg, mesh.nord, int(ldisp)
        s.freq0 = float(getattr(mesh, "freq0", 0.0)) if ldisp else 0.0
        for k, v in self.a.items():
            setattr(s, k, _np(v))
        s.xwidth, s.zwidth = mesh.xwidth, mesh.zwidth
        s.rcoeff_srf, s.rcoeff_bdy = mesh.rcoeff
        s.dmax_srf, s.dmax_bdy = mesh.dmax
        s.kappa_srf, s.kappa_bdy = mesh.kappa
        s.fcent_srf, s.fcent_bdy = mesh.fcent
        self.s = s
        self.ptr = C.cast(C.pointer(s), C.c_void_p)


def mesh_struct(mesh):
    return _MeshKeep(mesh)


class Graph:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def graph_build(mesh, cache=None):
    """GEN_GRAPH25: IEN, LM, IRPTR, JCPTR (1-based) and CNP of a mesh.  With
    ``cache`` (a file path) the graph is read from that file when it was made
    for this mesh, else built and written there."""
    L = lib()
    mk = _MeshKeep(mesh)
    h = C.c_void_p()
    if cache is not None and os.path.exists(cache):
        r = L.fem25_graph_load(mk.ptr, os.fsencode(cache), C.byref(h))
        if r:
            h = C.c_void_p()
    if not h:
        r = L.fem25_graph_build(mk.ptr, C.byref(h))
        if r:
            raise Fem25Error(r, "graph build failed")
        if cache is not None:
            r = L.fem25_graph_save(h, mk.ptr, os.fsencode(cache))
            if r:
                L.fem25_graph_free(h)
                raise Fem25Error(r, f"graph save to {cache} failed")
    nnp, ndof, nz = C.c_int(), C.c_int(), C.c_longlong()
    L.fem25_graph_info(h, C.byref(nnp), C.byref(ndof), C.byref(nz))
    nen = (mesh.nord + 1) ** 2
    ien = np.empty((mesh.nelem, nen), np.int32)
    lm = np.empty((mesh.nelem, nen, 3), np.int32)
    irptr = np.empty(ndof.value + 1, np.int32)
    jcptr = np.empty(nz.value, np.int32)
    cnp = np.empty(ndof.value, np.uint8)
    L.fem25_graph_copy(h, _np(ien), _np(lm), _np(irptr), _np(jcptr), _np(cnp))
    L.fem25_graph_free(h)
    return Graph(nnp=nnp.value, ndof=ndof.value, nzero=nz.value, ien=ien, lm=lm, irptr=irptr,
                 jcptr=jcptr, cnp=cnp)


def sparse_plan(mesh):
    """The nested dissection fem25_sparse_factor_dev would use for ``mesh``,
    planned on the host (fem25_sparse_plan): (fronts, levels, factor bytes,
    largest level work bytes, largest own count, largest front order, flops
    of one factorisation)."""
    L = lib()
    mk = _MeshKeep(mesh)
    h = C.c_void_p()
    r = L.fem25_graph_build(mk.ptr, C.byref(h))
    if r:
        raise Fem25Error(r, "graph build failed")
    out = np.zeros(7, np.int64)
    try:
        r = L.fem25_sparse_plan(mk.ptr, h, out.ctypes.data)
    finally:
        L.fem25_graph_free(h)
    if r:
        raise Fem25Error(r, "sparse plan failed")
    return tuple(int(v) for v in out)


def fazmod(xlatmin, xlonmin, xlatmax, xlonmax):
    """FAZMOD: model azimuth (degrees) of the Bielak/absorbing corners (WGS-84)."""
    az = C.c_double()
    r = lib().fem25_fazmod(xlatmin, xlonmin, xlatmax, xlonmax, C.byref(az))
    if r:
        raise Fem25Error(r, "fazmod: Vincenty iteration did not converge")
    return az.value


def read_mesh(projnm):
    """RDMESHBK: PROJNM.nodes + PROJNM.mesh -> (Mesh, info).  info holds INPTYP,
    IITYPE, IDISP, NELEME, NABS and the Bielak/absorbing corner latitudes and
    longitudes; the PML parameters keep the Mesh defaults (they come from the
    reference's parameter file, not the mesh files)."""
    from .synth import Mesh as PyMesh
    L = lib()
    h = C.c_void_p()
    r = L.fem25_read_mesh(os.fsencode(projnm), C.byref(h))
    if r and not h:
        raise Fem25Error(r, f"reading {projnm}.nodes / .mesh failed (see stderr)")
    try:
        m = Mesh()
        ints = np.zeros(5, np.int32)
        reals = np.zeros(4)
        L.fem25_mesh_file_get(h, C.byref(m), _np(ints), _np(reals))
        if r:
            raise Fem25Error(r, f"{projnm}: unsupported mesh (INPTYP {ints[0]}, IITYPE {ints[1]})")
        ne, nn = m.nelem, m.nnpg
        arr = lambda ptr, n, dt: np.ctypeslib.as_array(C.cast(ptr, C.POINTER(dt)), (n,)).copy()
        ldisp = bool(m.ldisp)
        mesh = PyMesh(nelem=ne, nnpg=nn, nord=m.nord,
                      ieng=arr(m.ieng, 4 * ne, C.c_int32).reshape(ne, 4),
                      cdomain=arr(m.cdomain, ne, C.c_uint8),
                      cnnpg=arr(m.cnnpg, 2 * nn, C.c_uint8).reshape(nn, 2),
                      xlocs=arr(m.xlocs, nn, C.c_double), zlocs=arr(m.zlocs, nn, C.c_double),
                      xd=arr(m.xd, nn, C.c_double), zd=arr(m.zd, nn, C.c_double),
                      ecoeff=arr(m.ecoeff, 2 * nn, C.c_double).reshape(2, nn),
                      dens=arr(m.dens, nn, C.c_double), xwidth=m.xwidth, zwidth=m.zwidth,
                      ldisp=ldisp, qp=arr(m.qp, nn, C.c_double) if ldisp else None,
                      qs=arr(m.qs, nn, C.c_double) if ldisp else None)
        info = dict(inptyp=int(ints[0]), iitype=int(ints[1]), idisp=int(ints[2]),
                    neleme=int(ints[3]), nabs=int(ints[4]), xlatmin=reals[0], xlonmin=reals[1],
                    xlatmax=reals[2], xlonmax=reals[3])
        return mesh, info
    finally:
        L.fem25_mesh_file_free(h)


class Context:
    """Device context for one mesh (fem25_create)."""

    def __init__(self, mesh, graph=None, device=0):
        L = lib()
        self.mesh = mesh
        self.g = graph_build(mesh) if graph is None else graph
        self._mk = _MeshKeep(mesh)
        h = C.c_void_p()
        g = self.g
        self._lm = np.ascontiguousarray(g.lm, np.int32)
        self._irptr = np.ascontiguousarray(g.irptr, np.int32)
        self._jcptr = np.ascontiguousarray(g.jcptr, np.int32)
        self._cnp = np.ascontiguousarray(g.cnp, np.uint8)
        r = L.fem25_create(self._mk.ptr, g.ndof, g.nzero, _np(self._lm), _np(self._irptr),
                           _np(self._jcptr), _np(self._cnp), device, C.byref(h))
        if r:
            raise Fem25Error(r, "fem25_create failed (see stderr)")
        self.h = h
        self.device = device
        self.ndof = g.ndof
        self.nzero = g.nzero
        nb = C.c_longlong()
        L.fem25_sizes(h, None, None, C.byref(nb))
        self.nblocks = nb.value

    def close(self):
        if getattr(self, "h", None):
            lib().fem25_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tuning(self):
        """Autotuner choices: {"stream_variant": v, "grad_tile": t} (-1 = not tuned)."""
        v, t = C.c_int(), C.c_int()
        lib().fem25_tuning(self.h, C.byref(v), C.byref(t))
        return {"stream_variant": v.value, "grad_tile": t.value}

    def _check(self, r):
        if r:
            buf = C.create_string_buffer(512)
            lib().fem25_last_error(self.h, buf, 512)
            raise Fem25Error(r, buf.value.decode(errors="replace"))

    # ---- profiling
    def profile(self, enable=True):
        self._check(lib().fem25_profile_enable(self.h, 1 if enable else 0))

    def profile_ms(self, which):
        v = C.c_double()
        self._check(lib().fem25_profile_ms(self.h, which, C.byref(v)))
        return v.value

    # ---- model
    def update_model(self, ecoeff, dens):
        e = np.ascontiguousarray(ecoeff, np.float64)
        d = np.ascontiguousarray(dens, np.float64)
        self._check(lib().fem25_update_model(self.h, _np(e), _np(d)))

    # ---- assembly
    def asmble_driver(self, cftype, freq, py, out=None):
        """ASMBLE_DRIVER: host COMPLEX*8 CDIST(NZLOC) (mid%A_LOC order)."""
        if out is None:
            out = np.empty(self.nzero, np.complex64)
        ptr = C.c_void_p(out.data_ptr()) if hasattr(out, "data_ptr") else _np(out)
        self._check(lib().fem25_asmble_driver(self.h, self.nzero, cftype.encode(), freq, py, ptr))
        return out

    def plain_fma(self, enable=True):
        """Benchmark option: assemble() with the FMA build of the element
        kernels (not bit-identical to the reference arithmetic)."""
        self._check(lib().fem25_plain_fma(self.h, 1 if enable else 0))

    def assemble(self, cftype, freq, py, out128=None, out64=None, stream=None):
        self._check(lib().fem25_assemble_dev(self.h, cftype.encode(), freq, py, _ptr(out128),
                                             _ptr(out64), _stream(stream)))

    def assemble_batch(self, cftypes, freqs, pys, ring, slot_stride, nslots, stream=None):
        """Systems k -> ring + (k % nslots) * slot_stride doubles (complex128)."""
        n = len(freqs)
        ct = np.frombuffer("".join(cftypes).encode(), np.uint8).copy() if isinstance(
            cftypes, (list, tuple)) else np.full(n, ord(cftypes), np.uint8)
        f = np.ascontiguousarray(freqs, np.float64)
        p = np.ascontiguousarray(pys, np.float64)
        self._check(lib().fem25_assemble_batch_dev(self.h, n, _np(ct), _np(f), _np(p), _ptr(ring),
                                                   slot_stride, nslots, _stream(stream)))

    # ---- Bielak effective force
    def asmb_peff(self, nsrc, a_loc, ue, peff, stream=None):
        self._check(lib().fem25_peff_dev(self.h, nsrc, _ptr(a_loc), _ptr(ue), _ptr(peff),
                                         _stream(stream)))

    def asmb_peff_host(self, ue, cdist=None):
        """ASMB_PEFF with host arrays: P_eff (COMPLEX*8 [NDOF]) of the host
        background field ue; cdist = host COMPLEX*8 CDIST, or None for the
        last asmble_driver system still on the device."""
        peff = np.zeros(self.ndof, np.complex64)
        cd = None if cdist is None else _np(np.ascontiguousarray(cdist, np.complex64))
        self._check(lib().fem25_asmb_peff(self.h, self.ndof, cd,
                                          _np(np.ascontiguousarray(ue, np.complex64)), _np(peff)))
        return peff

    def dense_factor(self, csr128, stream=None):
        """LU of the assembled complex128 CSR (device) for the small-mesh solve."""
        self._check(lib().fem25_dense_factor_dev(self.h, _ptr(csr128), _stream(stream)))

    def sparse_factor(self, csr128, stream=None):
        """Multifrontal LU of a complex128 CSR (device) -- fem25_sparse_factor_dev."""
        self._check(lib().fem25_sparse_factor_dev(self.h, _ptr(csr128), _stream(stream)))

    def sparse_solve(self, rhs, trans=0, stream=None):
        """op(A) X = B in place, rhs complex128 [nrhs, NDOF] (device); trans 0: A,
        1: A^T, 2: A^H -- fem25_sparse_solve_dev."""
        nrhs = 1 if rhs.dim() == 1 else rhs.shape[0]
        self._check(lib().fem25_sparse_solve_dev(self.h, nrhs, trans, _ptr(rhs), _stream(stream)))

    def sparse_info(self):
        """(fronts, levels, factor bytes, work bytes, largest k, largest front
        order, flops of one factorisation) -- fem25_sparse_info."""
        out = np.zeros(7, np.int64)
        self._check(lib().fem25_sparse_info(self.h, out.ctypes.data))
        return tuple(int(v) for v in out)

    def dense_solve(self, rhs, trans=0, stream=None):
        """op(A) X = B in place; rhs complex128 [nrhs][NDOF] on the device;
        trans 0: A, 1: A^T, 2: A^H."""
        nrhs = rhs.numel() // self.ndof if hasattr(rhs, "numel") else rhs.size // self.ndof
        self._check(lib().fem25_dense_solve_dev(self.h, nrhs, trans, _ptr(rhs), _stream(stream)))

    def addblk(self, nsrc, ue, sol, stream=None):
        """ADDBLK: sol += ue on the 'E' DOFs (COMPLEX*8 [nsrc][NDOF], in place)."""
        self._check(lib().fem25_addblk_dev(self.h, nsrc, _ptr(ue), _ptr(sol), _stream(stream)))

    # ---- gradients
    def gradient(self, freqs, pys, nsrc, u, lam, grad, prec=FEM25_PREC_FP64, stream=None):
        f = np.ascontiguousarray(freqs, np.float64)
        p = np.ascontiguousarray(pys, np.float64)
        self._check(lib().fem25_gradient_dev(self.h, len(f), _np(f), _np(p), nsrc, _ptr(u),
                                             _ptr(lam), prec, _ptr(grad), _stream(stream)))

    def gradient_accumulate(self, freqs, pys, nsrc, u, lam, stream=None):
        """Adds the field covariances of the pairs into the context's
        accumulators (split-precision gradient, see gradient_finalize)."""
        f = np.ascontiguousarray(freqs, np.float64)
        p = np.ascontiguousarray(pys, np.float64)
        self._check(lib().fem25_gradient_accumulate_dev(self.h, len(f), _np(f), _np(p), nsrc,
                                                        _ptr(u), _ptr(lam), _stream(stream)))

    def sync_status(self, stream=None):
        """Waits for the stream; raises Fem25Error for what kernels recorded
        on the device (Jacobian failures, timed-out pipeline waits)."""
        self._check(lib().fem25_sync_status(self.h, _stream(stream)))

    def test_waits(self, limit_cycles=0, inject=False):
        """Test hook of the tensor-core kernels' bounded waits: the limit in SM
        clocks (0: default) and whether launches withhold one producer arrival
        so that a wait runs out (see fem25_test_waits)."""
        self._check(lib().fem25_test_waits(self.h, int(limit_cycles), 1 if inject else 0))

    def gradient_finalize(self, grad, stream=None):
        """grad += the gradient of everything accumulated since the last
        finalize; empties the accumulators."""
        self._check(lib().fem25_gradient_finalize_dev(self.h, _ptr(grad), _stream(stream)))

    def ref_gradient_info(self):
        n, nz = C.c_int(), C.c_longlong()
        maskg = np.zeros(self.mesh.nnpg, np.int32)
        self._check(lib().fem25_ref_gradient_info(self.h, C.byref(n), C.byref(nz), _np(maskg)))
        return n.value, nz.value, maskg

    def cfmat_adjgrad(self, cinvtype, vpvs, freq, py, wave, adjlam, gradl, accumulate=False,
                      stream=None):
        self._check(lib().fem25_ref_gradient_dev(self.h, cinvtype.encode(), vpvs, freq, py,
                                                 _ptr(wave), _ptr(adjlam), 1 if accumulate else 0,
                                                 _ptr(gradl), _stream(stream)))

    def wtgrad(self, wgrad, grad, stream=None):
        """WTGRAD: grad *= wgrad (REAL*4 device arrays, in place)."""
        self._check(lib().fem25_wtgrad_dev(self.h, grad.numel(), _ptr(wgrad), _ptr(grad),
                                           _stream(stream)))

    def avgrad(self, nvinv, ncasc, grad, stream=None):
        """AVGRAD (REAL*4) or AVGRAD8 (REAL*8, by the tensor's dtype) on
        grad[NNPINV * nvinv] in place."""
        import torch
        fn = lib().fem25_avgrad8_dev if grad.dtype == torch.float64 else lib().fem25_avgrad_dev
        self._check(fn(self.h, nvinv, ncasc, _ptr(grad), _stream(stream)))

    def cfmat_adjgrad_host(self, cinvtype, vpvs, freq, py, wave, adjlam, gradl, accumulate=False):
        """CFMAT_DIST + ADJGRAD with host arrays; gradl (float32 numpy) updated in place."""
        self._check(lib().fem25_cfmat_adjgrad(
            self.h, cinvtype.encode(), vpvs, freq, py,
            _np(np.ascontiguousarray(wave, np.complex64)),
            _np(np.ascontiguousarray(adjlam, np.complex64)), 1 if accumulate else 0, _np(gradl)))

    def met225(self, cinvtype, freq, py, adjlam, nu, alpha, wave, p1buf, p2buf,
               accumulate=False, stream=None):
        """MET225_MOD Hessian-vector buffers (REAL*4 [nnpinv * nvinv] each)."""
        self._check(lib().fem25_ref_met225_dev(self.h, cinvtype.encode(), freq, py, _ptr(adjlam),
                                               _ptr(nu), _ptr(alpha), _ptr(wave),
                                               1 if accumulate else 0, _ptr(p1buf), _ptr(p2buf),
                                               _stream(stream)))

    def cadj_nu_alpha(self, cinvtype, freq, py, v, adjlam, wave, rhsbnu, rhsalp, p3,
                      accumulate=False, stream=None):
        """CADJ_NU_ALPHA right-hand sides and P3 (see fem25_ref_cadj_nu_alpha_dev)."""
        self._check(lib().fem25_ref_cadj_nu_alpha_dev(self.h, cinvtype.encode(), freq, py, _ptr(v),
                                                      _ptr(adjlam), _ptr(wave),
                                                      1 if accumulate else 0, _ptr(rhsbnu),
                                                      _ptr(rhsalp), _ptr(p3), _stream(stream)))

    def pchadj(self, nvinv, nrhs, grns, fmat, hessb, jacl=None, stream=None):
        """PCHADJ products: HESSB += REAL(JACL^H JACL) in place, JACL optional."""
        self._check(lib().fem25_ref_pchadj_dev(self.h, nvinv, nrhs, _ptr(grns), _ptr(fmat),
                                               _ptr(hessb), _ptr(jacl), _stream(stream)))

    def vforce2(self, cinvtype, freq, py, wave, fmat, stream=None):
        """VFORCE25_2 / DABMKISOB25 virtual forces into fmat (COMPLEX*8 [nvinv][nz])."""
        self._check(lib().fem25_ref_vforce2_dev(self.h, cinvtype.encode(), freq, py, _ptr(wave),
                                                _ptr(fmat), _stream(stream)))

    # ---- misfit
    def misfit_options(self, norm=2, irestp=3, ibphase=0, eps=0.0, thresh=0.0, dtmax=0.0,
                       dtmax_obj=0.0):
        """NORM, IRESTP, IBPHASE, COBJ4's EPS / THRESH and the DTMAX tests of the
        misfit entry points (see fem25_misfit_options); no arguments restore
        the defaults."""
        self._check(lib().fem25_misfit_options(self.h, norm, irestp, ibphase, eps, thresh, dtmax,
                                               dtmax_obj))

    def misfit(self, nsrc, mrdof, yrec, freq, py, azmod, recv, sol, obs, wghts, rhs, stream=None):
        nrec = mrdof.shape[0]
        est = np.zeros((nsrc, nrec, 3), np.complex64)
        mis = np.zeros(nsrc, np.float32)
        self._check(lib().fem25_misfit_dev(
            self.h, nsrc, nrec, _np(np.ascontiguousarray(mrdof, np.int32)),
            _np(np.ascontiguousarray(yrec, np.float64)), freq, py, azmod,
            _np(np.ascontiguousarray(recv, np.complex64)), _ptr(sol),
            _np(np.ascontiguousarray(obs, np.complex64)),
            _np(np.ascontiguousarray(wghts, np.float32)), _np(est), _ptr(rhs), _np(mis),
            _stream(stream)))
        return est, mis

    def postsolve(self, nsrc, mrdof, yrec, freq, py, azmod, recv, ue, sol, obs, wghts, rhs,
                  stream=None):
        """ADDBLK + EXRESP25D + misfit / adjoint source in one kernel: sol
        (device, COMPLEX*8 [nsrc][NDOF]) gets ue added on the 'E' DOFs in
        place; returns (est, misfit) like misfit()."""
        nrec = mrdof.shape[0]
        est = np.zeros((nsrc, nrec, 3), np.complex64)
        mis = np.zeros(nsrc, np.float32)
        self._check(lib().fem25_postsolve_dev(
            self.h, nsrc, nrec, _np(np.ascontiguousarray(mrdof, np.int32)),
            _np(np.ascontiguousarray(yrec, np.float64)), freq, py, azmod,
            _np(np.ascontiguousarray(recv, np.complex64)), _ptr(ue), _ptr(sol),
            _np(np.ascontiguousarray(obs, np.complex64)),
            _np(np.ascontiguousarray(wghts, np.float32)), _np(est), _ptr(rhs), _np(mis),
            _stream(stream)))
        return est, mis

    def misfit_noalloc(self, nsrc, mrdof, yrec, freq, py, azmod, recv, sol, obs, wghts, est, rhs,
                       misfit, stream=None):
        """fem25_misfit_noalloc_dev: obs, wghts, est, misfit are device tensors;
        mrdof, yrec, recv host arrays.  Allocates no device memory."""
        nrec = mrdof.shape[0]
        self._check(lib().fem25_misfit_noalloc_dev(
            self.h, nsrc, nrec, _np(np.ascontiguousarray(mrdof, np.int32)),
            _np(np.ascontiguousarray(yrec, np.float64)), freq, py, azmod,
            _np(np.ascontiguousarray(recv, np.complex64)), _ptr(sol), _ptr(obs), _ptr(wghts),
            _ptr(est), _ptr(rhs), _ptr(misfit), _stream(stream)))
