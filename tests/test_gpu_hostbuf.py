"""Host-buffer drop-ins of ASMB_PEFF (fem25_asmb_peff) and CFMAT_DIST +
ADJGRAD (fem25_cfmat_adjgrad): the call sites of the reference pass host
arrays (mid%A_LOC, UE, PEFF, WAVE, ADJLAM, GRADL).  Checked bit for bit
against the oracle (ASMB_PEFF on the oracle's COMPLEX*8 CDIST; the
CFMAT_DIST + ADJFLAM_DIST restatement), with P_eff taken both from the last
ASMBLE_DRIVER system kept on the device and from an uploaded CDIST."""
import numpy as np
import pytest

import oracle
from fem25_b200 import Context, synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_host_buffer_dropins_match_oracle():
    mesh, pairs, _ = synth.make_config(0)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    try:
        rng = np.random.default_rng(17)
        f, py = pairs[9]
        _, ref64 = oracle.asmble(mesh, g, "B", f, py)
        ue = (rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
        cdist = ctx.asmble_driver("B", f, py)
        assert np.array_equal(cdist.view(np.uint32), ref64.view(np.uint32))
        pe = oracle.peff(g, ref64, ue)
        got = ctx.asmb_peff_host(ue)  # CDIST of the last ASMBLE_DRIVER, on the device
        assert np.array_equal(got.view(np.uint32), pe.view(np.uint32))
        _, other64 = oracle.asmble(mesh, g, "S", *pairs[2])
        got2 = ctx.asmb_peff_host(ue, cdist=other64)  # an uploaded CDIST
        assert np.array_equal(got2.view(np.uint32), oracle.peff(g, other64, ue).view(np.uint32))
        # CFMAT_DIST + ADJGRAD with host arrays, accumulating into GRADL
        rg = oracle.RefGrad(mesh, g)
        wave = (rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
        lam = (rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
        g0 = rng.standard_normal(rg.nnpinv).astype(np.float32)
        for cinv in ("PP", "SS"):
            fm = rg.cfmat(f, py, wave, lisp=(cinv == "PP"))
            ref = rg.adjflam(fm, lam, gradl=g0.copy())
            gl = g0.copy()
            ctx.cfmat_adjgrad_host(cinv, 1.7320508075688772, f, py, wave, lam, gl)
            assert np.array_equal(gl.view(np.uint32), ref.view(np.uint32)), cinv
    finally:
        ctx.close()
