"""Generates tests/golden/oracle_small.npz: fixtures the oracle must keep
reproducing bit for bit (element matrices of an interior and a PML element,
the complex128 and COMPLEX*8 CSR of a 6x4-element mesh, its graph, an exact
gradient, and the same matrices and CSR for dispersive media).  The reference ships no golden vectors for this path; these
pin the oracle against unnoticed changes.

    python -m tests.golden.make_golden
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def compute():
    import oracle
    from fem25_b200 import synth
    mesh, pairs, _ = synth.make_config(0, nx=6, nz=4)
    g = oracle.graph_build(mesh)
    inner = [e for e in range(mesh.nelem) if chr(mesh.cdomain[e]) == "I"][0]
    pml = [e for e in range(mesh.nelem) if chr(mesh.cdomain[e]) == "A"][0]
    f, py = pairs[6]
    me_i, ce_i = oracle.element_matrix(mesh, inner, "B", f, py)
    me_a, ce_a = oracle.element_matrix(mesh, pml, "S", f, py)
    c128, c64 = oracle.asmble(mesh, g, "B", f, py)
    rng = np.random.default_rng(1234)
    u = rng.standard_normal((2, g.ndof)) + 1j * rng.standard_normal((2, g.ndof))
    lam = rng.standard_normal((2, g.ndof)) + 1j * rng.standard_normal((2, g.ndof))
    grad = oracle.grad_exact(mesh, g, f, py, u, lam)
    import hashlib

    def digest(a):
        return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)

    # dispersive media (KMDAMP / CMDAMP): the same mesh with seeded Q
    synth.make_dispersive(mesh, seed=3, freq0=1.0, qs_mean=30.0)
    dme_i, dce_i = oracle.element_matrix(mesh, inner, "B", f, py)
    dme_a, dce_a = oracle.element_matrix(mesh, pml, "S", f, py)
    d128, d64 = oracle.asmble(mesh, g, "B", f, py)
    # leading slices stored verbatim, whole arrays pinned by SHA-256
    return dict(me_i=me_i[:, :12], ce_i=ce_i[:, :12], me_a=me_a[:, :12], ce_a=ce_a[:, :12],
                c128=c128[:4096], c64=c64[:4096], irptr=g.irptr[:512], grad=grad,
                sha_me_i=digest(me_i), sha_ce_i=digest(ce_i), sha_me_a=digest(me_a),
                sha_ce_a=digest(ce_a), sha_c128=digest(c128), sha_c64=digest(c64),
                sha_jcptr=digest(g.jcptr), sha_lm=digest(g.lm), sha_cnp=digest(g.cnp),
                disp_ce_i=dce_i[:, :12], disp_ce_a=dce_a[:, :12], disp_c128=d128[:2048],
                sha_disp_me_i=digest(dme_i), sha_disp_ce_i=digest(dce_i),
                sha_disp_me_a=digest(dme_a), sha_disp_ce_a=digest(dce_a),
                sha_disp_c128=digest(d128), sha_disp_c64=digest(d64))


if __name__ == "__main__":
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **compute())
    print("written", os.path.join(HERE, "oracle_small.npz"))
