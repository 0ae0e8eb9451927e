"""The fused post-solve pass (fem25_postsolve_dev): ADDBLK + EXRESP25D +
misfit / adjoint source for all sources of a group in one kernel, against
the separate calls (fem25_addblk_dev then fem25_misfit_dev) and the oracle
(ADDBLK then the misfit restatement).  Tolerance: bit-identical, for two
receiver sets in a row (the receiver bitmap is rebuilt when MRDOF changes)
and with non-default misfit options."""
import numpy as np
import pytest

import oracle
from fem25_b200 import Context, synth
from tests import helpers

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_postsolve_matches_separate_calls_and_oracle():
    mesh, pairs, _ = synth.make_config(4, nx=24, nz=12)  # 4-element strip: many 'E' DOFs
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(314)
    nsrc = 5
    try:
        for rep, (nrec, opts) in enumerate(((20, {}), (31, dict(norm=1, ibphase=1)))):
            ctx.misfit_options(**opts)
            mrdof = helpers.surface_receivers(mesh, g, nrec)
            # receivers on the Bielak strip too, so that ADDBLK reaches them
            e_nodes = np.unique(g.lm[mesh.cdomain == ord("E")].reshape(-1, 3), axis=0)
            e_nodes = e_nodes[(e_nodes > 0).all(axis=1)]
            extra = e_nodes[rng.choice(len(e_nodes), 6, replace=False)]
            mrdof = np.unique(np.concatenate([mrdof, extra]), axis=0).astype(np.int32)
            nr = len(mrdof)
            yrec = rng.uniform(-900, 900, nr)
            recv = (1 + 0.1j * rng.standard_normal((nr, 3))).astype(np.complex64)
            sol = (rng.standard_normal((nsrc, g.ndof)) + 1j * rng.standard_normal((nsrc, g.ndof))).astype(np.complex64)
            ue = (rng.standard_normal((nsrc, g.ndof)) + 1j * rng.standard_normal((nsrc, g.ndof))).astype(np.complex64)
            obs = (rng.standard_normal((nsrc, nr, 3)) + 1j * rng.standard_normal((nsrc, nr, 3))).astype(np.complex64)
            obs[1, 2, 0] = 0
            w = rng.uniform(0.5, 1.5, (nsrc, nr, 3)).astype(np.float32)
            f, py = pairs[30 + rep]
            d_ue = torch.from_numpy(ue).to(dev)
            # separate calls
            s1 = torch.from_numpy(sol).to(dev)
            r1 = torch.zeros((nsrc, g.ndof), dtype=torch.complex64, device=dev)
            ctx.addblk(nsrc, d_ue, s1)
            e1, m1 = ctx.misfit(nsrc, mrdof, yrec, f, py, 11.0, recv, s1, obs, w, r1)
            # fused
            s2 = torch.from_numpy(sol).to(dev)
            r2 = torch.full((nsrc, g.ndof), float("nan"), dtype=torch.complex64, device=dev)
            e2, m2 = ctx.postsolve(nsrc, mrdof, yrec, f, py, 11.0, recv, d_ue, s2, obs, w, r2)
            torch.cuda.synchronize()
            for a, b in ((s1, s2), (r1, r2)):
                assert np.array_equal(a.cpu().numpy().view(np.uint32), b.cpu().numpy().view(np.uint32))
            assert np.array_equal(e1.view(np.uint32), e2.view(np.uint32))
            assert np.array_equal(m1.view(np.uint32), m2.view(np.uint32))
            # the oracle
            s2h, r2h = s2.cpu().numpy(), r2.cpu().numpy()
            for s in range(nsrc):
                so = oracle.addblk(g, ue[s], sol[s])
                assert np.array_equal(s2h[s].view(np.uint32), so.view(np.uint32))
                eo, ro, mo = oracle.misfit(g.ndof, mrdof, yrec, f, py, 11.0, recv, so, obs[s], w[s],
                                           **opts)
                assert np.array_equal(e2[s].view(np.uint32), eo.view(np.uint32))
                assert np.array_equal(r2h[s].view(np.uint32), ro.view(np.uint32))
                assert np.float32(m2[s]).view(np.uint32) == np.float32(mo).view(np.uint32)
    finally:
        ctx.close()
