"""The nested dissection of the sparse direct solve, planned on the host
(fem25_sparse_plan, no device): its front count, levels, factor and work
sizes and flop count against an independent numpy restatement of the same
dissection -- elements bisected along the longer side of their centroids'
bounding box (ties broken by element number), a separator of the DOFs both
halves share that no coarser separator took, leaves of at most two elements
owning their remaining DOFs, a front's boundary the DOFs of its subtree owned
by an ancestor.  Exact integer equality."""
import numpy as np
import pytest

from fem25_b200 import graph_build, sparse_plan, synth


def _numpy_plan(mesh, g, leaf=2):
    lm = np.asarray(g.lm).reshape(mesh.nelem, -1) - 1
    cx = mesh.xlocs[mesh.ieng - 1].mean(1)
    cz = mesh.zlocs[mesh.ieng - 1].mean(1)
    owner = np.full(g.ndof, -1, np.int64)
    fronts = []  # (own DOFs, elements, depth); postorder ids

    def rec(E, depth):
        if len(E) <= leaf:
            d = np.unique(lm[E])
            d = d[d >= 0]
            d = d[owner[d] == -1]
            owner[d] = len(fronts)
            fronts.append((d, E, depth))
            return
        x, z = cx[E], cz[E]
        ax = x if (x.max() - x.min()) >= (z.max() - z.min()) else z
        o = np.lexsort((E, ax))
        h = len(E) // 2
        E1, E2 = E[o[:h]], E[o[h:]]
        d1 = np.unique(lm[E1])
        d2 = np.unique(lm[E2])
        sep = np.intersect1d(d1[d1 >= 0], d2[d2 >= 0])
        sep = sep[owner[sep] == -1]
        owner[sep] = -2
        rec(E1, depth + 1)
        rec(E2, depth + 1)
        owner[sep] = len(fronts)
        fronts.append((sep, E, depth))

    rec(np.arange(mesh.nelem), 0)
    assert (owner >= 0).all()
    nlev = 1 + max(f[2] for f in fronts)
    lev_work = np.zeros(nlev, np.int64)
    fac = 0
    flops = 0.0
    kmax = nmax = 0
    for t, (own, E, depth) in enumerate(fronts):
        d = np.unique(lm[E])
        d = d[d >= 0]
        k = len(own)
        m = int(np.sum(owner[d] > t))
        n = k + m
        fac += n * k + k * m
        lev_work[depth] += n * n
        flops += 8.0 / 3.0 * k ** 3 + 8.0 * k * k * m + 8.0 * k * m * m
        kmax, nmax = max(kmax, k), max(nmax, n)
    return (len(fronts), nlev, fac * 16, int(lev_work.max()) * 16, kmax, nmax, int(flops))


@pytest.mark.parametrize("cfg, nx, nz", [(0, 12, 6), (0, None, None), (1, 48, 18), (4, 40, 16)])
def test_plan_matches_numpy_restatement(cfg, nx, nz):
    mesh, _, _ = synth.make_config(cfg, nx=nx, nz=nz)
    g = graph_build(mesh)
    got = sparse_plan(mesh)
    ref = _numpy_plan(mesh, g)
    assert got[:6] == ref[:6], (got, ref)
    assert abs(got[6] - ref[6]) <= 1e-9 * ref[6] + 8, (got[6], ref[6])


def test_plan_of_the_layered_benchmark_mesh():
    """The 400x120 mesh: sizes the factorisation tests and the bench report
    (63 231 fronts in 16 levels, 14.6 GB of factors, 2.5 TFLOP)."""
    mesh, _, _ = synth.make_config(1)
    fronts, levels, fbytes, wbytes, kmax, nmax, flops = sparse_plan(mesh)
    assert (fronts, levels, kmax, nmax) == (63231, 16, 1440, 4077)
    assert fbytes == 14562028656 and 2.4e12 < flops < 2.6e12
