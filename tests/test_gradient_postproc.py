"""Gradient post-processing of FUNCGRADH25 (funcgradh.f90:436-443): WTGRAD
(gengmask.f90:384-416) and AVGRAD / AVGRAD8 (gengmask.f90:1202-1332).

CPU: the oracle's AVGRAD pinned by closed forms -- a constant gradient is
unchanged, one cascade of AVGRAD8 equals a numpy restatement of the
neighbourhood mean, and cascades compose.  GPU: fem25_wtgrad_dev,
fem25_avgrad_dev and fem25_avgrad8_dev against the oracle, bit-identical
(ordered FP32 / FP64 sums and an IEEE division)."""
import numpy as np
import pytest

import oracle
from fem25_b200 import Context, synth


@pytest.fixture(scope="module")
def case():
    mesh, pairs, _ = synth.make_config(3, nx=14, nz=8)
    g = oracle.graph_build(mesh)
    rg = oracle.RefGrad(mesh, g)
    return mesh, g, rg


def _numpy_avg(mesh, rg, nvinv, grad):
    out = grad.copy()
    for p in range(mesh.nnpg):
        ip = rg.maskg[p]
        if ip <= 0:
            continue
        acc = np.zeros(nvinv)
        n = np.zeros(nvinv, int)
        for ic in range(rg.ncon):
            e = rg.mconn[ic, p]
            if e == 0:
                break
            for a in mesh.ieng[e - 1]:
                jp = rg.maskg[a - 1]
                if jp > 0:
                    acc += grad[(jp - 1) * nvinv:(jp - 1) * nvinv + nvinv]
                    n += 1
        m = n > 0
        out[(ip - 1) * nvinv:(ip - 1) * nvinv + nvinv][m] = acc[m] / n[m]
    return out


def test_avgrad_closed_forms(case):
    mesh, g, rg = case
    rng = np.random.default_rng(3)
    for nvinv in (1, 2):
        const = np.full(rg.nnpinv * nvinv, 2.5)
        assert np.array_equal(rg.avgrad(nvinv, 3, const), const)
        x = rng.standard_normal(rg.nnpinv * nvinv)
        one = rg.avgrad(nvinv, 1, x)
        assert np.abs(one - _numpy_avg(mesh, rg, nvinv, x)).max() <= 1e-14 * np.abs(x).max()
        assert np.array_equal(rg.avgrad(nvinv, 2, x), rg.avgrad(nvinv, 1, one))
        assert np.array_equal(rg.avgrad(nvinv, 0, x), x)
    w = rng.uniform(0, 1, 10).astype(np.float32)
    gr = rng.standard_normal(10).astype(np.float32)
    assert np.array_equal(oracle.wtgrad(w, gr), gr * w)


@pytest.mark.gpu
def test_gpu_postproc_matches_oracle(case):
    torch = pytest.importorskip("torch")
    mesh, g, rg = case
    dev = torch.device("cuda:0")
    ctx = Context(mesh, g)
    try:
        nnpinv, _, maskg = ctx.ref_gradient_info()
        assert nnpinv == rg.nnpinv and np.array_equal(maskg, rg.maskg)
        rng = np.random.default_rng(9)
        for nvinv in (1, 2):
            x32 = rng.standard_normal(nnpinv * nvinv).astype(np.float32)
            x64 = rng.standard_normal(nnpinv * nvinv)
            for ncasc in (1, 3):
                d32 = torch.from_numpy(x32).to(dev)
                ctx.avgrad(nvinv, ncasc, d32)
                assert np.array_equal(d32.cpu().numpy().view(np.uint32),
                                      rg.avgrad(nvinv, ncasc, x32).view(np.uint32))
                d64 = torch.from_numpy(x64).to(dev)
                ctx.avgrad(nvinv, ncasc, d64)
                assert np.array_equal(d64.cpu().numpy().view(np.uint64),
                                      rg.avgrad(nvinv, ncasc, x64).view(np.uint64))
        w = rng.uniform(0, 1, nnpinv).astype(np.float32)
        x = rng.standard_normal(nnpinv).astype(np.float32)
        dx = torch.from_numpy(x).to(dev)
        ctx.wtgrad(torch.from_numpy(w).to(dev), dx)
        assert np.array_equal(dx.cpu().numpy().view(np.uint32), oracle.wtgrad(w, x).view(np.uint32))
    finally:
        ctx.close()
