"""fem25_misfit_noalloc_dev, the misfit / adjoint-source entry point that
allocates no device memory, against fem25_misfit_dev on the same inputs.

The file name sorts last so that, in a full run, the entry point is first
called after every other test has used the library; run alone it is the
first call in a fresh process.  Tolerance: bit-identical (the misfit path of
fem25_misfit_dev is itself bit-exact against the oracle)."""
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from fem25_b200 import Context, Fem25Error, synth
from tests import helpers

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

_HDR = (Path(__file__).resolve().parents[1] / "include" / "fem25gpu.h").read_text()
MAX_REC = int(re.search(r"#define FEM25_NOALLOC_MAX_REC (\d+)", _HDR).group(1))
MAX_SRC_REC = int(re.search(r"#define FEM25_NOALLOC_MAX_SRC_REC (\d+)", _HDR).group(1))


@pytest.fixture(scope="module")
def case():
    mesh, pairs, _ = synth.make_config(0)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    yield mesh, pairs, g, ctx
    ctx.close()


def _inputs(mesh, g, nsrc, seed):
    rng = np.random.default_rng(seed)
    mrdof = helpers.surface_receivers(mesh, g, 20)
    nrec = len(mrdof)
    yrec = rng.uniform(-500, 500, nrec)
    recv = (1 + 0.1j * rng.standard_normal((nrec, 3))).astype(np.complex64)
    sol = (rng.standard_normal((nsrc, g.ndof)) + 1j * rng.standard_normal((nsrc, g.ndof))).astype(np.complex64)
    obs = (rng.standard_normal((nsrc, nrec, 3)) + 1j * rng.standard_normal((nsrc, nrec, 3))).astype(np.complex64)
    obs[0, 3, 1] = 0  # an absent observation
    w = rng.uniform(0.5, 1.5, (nsrc, nrec, 3)).astype(np.float32)
    return mrdof, yrec, recv, sol, obs, w


def test_noalloc_matches_misfit_dev_twice(case):
    mesh, pairs, g, ctx = case
    dev = torch.device("cuda:0")
    nsrc = 3
    f, py = pairs[6]
    mrdof, yrec, recv, sol, obs, w = _inputs(mesh, g, nsrc, 21)
    nrec = len(mrdof)
    d_sol = torch.from_numpy(sol).to(dev)
    # the existing entry point (host obs / wghts / est / misfit)
    d_rhs_ref = torch.zeros((nsrc, g.ndof), dtype=torch.complex64, device=dev)
    est_ref, mis_ref = ctx.misfit(nsrc, mrdof, yrec, f, py, 12.5, recv, d_sol, obs, w, d_rhs_ref)
    rhs_ref = d_rhs_ref.cpu().numpy()
    # the allocation-free one, device obs / wghts / est / misfit
    d_obs = torch.from_numpy(obs).to(dev)
    d_w = torch.from_numpy(w).to(dev)
    d_est = torch.empty((nsrc, nrec, 3), dtype=torch.complex64, device=dev)
    d_mis = torch.empty(nsrc, dtype=torch.float32, device=dev)
    d_rhs = torch.empty((nsrc, g.ndof), dtype=torch.complex64, device=dev)
    for call in range(2):
        for t in (d_est, d_mis, d_rhs):  # every output must be written by the call
            t.fill_(float("nan"))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        ctx.misfit_noalloc(nsrc, mrdof, yrec, f, py, 12.5, recv, d_sol, d_obs, d_w, d_est, d_rhs,
                           d_mis)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info(dev)[0]
        if call == 1:  # set-up (first call) done: free device memory must not move
            assert free1 == free0, (free0, free1)
        est = d_est.cpu().numpy()
        assert np.array_equal(est.view(np.uint32), est_ref.view(np.uint32)), call
        assert np.array_equal(d_rhs.cpu().numpy().view(np.uint32), rhs_ref.view(np.uint32)), call
        assert np.array_equal(d_mis.cpu().numpy().view(np.uint32), mis_ref.view(np.uint32)), call


def test_noalloc_rejects_sizes_beyond_scratch(case):
    mesh, pairs, g, ctx = case
    dev = torch.device("cuda:0")
    f, py = pairs[2]
    buf = torch.zeros(16, dtype=torch.complex64, device=dev)
    # too many receivers
    nrec = MAX_REC + 1
    mrdof = np.zeros((nrec, 3), np.int32)
    with pytest.raises(Fem25Error) as ei:
        ctx.misfit_noalloc(1, mrdof, np.zeros(nrec), f, py, 0.0, np.zeros((nrec, 3), np.complex64),
                           buf, buf, buf, buf, buf, buf)
    assert ei.value.code == 1 and "FEM25_NOALLOC_MAX_REC" in str(ei.value)
    # too many (source, receiver) pairs
    nrec = 20
    nsrc = MAX_SRC_REC // nrec + 1
    mrdof = np.zeros((nrec, 3), np.int32)
    with pytest.raises(Fem25Error) as ei:
        ctx.misfit_noalloc(nsrc, mrdof, np.zeros(nrec), f, py, 0.0, np.zeros((nrec, 3), np.complex64),
                           buf, buf, buf, buf, buf, buf)
    assert ei.value.code == 1 and "FEM25_NOALLOC_MAX_SRC_REC" in str(ei.value)


def _node_receivers(g, nrec):
    """nrec receivers at distinct unconstrained GLL nodes (MRDOF(3,NREC)),
    spread over the mesh: more than the free surface holds."""
    trip = np.unique(g.lm.reshape(-1, 3), axis=0)
    trip = trip[(trip > 0).all(axis=1)]
    assert len(trip) >= nrec, (len(trip), nrec)
    idx = np.linspace(0, len(trip) - 1, nrec).round().astype(int)
    return np.ascontiguousarray(trip[idx], np.int32)


@pytest.mark.parametrize("nrec", [300, MAX_REC])
def test_noalloc_many_receivers_match_misfit_dev(case, nrec):
    """Receiver counts beyond one 256-receiver staging chunk (and at the
    limit): every chunk's table offsets reach the kernels."""
    mesh, pairs, g, ctx = case
    dev = torch.device("cuda:0")
    nsrc = 2
    f, py = pairs[9]
    rng = np.random.default_rng(nrec)
    mrdof = _node_receivers(g, nrec)
    yrec = rng.uniform(-800, 800, nrec)
    recv = (1 + 0.1j * rng.standard_normal((nrec, 3))).astype(np.complex64)
    sol = (rng.standard_normal((nsrc, g.ndof)) + 1j * rng.standard_normal((nsrc, g.ndof))).astype(np.complex64)
    obs = (rng.standard_normal((nsrc, nrec, 3)) + 1j * rng.standard_normal((nsrc, nrec, 3))).astype(np.complex64)
    w = rng.uniform(0.5, 1.5, (nsrc, nrec, 3)).astype(np.float32)
    d_sol = torch.from_numpy(sol).to(dev)
    d_rhs_ref = torch.zeros((nsrc, g.ndof), dtype=torch.complex64, device=dev)
    est_ref, mis_ref = ctx.misfit(nsrc, mrdof, yrec, f, py, -31.0, recv, d_sol, obs, w, d_rhs_ref)
    d_obs = torch.from_numpy(obs).to(dev)
    d_w = torch.from_numpy(w).to(dev)
    d_est = torch.full((nsrc, nrec, 3), float("nan"), dtype=torch.complex64, device=dev)
    d_mis = torch.full((nsrc,), float("nan"), dtype=torch.float32, device=dev)
    d_rhs = torch.full((nsrc, g.ndof), float("nan"), dtype=torch.complex64, device=dev)
    ctx.misfit_noalloc(nsrc, mrdof, yrec, f, py, -31.0, recv, d_sol, d_obs, d_w, d_est, d_rhs, d_mis)
    torch.cuda.synchronize()
    assert np.array_equal(d_est.cpu().numpy().view(np.uint32), est_ref.view(np.uint32))
    assert np.array_equal(d_rhs.cpu().numpy().view(np.uint32), d_rhs_ref.cpu().numpy().view(np.uint32))
    assert np.array_equal(d_mis.cpu().numpy().view(np.uint32), mis_ref.view(np.uint32))


def test_noalloc_refuses_a_capturing_stream(case):
    """The receiver tables are staged from host buffers that live only during
    the call, so a call on a stream under capture is refused (nothing is
    enqueued) instead of recording copies from dead host memory."""
    mesh, pairs, g, ctx = case
    dev = torch.device("cuda:0")
    f, py = pairs[1]
    mrdof, yrec, recv, sol, obs, w = _inputs(mesh, g, 1, 5)
    nrec = len(mrdof)
    d_sol = torch.from_numpy(sol).to(dev)
    d_obs = torch.from_numpy(obs).to(dev)
    d_w = torch.from_numpy(w).to(dev)
    d_est = torch.zeros((1, nrec, 3), dtype=torch.complex64, device=dev)
    d_mis = torch.zeros(1, dtype=torch.float32, device=dev)
    d_rhs = torch.zeros((1, g.ndof), dtype=torch.complex64, device=dev)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    code = None
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            d_mis.add_(1.0)  # keeps the captured graph non-empty
            try:
                ctx.misfit_noalloc(1, mrdof, yrec, f, py, 0.0, recv, d_sol, d_obs, d_w, d_est,
                                   d_rhs, d_mis, stream=torch.cuda.current_stream(dev))
            except Fem25Error as e:
                code = e.code
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize()
    del graph
    assert code == 1
    # the context and the entry point still work after the refusal
    ctx.misfit_noalloc(1, mrdof, yrec, f, py, 0.0, recv, d_sol, d_obs, d_w, d_est, d_rhs, d_mis)
    torch.cuda.synchronize()
    assert np.isfinite(d_mis.cpu().numpy()).all()
