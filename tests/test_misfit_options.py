"""Misfit / adjoint-source options: NORM (COBJ4 objfn.f:5-175, BPRESID4
objfn.f:757-847), IRESTP (CRESID objfn.f:953-1012), IBPHASE (HDIFFER
adjgrad.f90:528-566) and the DTMAX phase-jump tests.

CPU part: the oracle's restatement pinned against closed forms written here
in numpy (HDIFFER's half differentiators, the amplitude- and phase-only
residuals, the L1 / Huber / combination terms, the back-propagation filter
as a scaling of the right-hand side, DTMAX switching residuals off).
GPU part: fem25_misfit_dev and fem25_misfit_noalloc_dev against the oracle
for every option set.  Tolerances: bit-identical wherever the arithmetic is
+ - * / sqrt (IRESTP 2, 3 without DTMAX), NaN where the reference's NORM 4
residual is NaN; where phases are taken (IRESTP 1, DTMAX), 1e-6 of the
larger of the largest magnitude and w_max^2 = 2.25 (the phase-only residual
is a difference of unit phasors times w^2), and 1e-4 for the L1 norm with
phase-only residuals, whose normalisation by |DIF| magnifies the rounding of
nearly equal phases -- because atan2f / cosf / sinf of the device and the
host library differ in the last bits."""
import numpy as np
import pytest

import oracle
from fem25_b200 import Context, synth
from tests import helpers


@pytest.fixture(scope="module")
def case():
    mesh, pairs, _ = synth.make_config(0)
    g = oracle.graph_build(mesh)
    rng = np.random.default_rng(88)
    mrdof = helpers.surface_receivers(mesh, g, 20)
    nrec = len(mrdof)
    yrec = rng.uniform(-500, 500, nrec)
    recv = (1 + 0.1j * rng.standard_normal((nrec, 3))).astype(np.complex64)
    nsrc = 3
    sol = (rng.standard_normal((nsrc, g.ndof)) + 1j * rng.standard_normal((nsrc, g.ndof))).astype(np.complex64)
    obs = (rng.standard_normal((nsrc, nrec, 3)) + 1j * rng.standard_normal((nsrc, nrec, 3))).astype(np.complex64)
    obs[0, 4, 2] = 0  # an absent observation
    w = rng.uniform(0.5, 1.5, (nsrc, nrec, 3)).astype(np.float32)
    f, py = pairs[6]
    return mesh, g, mrdof, yrec, recv, sol, obs, w, f, py


def _orc(c, s, **kw):
    mesh, g, mrdof, yrec, recv, sol, obs, w, f, py = c
    return oracle.misfit(g.ndof, mrdof, yrec, f, py, 23.0, recv, sol[s], obs[s], w[s], **kw)


def test_hdiffer_closed_forms():
    f = 0.37
    om = 2 * np.pi * f
    h = {k: oracle.hdiffer(k, f) for k in range(7)}
    r = np.sqrt(om / 2)
    exp = {0: 1, 1: r * (1 - 1j), 2: -r * (1 - 1j), 3: r * (1 + 1j), 4: -r * (1 + 1j),
           5: 1j * om, 6: 1j}
    for k in range(7):
        assert abs(h[k] - exp[k]) <= 1e-6 * abs(exp[k]), (k, h[k], exp[k])


def test_ibphase_scales_the_adjoint_source(case):
    _, rhs0, m0 = _orc(case, 0)
    f = case[-2]
    for k in range(1, 7):
        _, rk, mk = _orc(case, 0, ibphase=k)
        h = oracle.hdiffer(k, f)
        # RESID_DRHS: RHS = conj(HFACT * RESID) = conj(HFACT) * conj(RESID)
        ref = np.conj(h) * rhs0.astype(np.complex128)
        assert np.abs(rk - ref).max() <= 1e-6 * np.abs(ref).max(), k
        assert mk == m0  # the objective does not see the filter


def _pairs(case, s):
    """(obs, est) in the objective's frame and the shifted (u, v, w) frame."""
    mesh, g, mrdof, yrec, recv, sol, obs, w, f, py = case
    est, _, _ = _orc(case, s)
    th = np.float32(23.0) * np.float32(0.017453292519943295)
    ct, st = np.cos(th), np.sin(th)
    er = est.astype(np.complex128).copy()
    er[:, 0] = est[:, 0] * ct - est[:, 1] * st
    er[:, 1] = est[:, 0] * st + est[:, 1] * ct
    sh = np.exp(-1j * 2 * np.pi * f * py * yrec)[:, None]
    return obs[s].astype(np.complex128), er, sh


def test_objective_norms_closed_forms(case):
    mesh, g, mrdof, yrec, recv, sol, obs, w, f, py = case
    o, er, _ = _pairs(case, 1)
    ww = w[1].astype(np.float64)
    pres = o != 0
    dif = (o - er)[pres]
    sw = np.abs(ww[pres])
    l1 = np.sum(np.abs(sw * dif))
    _, _, m1 = _orc(case, 1, norm=1)
    assert abs(m1 - l1) <= 1e-5 * l1
    eps, thr = 0.7, 1.1
    a = np.abs(sw * dif)
    hub = np.sum(np.where(a <= eps, a * a / (2 * eps), a - eps / 2))
    _, _, m3 = _orc(case, 1, norm=3, eps=eps)
    assert abs(m3 - hub) <= 1e-5 * hub
    comb = np.sum(np.where(np.abs(dif) <= thr, a * a / (2 * eps * eps), a / eps))
    _, _, m4 = _orc(case, 1, norm=4, eps=eps, thresh=thr)
    assert abs(m4 - comb) <= 1e-5 * comb
    # amplitude-only and phase-only L2 terms
    _, _, ma = _orc(case, 1, irestp=2)
    ra = np.sum(sw ** 2 * (np.abs(o[pres]) - np.abs(er[pres])) ** 2)
    assert abs(ma - ra) <= 1e-5 * ra
    _, _, mp = _orc(case, 1, irestp=1)
    rp = np.sum(sw ** 2 * np.abs(np.exp(1j * np.angle(o[pres])) - np.exp(1j * np.angle(er[pres]))) ** 2)
    assert abs(mp - rp) <= 1e-5 * rp


def _unrot_conj(res, mrdof, ndof):
    th = np.float32(-23.0) * np.float32(0.017453292519943295)
    ct, st = np.cos(th), np.sin(th)
    rr = res.copy()
    rr[:, 0] = res[:, 0] * ct - res[:, 1] * st
    rr[:, 1] = res[:, 0] * st + res[:, 1] * ct
    rhs = np.zeros(ndof, np.complex128)
    rhs[mrdof.reshape(-1) - 1] = rr.reshape(-1)
    return np.conj(rhs)


def test_backprop_residuals_closed_forms(case):
    mesh, g, mrdof, yrec, recv, sol, obs, w, f, py = case
    o, er, sh = _pairs(case, 2)
    ww = w[2].astype(np.float64)
    ob, es = o * sh, er * sh
    dif = np.where(o != 0, ob - es, 0)
    forms = {
        dict(norm=1).__repr__(): np.where(o != 0, ww * dif / np.where(dif != 0, np.abs(dif), 1), 0),
        dict(irestp=2).__repr__(): np.where(o != 0, ww ** 2 * (np.abs(ob) - np.abs(es)), 0),
        dict(irestp=1).__repr__(): np.where(o != 0, ww ** 2 * (np.exp(1j * np.angle(ob)) -
                                                               np.exp(1j * np.angle(es))), 0),
    }
    for kw in (dict(norm=1), dict(irestp=2), dict(irestp=1)):
        _, rhs, _ = _orc(case, 2, **kw)
        ref = _unrot_conj(forms[repr(kw)], mrdof, g.ndof)
        assert np.abs(rhs - ref).max() <= 2e-6 * np.abs(ref).max(), kw
    # BPRESID4 keeps EPS = 0 for NORM > 2: Huber is the L1 residual, the
    # combination norm is not finite where there are observations
    _, r1, _ = _orc(case, 2, norm=1)
    _, r3, _ = _orc(case, 2, norm=3, eps=0.5)
    assert np.array_equal(r1.view(np.uint32), r3.view(np.uint32))
    _, r4, _ = _orc(case, 2, norm=4, eps=0.5, thresh=1.0)
    rows = mrdof.reshape(-1)[(o != 0).reshape(-1)] - 1
    assert not np.isfinite(r4[rows]).any()
    # DTMAX: a tiny limit zeroes every residual, a huge one changes nothing
    _, rz, _ = _orc(case, 2, dtmax=1e-9)
    assert np.abs(rz).max() == 0.0
    _, r2, _ = _orc(case, 2)
    _, rbig, _ = _orc(case, 2, dtmax=1e9)
    assert np.array_equal(r2.view(np.uint32), rbig.view(np.uint32))


OPTION_SETS = (
    [dict(norm=n, irestp=r, ibphase=b) for n in (1, 2, 3) for r in (2, 3) for b in (0, 1, 4)] +
    [dict(norm=3, irestp=3, eps=0.8), dict(norm=4, irestp=3, eps=0.8, thresh=1.2),
     dict(norm=4, irestp=2, eps=0.5, thresh=0.9, ibphase=5)] +
    [dict(irestp=1, ibphase=2), dict(norm=1, irestp=1, ibphase=6), dict(dtmax=0.05),
     dict(dtmax_obj=0.05, ibphase=3), dict(irestp=1, dtmax=0.05, dtmax_obj=0.05)])


def _phase(kw):
    return kw.get("irestp") == 1 or kw.get("dtmax", 0) > 0 or kw.get("dtmax_obj", 0) > 0


def _same(a, b, tol):
    a, b = np.asarray(a), np.asarray(b)
    na, nb = np.isnan(a.view(np.float32)), np.isnan(b.view(np.float32))
    assert np.array_equal(na, nb)
    av, bv = a.view(np.float32)[~na], b.view(np.float32)[~nb]
    if tol == 0:
        assert np.array_equal(av.view(np.uint32), bv.view(np.uint32))
    else:
        fin = np.isfinite(bv)
        assert np.array_equal(np.isfinite(av), fin)
        # phase-only residuals are differences of unit phasors scaled by w^2
        # (w <= 1.5): rounding is relative to that scale, not to the result
        scale = max(np.abs(bv[fin]).max() if fin.any() else 0.0, 2.25)
        assert np.abs(av[fin] - bv[fin]).max() <= tol * scale


@pytest.mark.gpu
@pytest.mark.parametrize("kw", OPTION_SETS, ids=lambda k: "-".join(f"{a}{v}" for a, v in k.items()))
def test_gpu_misfit_options_match_oracle(case, kw):
    torch = pytest.importorskip("torch")
    mesh, g, mrdof, yrec, recv, sol, obs, w, f, py = case
    dev = torch.device("cuda:0")
    ctx = Context(mesh, g)
    try:
        ctx.misfit_options(**kw)
        nsrc = sol.shape[0]
        d_sol = torch.from_numpy(sol).to(dev)
        d_rhs = torch.zeros((nsrc, g.ndof), dtype=torch.complex64, device=dev)
        est, mis = ctx.misfit(nsrc, mrdof, yrec, f, py, 23.0, recv, d_sol, obs, w, d_rhs)
        rhs = d_rhs.cpu().numpy()
        # the L1 residual normalises DIF (objfn.f:803-804): with phases its
        # rounding grows as 1 / |DIF| for nearly equal phases
        tol = (1e-4 if kw.get("norm") == 1 and kw.get("irestp") == 1 else 1e-6) if _phase(kw) else 0
        for s in range(nsrc):
            e_o, r_o, m_o = _orc(case, s, **kw)
            _same(est[s].reshape(-1).view(np.float32), e_o.reshape(-1).view(np.float32), 0)
            _same(rhs[s].view(np.float32), r_o.view(np.float32), tol)
            _same(np.float32(mis[s]).reshape(1), np.float32(m_o).reshape(1), tol)
        # the allocation-free entry point follows the same options, bit for bit
        d_obs, d_w = torch.from_numpy(obs).to(dev), torch.from_numpy(w).to(dev)
        d_est = torch.empty((nsrc, len(mrdof), 3), dtype=torch.complex64, device=dev)
        d_mis = torch.empty(nsrc, dtype=torch.float32, device=dev)
        d_rhs2 = torch.empty_like(d_rhs)
        ctx.misfit_noalloc(nsrc, mrdof, yrec, f, py, 23.0, recv, d_sol, d_obs, d_w, d_est, d_rhs2,
                           d_mis)
        torch.cuda.synchronize()
        _same(d_rhs2.cpu().numpy().view(np.float32), rhs.view(np.float32), 0)
        _same(d_mis.cpu().numpy(), mis.astype(np.float32), 0)
    finally:
        ctx.close()
