"""CPU checks of the oracle (the CPU restatement of the reference hot path).

The reference ships no golden vectors for this path, so the oracle is pinned
by closed-form properties of its tables, element invariants, its own
committed fixtures (tests/golden) and a finite-difference check of the
gradient through a full assemble + direct solve."""
import os

import numpy as np
import pytest

import oracle
from fem25_b200 import synth
from tests import helpers

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_lobatto_rule_closed_form():
    for n in (5, 13):
        x, w = oracle.lobatto(n)
        # interior nodes are the roots of P'_{n-1}
        P = np.polynomial.legendre.Legendre.basis(n - 1)
        roots = np.sort(P.deriv().roots().real)
        assert np.allclose(x[1:-1], roots, atol=1e-14)
        assert x[0] == -1.0 and x[-1] == 1.0
        assert abs(w.sum() - 2.0) < 1e-14
        # exact for polynomials up to degree 2n-3
        for k in range(0, 2 * n - 2):
            exact = 0.0 if k % 2 else 2.0 / (k + 1)
            assert abs(np.sum(w * x ** k) - exact) < 1e-13


def test_shape_function_tables():
    xw, shl = oracle.tables(4)
    xi = xw[0]
    assert xi[6] == 0.0  # midpoint forced to zero (dshl.f:145)
    gll, _ = oracle.lobatto(5)
    gll[2] = 0.0
    # N_a = l_i(xi) l_j(eta), a = j*5 + i  (dshl.f:41-62)
    def lag(k, t, deriv=False):
        others = [gll[m] for m in range(5) if m != k]
        p = np.poly1d(np.poly(others)) / np.prod([gll[k] - o for o in others])
        return (p.deriv() if deriv else p)(t)
    for iz in (0, 3, 12):
        for ix in (0, 5, 6):
            for a in (0, 7, 24):
                i, j = a % 5, a // 5
                ref_n = lag(i, xi[ix]) * lag(j, xi[iz])
                ref_dx = lag(i, xi[ix], True) * lag(j, xi[iz])
                ref_dz = lag(i, xi[ix]) * lag(j, xi[iz], True)
                got = shl[iz, ix, a]
                assert abs(got[2] - ref_n) < 1e-13
                assert abs(got[0] - ref_dx) < 1e-12
                assert abs(got[1] - ref_dz) < 1e-12
    # partition of unity and zero-sum derivatives at every quadrature point
    assert np.allclose(shl[..., 2].sum(-1), 1.0, atol=1e-13)
    assert np.allclose(shl[..., 0].sum(-1), 0.0, atol=1e-12)
    assert np.allclose(shl[..., 1].sum(-1), 0.0, atol=1e-12)


def test_element_matrix_invariants(small_case):
    mesh, _ = small_case
    ie = [e for e in range(mesh.nelem) if chr(mesh.cdomain[e]) == "I"][0]
    f, py = 0.5, 1.3e-4
    me, ce = oracle.element_matrix(mesh, ie, "B", f, py)
    A = me + ce
    # KM25ISOQ is Hermitian for real media (estiff25.f:142-150)
    assert np.abs(A - A.conj().T).max() < 1e-9 * np.abs(A).max()
    # static (omega = 0): rigid translations in x, y, z are in the null space
    me0, ce0 = oracle.element_matrix(mesh, ie, "B", 1e-12, 0.0)
    K0 = me0 + ce0
    for comp in range(3):
        t = np.zeros(75)
        t[comp::3] = 1.0
        assert np.abs(K0 @ t).max() < 1e-9 * np.abs(K0).max()
    # mass: -omega^2 sum_ab M_ab over one component = -omega^2 int rho dA
    me1, _ = oracle.element_matrix(mesh, ie, "B", 1.0, 0.0)
    mass = -me1[0::3, 0::3].sum() / (2 * np.pi) ** 2
    ia = mesh.ieng[ie] - 1
    x, z = mesh.xlocs[ia], mesh.zlocs[ia]
    area = 0.5 * abs(np.dot(x, np.roll(z, -1)) - np.dot(z, np.roll(x, -1)))
    rho_mean = mesh.dens[ia].mean()
    assert abs(mass / (area * rho_mean) - 1.0) < 1e-12


def test_oracle_c64_is_fp32_of_c128(small_case):
    mesh, pairs = small_case
    g = oracle.graph_build(mesh)
    c128, c64 = oracle.asmble(mesh, g, "B", *pairs[3])
    err = helpers.row_norm_err(c64.astype(np.complex128), c128, g.irptr)
    assert err < 5e-7


def test_graph_structure(small_case):
    mesh, _ = small_case
    g = oracle.graph_build(mesh)
    assert g.irptr[0] == 1 and g.irptr[-1] - 1 == g.nzero
    rows = np.repeat(np.arange(g.ndof), np.diff(g.irptr))
    cols = g.jcptr - 1
    # sorted, distinct columns per row and a symmetric pattern
    assert np.all((np.diff(cols) > 0) | (np.diff(rows) > 0))
    s = set(zip(rows.tolist(), cols.tolist()))
    assert all((c, r) in s for r, c in list(s)[:2000])
    # every DOF classified A/E/I/B
    assert set(bytes(g.cnp)) <= set(b"AEIB")


def test_golden_fixtures():
    path = os.path.join(GOLDEN, "oracle_small.npz")
    if not os.path.exists(path):
        pytest.skip("golden fixtures not generated")
    ref = np.load(path)
    from tests.golden.make_golden import compute
    got = compute()
    for k in ref.files:
        a, b = np.ascontiguousarray(ref[k]), np.ascontiguousarray(got[k])
        assert a.shape == b.shape, k
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), k


def test_oracle_gradient_finite_difference(small_case):
    """Exact lambda/mu/rho adjoint of the oracle vs central differences of the
    L2 misfit through assemble + direct solve (h = 1e-4 relative)."""
    mesh, pairs = small_case
    g = oracle.graph_build(mesh)
    mrdof = helpers.surface_receivers(mesh, g, 6)
    fwi = helpers.DirectFWI(g, mrdof)
    use = [pairs[2], pairs[9]]
    rng = np.random.default_rng(5)
    f_src = helpers.point_force_rhs(g, mrdof[len(mrdof) // 2])
    obs = [rng.standard_normal(len(fwi.rdofs)) * 1e-9 + 1j * rng.standard_normal(len(fwi.rdofs)) * 1e-9
           for _ in use]

    def chi_grad(m, want_grad):
        chi = 0.0
        grad = np.zeros((3, mesh.nnpg))
        for (f, py), ob in zip(use, obs):
            c128, _ = oracle.asmble(m, g, "B", f, py, want64=False)
            c, u, lam = fwi.misfit_and_fields(c128, f_src, ob)
            chi += c
            if want_grad:
                oracle.grad_exact(m, g, f, py, u[None], lam[None], out=grad)
        return chi, grad

    chi0, grad = chi_grad(mesh, True)
    # perturb anchors that touch no PML element
    touch = np.zeros(mesh.nnpg, bool)
    for e in range(mesh.nelem):
        if chr(mesh.cdomain[e]) == "A":
            touch[mesh.ieng[e] - 1] = True
    base = np.stack([mesh.ecoeff[0], mesh.ecoeff[1], mesh.dens])
    h = 1e-4

    def cfd(dm, hh):
        mp, mm = _perturbed(mesh, base + hh * dm), _perturbed(mesh, base - hh * dm)
        return (chi_grad(mp, False)[0] - chi_grad(mm, False)[0]) / (2 * hh)

    for trial in range(3):
        d = rng.standard_normal((3, mesh.nnpg)) * ~touch
        dm = d * base
        an = float(np.sum(grad * dm))
        # central differences at h and h/2, Richardson-extrapolated to remove
        # the O(h^2) truncation term
        fd = (4.0 * cfd(dm, h / 2) - cfd(dm, h)) / 3.0
        assert abs(fd - an) <= 1e-6 * abs(an), (trial, fd, an)


def _perturbed(mesh, m3):
    import copy
    m = copy.copy(mesh)
    m.ecoeff = np.ascontiguousarray(m3[:2])
    m.dens = np.ascontiguousarray(m3[2])
    return m


# ---------------------------------------------------------------------------
# dispersive media (KMDAMP / CMDAMP with VCMPLX complex velocities)
# ---------------------------------------------------------------------------
def _homogeneous(nx=6, nz=4):
    mesh, pairs, _ = synth.make_config(0, nx=nx, nz=nz)
    synth.set_model_from_velocities(mesh, np.full(mesh.nnpg, 3000.0), np.full(mesh.nnpg, 1730.0),
                                    np.full(mesh.nnpg, 2500.0))
    return mesh, pairs


@pytest.mark.parametrize("dom", ["I", "A"])
def test_dispersive_without_damping_is_density_normalised(dom):
    """All Q = 9999 (the reference's 'no damping'), homogeneous medium:
    KMDAMP / CMDAMP interpolate velocities instead of moduli and leave out
    the density, so A_disp = A_standard / rho up to rounding (all 9 blocks,
    stiffness, mass and the i omega py terms, PML stretching included)."""
    mesh, pairs = _homogeneous()
    e = int(np.flatnonzero(mesh.cdomain == ord(dom))[0])
    f, py = pairs[9]
    me, ce = oracle.element_matrix(mesh, e, "B", f, py)
    ref = (me + ce) / 2500.0
    mesh.qp = np.full(mesh.nnpg, 9999.0)
    mesh.qs = np.full(mesh.nnpg, 9999.0)
    mesh.freq0, mesh.ldisp = 1.0, True
    me_d, ce_d = oracle.element_matrix(mesh, e, "B", f, py)
    got = me_d + ce_d
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_dispersive_damping_scales_with_inverse_q():
    """Finite Q: the operator departs from the undamped one by O(1/Q)
    (Aki & Richards 5.94: v (1 + ln(f/f0)/(pi Q)) - i v / (2Q)); doubling Q
    halves the departure to first order, and Q = 9999 gives none."""
    mesh, pairs = _homogeneous()
    e = int(np.flatnonzero(mesh.cdomain == ord("I"))[0])
    f, py = 0.5, pairs[5][1]
    mesh.freq0, mesh.ldisp = 1.0, True

    def op(qp, qs):
        mesh.qp = np.full(mesh.nnpg, qp)
        mesh.qs = np.full(mesh.nnpg, qs)
        me, ce = oracle.element_matrix(mesh, e, "B", f, py)
        return me + ce

    a0 = op(9999.0, 9999.0)
    d1 = np.abs(op(2.25 * 200.0, 200.0) - a0).max()
    d2 = np.abs(op(2.25 * 400.0, 400.0) - a0).max()
    assert d1 > 0 and abs(d1 / d2 - 2.0) < 0.05


# ---------------------------------------------------------------------------
# DABMKISOB25: alpha / beta derivatives of the density-normalised operator
# ---------------------------------------------------------------------------
def test_dabmkisob25_matches_central_difference():
    """With rho = 1 the KM25ISOQ operator interpolates alpha^2 = lambda + 2 mu
    and beta^2 = mu, the model DABMKISOB25 differentiates (DAB = 2 alpha N_p,
    2 beta N_p).  The operator is quadratic in alpha_p and beta_p, so a
    central difference reproduces dM/dalpha + dK/dalpha and the beta pair up
    to rounding (all 9 blocks, mass and the i omega py terms)."""
    mesh, pairs, _ = synth.make_config(0, nx=6, nz=4)
    rng = np.random.default_rng(4)
    vp = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, mesh.nnpg))
    vs = 1730.0 * (1 + 0.05 * rng.uniform(-1, 1, mesh.nnpg))
    synth.set_model_from_velocities(mesh, vp, vs, np.ones(mesh.nnpg))
    e = int(np.flatnonzero(mesh.cdomain == ord("I"))[0])
    inpg = int(mesh.ieng[e, 2])          # an anchor of the element (1-based)
    f, py = pairs[7]
    dmda, dkda, dmdb, dkdb = oracle.dabm_element(mesh, e, inpg, f, py)
    p = inpg - 1
    a0, b0 = vp[p], vs[p]

    def op(alpha, beta):
        m = synth.make_config(0, nx=6, nz=4)[0]
        a, b = vp.copy(), vs.copy()
        a[p], b[p] = alpha, beta
        synth.set_model_from_velocities(m, a, b, np.ones(m.nnpg))
        me, ce = oracle.element_matrix(m, e, "B", f, py)
        return me + ce

    h = 1e-3 * a0
    fd_a = (op(a0 + h, b0) - op(a0 - h, b0)) / (2 * h)
    got_a = dmda + dkda
    assert np.abs(got_a - fd_a).max() <= 1e-8 * np.abs(fd_a).max()
    h = 1e-3 * b0
    fd_b = (op(a0, b0 + h) - op(a0, b0 - h)) / (2 * h)
    got_b = dmdb + dkdb
    assert np.abs(got_b - fd_b).max() <= 1e-8 * np.abs(fd_b).max()


def test_addblk_touches_only_exterior_dofs(small_case):
    """ADDBLK adds the background field on the 'E' DOFs only, in COMPLEX*8."""
    mesh, _ = small_case
    g = oracle.graph_build(mesh)
    rng = np.random.default_rng(9)
    ue = (rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
    sol = (rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
    out = oracle.addblk(g, ue, sol)
    ext = g.cnp == ord("E")
    assert ext.any() and (~ext).any()
    assert np.array_equal(out[~ext], sol[~ext])
    assert np.array_equal(out[ext], (sol + ue)[ext])


@pytest.mark.parametrize("accumulate", [False, True])
def test_met225_matches_numpy_restatement(small_case, accumulate):
    """MET225_MOD's FP32 Hessian-vector buffers against an FP64 numpy
    evaluation of the same sums built from the oracle's DABMKISOB25 element
    matrices (weights ELEM_WTS, CONJG dot products, only the last connected
    element unless accumulate)."""
    mesh, pairs = small_case
    g = oracle.graph_build(mesh)
    rg = oracle.RefGrad(mesh, g)
    f, py = pairs[1]
    rng = np.random.default_rng(21)
    vec = [(rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
           for _ in range(4)]
    adjlam, nu, alpha, wave = vec
    p1, p2 = rg.met225(f, py, adjlam, nu, alpha, wave, cinvtype="PS", accumulate=accumulate)
    lm = g.lm.reshape(mesh.nelem, -1)
    r1 = np.zeros_like(p1, dtype=np.float64)
    r2 = np.zeros_like(r1)
    col = 0
    for p in range(mesh.nnpg):
        if rg.maskg[p] <= 0:
            continue
        rows = rg.icsc[rg.jcsc[col] - 1:rg.jcsc[col + 1] - 1]
        pos = {int(d): k for k, d in enumerate(rows)}
        t1 = np.zeros((2, len(rows)), np.complex128)
        t2 = np.zeros_like(t1)
        for ic in range(rg.ncon):
            e = rg.mconn[ic, p]
            if e <= 0:
                break
            if not accumulate:
                t1[:] = 0
                t2[:] = 0
            dmda, dkda, dmdb, dkdb = oracle.dabm_element(mesh, e - 1, p + 1, f, py)
            dofs = lm[e - 1]
            ok = dofs > 0
            w = float(np.float32(rg.elem_wts[e - 1]))
            for v, cm in enumerate((dmda + dkda, dmdb + dkdb)):
                sub = cm[np.ix_(ok, ok)]
                idx = [pos[int(d)] for d in dofs[ok]]
                t1[v, idx] += w * sub @ wave.astype(np.complex128)[dofs[ok] - 1]
                t2[v, idx] += w * sub @ alpha.astype(np.complex128)[dofs[ok] - 1]
        for v in range(2):
            ia = (rg.maskg[p] - 1) * 2 + v
            r1[ia] = -np.real(np.sum(np.conj(t1[v]) * nu[rows - 1]))
            r2[ia] = -np.real(np.sum(np.conj(t2[v]) * adjlam[rows - 1]))
        col += 1
    assert col == rg.nnpinv
    for got, ref in ((p1, r1), (p2, r2)):
        assert np.max(np.abs(got - ref)) <= 2e-4 * np.max(np.abs(ref))


@pytest.mark.parametrize("accumulate", [False, True])
def test_cadj_nu_alpha_matches_numpy_restatement(small_case, accumulate):
    """CADJ_NU_ALPHA's FP32 right-hand sides (nu and alpha fields) and P3
    buffer against an FP64 numpy evaluation from the oracle's DABMKISOB25
    element matrices: RHSALP = sum w_e V_p C_e WAVE, RHSBNU = sum conj(w_e V_p
    C_e)^T ADJLAM, P3 from the last connected element unless accumulate."""
    mesh, pairs = small_case
    g = oracle.graph_build(mesh)
    rg = oracle.RefGrad(mesh, g)
    f, py = pairs[0]
    rng = np.random.default_rng(31)
    adjlam, wave = [(rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof))
                    .astype(np.complex64) for _ in range(2)]
    v = rng.standard_normal(2 * rg.nnpinv).astype(np.float32)
    rb, ra, p3 = rg.cadj_nu_alpha(f, py, v, adjlam, wave, cinvtype="PS", accumulate=accumulate)
    lm = g.lm.reshape(mesh.nelem, -1)
    adj64, wave64 = adjlam.astype(np.complex128), wave.astype(np.complex128)
    ref_b = np.zeros(g.ndof, np.complex128)
    ref_a = np.zeros(g.ndof, np.complex128)
    ref_p3 = np.zeros(p3.shape)
    col = 0
    for p in range(mesh.nnpg):
        if rg.maskg[p] <= 0:
            continue
        rows = rg.icsc[rg.jcsc[col] - 1:rg.jcsc[col + 1] - 1]
        pos = {int(d): k for k, d in enumerate(rows)}
        temp = np.zeros((2, len(rows)), np.complex128)
        for ic in range(rg.ncon):
            e = rg.mconn[ic, p]
            if e <= 0:
                break
            if not accumulate:
                temp[:] = 0
            dmda, dkda, dmdb, dkdb = oracle.dabm_element(mesh, e - 1, p + 1, f, py)
            dofs = lm[e - 1]
            ok = dofs > 0
            d = dofs[ok] - 1
            for var, cm in enumerate((dmda + dkda, dmdb + dkdb)):
                wv = float(np.float32(rg.elem_wts[e - 1])) * float(v[(rg.maskg[p] - 1) * 2 + var])
                sub = wv * cm[np.ix_(ok, ok)]
                y = sub @ wave64[d]
                ref_a[d] += y
                ref_b[d] += np.conj(sub).T @ adj64[d]
                temp[var, [pos[int(x)] for x in dofs[ok]]] += y
        for var in range(2):
            ref_p3[(rg.maskg[p] - 1) * 2 + var] = -np.real(np.sum(np.conj(temp[var]) *
                                                                  adj64[rows - 1]))
        col += 1
    for got, ref in ((ra, ref_a), (rb, ref_b), (p3, ref_p3)):
        assert np.max(np.abs(got - ref)) <= 2e-4 * np.max(np.abs(ref))


def test_pchadj_matches_numpy_restatement(small_case):
    """PCHADJ's Jacobian block JACL = G^T F and the preconditioner update
    HESSB += REAL(JACL^H JACL) (FP32) against FP64 numpy, 'PS' layout."""
    mesh, pairs = small_case
    g = oracle.graph_build(mesh)
    rg = oracle.RefGrad(mesh, g)
    rng = np.random.default_rng(41)
    nrhs = 6
    grns = (rng.standard_normal((nrhs, g.ndof)) + 1j * rng.standard_normal((nrhs, g.ndof))
            ).astype(np.complex64)
    fmat = (rng.standard_normal((2, rg.nz)) + 1j * rng.standard_normal((2, rg.nz))
            ).astype(np.complex64)
    hess0 = rng.standard_normal(rg.nnpinv * 4).astype(np.float32)
    hess = hess0.copy()
    jacl = rg.pchadj(grns, fmat, hess)
    ref_h = hess0.astype(np.float64)
    for col in range(rg.nnpinv):
        i1, i2 = rg.jcsc[col] - 1, rg.jcsc[col + 1] - 1
        rows = rg.icsc[i1:i2] - 1
        j = grns[:, rows].astype(np.complex128) @ fmat[:, i1:i2].T.astype(np.complex128)
        assert np.allclose(jacl[2 * col:2 * col + 2].T, j, rtol=0, atol=1e-4 * np.abs(j).max())
        ref_h[4 * col:4 * col + 4] += np.real(j.conj().T @ j).reshape(-1)
    assert np.max(np.abs(hess - ref_h)) <= 2e-5 * np.max(np.abs(ref_h))


def test_gradient_covariance_form():
    """The algebra of the covariance gradient (k_grad_cov.cu) restated in
    numpy: per element the 15 weighted blocks of sum conj(lam) u^T, the 9
    combined blocks and the sum-factorised contraction with the 1D Lagrange
    factors of SHL, against the oracle's exact gradient (grad_exact) on a
    jittered, topographic layout, several pairs and sources."""
    mesh, pairs, _ = synth.make_config(4, nx=8, nz=6)
    g = oracle.graph_build(mesh)
    lm = np.asarray(g.lm).reshape(mesh.nelem, 75)
    use = [pairs[1], pairs[len(pairs) // 2], pairs[-1]]
    nsrc = 3
    rng = np.random.default_rng(91)
    shape = (len(use), nsrc, g.ndof)
    u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    lam = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ref = np.zeros((3, mesh.nnpg))
    for p, (f, py) in enumerate(use):
        oracle.grad_exact(mesh, g, f, py, u[p], lam[p], out=ref)
    xig, shl = oracle.tables()
    xq, wq = xig[0], xig[1]
    xn, _ = oracle.lobatto(5)
    xn[2] = 0.0
    # 1D Lagrange values l[q][i] and derivatives d[q][i] on the 5 GLL nodes
    lg = np.ones((13, 5))
    dg = np.zeros((13, 5))
    for i in range(5):
        oth = [k for k in range(5) if k != i]
        for k in oth:
            lg[:, i] *= (xq - xn[k]) / (xn[i] - xn[k])
        for m in oth:
            t = np.full(13, 1.0 / (xn[i] - xn[m]))
            for k in oth:
                if k != m:
                    t *= (xq - xn[k]) / (xn[i] - xn[k])
            dg[:, i] += t
    # SHL is the tensor product (node a = ix + 5 ie, point q = qx + 13 qz)
    assert np.allclose(np.einsum("xi,ze->zxei", lg, lg).reshape(13, 13, 25), shl[:, :, :, 2],
                       atol=1e-14)
    fx = {"N": lg, "X": dg, "E": lg}  # factor on xi for T_N, T_xi, T_eta
    fe = {"N": lg, "X": lg, "E": dg}  # factor on eta

    def Y(B, t):  # [ie][ix][qz][qx]
        return np.einsum("iej,ze,xj->izx", B.reshape(25, 5, 5), fe[t], fx[t]).reshape(5, 5, 13, 13)

    def F(Yt, t1):  # T_t1(q)^T Y(q)
        return np.einsum("eizx,xi,ze->zx", Yt, fx[t1], fe[t1])

    X, Z = np.meshgrid(xq, xq)  # [qz][qx]: X = xi, Z = eta
    W = np.outer(wq, wq)
    sf = 0.25 * np.array([(1 - X) * (1 - Z), (1 + X) * (1 - Z), (1 + X) * (1 + Z), (1 - X) * (1 + Z)])
    dsx = 0.25 * np.array([-(1 - Z), (1 - Z), (1 + Z), -(1 + Z)])
    dse = 0.25 * np.array([-(1 - X), -(1 + X), (1 + X), (1 - X)])
    out = np.zeros((3, mesh.nnpg))
    for e in range(mesh.nelem):
        if chr(mesh.cdomain[e]) == "A":
            continue
        dofs = lm[e]
        on = dofs > 0

        def gather(fld):
            v = np.zeros((len(use), nsrc, 75), complex)
            v[:, :, on] = fld[:, :, dofs[on] - 1]
            return v.reshape(len(use), nsrc, 25, 3).transpose(0, 1, 3, 2)  # [p][s][comp][node]

        U, L = gather(u), gather(lam)
        blk = {k: np.zeros((25, 25)) for k in ("R00", "R02", "R20", "R22", "R11", "P0", "P1",
                                               "P2", "W0", "W1", "W2", "I01", "I21", "I10", "I12")}
        for p, (f, py) in enumerate(use):
            om = 2.0 * np.pi * f
            wpy = om * py
            C = np.einsum("sci,sdj->cdij", np.conj(L[p]), U[p])
            for c, d in ((0, 0), (0, 2), (2, 0), (2, 2), (1, 1)):
                blk[f"R{c}{d}"] += C[c, d].real
            for c in range(3):
                blk[f"P{c}"] += wpy * wpy * C[c, c].real
                blk[f"W{c}"] += om * om * C[c, c].real
            for c, d in ((0, 1), (2, 1), (1, 0), (1, 2)):
                blk[f"I{c}{d}"] += wpy * C[c, d].imag
        sym = [0.5 * (blk[k] + blk[k].T) for k in ("R00", "R22", "R11")]
        S = blk["R02"] + blk["R20"].T
        G = [blk["I01"] - blk["I10"].T, blk["I21"] - blk["I12"].T]
        VA, VB, VC = blk["P1"], blk["P0"] + blk["P2"], blk["W0"] + blk["W1"] + blk["W2"]
        ie = mesh.ieng[e] - 1
        xa, za = mesh.xlocs[ie], mesh.zlocs[ie]
        dxdxi, dxdeta = np.tensordot(xa, dsx, 1), np.tensordot(xa, dse, 1)
        dzdxi, dzdeta = np.tensordot(za, dsx, 1), np.tensordot(za, dse, 1)
        rj = dxdxi * dzdeta - dxdeta * dzdxi
        ax, bx, az, bz = dzdeta / rj, -dzdxi / rj, -dxdeta / rj, dxdxi / rj
        xx, zz = [], []
        for B in sym:
            yx, ye = Y(B, "X"), Y(B, "E")
            fxx, fxe, fee = F(yx, "X"), F(ye, "X"), F(ye, "E")
            xx.append(ax * ax * fxx + 2 * ax * bx * fxe + bx * bx * fee)
            zz.append(az * az * fxx + 2 * az * bz * fxe + bz * bz * fee)
        yx, ye = Y(S, "X"), Y(S, "E")
        sxx, sxe, sex, see = F(yx, "X"), F(ye, "X"), F(yx, "E"), F(ye, "E")
        xsz = ax * az * sxx + ax * bz * sxe + bx * az * sex + bx * bz * see
        zsx = az * ax * sxx + az * bx * sxe + bz * ax * sex + bz * bx * see
        gl, gm = 0.0, 0.0
        for Gk, (c1, c2) in zip(G, ((ax, bx), (az, bz))):
            yn, yx, ye = Y(Gk, "N"), Y(Gk, "X"), Y(Gk, "E")
            gl = gl + c1 * F(yn, "X") + c2 * F(yn, "E")
            gm = gm - (c1 * F(yx, "N") + c2 * F(ye, "N"))
        va, vb, vc = (F(Y(V, "N"), "N") for V in (VA, VB, VC))
        tl = xx[0] + xsz + zz[1] + gl + va
        tm = 2 * xx[0] + zz[0] + zsx + xx[1] + 2 * zz[1] + xx[2] + zz[2] + gm + 2 * va + vb
        tr = -vc
        wgt = W * rj
        for a in range(4):
            out[:, ie[a]] += [np.sum(sf[a] * wgt * t) for t in (tl, tm, tr)]
    for m in range(3):
        assert np.linalg.norm(out[m] - ref[m]) <= 1e-12 * np.linalg.norm(ref[m]), m
