"""GPU parity of libfem25gpu (through its C ABI) against the CPU oracle.

Tolerances (CSR values are compared per row against the row's largest
magnitude, the definition used for every CSR error in this repository):
  * plain FP64 assembly vs oracle FP64:            <= 1e-12 (expected bit-exact)
  * COMPLEX*8 CDIST (reference FP32 accumulation): bit-exact
  * batched affine assembly vs oracle FP64:        <= 1e-12
  * exact gradient FP64 vs oracle:                 <= 1e-10 relative (2-norm)
  * exact gradient 3xTF32 tensor cores vs oracle:  <= 2e-5 relative (2-norm)
  * reference-compatible gradient, VFORCE25_2 forces, P_eff, misfit: bit-exact
"""
import numpy as np
import pytest

import oracle
from fem25_b200 import (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE,
                        Context, Fem25Error, synth)
from tests import helpers

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dev():
    return torch.device("cuda:0")


@pytest.fixture(scope="module")
def case0():
    mesh, pairs, _ = synth.make_config(0)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    yield mesh, pairs, g, ctx
    ctx.close()


def test_plain_assembly_matches_oracle(case0):
    mesh, pairs, g, ctx = case0
    for (f, py) in (pairs[0], pairs[7], pairs[15]):
        ref128, ref64 = oracle.asmble(mesh, g, "B", f, py)
        o128 = torch.zeros(g.nzero, dtype=torch.complex128, device=_dev())
        o64 = torch.zeros(g.nzero, dtype=torch.complex64, device=_dev())
        ctx.assemble("B", f, py, o128, o64)
        torch.cuda.synchronize()
        a128 = o128.cpu().numpy()
        a64 = o64.cpu().numpy()
        err = helpers.row_norm_err(a128, ref128, g.irptr)
        assert err <= 1e-12, err
        exact = np.mean(a128 == ref128)
        assert exact == 1.0, f"bit-identical fraction {exact}"
        assert np.array_equal(a64.view(np.uint32), ref64.view(np.uint32))


def test_asmble_driver_host_buffer(case0):
    mesh, pairs, g, ctx = case0
    f, py = pairs[4]
    _, ref64 = oracle.asmble(mesh, g, "S", f, py)
    out = ctx.asmble_driver("S", f, py)
    assert np.array_equal(out.view(np.uint32), ref64.view(np.uint32))


def test_asmble_driver_chunked_pinned_and_pageable():
    """fem25_asmble_driver computes elements in up to 16 chunks and copies each chunk's
    completed CSR rows while the next computes: the jittered, topographic
    layout at 48x20 elements (960 elements, 6 chunks) into pinned and
    pageable host buffers, both bit-exact to the oracle's COMPLEX*8 CDIST,
    twice in a row."""
    mesh, pairs, _ = synth.make_config(4, nx=48, nz=20)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    f, py = pairs[5]
    _, ref64 = oracle.asmble(mesh, g, "B", f, py)
    pinned = torch.empty(g.nzero, dtype=torch.complex64, pin_memory=True)
    for _ in range(2):
        pinned.fill_(float("nan"))
        ctx.asmble_driver("B", f, py, out=pinned)
        assert np.array_equal(pinned.numpy().view(np.uint32), ref64.view(np.uint32))
        page = ctx.asmble_driver("B", f, py)
        assert np.array_equal(page.view(np.uint32), ref64.view(np.uint32))
    ctx.close()


def test_batched_matches_oracle(case0):
    mesh, pairs, g, ctx = case0
    sel = [pairs[0], pairs[5], pairs[11], pairs[15], (0.8, 2.0e-4), (0.3, 0.0)]
    n = len(sel)
    stride = 2 * g.nzero
    ring = torch.zeros(n * stride, dtype=torch.float64, device=_dev())
    ctx.assemble_batch(["B"] * n, [p[0] for p in sel], [p[1] for p in sel], ring, stride, n)
    torch.cuda.synchronize()
    r = ring.view(n, g.nzero, 2).cpu().numpy()
    for k, (f, py) in enumerate(sel):
        ref128, _ = oracle.asmble(mesh, g, "B", f, py, want64=False)
        got = r[k, :, 0] + 1j * r[k, :, 1]
        err = helpers.row_norm_err(got, ref128, g.irptr)
        assert err <= 1e-12, (k, err)


def test_batched_ring_wraps(case0):
    mesh, pairs, g, ctx = case0
    sel = pairs[:7]
    stride = 2 * g.nzero + 2  # padded slots
    ring = torch.zeros(3 * stride, dtype=torch.float64, device=_dev())
    ctx.assemble_batch("S", [p[0] for p in sel], [p[1] for p in sel], ring, stride, 3)
    torch.cuda.synchronize()
    r = ring.view(3, stride).cpu().numpy()
    # system 6 lands in slot 0, system 4 in slot 1, system 5 in slot 2
    for k in (4, 5, 6):
        ref128, _ = oracle.asmble(mesh, g, "S", *sel[k], want64=False)
        got = r[k % 3, :2 * g.nzero:2] + 1j * r[k % 3, 1:2 * g.nzero:2]
        assert helpers.row_norm_err(got, ref128, g.irptr) <= 1e-12


_VARIANT_OUT = {}


@pytest.mark.parametrize("variant", range(10))
def test_stream_variants_agree(case0, variant, monkeypatch):
    """Every streaming variant the autotuner can pick (forced through
    FEM25_STREAM_VARIANT) writes the same bits: 19 systems = one launch of 16
    and one of 3, mixed CFTYPE and frequencies, slots that start 16 bytes past
    a 128-byte boundary with a stride that is not a multiple of 16."""
    mesh, pairs, g, _ = case0
    monkeypatch.setenv("FEM25_STREAM_VARIANT", str(variant))
    ctx = Context(mesh, g)
    n = 19
    sel = [(pairs[k % len(pairs)][0] * (1.0 + 0.05 * (k // 5)), pairs[(3 * k) % len(pairs)][1])
           for k in range(n)]
    cft = ["B" if k % 3 else "S" for k in range(n)]
    stride = 2 * g.nzero + 2
    buf = torch.zeros(2 + n * stride, dtype=torch.float64, device=_dev())
    ctx.assemble_batch(cft, [p[0] for p in sel], [p[1] for p in sel], buf[2:], stride, n)
    torch.cuda.synchronize()
    r = buf[2:].view(n, stride)
    if variant == 0:
        for k in (0, 15, 16, 18):
            ref128, _ = oracle.asmble(mesh, g, cft[k], *sel[k], want64=False)
            got = r[k, :2 * g.nzero].cpu().numpy()
            assert helpers.row_norm_err(got[0::2] + 1j * got[1::2], ref128, g.irptr) <= 1e-12, k
        _VARIANT_OUT[0] = r.clone()
    elif 0 in _VARIANT_OUT:
        assert torch.equal(r, _VARIANT_OUT[0])
    assert torch.count_nonzero(buf[:2]) == 0
    ctx.close()


@pytest.mark.parametrize("variant", [8, 9])
@pytest.mark.parametrize("nslots", [1, 3, 19])
def test_large_ring_variants_small_rings(case0, variant, nslots, monkeypatch):
    """The large-ring streaming variants take up to min(1024, nslots) systems
    per launch: with small rings each slot must still end with its last
    system, bit-identical to variant 0."""
    mesh, pairs, g, _ = case0
    n = 19
    sel = [(pairs[k % len(pairs)][0] * (1.0 + 0.03 * (k // 4)), pairs[(5 * k) % len(pairs)][1])
           for k in range(n)]
    cft = ["S" if k % 4 == 1 else "B" for k in range(n)]
    stride = 2 * g.nzero
    out = {}
    for v in (0, variant):
        monkeypatch.setenv("FEM25_STREAM_VARIANT", str(v))
        ctx = Context(mesh, g)
        ring = torch.full((nslots * stride,), float("nan"), dtype=torch.float64, device=_dev())
        ctx.assemble_batch(cft, [p[0] for p in sel], [p[1] for p in sel], ring, stride, nslots)
        torch.cuda.synchronize()
        assert ctx.tuning()["stream_variant"] == v
        out[v] = ring.clone()
        ctx.close()
    assert torch.equal(out[0], out[variant])
    k = n - 1
    ref128, _ = oracle.asmble(mesh, g, cft[k], *sel[k], want64=False)
    got = out[variant].view(nslots, stride)[k % nslots].cpu().numpy()
    assert helpers.row_norm_err(got[0::2] + 1j * got[1::2], ref128, g.irptr) <= 1e-12


def test_peff_matches_oracle(case0):
    mesh, pairs, g, ctx = case0
    _, a64 = oracle.asmble(mesh, g, "B", *pairs[3])
    rng = np.random.default_rng(3)
    nsrc = 3
    ue = (rng.standard_normal((nsrc, g.ndof)) + 1j * rng.standard_normal((nsrc, g.ndof))).astype(np.complex64)
    d_a = torch.from_numpy(a64).to(_dev())
    d_u = torch.from_numpy(ue).to(_dev())
    d_p = torch.zeros((nsrc, g.ndof), dtype=torch.complex64, device=_dev())
    ctx.asmb_peff(nsrc, d_a, d_u, d_p)
    got = d_p.cpu().numpy()
    for s in range(nsrc):
        ref = oracle.peff(g, a64, ue[s])
        assert np.array_equal(got[s].view(np.uint32), ref.view(np.uint32))


def test_addblk_matches_oracle(case0):
    mesh, pairs, g, ctx = case0
    rng = np.random.default_rng(4)
    nsrc = 3
    shape = (nsrc, g.ndof)
    ue = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    sol = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    d_u = torch.from_numpy(ue).to(_dev())
    d_s = torch.from_numpy(sol).to(_dev())
    ctx.addblk(nsrc, d_u, d_s)
    got = d_s.cpu().numpy()
    assert np.count_nonzero(g.cnp == ord("E")) > 0
    for s in range(nsrc):
        ref = oracle.addblk(g, ue[s], sol[s])
        assert np.array_equal(got[s].view(np.uint32), ref.view(np.uint32))


def test_gradient_fp64_matches_oracle():
    mesh, pairs, _ = synth.make_config(0, nx=10, nz=6)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    rng = np.random.default_rng(11)
    use = [pairs[1], pairs[6], pairs[13]]
    nsrc = 3
    u = rng.standard_normal((len(use), nsrc, g.ndof)) + 1j * rng.standard_normal((len(use), nsrc, g.ndof))
    lam = rng.standard_normal((len(use), nsrc, g.ndof)) + 1j * rng.standard_normal((len(use), nsrc, g.ndof))
    ref = np.zeros((3, mesh.nnpg))
    for p, (f, py) in enumerate(use):
        oracle.grad_exact(mesh, g, f, py, u[p], lam[p], out=ref)
    d_u = torch.from_numpy(u).to(_dev())
    d_l = torch.from_numpy(lam).to(_dev())
    d_g = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
    ctx.gradient([p[0] for p in use], [p[1] for p in use], nsrc, d_u, d_l, d_g, FEM25_PREC_FP64)
    got = d_g.cpu().numpy()
    for m in range(3):
        rel = np.linalg.norm(got[m] - ref[m]) / np.linalg.norm(ref[m])
        assert rel <= 1e-10, (m, rel)
    ctx.close()


_TILE_OUT = {}


@pytest.mark.parametrize("tile", [4, 2, 8])
def test_gradient_fp64_source_tiles_agree(tile, monkeypatch):
    """Every source-tile width the FP64 gradient's autotuner can pick gives
    the same gradient (sources are summed in the same order; only the
    cross-element atomics differ): 9 sources = 4 full tiles of 2 and a
    ragged one, a ragged tile of 4, a ragged tile of 8."""
    monkeypatch.setenv("FEM25_GRAD_TILE", str(tile))
    mesh, pairs, _ = synth.make_config(0, nx=10, nz=6)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    rng = np.random.default_rng(19)
    use = [pairs[2], pairs[11]]
    shape = (len(use), 9, g.ndof)
    u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    lam = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    d_g = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
    ctx.gradient([p[0] for p in use], [p[1] for p in use], 9, torch.from_numpy(u).to(_dev()),
                 torch.from_numpy(lam).to(_dev()), d_g, FEM25_PREC_FP64)
    assert ctx.tuning()["grad_tile"] == tile
    got = d_g.cpu().numpy()
    if tile == 4:
        ref = np.zeros((3, mesh.nnpg))
        for p, (f, py) in enumerate(use):
            oracle.grad_exact(mesh, g, f, py, u[p], lam[p], out=ref)
        for m in range(3):
            assert np.linalg.norm(got[m] - ref[m]) <= 1e-10 * np.linalg.norm(ref[m])
        _TILE_OUT[4] = got
    elif 4 in _TILE_OUT:
        for m in range(3):
            ref = _TILE_OUT[4][m]
            assert np.linalg.norm(got[m] - ref) <= 1e-13 * np.linalg.norm(ref), m
    ctx.close()


@pytest.mark.parametrize("prec", [FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE],
                         ids=["covariance", "pointwise"])
@pytest.mark.parametrize("nsrc", [1, 7])
def test_gradient_tf32x3_matches_oracle(nsrc, prec):
    """Split-precision tensor-core gradients.  Pointwise form: 3 pairs x 7
    sources = 21 combos exercises four full stages of 5 combos and a ragged
    one, nsrc=1 a stage of 3.  Covariance form: a partly filled 8-source
    stage per pair."""
    mesh, pairs, _ = synth.make_config(0, nx=10, nz=6)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    rng = np.random.default_rng(12 + nsrc)
    use = [pairs[2], pairs[9], pairs[14]]
    shape = (len(use), nsrc, g.ndof)
    u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    lam = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ref = np.zeros((3, mesh.nnpg))
    for p, (f, py) in enumerate(use):
        oracle.grad_exact(mesh, g, f, py, u[p], lam[p], out=ref)
    d_u = torch.from_numpy(u).to(_dev())
    d_l = torch.from_numpy(lam).to(_dev())
    for rep in range(2):
        d_g = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
        ctx.gradient([p[0] for p in use], [p[1] for p in use], nsrc, d_u, d_l, d_g, prec)
        got = d_g.cpu().numpy()
        for m in range(3):
            rel = np.linalg.norm(got[m] - ref[m]) / np.linalg.norm(ref[m])
            assert rel <= 2e-5, (rep, m, rel)
    ctx.close()


def test_gradient_finite_difference_gpu_pipeline():
    """GPU assembly + host direct solve + GPU misfit + GPU gradient vs central
    finite differences (h = 1e-4 relative, Richardson-extrapolated)."""
    mesh, pairs, _ = synth.make_config(0, nx=12, nz=6)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    mrdof = helpers.surface_receivers(mesh, g, 8)
    fwi = helpers.DirectFWI(g, mrdof)
    use = [pairs[3], pairs[10]]
    rng = np.random.default_rng(8)
    f_src = helpers.point_force_rhs(g, mrdof[len(mrdof) // 2])
    obs = [(rng.standard_normal(len(fwi.rdofs)) + 1j * rng.standard_normal(len(fwi.rdofs))) * 1e-9
           for _ in use]

    def chi_grad(want):
        chi, grad = 0.0, torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
        for (f, py), ob in zip(use, obs):
            o128 = torch.zeros(g.nzero, dtype=torch.complex128, device=_dev())
            ctx.assemble("B", f, py, o128)
            c, u, lam = fwi.misfit_and_fields(o128.cpu().numpy(), f_src, ob)
            chi += c
            if want:
                ctx.gradient([f], [py], 1, torch.from_numpy(u[None, None]).to(_dev()),
                             torch.from_numpy(lam[None, None]).to(_dev()), grad)
        return chi, grad.cpu().numpy()

    _, grad = chi_grad(True)
    touch = np.zeros(mesh.nnpg, bool)
    for e in range(mesh.nelem):
        if chr(mesh.cdomain[e]) == "A":
            touch[mesh.ieng[e] - 1] = True
    base = np.stack([mesh.ecoeff[0], mesh.ecoeff[1], mesh.dens])

    def chi_at(m3):
        ctx.update_model(m3[:2], m3[2])
        return chi_grad(False)[0]

    h = 1e-4
    for trial in range(3):
        dm = rng.standard_normal((3, mesh.nnpg)) * ~touch * base
        an = float(np.sum(grad * dm))
        fd1 = (chi_at(base + h * dm) - chi_at(base - h * dm)) / (2 * h)
        fd2 = (chi_at(base + h / 2 * dm) - chi_at(base - h / 2 * dm)) / h
        fd = (4 * fd2 - fd1) / 3
        assert abs(fd - an) <= 1e-6 * abs(an), (trial, fd, an)
    ctx.update_model(base[:2], base[2])
    ctx.close()


@pytest.mark.parametrize("cinv,accumulate", [("PP", False), ("SS", False), ("PP", True)])
def test_reference_gradient_matches_oracle(case0, cinv, accumulate):
    mesh, pairs, g, ctx = case0
    rg = oracle.RefGrad(mesh, g)
    nnpinv, nz, maskg = ctx.ref_gradient_info()
    assert nnpinv == rg.nnpinv and nz == rg.nz and np.array_equal(maskg, rg.maskg)
    rng = np.random.default_rng(4)
    wave = (rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
    lam = (rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
    f, py = pairs[5]
    fm = rg.cfmat(f, py, wave, lisp=(cinv == "PP"), accumulate=accumulate)
    ref = rg.adjflam(fm, lam)
    d_g = torch.zeros(nnpinv, dtype=torch.float32, device=_dev())
    ctx.cfmat_adjgrad(cinv, 1.7320508075688772, f, py, torch.from_numpy(wave).to(_dev()),
                      torch.from_numpy(lam).to(_dev()), d_g, accumulate=accumulate)
    got = d_g.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("cinv", ["PP", "SS", "PS"])
def test_vforce2_matches_oracle(case0, cinv):
    """VFORCE25_2 virtual forces with the DABMKISOB25 alpha / beta matrices:
    every COMPLEX*8 value bit-identical to the oracle."""
    mesh, pairs, g, ctx = case0
    rg = oracle.RefGrad(mesh, g)
    rng = np.random.default_rng(8)
    wave = (rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
    f, py = pairs[10]
    ref = rg.vforce2(f, py, wave, cinv)
    d_f = torch.full(ref.shape, float("nan"), dtype=torch.complex64, device=_dev())
    ctx.vforce2(cinv, f, py, torch.from_numpy(wave).to(_dev()), d_f)
    got = d_f.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("cinv,accumulate", [("PP", False), ("SS", False), ("PS", False),
                                             ("PS", True)])
def test_met225_matches_oracle(case0, cinv, accumulate):
    """MET225_MOD Hessian-vector buffers: every REAL*4 value bit-identical to
    the oracle, twice in a row (the buffers are overwritten, not added to)."""
    mesh, pairs, g, ctx = case0
    rg = oracle.RefGrad(mesh, g)
    rng = np.random.default_rng(23)
    vec = [(rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof)).astype(np.complex64)
           for _ in range(4)]
    f, py = pairs[6]
    r1, r2 = rg.met225(f, py, *vec, cinvtype=cinv, accumulate=accumulate)
    d = [torch.from_numpy(v).to(_dev()) for v in vec]
    p1 = torch.full(r1.shape, float("nan"), dtype=torch.float32, device=_dev())
    p2 = torch.full(r2.shape, float("nan"), dtype=torch.float32, device=_dev())
    for _ in range(2):
        ctx.met225(cinv, f, py, *d, p1, p2, accumulate=accumulate)
        assert np.array_equal(p1.cpu().numpy().view(np.uint32), r1.view(np.uint32))
        assert np.array_equal(p2.cpu().numpy().view(np.uint32), r2.view(np.uint32))


@pytest.mark.parametrize("cinv,accumulate", [("PP", False), ("SS", False), ("PS", False),
                                             ("PS", True)])
def test_cadj_nu_alpha_matches_oracle(case0, cinv, accumulate):
    """CADJ_NU_ALPHA right-hand sides and P3: every COMPLEX*8 / REAL*4 value
    bit-identical to the oracle, twice in a row."""
    mesh, pairs, g, ctx = case0
    rg = oracle.RefGrad(mesh, g)
    rng = np.random.default_rng(29)
    adjlam, wave = [(rng.standard_normal(g.ndof) + 1j * rng.standard_normal(g.ndof))
                    .astype(np.complex64) for _ in range(2)]
    nv = 2 if cinv == "PS" else 1
    v = rng.standard_normal(rg.nnpinv * nv).astype(np.float32)
    f, py = pairs[9]
    rb, ra, p3 = rg.cadj_nu_alpha(f, py, v, adjlam, wave, cinvtype=cinv, accumulate=accumulate)
    d_b = torch.full((g.ndof,), float("nan"), dtype=torch.complex64, device=_dev())
    d_a = torch.full((g.ndof,), float("nan"), dtype=torch.complex64, device=_dev())
    d_p = torch.full(p3.shape, float("nan"), dtype=torch.float32, device=_dev())
    for _ in range(2):
        ctx.cadj_nu_alpha(cinv, f, py, torch.from_numpy(v).to(_dev()),
                          torch.from_numpy(adjlam).to(_dev()), torch.from_numpy(wave).to(_dev()),
                          d_b, d_a, d_p, accumulate=accumulate)
        assert np.array_equal(d_b.cpu().numpy().view(np.uint32), rb.view(np.uint32))
        assert np.array_equal(d_a.cpu().numpy().view(np.uint32), ra.view(np.uint32))
        assert np.array_equal(d_p.cpu().numpy().view(np.uint32), p3.view(np.uint32))


@pytest.mark.parametrize("nvinv", [1, 2])
def test_pchadj_matches_oracle(case0, nvinv):
    """PCHADJ Jacobian blocks and preconditioner update: bit-identical to the
    oracle; HESSB is updated in place, so a second call adds the same block."""
    mesh, pairs, g, ctx = case0
    rg = oracle.RefGrad(mesh, g)
    rng = np.random.default_rng(43)
    nrhs = 9
    grns = (rng.standard_normal((nrhs, g.ndof)) + 1j * rng.standard_normal((nrhs, g.ndof))
            ).astype(np.complex64)
    fmat = (rng.standard_normal((nvinv, rg.nz)) + 1j * rng.standard_normal((nvinv, rg.nz))
            ).astype(np.complex64)
    hess = rng.standard_normal(rg.nnpinv * nvinv * nvinv).astype(np.float32)
    d_h = torch.from_numpy(hess.copy()).to(_dev())
    d_j = torch.full((rg.nnpinv * nvinv, nrhs), float("nan"), dtype=torch.complex64,
                     device=_dev())
    d_g, d_f = torch.from_numpy(grns).to(_dev()), torch.from_numpy(fmat).to(_dev())
    for rep in range(2):
        jacl = rg.pchadj(grns, fmat, hess)
        ctx.pchadj(nvinv, nrhs, d_g, d_f, d_h, d_j)
        assert np.array_equal(d_j.cpu().numpy().view(np.uint32), jacl.view(np.uint32)), rep
        assert np.array_equal(d_h.cpu().numpy().view(np.uint32), hess.view(np.uint32)), rep


def test_reference_gradient_rejects_ps(case0):
    mesh, pairs, g, ctx = case0
    d = torch.zeros(g.ndof, dtype=torch.complex64, device=_dev())
    gl = torch.zeros(16, dtype=torch.float32, device=_dev())
    with pytest.raises(Fem25Error) as ei:
        ctx.cfmat_adjgrad("PS", 1.7, 0.5, 0.0, d, d, gl)
    assert ei.value.code == 7


def test_misfit_matches_oracle(case0):
    mesh, pairs, g, ctx = case0
    mrdof = helpers.surface_receivers(mesh, g, 20)
    nrec = len(mrdof)
    rng = np.random.default_rng(9)
    nsrc = 2
    f, py = pairs[6]
    yrec = rng.uniform(-500, 500, nrec)
    recv = (1 + 0.1j * rng.standard_normal((nrec, 3))).astype(np.complex64)
    sol = (rng.standard_normal((nsrc, g.ndof)) + 1j * rng.standard_normal((nsrc, g.ndof))).astype(np.complex64)
    obs = (rng.standard_normal((nsrc, nrec, 3)) + 1j * rng.standard_normal((nsrc, nrec, 3))).astype(np.complex64)
    obs[0, 3, 1] = 0  # an absent observation
    w = rng.uniform(0.5, 1.5, (nsrc, nrec, 3)).astype(np.float32)
    d_sol = torch.from_numpy(sol).to(_dev())
    d_rhs = torch.zeros((nsrc, g.ndof), dtype=torch.complex64, device=_dev())
    est, mis = ctx.misfit(nsrc, mrdof, yrec, f, py, 12.5, recv, d_sol, obs, w, d_rhs)
    rhs = d_rhs.cpu().numpy()
    for s in range(nsrc):
        e_ref, r_ref, m_ref = oracle.misfit(g.ndof, mrdof, yrec, f, py, 12.5, recv, sol[s], obs[s], w[s])
        assert np.array_equal(est[s].view(np.uint32), e_ref.view(np.uint32))
        assert np.array_equal(rhs[s].view(np.uint32), r_ref.view(np.uint32))
        assert np.float32(m_ref) == mis[s]


def test_jacobian_error_is_reported():
    mesh, _, _ = synth.make_config(0, nx=6, nz=4)
    g = oracle.graph_build(mesh)
    # fold one interior element: swap two anchors
    bad = mesh.ieng.copy()
    e = [k for k in range(mesh.nelem) if chr(mesh.cdomain[k]) == "I"][0]
    bad[e, [1, 3]] = bad[e, [3, 1]]
    mesh.ieng = bad
    with pytest.raises(Fem25Error) as ei:
        Context(mesh, g)
    assert ei.value.code == 2


def test_nzloc_mismatch_is_rejected(case0):
    mesh, pairs, g, ctx = case0
    from fem25_b200.lib import lib as L
    import ctypes
    buf = np.zeros(4, np.complex64)
    r = L().fem25_asmble_driver(ctx.h, 4, b"B", 0.5, 0.0, buf.ctypes.data_as(ctypes.c_void_p))
    assert r == 1


# ---------------------------------------------------------------------------
# dispersive media (KMDAMP / CMDAMP): plain path only
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def case_disp():
    mesh, pairs, _ = synth.make_config(0, nx=8, nz=5)
    synth.make_dispersive(mesh, seed=5, freq0=1.0, qs_mean=30.0)
    g = oracle.graph_build(mesh)
    ctx = Context(mesh, g)
    yield mesh, pairs, g, ctx
    ctx.close()


def test_dispersive_plain_assembly_matches_oracle(case_disp):
    """KMDAMP (interior, Bielak) and CMDAMP (PML) elements: complex128 CSR and
    the COMPLEX*8 CDIST bit-identical to the oracle, below and above FREQ0."""
    mesh, pairs, g, ctx = case_disp
    for (f, py, cft) in ((0.5, pairs[6][1], "B"), (1.7, pairs[11][1], "S")):
        ref128, ref64 = oracle.asmble(mesh, g, cft, f, py)
        o128 = torch.zeros(g.nzero, dtype=torch.complex128, device=_dev())
        o64 = torch.zeros(g.nzero, dtype=torch.complex64, device=_dev())
        ctx.assemble(cft, f, py, o128, o64)
        torch.cuda.synchronize()
        a128 = o128.cpu().numpy()
        assert np.array_equal(a128.view(np.uint64), ref128.view(np.uint64)), f
        assert np.array_equal(o64.cpu().numpy().view(np.uint32), ref64.view(np.uint32)), f
    out = ctx.asmble_driver("B", 0.5, pairs[6][1])
    _, ref64 = oracle.asmble(mesh, g, "B", 0.5, pairs[6][1])
    assert np.array_equal(out.view(np.uint32), ref64.view(np.uint32))


def test_dispersive_batched_and_gradient_rejected(case_disp):
    mesh, pairs, g, ctx = case_disp
    ring = torch.zeros(2 * g.nzero, dtype=torch.float64, device=_dev())
    with pytest.raises(Fem25Error) as ei:
        ctx.assemble_batch(["B"], [0.5], [0.0], ring, 2 * g.nzero, 1)
    assert ei.value.code == 7
    u = torch.zeros((1, 1, g.ndof), dtype=torch.complex128, device=_dev())
    d_g = torch.zeros((3, mesh.nnpg), dtype=torch.float64, device=_dev())
    for prec in (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE):
        with pytest.raises(Fem25Error) as ei:
            ctx.gradient([0.5], [0.0], 1, u, u, d_g, prec)
        assert ei.value.code == 7
    with pytest.raises(Fem25Error) as ei:
        ctx.gradient_accumulate([0.5], [0.0], 1, u, u)
    assert ei.value.code == 7
    with pytest.raises(Fem25Error) as ei:
        ctx.gradient_finalize(d_g)
    assert ei.value.code == 7
